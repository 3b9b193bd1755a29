"""The multi-rank path of the domain split (fastice_b200.distributed.Slab over
TorchTransport) on CPU: world-size 2 and 3 gloo process groups, each rank holding
one slab of a periodic line of cells.  The slab model here is a host-side stand-in
with the library's halo layers (Center fields: one layer each way; Vertex fields:
nodes 1 and 2 toward the low neighbour, node n toward the high one) and a sweep
that, like the fused sweep, recomputes its ghost cells from ghost nodes and writes
periodic images of its own nodes.  The split run must equal the undivided one."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import load_fastice

N_LOCAL, STEPS = 7, 9


class LineSlab:
    """c: cells 1..n (ghosts 0, n+1); v: nodes 1..n+1 (ghosts 0, n+2)."""

    halo_takes_tensors = True

    def __init__(self, c, v):
        self.n = len(c)
        self.c = np.zeros(self.n + 3)
        self.v = np.zeros(self.n + 3)
        self.c[1:self.n + 1] = c
        self.v[1:self.n + 2] = v
        self._images()
        self.c[0], self.c[self.n + 1] = self.c[self.n], self.c[1]

    def _images(self):
        n = self.n
        self.v[0], self.v[n + 1], self.v[n + 2] = self.v[n], self.v[1], self.v[2]

    def advance(self, k):
        n = self.n
        for _ in range(k):
            c = self.c.copy()
            c[0:n + 2] = self.c[0:n + 2] + 0.3 * (self.v[1:n + 3] - self.v[0:n + 2]) - 0.1 * self.c[0:n + 2] ** 2
            v = self.v.copy()
            v[1:n + 1] = self.v[1:n + 1] + 0.2 * (c[1:n + 1] - c[0:n])
            self.c, self.v = c, v
            self._images()

    def _layers(self, side, pack, what):
        n = self.n
        out = []
        if what == "state":
            out.append((self.c, (1,) if pack and side == 0 else (n,) if pack else (0,) if side == 0 else (n + 1,)))
        out.append((self.v, ((1, 2) if side == 0 else (n,)) if pack else ((0,) if side == 0 else (n + 1, n + 2))))
        return out

    def residual_norms(self):
        """A norm vector in the library's layout from the slab's own cells and nodes:
        ∞-norms of c (slot 0) and v (slot 1), L2 of c (slot 4), max|v| (slot 8), flag."""
        n = self.n
        c, v = self.c[1:n + 1], self.v[1:n + 2]
        out = np.zeros(12)
        out[0], out[1] = np.max(np.abs(c)), np.max(np.abs(v))
        out[4] = np.sqrt(np.sum(c * c))
        out[8] = np.max(np.abs(v))
        out[11] = 0.0 if np.isfinite(c).all() and np.isfinite(v).all() else 1.0
        return out

    def halo_bytes(self, dim, side, what="iteration"):
        return 8 * sum(len(ix) for _, ix in self._layers(side, True, what))

    def halo_pack(self, dim, side, buf, what="iteration"):
        vals = [a[i] for a, ix in self._layers(side, True, what) for i in ix]
        buf.view(torch.float64)[:] = torch.tensor(vals, dtype=torch.float64)

    def halo_unpack(self, dim, side, buf, what="iteration"):
        vals = buf.view(torch.float64).tolist()
        q = 0
        for a, ix in self._layers(side, False, what):
            for i in ix:
                a[i] = vals[q]
                q += 1


def _globals(R, scale=0.5):
    rng = np.random.default_rng(3)
    n = N_LOCAL * R
    return scale * rng.standard_normal(n), scale * rng.standard_normal(n + 1)


def _rank(rank, R, port, out):
    import torch.distributed as dist
    fi = load_fastice()
    from fastice_b200 import distributed as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=R)
    try:
        c, v = _globals(R)
        s = LineSlab(D.slab_of(c, 0, rank, R, False), D.slab_of(v, 0, rank, R, True))
        slab = D.Slab(s, 0, D.TorchTransport(), alloc=lambda nb: torch.empty(nb, dtype=torch.uint8))
        slab.exchange("state")
        slab.advance(STEPS)
        out.put((rank, s.c[1:s.n + 1].copy(), s.v[1:s.n + 2].copy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("R", [2, 3])
def test_gloo_ranks_reproduce_the_undivided_line(R):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, R, port, out)) for r in range(R)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(R):
        rank, c, v = out.get(timeout=120)
        got[rank] = (c, v)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    c, v = _globals(R)
    whole = LineSlab(c, v)
    whole.advance(STEPS)
    n = N_LOCAL
    for r in range(R):
        np.testing.assert_array_equal(got[r][0], whole.c[1 + r * n:1 + (r + 1) * n])
        np.testing.assert_array_equal(got[r][1], whole.v[1 + r * n:2 + (r + 1) * n])


# ---- the distributed driver loop: reduced norms, the same decision on every rank
NCHECK = 3
SOLVE_SCALE = 0.05  # small enough that the line's quadratic term keeps the 24 iterations finite


class _Single:
    size = 1


def _whole_measures(R, checks):
    load_fastice()
    from fastice_b200 import distributed as D
    c, v = _globals(R, SOLVE_SCALE)
    whole = LineSlab(c, v)
    out = []
    for _ in range(checks):
        whole.advance(NCHECK)
        out.append(D.measure_of(whole.residual_norms(), "abs_inf"))
    return out


def _solve_rank(rank, R, port, tol, out):
    import torch.distributed as dist
    load_fastice()
    from fastice_b200 import distributed as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=R)
    try:
        c, v = _globals(R, SOLVE_SCALE)
        s = LineSlab(D.slab_of(c, 0, rank, R, False), D.slab_of(v, 0, rank, R, True))
        slab = D.Slab(s, 0, D.TorchTransport(), alloc=lambda nb: torch.empty(nb, dtype=torch.uint8))
        slab.exchange("state")
        rep = slab.solve(max_iter=8 * NCHECK, ncheck=NCHECK, tol=tol, measure="abs_inf")
        out.put((rank, rep["iterations"], rep["measure"], rep["converged"], rep["norms"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("R", [2, 3])
def test_gloo_ranks_take_the_undivided_convergence_decision(R):
    load_fastice()
    from fastice_b200 import distributed as D
    meas = _whole_measures(R, 8)
    # converge at the first check whose measure is below the third check's (inclusive)
    tol = meas[2] * (1 + 1e-12)
    k = next(q for q, m in enumerate(meas) if m < tol)
    # the same loop on the undivided line (one rank, no exchange) decides at check k
    c, v = _globals(R, SOLVE_SCALE)
    whole = D.Slab(LineSlab(c, v), 0, _Single(), alloc=lambda nb: torch.empty(nb, dtype=torch.uint8))
    ref = whole.solve(max_iter=8 * NCHECK, ncheck=NCHECK, tol=tol, measure="abs_inf")
    assert ref["converged"] and ref["iterations"] == (k + 1) * NCHECK
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_solve_rank, args=(r, R, port, tol, out)) for r in range(R)]
    for p in procs:
        p.start()
    got = [out.get(timeout=120) for _ in range(R)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, its, m, conv, norms in got:
        assert conv and its == ref["iterations"], (rank, its, ref)
        assert m == ref["measure"]
        # ∞-norms and max|V| reduce by maximum: equal to the undivided line's
        np.testing.assert_array_equal(np.asarray(norms)[[0, 1, 8, 11]], np.asarray(ref["norms"])[[0, 1, 8, 11]])
        # the L2 norm of the cells (no shared cells) is the root of the summed squares
        np.testing.assert_allclose(norms[4], ref["norms"][4], rtol=1e-14)


def test_combine_norms_slots():
    load_fastice()
    from fastice_b200 import distributed as D
    a = np.arange(12, dtype=float)
    b = a[::-1].copy()
    c = D.combine_norms([a, b])
    for q in (0, 1, 2, 3, 8, 9, 10, 11):
        assert c[q] == max(a[q], b[q])
    for q in (4, 5, 6, 7):
        assert c[q] == pytest.approx(np.hypot(a[q], b[q]))


def test_halo_messages_fit_one_pack_launch():
    """Every message's layers go to one pack or unpack launch whose layer table holds
    16 entries: the longest plan (3D state, split along x or y) has 14 layers, and a
    message's byte count is its layers times one storage plane."""
    load_fastice()
    from fastice_b200 import distributed as D
    n = (7, 6, 5)
    longest = 0
    for nd in (2, 3):
        for dim in (0, 1):
            for side in (0, 1):
                for what in ("iteration", "state"):
                    for pack in (True, False):
                        plan = D.halo_plan(nd, n[:nd], dim, side, what, pack)
                        longest = max(longest, len(plan))
                        assert len(plan) <= 16
                        assert all(name in ("Vx", "Vy", "Vz", "eta") for name, _ in plan) or what == "state"
    assert longest == 14


# ---- the library's own halo layer plan (fi_halo_plan) over gloo ranks
SHAPE_LOCAL = (6, 5, 4)


def _field_global(name, dim, R, seed, extra=0):
    """Values of a field along a split dimension: positions 1..N (N = R * n; one more
    node for a vertex field of a bounded dimension, extra=1), every storage
    position (ghosts included) along the other dims."""
    rng = np.random.default_rng(seed)
    nl = list(SHAPE_LOCAL)
    e = [x + 3 for x in nl]
    e[dim] = nl[dim] * R + extra
    return rng.standard_normal(tuple(reversed(e)))  # numpy order (z, y, x)


def _local_index(r, n, N, i, periodic=True):
    """Position index (0-based) in the global array of a slab's index i; None past a
    bounded dimension's ends."""
    q = r * n + i - 1
    if periodic:
        return q % N
    return q if 0 <= q < N else None


def _layer(a, dim, i):
    return a[:, :, i] if dim == 0 else a[:, i, :]


def _plan_rank(rank, R, dim, what, port, out, periodic=True):
    import torch.distributed as dist
    fi = load_fastice()
    from fastice_b200 import distributed as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=R)
    try:
        n = SHAPE_LOCAL[dim]
        N = n * R
        plans = {(side, pk): D.halo_plan(3, SHAPE_LOCAL, dim, side, what, pack=pk) for side in (0, 1)
                 for pk in (True, False)}
        names = sorted({f for pl in plans.values() for f, _ in pl})
        local = {}
        glob = {}
        for k, name in enumerate(names):
            vert = fi._lib.FIELD_LOC[name][dim] == 1
            extra = 1 if (vert and not periodic) else 0
            g = glob[name] = _field_global(name, dim, R, 100 + k, extra)
            shape = list(reversed([x + 3 for x in SHAPE_LOCAL]))
            a = np.full(shape, np.nan)
            for i in range(1, n + (2 if vert else 1)):
                _layer(a, dim, i)[...] = np.take(g, _local_index(rank, n, N + extra, i, periodic), axis=2 - dim)
            local[name] = a

        class Host:
            halo_takes_tensors = True

            def halo_bytes(self, d, side, what_):
                return 8 * len(plans[(side, True)]) * _layer(local[names[0]], d, 0).size

            def halo_pack(self, d, side, buf, what_):
                vals = np.concatenate([_layer(local[f], d, i).ravel() for f, i in plans[(side, True)]])
                buf.view(torch.float64)[:] = torch.from_numpy(vals)

            def halo_unpack(self, d, side, buf, what_):
                vals = buf.view(torch.float64).numpy()
                q = 0
                for f, i in plans[(side, False)]:
                    L = _layer(local[f], d, i)
                    L[...] = vals[q:q + L.size].reshape(L.shape)
                    q += L.size

        slab = D.Slab(Host(), dim, D.TorchTransport(periodic=periodic),
                      alloc=lambda nb: torch.empty(nb, dtype=torch.uint8))
        slab.exchange(what)
        bad = []
        for k, name in enumerate(names):
            g = glob[name]
            vert = fi._lib.FIELD_LOC[name][dim] == 1
            extra = 1 if (vert and not periodic) else 0
            for i in range(0, n + (3 if vert else 2)):
                q = _local_index(rank, n, N + extra, i, periodic)
                got = _layer(local[name], dim, i)
                if q is None:  # past a chain's end: no neighbour wrote it
                    if not np.isnan(got).all():
                        bad.append((name, i, "written"))
                elif not np.array_equal(got, np.take(g, q, axis=2 - dim)):
                    bad.append((name, i))
        out.put((rank, bad, names))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("R,dim,what,periodic", [(2, 0, "iteration", True), (3, 0, "state", True),
                                                 (3, 1, "iteration", True), (2, 1, "state", True),
                                                 (3, 0, "iteration", False), (2, 1, "state", False)])
def test_gloo_ranks_fill_ghost_layers_by_the_library_plan(R, dim, what, periodic):
    # every slab's ghost layers (and node n+1, which the high neighbour owns) must
    # hold the domain's values after one exchange by the library's plan: a ring over
    # a periodic dimension, or a chain over a bounded one (whose outer ghosts stay)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_plan_rank, args=(r, R, dim, what, port, out, periodic)) for r in range(R)]
    for p in procs:
        p.start()
    got = [out.get(timeout=120) for _ in range(R)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, bad, names in got:
        assert not bad, (rank, bad)
        assert ("P" in names) == (what == "state") and "Vx" in names and "eta" in names
