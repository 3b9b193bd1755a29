"""Domain decomposition into slabs with a halo exchange after every PT iteration.

The reference's distributed architecture (Chmy.Distributed with a Cartesian
topology; src/Models/FullStokes/Isothermal/Isothermal.jl:101-107) splits the
grid into per-rank subdomains and exchanges the halos of V and η_next after
update_V!.  Here a domain is split into R slabs along x (or y), one model per
rank.  Along a periodic dimension the slabs form a ring and each is declared
periodic along it; along a bounded one they form a chain: the sides between
ranks are FI_BC_HALO (the neighbour's values arrive by the exchange) and the two
outer sides keep the domain's own conditions.  After every iteration each slab
sends its boundary layers to its neighbours and unpacks what it receives into its
ghost layers (fi_model_halo_*).  The sweep recomputes the ghost stresses from the
exchanged velocities, so the split run reproduces the undivided domain exactly.

Transport: ``TorchTransport`` moves the messages with torch.distributed
point-to-point operations (NCCL between GPUs, gloo on CPU), grouped in one
``batch_isend_irecv`` so no ordering of blocking calls can deadlock.  Every rank
posts its operations in the same order: send to the low neighbour, receive from
the high one, send to the high neighbour, receive from the low one.  With two
ranks both neighbours are the same peer; the messages still match because each
pair of sends and receives is posted in that order (and tagged, for gloo).

A slab needs an ``exchange`` step only when R > 1: with one rank the sweep's own
periodic images are already the neighbour's values.

Convergence.  The driver's check (tm_stokes_chmy.jl:283-305) takes the residual
norms every ncheck iterations; the reference's distributed driver reduces them
over the ranks with MPI.Allreduce(MAX) (tm_stokes_mpi_wip.jl:21-22,157-163).
``reduce_norms`` does the same over the FI_NORMS_LEN slots: the ∞-norms of r_P and
r_V, max|V| and the non-finite flag by maximum (each equals the undivided
domain's value exactly), the L2 norms as the root of the summed squares (the node
layer two slabs share along the split dimension then counts on both sides).
``Slab.solve`` is the driver loop on top: every rank takes the same checks and, from
the same reduced norms, the same decision.

Streams.  With device buffers the pack, the point-to-point operations and the
unpack are all ordered on the model's own stream (the transfers are issued with it
as torch's current stream, and waiting on them orders that stream after them), so
an exchange needs no host synchronisation.
"""
from __future__ import annotations

import math
from typing import Callable, Optional

import numpy as np

TAG_TO_LOW, TAG_TO_HIGH = 11, 12
NORMS_LEN = 12
NORM_MAX_SLOTS = (0, 1, 2, 3, 8, 9, 10, 11)  # ∞-norms of r_P, r_Vx..z; max|V|; non-finite flag
NORM_L2_SLOTS = (4, 5, 6, 7)                  # L2 norms of r_P, r_Vx..z


def combine_norms(per_rank) -> np.ndarray:
    """The norm vector of the whole domain from the ranks' vectors (what
    ``TorchTransport.allreduce_norms`` computes with collectives)."""
    per_rank = [np.asarray(r, dtype=np.float64) for r in per_rank]
    out = np.zeros(NORMS_LEN)
    for q in NORM_MAX_SLOTS:
        out[q] = max(r[q] for r in per_rank)
    for q in NORM_L2_SLOTS:
        out[q] = math.sqrt(sum(r[q] * r[q] for r in per_rank))
    return out


def measure_of(norms, measure: str = "abs_inf", nd: int = 3, rho_g_inf: float = 1.0, length_z: float = 1.0) -> float:
    """Convergence measure of a norm vector, as fi_model_solve computes it:
    abs_inf = max ∞-norm of r_P and r_V; rel_slab = max(|r_V|∞ / |ρg|∞,
    |r_P|∞ · L_z / max|V|)."""
    n = norms
    if measure == "rel_slab":
        rv = max(n[1], n[2], n[3] if nd == 3 else 0.0)
        vmax = max(n[8], n[9], n[10])
        a = rv / (rho_g_inf if rho_g_inf > 0 else 1.0)
        b = n[0] * length_z / vmax if vmax > 0 else n[0]
        return max(a, b)
    if measure != "abs_inf":
        raise ValueError(measure)
    return max(n[0], n[1], n[2], n[3])


class TorchTransport:
    """Point-to-point exchange over torch.distributed (NCCL or gloo) between the
    slabs of a split dimension: a ring when the dimension is periodic, else a chain
    (the first rank has no low neighbour, the last no high one)."""

    def __init__(self, group=None, periodic: bool = True):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.periodic = periodic

    def neighbours(self):
        """(low, high) neighbour ranks, None where a chain ends."""
        if self.periodic:
            return (self.rank - 1) % self.size, (self.rank + 1) % self.size
        return (self.rank - 1 if self.rank > 0 else None, self.rank + 1 if self.rank < self.size - 1 else None)

    def _global(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def allreduce_norms(self, norms) -> np.ndarray:
        """``combine_norms`` over the ranks: one MAX and one SUM all-reduce, taken
        in the same order on every rank."""
        import torch
        d = self.dist
        dev = "cuda" if d.get_backend(self.group) == "nccl" else "cpu"
        n = np.asarray(norms, dtype=np.float64)
        mx = torch.tensor([n[q] for q in NORM_MAX_SLOTS], dtype=torch.float64, device=dev)
        sq = torch.tensor([n[q] * n[q] for q in NORM_L2_SLOTS], dtype=torch.float64, device=dev)
        d.all_reduce(mx, op=d.ReduceOp.MAX, group=self.group)
        d.all_reduce(sq, op=d.ReduceOp.SUM, group=self.group)
        out = np.zeros(NORMS_LEN)
        out[list(NORM_MAX_SLOTS)] = mx.cpu().numpy()
        out[list(NORM_L2_SLOTS)] = np.sqrt(sq.cpu().numpy())
        return out

    def exchange(self, send_low, send_high, recv_low, recv_high) -> None:
        """send_low -> low neighbour (its recv_high), send_high -> high neighbour
        (its recv_low); the operations toward a missing neighbour (a chain's end) are
        left out.  Waiting on the operations orders torch's current stream after them
        (device tensors) or blocks until they completed (host tensors)."""
        d = self.dist
        low, high = self.neighbours()
        ops = []
        if low is not None:
            ops.append(d.P2POp(d.isend, send_low, self._global(low), self.group, TAG_TO_LOW))
        if high is not None:
            ops.append(d.P2POp(d.irecv, recv_high, self._global(high), self.group, TAG_TO_LOW))
            ops.append(d.P2POp(d.isend, send_high, self._global(high), self.group, TAG_TO_HIGH))
        if low is not None:
            ops.append(d.P2POp(d.irecv, recv_low, self._global(low), self.group, TAG_TO_HIGH))
        if not ops:
            return
        for req in d.batch_isend_irecv(ops):
            req.wait()


class Slab:
    """One rank's subdomain: a model plus its halo buffers and transport.

    ``model`` provides ``halo_bytes(dim, side, what)``, ``halo_pack(dim, side, ptr,
    what)``, ``halo_unpack(dim, side, ptr, what)`` and ``advance(n)`` (a library
    model, or any object with the same methods); ``alloc(nbytes)`` returns a buffer
    tensor for messages (device memory for a library model) and ``ptr(t)`` its
    address.
    """

    def __init__(self, model, dim: int, transport, alloc: Optional[Callable] = None):
        self.model, self.dim, self.transport = model, int(dim), transport
        self.iterations = 0
        if alloc is None:
            import torch
            dev = torch.device("cuda", torch.cuda.current_device())
            alloc = (lambda nb: torch.empty(nb, dtype=torch.uint8, device=dev))
        # the sides with a neighbour (both in a ring; a chain's ends have one)
        low, high = transport.neighbours() if transport.size > 1 else (None, None)
        self.sides = tuple(s for s, nb in ((0, low), (1, high)) if nb is not None)
        self.buf = {}
        for what in ("iteration", "state"):
            nb_low, nb_high = model.halo_bytes(self.dim, 0, what), model.halo_bytes(self.dim, 1, what)
            # messages sent toward a side and received from the opposite one have equal sizes
            self.buf[what] = {"send_low": alloc(nb_low), "send_high": alloc(nb_high),
                              "recv_high": alloc(nb_low), "recv_low": alloc(nb_high)}

    def _ptr(self, t):
        # a host-side model (halo_takes_tensors) packs into the tensor itself
        return t if getattr(self.model, "halo_takes_tensors", False) else t.data_ptr()

    def _steps(self, what):
        b, m, d = self.buf[what], self.model, self.dim
        for side, key in ((0, "send_low"), (1, "send_high")):
            if side in self.sides:
                m.halo_pack(d, side, self._ptr(b[key]), what)
        yield
        self.transport.exchange(b["send_low"], b["send_high"], b["recv_low"], b["recv_high"])
        for side, key in ((0, "recv_low"), (1, "recv_high")):
            if side in self.sides:
                m.halo_unpack(d, side, self._ptr(b[key]), what)

    def exchange(self, what: str = "iteration") -> None:
        if self.transport.size == 1:
            return
        b, m = self.buf[what], self.model
        on_device = hasattr(b["send_low"], "is_cuda") and b["send_low"].is_cuda and hasattr(m, "stream_ptr")
        steps = self._steps(what)
        if on_device:
            # pack, transfers and unpack in order on the model's stream
            import torch
            with torch.cuda.stream(torch.cuda.ExternalStream(m.stream_ptr)):
                for _ in steps:
                    pass
        else:
            next(steps)
            if hasattr(m, "synchronize"):
                m.synchronize()  # the packed messages are complete before a host transport reads them
            for _ in steps:
                pass

    def advance(self, niter: int, overlap: bool = False) -> None:
        """niter PT iterations, each followed by the halo exchange of V and η.  With
        ``overlap`` (a library model) each iteration runs in two halves: the tiles of
        the split faces, then the others on a second stream while the halo moves on
        the model's stream (fi_model_advance_begin / _end).  The overlap pays only
        where the transfer takes longer than the second launch's tail: at 511^3 FP64
        per rank the two launches cost 64-85 us more than one sweep, against about
        25 us of NVLink transfer, so the default is the plain iteration."""
        for _ in range(int(niter)):
            if overlap and self.transport.size > 1:
                self.model.advance_begin(self.dim)
                self.model.advance_end()
            else:
                self.model.advance(1)
            self.exchange("iteration")
            self.iterations += 1

    def residual_norms(self) -> np.ndarray:
        """The residual norms of the whole domain (every rank gets the same vector)."""
        local = self.model.residual_norms()
        if self.transport.size == 1:
            return np.asarray(local, dtype=np.float64)
        return self.transport.allreduce_norms(local)

    def solve(self, *, max_iter: int, ncheck: int, tol: float, measure: str = "abs_inf", rho_g_inf: float = 1.0,
              length_z: float = 1.0, nd: int = 3, overlap: bool = False) -> dict:
        """The driver loop (tm_stokes_chmy.jl:283-305) over the split domain: ncheck
        iterations with their exchanges, then the reduced norms and the decision,
        which every rank takes alike; stops on convergence (measure < tol), on a
        non-finite residual or after max_iter iterations (as fi_model_solve)."""
        it, rep = 0, {"converged": False, "diverged": False, "measure": float("nan"), "norms": None}
        while it < max_iter:
            k = min(ncheck, max_iter - it)
            self.advance(k, overlap=overlap)
            it += k
            norms = self.residual_norms()
            meas = measure_of(norms, measure, nd, rho_g_inf, length_z)
            rep.update(measure=meas, norms=norms.tolist())
            if norms[11] != 0.0 or not math.isfinite(meas):
                rep["diverged"] = True
                break
            if meas < tol:
                rep["converged"] = True
                break
        rep["iterations"] = it
        return rep


def advance_local(slabs, dim: int, niter: int, overlap: bool = False, periodic: bool = True) -> None:
    """``Slab.advance`` for a ring (periodic) or chain of slabs held by one process
    (one device): every slab's iteration (in two halves with ``overlap``), then
    ``exchange_local``."""
    for _ in range(int(niter)):
        for m in slabs:
            if overlap:
                m.advance_begin(dim)
            else:
                m.advance(1)
        if overlap:
            for m in slabs:
                m.advance_end()
        exchange_local(slabs, dim, periodic=periodic)


def exchange_local(slabs, dim: int, what: str = "iteration", periodic: bool = True) -> None:
    """The halo exchange of a ring (periodic) or chain of slabs held by one process
    (one device): every slab packs its messages toward its neighbours, each is
    copied to the neighbour that expects it, every slab unpacks.  The same messages
    and layers as a multi-rank run over ``TorchTransport``."""
    import torch
    R = len(slabs)
    if R == 1:
        return

    def has(r, side):
        return periodic or (r > 0 if side == 0 else r < R - 1)

    bufs = []
    for r, m in enumerate(slabs):
        lo = torch.empty(m.halo_bytes(dim, 0, what), dtype=torch.uint8, device="cuda")
        hi = torch.empty(m.halo_bytes(dim, 1, what), dtype=torch.uint8, device="cuda")
        if has(r, 0):
            m.halo_pack(dim, 0, lo.data_ptr(), what)
        if has(r, 1):
            m.halo_pack(dim, 1, hi.data_ptr(), what)
        m.synchronize()
        bufs.append((lo, hi))
    for r, m in enumerate(slabs):
        torch.cuda.synchronize()
        if has(r, 0):
            from_low = bufs[(r - 1) % R][1].clone()   # the low neighbour's message toward its high side
            torch.cuda.synchronize()
            m.halo_unpack(dim, 0, from_low.data_ptr(), what)
        if has(r, 1):
            from_high = bufs[(r + 1) % R][0].clone()  # the high neighbour's message toward its low side
            torch.cuda.synchronize()
            m.halo_unpack(dim, 1, from_high.data_ptr(), what)
        m.synchronize()


def halo_plan(nd: int, n, dim: int, side: int, what: str = "iteration", pack: bool = True, library: str = "fast"):
    """The library's layer plan of a halo message (fi_halo_plan, host only): a list
    of (field name, layer index along ``dim``) in message order, each one whole
    storage plane of the other dimensions."""
    import ctypes as C
    from . import _lib as L
    lib = L.load(library)
    nn = (C.c_int32 * 3)(*(list(n) + [0] * (3 - len(n))))
    w = {"iteration": 0, "state": 1}[what]
    cnt = C.c_int32()
    L.check(lib, lib.fi_halo_plan(nd, nn, dim, side, w, int(pack), None, None, 0, C.byref(cnt)))
    f, l = (C.c_int32 * cnt.value)(), (C.c_int32 * cnt.value)()
    L.check(lib, lib.fi_halo_plan(nd, nn, dim, side, w, int(pack), f, l, cnt.value, C.byref(cnt)))
    return [(L.FIELD_NAMES[f[k]], l[k]) for k in range(cnt.value)]


def solve_local(slabs, dim: int, *, max_iter: int, ncheck: int, tol: float, measure: str = "abs_inf",
                rho_g_inf: float = 1.0, length_z: float = 1.0, overlap: bool = False, periodic: bool = True) -> dict:
    """``Slab.solve`` for a ring of slabs held by one process (one device): the same
    iterations, exchanges (``exchange_local``), norm reduction (``combine_norms``)
    and decision as a multi-rank run."""
    nd = slabs[0].grid.ndims if hasattr(slabs[0], "grid") else 3
    it, rep = 0, {"converged": False, "diverged": False, "measure": float("nan"), "norms": None}
    while it < max_iter:
        k = min(ncheck, max_iter - it)
        advance_local(slabs, dim, k, overlap=overlap, periodic=periodic)
        it += k
        norms = combine_norms([m.residual_norms() for m in slabs])
        meas = measure_of(norms, measure, nd, rho_g_inf, length_z)
        rep.update(measure=meas, norms=norms.tolist())
        if norms[11] != 0.0 or not math.isfinite(meas):
            rep["diverged"] = True
            break
        if meas < tol:
            rep["converged"] = True
            break
    rep["iterations"] = it
    return rep


def slab_of(global_interior, dim: int, rank: int, size: int, vertex: bool):
    """The part of a global interior array (numpy order (z, y, x) / (y, x)) that
    slab ``rank`` of ``size`` holds along ``dim``: its n cells, or its n+1 nodes for
    a field Vertex-located along ``dim`` (a slab's last node is its high
    neighbour's first)."""
    axis = global_interior.ndim - 1 - dim
    ncells = global_interior.shape[axis] - (1 if vertex else 0)
    if ncells % size:
        raise ValueError("the split dimension must divide evenly among the ranks")
    n = ncells // size
    sl = [slice(None)] * global_interior.ndim
    sl[axis] = slice(rank * n, (rank + 1) * n + (1 if vertex else 0))
    return global_interior[tuple(sl)]


__all__ = ["TorchTransport", "Slab", "advance_local", "exchange_local", "solve_local", "slab_of", "combine_norms", "measure_of", "halo_plan"]
