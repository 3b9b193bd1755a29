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


def _globals(R):
    rng = np.random.default_rng(3)
    n = N_LOCAL * R
    return 0.5 * rng.standard_normal(n), 0.5 * rng.standard_normal(n + 1)


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
