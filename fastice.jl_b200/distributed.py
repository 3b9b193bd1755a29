"""Domain decomposition into slabs with a halo exchange after every PT iteration.

The reference's distributed architecture (Chmy.Distributed with a Cartesian
topology; src/Models/FullStokes/Isothermal/Isothermal.jl:101-107) splits the
grid into per-rank subdomains and exchanges the halos of V and η_next after
update_V!.  Here a domain that is periodic along x (or y) is split into R slabs
along that dimension, one model per rank, each declared periodic along the split
dimension; after every iteration each slab sends its boundary layers to its two
neighbours (a ring) and unpacks what it receives into its ghost layers
(fi_model_halo_*).  The sweep recomputes the ghost stresses from the exchanged
velocities, so the split run reproduces the undivided domain exactly.

Transport: ``TorchTransport`` moves the messages with torch.distributed
point-to-point operations (NCCL between GPUs, gloo on CPU), grouped in one
``batch_isend_irecv`` so no ordering of blocking calls can deadlock.  Every rank
posts its operations in the same order: send to the low neighbour, receive from
the high one, send to the high neighbour, receive from the low one.  With two
ranks both neighbours are the same peer; the messages still match because each
pair of sends and receives is posted in that order (and tagged, for gloo).

A slab needs an ``exchange`` step only when R > 1: with one rank the sweep's own
periodic images are already the neighbour's values.
"""
from __future__ import annotations

from typing import Callable, Optional

TAG_TO_LOW, TAG_TO_HIGH = 11, 12


class TorchTransport:
    """Ring point-to-point exchange over torch.distributed (NCCL or gloo)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def neighbours(self):
        return (self.rank - 1) % self.size, (self.rank + 1) % self.size

    def _global(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def exchange(self, send_low, send_high, recv_low, recv_high) -> None:
        """send_low -> low neighbour (its recv_high), send_high -> high neighbour
        (its recv_low); blocks until all four operations completed."""
        d = self.dist
        low, high = (self._global(r) for r in self.neighbours())
        ops = [d.P2POp(d.isend, send_low, low, self.group, TAG_TO_LOW),
               d.P2POp(d.irecv, recv_high, high, self.group, TAG_TO_LOW),
               d.P2POp(d.isend, send_high, high, self.group, TAG_TO_HIGH),
               d.P2POp(d.irecv, recv_low, low, self.group, TAG_TO_HIGH)]
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

    def __init__(self, model, dim: int, transport, alloc: Optional[Callable] = None, stream_ctx=None):
        self.model, self.dim, self.transport = model, int(dim), transport
        self.stream_ctx = stream_ctx
        if alloc is None:
            import torch
            dev = torch.device("cuda", torch.cuda.current_device())
            alloc = (lambda nb: torch.empty(nb, dtype=torch.uint8, device=dev))
        self.buf = {}
        for what in ("iteration", "state"):
            nb_low, nb_high = model.halo_bytes(self.dim, 0, what), model.halo_bytes(self.dim, 1, what)
            # messages sent toward a side and received from the opposite one have equal sizes
            self.buf[what] = {"send_low": alloc(nb_low), "send_high": alloc(nb_high),
                              "recv_high": alloc(nb_low), "recv_low": alloc(nb_high)}

    def _ptr(self, t):
        # a host-side model (halo_takes_tensors) packs into the tensor itself
        return t if getattr(self.model, "halo_takes_tensors", False) else t.data_ptr()

    def exchange(self, what: str = "iteration") -> None:
        if self.transport.size == 1:
            return
        b, m, d = self.buf[what], self.model, self.dim
        m.halo_pack(d, 0, self._ptr(b["send_low"]), what)
        m.halo_pack(d, 1, self._ptr(b["send_high"]), what)
        if self.stream_ctx is not None:
            with self.stream_ctx():
                self.transport.exchange(b["send_low"], b["send_high"], b["recv_low"], b["recv_high"])
        else:
            if hasattr(m, "synchronize"):
                m.synchronize()
            self.transport.exchange(b["send_low"], b["send_high"], b["recv_low"], b["recv_high"])
        m.halo_unpack(d, 0, self._ptr(b["recv_low"]), what)
        m.halo_unpack(d, 1, self._ptr(b["recv_high"]), what)

    def advance(self, niter: int) -> None:
        """niter PT iterations, each followed by the halo exchange of V and η."""
        for _ in range(int(niter)):
            self.model.advance(1)
            self.exchange("iteration")


def exchange_local(slabs, dim: int, what: str = "iteration") -> None:
    """The halo exchange of a ring of slabs held by one process (one device):
    every slab packs its two messages, each is copied to the neighbour that
    expects it, every slab unpacks.  The same messages and layers as a
    multi-rank run over ``TorchTransport``."""
    import torch
    R = len(slabs)
    if R == 1:
        return
    bufs = []
    for m in slabs:
        lo = torch.empty(m.halo_bytes(dim, 0, what), dtype=torch.uint8, device="cuda")
        hi = torch.empty(m.halo_bytes(dim, 1, what), dtype=torch.uint8, device="cuda")
        m.halo_pack(dim, 0, lo.data_ptr(), what)
        m.halo_pack(dim, 1, hi.data_ptr(), what)
        m.synchronize()
        bufs.append((lo, hi))
    for r, m in enumerate(slabs):
        from_low = bufs[(r - 1) % R][1].clone()   # the low neighbour's message toward its high side
        from_high = bufs[(r + 1) % R][0].clone()  # the high neighbour's message toward its low side
        torch.cuda.synchronize()
        m.halo_unpack(dim, 0, from_low.data_ptr(), what)
        m.halo_unpack(dim, 1, from_high.data_ptr(), what)
        m.synchronize()


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


__all__ = ["TorchTransport", "Slab", "exchange_local", "slab_of"]
