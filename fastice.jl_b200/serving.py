"""Continuous-batching solve server: a request loop that admits PT solves of
different sizes by a device-memory budget, keeps their fields resident until
they converge, and overlaps their work on the GPU.

No counterpart in the reference, whose drivers run one model to convergence per
process (scripts_future_API/tm_stokes_chmy.jl:283-305).  Every request follows
its own model's PT iteration and check cadence exactly, so its result is the same
served alone or in the mix:

* 2D requests join one :class:`BatchedStokes2D`; each loop turn runs one
  check-to-check round (ncheck iterations, device-side check, retirement and
  work-list compaction) of every 2D member still iterating;
* 3D requests (immersed-boundary models) each keep their own model and CUDA
  stream; each loop turn queues ncheck iterations on every 3D stream before the 2D
  round runs, so their sweeps overlap each other's and the batch's, then takes each
  3D model's residual check.  ``share3d=True`` advances them instead by shared
  launches (:class:`BatchedIB3D`), which on the scaled request stream served 6.1
  against 7.8 solves/s (two runs each, one box): requests join and leave the batch
  at every turn, and each change rebuilds its launch table and graphs.

Admission is first come, first served: the head of the queue is admitted once its
estimated device footprint fits the budget beside the requests in flight;
finished requests release their memory at the end of the turn.  Latency is
completion time minus arrival time.
"""
from __future__ import annotations

import dataclasses
import math
import time
from collections import deque
from typing import Callable, List, Optional

import numpy as np

from .models import BatchedIB3D, BatchedStokes2D


@dataclasses.dataclass
class SolveRequest:
    """One solve: ``build()`` returns a ready model (fields set, ghosts filled)."""
    rid: int
    arrival: float          # seconds after the stream starts
    kind: str               # "2d" (batched) or "3d" (own stream)
    build: Callable
    bytes: int              # estimated device footprint, for admission
    tol: float
    max_iter: int
    meta: dict = dataclasses.field(default_factory=dict)
    # filled in by the server
    admitted: Optional[float] = None
    finished: Optional[float] = None
    status: str = "queued"
    iterations: int = 0
    measure: float = math.inf

    @property
    def latency(self) -> float:
        return self.finished - self.arrival if self.finished is not None else math.inf


def footprint_2d(n, esz: int) -> int:
    """Device bytes of a batched 2D member: 15 state-sized arrays (P, τ×3, V×2 in
    two buffers, η, η_next, the rheology's η field), rows padded to 32."""
    pitch = ((31 + n[0] + 3 + 31) // 32) * 32
    return 15 * pitch * (n[1] + 3) * esz + 4096


def footprint_3d_ib(n, esz: int) -> int:
    """Device bytes of a 3D immersed-boundary model: 10 state fields, η, η_next,
    16 volume fractions, 4 residual fields, rows padded to 32."""
    pitch = ((31 + n[0] + 3 + 31) // 32) * 32
    return 30 * pitch * (n[1] + 3) * (n[2] + 3) * esz + (1 << 20)


def rel_measure_3d(norms: np.ndarray, rho_g_inf: float, length_z: float) -> float:
    """max(||r_V||∞ / ||ρg||∞, ||r_P||∞ L_z / ||V||∞) from a residual-norm vector."""
    rv = float(np.max(norms[1:4]))
    vmax = float(np.max(norms[8:11]))
    b = norms[0] * length_z / vmax if vmax > 0 else float(norms[0])
    return max(rv / rho_g_inf, b)


class SolveServer:
    """Serve a list of :class:`SolveRequest` in arrival order.

    ``max_active`` caps the requests in flight (1 gives one-at-a-time serving with
    the same numerics); ``realtime`` releases requests at their arrival times on
    the wall clock, otherwise all are available at once.
    """

    def __init__(self, budget_bytes: int, ncheck: int = 200, window: int = 0, max_active: int = 1 << 30,
                 realtime: bool = True, rho_g_inf: float = 1.0, length_z: float = 1.0, share3d: bool = False):
        if ncheck <= 0 or ncheck % 2:
            raise ValueError("ncheck must be a positive even number")
        self.budget = int(budget_bytes)
        self.ncheck = int(ncheck)
        self.window = int(window)
        self.max_active = int(max_active)
        self.realtime = realtime
        self.rho_g_inf = rho_g_inf
        self.length_z = length_z
        self.share3d = bool(share3d)  # True: 3D requests advance by shared launches (BatchedIB3D)
        self.peak_bytes = 0
        self.turns = 0

    def run(self, requests: List[SolveRequest]) -> List[SolveRequest]:
        two = [r for r in requests if r.kind == "2d"]
        if two and len({(r.tol, r.max_iter) for r in two}) != 1:
            raise ValueError("2D requests share one batch: give them one tol and one max_iter")
        tol2, max2 = (two[0].tol, two[0].max_iter) if two else (0.0, 0)
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        queue: deque = deque()
        active2d = {}   # rid -> (request, model)
        active3d = {}
        used = 0
        batch: Optional[BatchedStokes2D] = None
        batch3: Optional[BatchedIB3D] = None
        t0 = time.perf_counter()
        done: List[SolveRequest] = []

        def now():
            return time.perf_counter() - t0

        while pending or queue or active2d or active3d:
            t = now()
            while pending and (not self.realtime or pending[0].arrival <= t):
                queue.append(pending.popleft())
            # admission by budget, first come first served
            while queue and len(active2d) + len(active3d) < self.max_active and used + queue[0].bytes <= self.budget:
                r = queue.popleft()
                m = r.build()
                r.admitted = now()
                r.status = "running"
                used += r.bytes
                self.peak_bytes = max(self.peak_bytes, used)
                if r.kind == "2d":
                    if batch is None:
                        batch = BatchedStokes2D([m])
                    else:
                        batch.add(m)
                    active2d[r.rid] = (r, m)
                else:
                    if self.share3d:
                        if batch3 is None:
                            batch3 = BatchedIB3D([m])
                        else:
                            batch3.add(m)
                    active3d[r.rid] = (r, m)
            if queue and not active2d and not active3d and used + queue[0].bytes > self.budget:
                raise RuntimeError(f"request {queue[0].rid} needs {queue[0].bytes} bytes, over the budget")
            if not active2d and not active3d:
                if pending and self.realtime:
                    time.sleep(max(0.0, min(pending[0].arrival - now(), 0.01)))
                continue
            self.turns += 1
            # 3D: ncheck iterations of every 3D request, shared launches on the batch's
            # stream (asynchronous; each model's stream then waits for them), or each
            # on its own stream
            if active3d:
                if self.share3d:
                    batch3.advance(self.ncheck)
                else:
                    for r, m in active3d.values():
                        m.advance(self.ncheck)
                for r, m in active3d.values():
                    r.meta["_k"] = self.ncheck
            # 2D: one check round of the batch (its own stream, overlapping the 3D sweeps)
            retired = []
            if active2d:
                items, _ = batch.step(max_iter=max2, ncheck=self.ncheck, tol=tol2, rounds=1, window=self.window)
                by_model = {id(m): it for m, it in zip(batch.models, items)}
                for rid, (r, m) in list(active2d.items()):
                    it = by_model[id(m)]
                    r.iterations, r.measure = it["iterations"], it["measure"]
                    if it["status"] != "active" or r.iterations >= r.max_iter:
                        r.status = it["status"] if it["status"] != "active" else "max_iter"
                        retired.append((r, m))
                        del active2d[rid]
            # 3D checks (each synchronises its own stream)
            for rid, (r, m) in list(active3d.items()):
                k = r.meta.pop("_k")
                r.iterations += k
                norms = m.residual_norms()
                r.measure = rel_measure_3d(norms, self.rho_g_inf, r.meta.get("length_z", self.length_z))
                if r.measure < 0.5 * r.meta.get("_best", math.inf):
                    r.meta["_best"], r.meta["_since"] = r.measure, 0
                else:
                    r.meta["_since"] = r.meta.get("_since", 0) + k
                if norms[11] != 0.0 or not np.isfinite(r.measure):
                    r.status = "diverged"
                elif r.measure < r.tol:
                    r.status = "converged"
                elif self.window and r.meta["_since"] >= self.window:
                    r.status = "stalled"
                elif r.iterations >= r.max_iter:
                    r.status = "max_iter"
                if r.status != "running":
                    retired.append((r, m))
                    del active3d[rid]
            t = now()
            for r, m in retired:
                r.finished = t
                used -= r.bytes
                if r.kind == "2d":
                    batch.remove(m)
                else:
                    if self.share3d:
                        batch3.remove(m)
                r.meta["result"] = self._keep(m)
                m.close()
                done.append(r)
        if batch is not None:
            batch.close()
        if batch3 is not None:
            batch3.close()
        return done

    def _keep(self, m):
        """What a request returns: its velocity field (x component) and pressure."""
        return {"Vx": m.get_field("Vx"), "P": m.get_field("P")}


def summarize(done: List[SolveRequest], makespan: Optional[float] = None) -> dict:
    lat = np.array([r.latency for r in done])
    fin = [r.finished for r in done if r.finished is not None]
    span = makespan if makespan is not None else (max(fin) if fin else 0.0)
    status = {}
    for r in done:
        status[r.status] = status.get(r.status, 0) + 1
    return {"requests": len(done), "status": status, "makespan_s": span,
            "solves_per_s": len(done) / span if span > 0 else 0.0,
            "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else None}


__all__ = ["SolveRequest", "SolveServer", "summarize", "footprint_2d", "footprint_3d_ib", "rel_measure_3d"]
