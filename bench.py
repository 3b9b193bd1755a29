#!/usr/bin/env python3
"""Benchmark: pseudo-transient Stokes T_eff on one B200 (or N replicas).

Workload (one "step" = one PT iteration, advance_iteration!): the 3D
gravity-driven ice slab at 511^3 cells -- extent 1 x 1 x 0.25, tilted 10 degrees
(rho*g = (-sin a, 0, cos a)), Glen's law n=3, A=1 regularised at
strain rate 1e-6 (ViscoplasticRegularisation(PowerLawRheology(1, 3), 5000)),
free-slip bed, stress-free top, periodic x/y, zero initial fields; FP64 is the
headline, FP32 is measured in the same run.  Inputs are synthetic (the
reference publishes no dataset for this path).

T_eff = A_eff / t_iter with A_eff the minimum field bytes of one iteration:
P, tau(6), V(3) read and written, eta read, eta_next written, each at its exact
staggered interior size.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs an independent replica of the workload
("replicas only": the single-GPU path has no data-path collective); the time is
the max over ranks and ``value`` is the whole-job throughput.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))

# DRAM bytes per cell of one fused-sweep launch: dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu-captured 255^3 launch (32x8 tiles, z-blocks of
# 32, summarised in profiles/fused3d_slab255_ncu_full.md, v6) divided by its cell
# count; traffic grows with the cell count, so it scales to 511^3.
TRAFFIC_BYTES_PER_CELL = {"f64": 233.3, "f32": None}
# DRAM bytes per cell of one steady-state immersed-boundary iteration (update_σ!,
# update_V! and their six boundary launches, inactive zeros no longer stored,
# block list in use): dram__bytes_read.sum + dram__bytes_write.sum of one
# ncu-captured iteration of the 191^3 glacier divided by its cell count
# (profiles/ib_glacier191_dram.md); the same geometry scales to 383^3.
IB_TRAFFIC_BYTES_PER_CELL = {"f64": 109.5, "f32": 74.9}


def load_fastice():
    name = "fastice_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "fastice.jl_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def a_eff_elements(n):
    """Minimum field elements moved by one iteration (22 array passes)."""
    nx, ny, nz = n
    C = nx * ny * nz
    txy, txz, tyz = (nx + 1) * (ny + 1) * nz, (nx + 1) * ny * (nz + 1), nx * (ny + 1) * (nz + 1)
    vx, vy, vz = (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)
    return 2 * (4 * C + txy + txz + tyz + vx + vy + vz) + 2 * C


def slab_problem(fi, n, alpha_deg=10.0):
    grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=(1.0, 1.0, 0.25), dims=n)
    a = math.radians(alpha_deg)
    gravity = {"x": -math.sin(a), "y": 0.0, "z": math.cos(a)}
    bcs = {"x": (fi.PBC(), fi.PBC()), "y": (fi.PBC(), fi.PBC()),
           "z": (fi.SBC(0.0, 0.0, 0.0), fi.TBC(0.0, 0.0, 0.0))}
    rheology = fi.glen_regularised(A=1.0, n=3, strain_rate_0=1e-6)
    sp = fi.pt_params(grid, r=0.7, re_mech=8 * math.pi, vdtau_factor=1.1)
    return grid, bcs, gravity, rheology, sp


def make_model(fi, n, dtype, device, path="auto"):
    grid, bcs, gravity, rheology, sp = slab_problem(fi, n)
    m = fi.IsothermalFullStokesModel(arch=fi.Arch("cuda", device), grid=grid, boundary_conditions=bcs,
                                     gravity=gravity, rheology=rheology, solver_params=sp, dtype=dtype, path=path)
    # zero initial P, tau, V (allocation zero-fills); eta from the regularised law at tau = 0
    m.set_field("eta", rheology.eta_reg)
    m.set_field("eta_next", rheology.eta_reg)
    m.apply_bcs()
    return m


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in self.rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def time_advance(fi, model, steps, torch):
    """CUDA-event time of `steps` PT iterations on the model's stream (ms)."""
    stream = torch.cuda.ExternalStream(model.stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    model.synchronize()
    e0.record(stream)
    model.advance(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def e2e_run(fi, n, dtype, device, steps, torch, variant=None):
    """End to end through the public API with pinned host buffers: upload the
    state, run the iterations, read the residual norms and download the state."""
    names = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta")
    m = make_model(fi, n, dtype, device)
    npd = np.float64 if dtype == "f64" else np.float32
    host = {}
    for nm in names:
        shape = m.field_shape(nm)
        t = torch.empty(int(np.prod(shape)), dtype=torch.float64 if dtype == "f64" else torch.float32, pin_memory=True)
        a = t.numpy().reshape(shape)
        a[...] = 0.0 if nm != "eta" else 5000.0
        host[nm] = (t, a)
    h2d = sum(a.nbytes for _, a in host.values())
    d2h = sum(a.nbytes for nm, (_, a) in host.items() if nm != "eta") + 8 * 12
    if variant is not None:
        m.set_variant(variant)
    m.advance(2)
    m.synchronize()
    t0 = time.perf_counter()
    for nm, (_, a) in host.items():
        m.set_field(nm, a)
    m.copy_field("eta_next", "eta")  # η_next = η on the device, as drivers do before iterating
    m.apply_bcs()
    m.advance(steps)
    norms = m.residual_norms()
    for nm, (_, a) in host.items():
        if nm != "eta":
            m.get_field(nm, out=a)
    dt = time.perf_counter() - t0
    m.close()
    return dt, h2d, d2h, norms


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    return O


def oracle_slab(O, fi, n):
    """The slab workload on the CPU oracle (C restatement), at its initial state."""
    grid, bcs, gravity, rheology, sp = slab_problem(fi, n)
    dt = sp["Δτ"]
    taus = ("xx", "yy", "zz", "xy", "xz", "yz")
    per, z = (O.BC_PERIODIC, (0, 0, 0)), ((O.BC_SLIP, (0, 0, 0)), (O.BC_TRACTION, (0, 0, 0)))
    spec = O.Spec(nd=3, n=n, extent=grid.extent, origin=grid.origin, bcs=((per, per), (per, per), z),
                  dt_P=dt["Pr"], dt_tau=tuple(dt["τ"][k] for k in taus), dt_V=tuple(dt["V"][k] for k in "xyz"),
                  g_val=(gravity["x"], gravity["y"], gravity["z"]), rheo_inner=O.RHEO_POWER, rheo_A=1.0, rheo_n=3,
                  rheo_has_reg=1, rheo_inv_eta_reg=1.0 / rheology.eta_reg)
    m = O.OracleStokes(spec)
    m.a["eta"][...] = rheology.eta_reg
    m.a["eta_next"][...] = rheology.eta_reg
    m.apply_initial_bcs()
    return m


OMP_PIN = {"OMP_PROC_BIND": "close", "OMP_PLACES": "cores"}


def cpu_baseline(n, seconds=12.0, warm=1):
    """The CPU oracle (C restatement, OpenMP) on the same workload: whole
    iterations at the full grid, as many as fit in `seconds` (at least one).
    Runs in a fresh process with the OpenMP threads pinned (one per host core,
    bound close), so that both arms of the benchmark time it the same way and no
    runtime already initialised in this process (torch's) decides its threads."""
    env = dict(os.environ)
    env.update(OMP_PIN)
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    env["OMP_NUM_THREADS"] = str(threads)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-baseline-only", "--n", str(n[0]),
           "--cpu-seconds", str(seconds), "--warmup", str(warm)]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, check=True)
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return d["iterations"], d["seconds"], d["threads"]


def _cpu_baseline_inproc(n, seconds, warm):
    O = load_oracle()
    fi = load_fastice()
    m = oracle_slab(O, fi, n)
    for _ in range(warm):
        m.advance(1)
    its, t0 = 0, time.perf_counter()
    while True:
        m.advance(1)
        its += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    cores = os.cpu_count()
    try:
        cores = int(os.environ.get("OMP_NUM_THREADS", cores))
    except ValueError:
        pass
    return its, el, cores


def oracle_parity(fi, n, device, variants, iters=3):
    """Error of the GPU sweeps against the FP64 oracle at the workload's own size:
    a fresh model of each precision and the oracle advance `iters` PT iterations
    from the workload's initial state; per field, max |gpu - oracle| / max |oracle|
    over the interior, and the worst field."""
    O = load_oracle()
    om = oracle_slab(O, fi, n)
    om.advance(iters)
    names = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta")
    out = {"iterations": iters, "oracle": "C restatement (FP64) of the reference's kernels"}
    for dtype, variant in variants.items():
        m = make_model(fi, n, dtype, device)
        if variant is not None:
            m.set_variant(variant)
        m.advance(iters)
        per = {}
        for nm in names:
            b = om.interior(nm)
            a = m.get_field(nm).astype(np.float64)
            a -= b
            per[nm] = float(np.max(np.abs(a)) / max(float(np.max(np.abs(b))), 1e-300))
            del a, b
        m.close()
        out[dtype] = {"max_rel_diff": max(per.values()), "per_field": per}
    return out


def mms_errors(fi):
    """Manufactured-solution discretisation errors of this build: the 3D free-slip
    solution (stokes_manufactured_solution_free_slip_3D.jl) at 127^3 and the 2D one of
    the 128^2 unit-square case, each solved to |R|inf < 1e-8 in FP64; the 2D case
    also runs 1000 iterations of the no-FMA build against the oracle, bit for bit."""
    from fastice_b200 import scenarios
    res = {}
    grid, m = scenarios.mms3d_model(127)
    r = m.solve(max_iter=400 * 127, ncheck=127, tol=1e-8)
    res["mms3d_127"] = {"l2_rel_error": scenarios.mms3d_error(grid, m), "converged": bool(r["converged"]),
                        "iterations": r["iterations"]}
    m.close()
    for lib_name in ("fast", "strict"):
        grid, m, gravity = scenarios.mms2d_model(128, library=lib_name)
        if lib_name == "fast":
            r = m.solve(max_iter=200 * 128, ncheck=128, tol=1e-8)
            res["mms2d_128"] = {"l2_rel_error": scenarios.mms2d_error(grid, m), "converged": bool(r["converged"]),
                                "iterations": r["iterations"]}
        else:
            O = load_oracle()
            om = scenarios_mms2d_oracle(fi, O, grid, gravity)
            m.advance(1000)
            om.advance(1000)
            same = all(np.array_equal(m.get_field(nm).view(np.uint64), om.interior(nm).view(np.uint64))
                       for nm in ("P", "txx", "tyy", "txy", "Vx", "Vy"))
            res["mms2d_128"]["bitwise_vs_oracle_after_1000_iterations"] = bool(same)
        m.close()
    return res


def scenarios_mms2d_oracle(fi, O, grid, gravity):
    """The 2D manufactured-solution case on the CPU oracle."""
    sp = fi.pt_params(grid)["Δτ"]
    slip = (O.BC_SLIP, (0, 0, 0))
    spec = O.Spec(nd=2, n=grid.dims, extent=grid.extent, origin=grid.origin, bcs=((slip, slip), (slip, slip)),
                  dt_P=sp["Pr"], dt_tau=(sp["τ"]["xx"], sp["τ"]["yy"], 0.0, sp["τ"]["xy"], 0.0, 0.0),
                  dt_V=(sp["V"]["x"], sp["V"]["y"], 0.0))
    o = O.OracleStokes(spec, gravity_arrays={"gx": gravity["x"].sample(), "gy": gravity["y"].sample()})
    o.a["eta"][...] = 1.0
    o.a["eta_next"][...] = 1.0
    o.apply_initial_bcs()
    return o


def _base_line(metric, value, unit, steps, warmup, ms, dtype, cfg, hib=True):
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic", "config": cfg}


def run_batched(args):
    """Batched 2D solves: `instances` pure-shear inclusion problems (seeds 0..k-1,
    63-511 cells per side, 1-16 inclusions, contrasts up to 1e4) in one batch:
    autotuned tile shape, CUDA-graph replay of each check round, one step = one
    check round.  With --storage f32 (the default) every PT sweep runs on FP32
    storage inside a per-member FP64 defect correction (FP64 solution and
    residuals) to the FP64 measure --tol (1e-6); --storage f64 runs plain FP64
    sweeps.  value = instances solved / wall time of the solve.  The same method
    solving members one at a time (a batch of one each) is timed on the first
    --alone members, and the first --errcheck members are compared with a plain
    FP64 solve taken to 1e-9."""
    import torch
    fi = load_fastice()
    from fastice_b200 import scenarios
    storage = args.storage
    mode = "mixed" if storage == "f32" else "plain"
    tol = args.tol or 1e-6
    ncheck = 200
    window = args.window

    def members(seeds):
        return [scenarios.inclusion_model(s, dtype="f64", smooth=args.smooth)[0] for s in seeds]

    models = members(range(args.instances))
    cells = sum(m.grid.dims[0] * m.grid.dims[1] for m in models)
    batch = fi.BatchedStokes2D(models)
    best, per = batch.autotune(iters=10)
    sweep_gbs = {k: 13 * 8 * cells / (v * 1e-3) / 1e9 for k, v in per.items()}
    clocks = ClockSampler(0)
    clocks.start()
    max_iter = args.rounds * ncheck if args.rounds > 0 else 400000
    items, sec = batch.solve(max_iter=max_iter, ncheck=ncheck, tol=tol, window=window, use_graph=True, mode=mode)
    ck = clocks.stop()
    batch.close()
    status = {}
    for it in items:
        status[it["status"]] = status.get(it["status"], 0) + 1
    iters = [it["iterations"] for it in items]
    done = sum(1 for it in items if it["status"] == "converged")
    # one at a time: the same method, each member alone in its own batch
    alone = {"members": 0, "seconds": 0.0, "status": {}}
    for q in range(min(args.alone, len(models))):
        mq = members([q])
        b1 = fi.BatchedStokes2D(mq)
        b1.set_variant(best)
        it1, s1 = b1.solve(max_iter=max_iter, ncheck=ncheck, tol=tol, window=window, use_graph=True, mode=mode)
        b1.close()
        mq[0].close()
        alone["members"] += 1
        alone["seconds"] += s1
        alone["status"][it1[0]["status"]] = alone["status"].get(it1[0]["status"], 0) + 1
    alone["solves_per_s"] = alone["members"] / alone["seconds"] if alone["seconds"] > 0 else None
    # error against a plain FP64 solve of the same members, to 1e-9
    errs = []
    if args.errcheck > 0:
        k = min(args.errcheck, len(models))
        ref = members(range(k))
        rb = fi.BatchedStokes2D(ref)
        ritems, _ = rb.solve(max_iter=4 * max_iter, ncheck=ncheck, tol=1e-9, window=0, use_graph=True)
        rb.close()
        for q in range(k):
            if ritems[q]["status"] != "converged" or items[q]["status"] != "converged":
                errs.append(None)
                continue
            vmax = max(float(np.max(np.abs(ref[q].get_field(c)))) for c in ("Vx", "Vy"))
            d = max(float(np.max(np.abs(models[q].get_field(c) - ref[q].get_field(c)))) for c in ("Vx", "Vy"))
            errs.append(d / vmax)
        for m in ref:
            m.close()
    for m in models:
        m.close()
    smooth = f"viscosity smoothed by {args.smooth} log-space passes" if args.smooth else "sharp inclusions"
    cfg = {"workload": f"{args.instances} independent 2D pure-shear inclusion problems (seeds 0..{args.instances - 1}, "
                       "63-511 cells per side, 1-16 circles r~U(0.02,0.15), log-normal contrast clipped to 1e4, "
                       f"{smooth}, free-slip walls with pure shear)",
           "instances": args.instances, "cells_total": cells, "tol": tol, "ncheck": ncheck, "window": window,
           "measure": "cell-scaled relative residual max(|r_V|inf h/max|P,tau|, |r_P|inf h/max|V|), FP64",
           "storage": "FP32 sweeps inside an FP64 defect correction (FP64 solution and residuals)" if mode == "mixed"
           else "FP64", "tile_shape": list(per)[best], "graph": True}
    line = _base_line(f"batched 2D PT solves/s ({args.instances} instances)", done / sec, "solves/s",
                      len(iters), 10 * 3, 1e3 * sec / max(1, max(iters) // ncheck), "f32+f64" if mode == "mixed"
                      else "f64", cfg)
    line.update({"status": status, "iterations": {"min": min(iters), "max": max(iters), "mean": float(np.mean(iters))},
                 "seconds": sec, "sweep_teff_gbs_fp64_members": sweep_gbs, "clocks": ck,
                 "one_at_a_time": alone,
                 "speedup_vs_one_at_a_time": (done / sec) / alone["solves_per_s"] if alone["solves_per_s"] else None,
                 "error_vs_fp64_solve": errs,
                 "gpu_launches": "k sweeps + 4 bookkeeping kernels per check round, replayed as one graph; per outer "
                                 "step of the defect correction a few FP64 kernels per member"})
    return line


def _serving_requests(fi, scale, duration, rate, seed=0):
    from fastice_b200 import scenarios, serving
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        rid = len(reqs)
        if rng.random() < 0.7:
            n = int(round(rng.integers(128, 1025) * scale))
            n = (max(n, 16), max(n, 16))
            build = (lambda s=rid, n=n: scenarios.inclusion_model(s, n=n, dtype="f64")[0])
            reqs.append(serving.SolveRequest(rid=rid, arrival=t, kind="2d", build=build,
                                             bytes=serving.footprint_2d(n, 8), tol=1e-6, max_iter=400000))
        else:
            n = max(int(round(rng.integers(64, 256) * scale)), 12)
            build = (lambda s=rid, n=n: scenarios.bed_model(s, n)[0])
            reqs.append(serving.SolveRequest(rid=rid, arrival=t, kind="3d", build=build,
                                             bytes=serving.footprint_3d_ib((n, n, n), 8), tol=1e-6, max_iter=200000,
                                             meta={"length_z": 0.6}))
    return reqs


def run_serving(args):
    """Continuous-batching server against one-at-a-time solves on the same
    seeded Poisson stream (70 % 2D inclusion problems, 30 % 3D immersed-boundary
    glaciers; sizes scaled by --scale from 128-1024 and 64-255 cells per side),
    admission by a 150 GB device-memory budget, every request to 1e-6.  value =
    requests / makespan with every request available at once; the latencies come
    from a run that releases requests at their Poisson arrival times."""
    fi = load_fastice()
    from fastice_b200 import serving
    rate, budget = 50.0, 150 << 30
    out = {}
    for mode, kw in (("batched", {"share3d": args.shared3d}), ("sequential", {"max_active": 1})):
        srv = serving.SolveServer(budget_bytes=budget, ncheck=200, window=100000, realtime=False, **kw)
        t0 = time.perf_counter()
        done = srv.run(_serving_requests(fi, args.scale, args.duration, rate))
        span = time.perf_counter() - t0
        thr = serving.summarize(done, makespan=span)
        srv = serving.SolveServer(budget_bytes=budget, ncheck=200, window=100000, realtime=True, **kw)
        done_rt = srv.run(_serving_requests(fi, args.scale, args.duration, rate))
        lat = serving.summarize(done_rt)
        out[mode] = {"solves_per_s": thr["solves_per_s"], "makespan_s": span, "status": thr["status"],
                     "p50_latency_s": lat["p50_latency_s"], "p99_latency_s": lat["p99_latency_s"],
                     "peak_bytes": srv.peak_bytes, "requests": thr["requests"]}
    cfg = {"workload": f"Poisson stream lambda={rate}/s for {args.duration} s: 70% 2D inclusion problems "
                       f"(128-1024 cells per side x {args.scale}), 30% 3D immersed-boundary glaciers over a seeded "
                       f"64-bump bed (64-255 cells per side x {args.scale}); FP64; stop at 1e-6",
           "budget_bytes": budget, "ncheck": 200,
           "3d_requests": "shared launches (BatchedIB3D)" if args.shared3d else "each on its own stream",
           "scaled": "the full stream (60 s, unscaled sizes) needs about an hour of GPU time per arm at the "
                     "reference PT scheme's iteration counts"}
    b = out["batched"]
    line = _base_line("serving solves/s (continuous batching, scaled Poisson stream)", b["solves_per_s"], "solves/s",
                      b["requests"], 0, 1e3 * b["makespan_s"] / max(1, b["requests"]), "f64", cfg)
    line.update({"batched": b, "sequential": out["sequential"],
                 "speedup_vs_sequential": b["solves_per_s"] / out["sequential"]["solves_per_s"]})
    return line


def run_mixed(args):
    """Mixed-precision refined solve against the plain FP64 solve, both to the same
    tolerance; one step = one solve.  Scenarios: the 3D manufactured solution
    (stokes_manufactured_solution_free_slip_3D.jl) at n^3, |R|inf < tol, or the
    immersed-boundary glacier (seeded 64-bump bed) at n^3, relative residual < tol."""
    fi = load_fastice()
    from fastice_b200 import scenarios
    n = args.n if args.n != 511 else (255 if args.scenario == "mms" else 127)
    tol = args.tol or 1e-8
    res = {}
    fields = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz")
    rheo, eta0, rdesc, pt = glacier_rheology(fi, args.rheology)
    if args.scenario == "mms":
        eta0 = 1.0
    if args.scenario == "glacier" and args.rheology == "glen":
        eta0 = 1.0  # the continuation starts from the linear problem
        rdesc += ("; solved by continuation: linear, then the cap 10, 100, 1000, 5000 (PT velocity step factor 4.4 "
                  "from 1000; a diverged stage is retried from its start with the factor doubled)")
    for mode in ("plain", "mixed"):
        if args.scenario == "mms":
            grid, m = scenarios.mms3d_model(n)
            kw = dict(max_iter=400 * n, ncheck=n, tol=tol)
        else:
            m, _ = scenarios.bed_model(0, n, rheology=rheo, pt=pt)
            m.set_field("eta", eta0)
            m.set_field("eta_next", eta0)
            m.apply_bcs()
            grid = m.grid
            kw = dict(max_iter=1000 * n, ncheck=n, tol=tol, measure="rel_slab", rho_g_inf=1.0, length_z=0.6)
        glen = args.scenario == "glacier" and args.rheology == "glen"
        if glen:
            # from rest only the continuation's first (linear) stage is stable
            stages = scenarios.glacier_glen_stages(grid, tol=tol)
            m.set_params(stages[0][0], stages[0][1](0))
        m.solve(mode=mode, **dict(kw, max_iter=2 * n, tol=1e-30))  # warm-up (shadow model, launch shapes)
        for f in fields:
            m.set_field(f, 0.0)
        m.set_field("eta", eta0)
        m.set_field("eta_next", eta0)
        m.apply_bcs()
        m.synchronize()
        t0 = time.perf_counter()
        if glen:
            # Glen's law needs a continuation: linear, then the viscosity cap raised stage by stage
            r = m.solve_continuation(stages, retries=2, mode=mode, **{k: v for k, v in kw.items() if k != "tol"})
        else:
            r = m.solve(mode=mode, **kw)
        sec = time.perf_counter() - t0
        res[mode] = {"seconds": sec, "iterations": r["iterations"], "outer": r["outer"], "measure": r["measure"],
                     "converged": bool(r["converged"]), "V": [m.get_field(c) for c in ("Vx", "Vy", "Vz")]}
        if "stages" in r:
            res[mode]["stages"] = r["stages"]
        if args.scenario == "mms":
            res[mode]["mms_l2_error"] = scenarios.mms3d_error(grid, m)
        m.close()
    vmax = max(float(np.max(np.abs(v))) for v in res["plain"]["V"])
    dv = max(float(np.max(np.abs(a - b))) for a, b in zip(res["mixed"]["V"], res["plain"]["V"])) / vmax
    for r in res.values():
        r.pop("V")
    if args.scenario == "mms":
        cfg = {"workload": f"3D free-slip manufactured solution (eta=1) on [-1,1]^3, {n}^3 cells, to |R|inf < {tol}",
               "n": n, "tol": tol}
    else:
        cfg = {"workload": f"3D immersed-boundary glacier {n}^3 cells (seeded 64-bump bed, surface 0.6 + 0.05 "
                           f"sin(2 pi x), traction-free box, {rdesc}) to relative residual < {tol}",
               "n": n, "tol": tol, "measure": "max(|r_V|inf / |rho g|inf, |r_P|inf * 0.6 / max|V|)"}
    # a speed-up is only a speed-up between two solves that both reached the tolerance
    both = res["plain"]["converged"] and res["mixed"]["converged"]
    sp = res["plain"]["seconds"] / res["mixed"]["seconds"] if both else None
    line = _base_line("mixed-precision solve speedup vs plain FP64", sp, "x", 1, 1, 1e3 * res["mixed"]["seconds"],
                      "f32+f64", cfg)
    line.update({"plain_fp64": res["plain"], "mixed": res["mixed"], "max_rel_diff_V_vs_fp64": dv})
    if not both:
        line["invalid"] = "a solve stopped before reaching the tolerance; no speed-up is reported"
    return line


def glacier_rheology(fi, kind):
    """(rheology or None for the default linear viscosity 1, initial η, description,
    PT steps (r, re, factor))."""
    if kind in ("glen", "glen_relaxed"):
        r = fi.glen_regularised(A=1.0, n=3, strain_rate_0=1e-6)
        eta0 = r.eta_reg
        desc = "Glen n=3, A=1, regularised at strain rate 1e-6 (viscosity cap 5000)"
        if kind == "glen_relaxed":
            r = fi.Relaxation(r, 0.1, scale="log")
            desc += ", relaxed in log scale at rate 0.1"
        return r, eta0, desc, (0.7, 8 * math.pi, 1.1)
    return None, 1.0, "linear viscosity", (0.9, 5 * math.pi, 1.1)


def ib_a_eff_elements(n):
    """Minimum elements one immersed-boundary iteration moves: the 22 state passes
    plus a read of the seven mask components of each of ω.na and ω.ns that the
    masked kernels use (ccc, vcc, cvc, ccv, vvc, vcv, cvv), at their staggered sizes."""
    nx, ny, nz = n
    masks = nx * ny * nz + (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1) + \
        (nx + 1) * (ny + 1) * nz + (nx + 1) * ny * (nz + 1) + nx * (ny + 1) * (nz + 1)
    return a_eff_elements(n) + 2 * masks


def run_glacier(args):
    """Immersed-boundary glacier: seeded 64-bump bed and the sinusoidal surface on
    the unit cube at n^3 cells (383^3 by default), level sets from the DEMs, volume
    fractions from the level sets, linear viscosity; one step = one PT iteration
    (advance_iteration! of the immersed-boundary model).  value = T_eff in the
    reference's convention: 36 array passes over the whole box per iteration (FP64;
    FP32 in the same line).  About three quarters of the box are ice-free, where the
    masked kernels read only the activity byte and, once the zeros are stored, write
    nothing, so this figure can exceed the copy bandwidth; the DRAM bytes an iteration
    really moves (ncu) and the bandwidth they imply are reported beside it."""
    import torch
    fi = load_fastice()
    from fastice_b200 import scenarios
    n = args.n if args.n != 511 else 383
    dims = (n, n, n)
    A = ib_a_eff_elements(dims)
    peak, peak_kind = measured_peak_hbm()
    res = {}
    clocks = None
    rheo, eta0, rdesc, pt = glacier_rheology(fi, args.rheology)
    for dtype in [d for d in args.dtypes.split(",") if d in ("f64", "f32")]:
        t0 = time.perf_counter()
        m, prm = scenarios.bed_model(0, n, dtype=dtype, rheology=rheo, pt=pt)
        if rheo is not None:
            m.set_field("eta", eta0)
            m.set_field("eta_next", eta0)
            m.apply_bcs()
        setup = time.perf_counter() - t0
        m.advance(args.warmup)
        m.synchronize()
        sampler = ClockSampler(0) if dtype == "f64" else None
        if sampler:
            sampler.start()
            time.sleep(0.15)
        ms = time_advance(fi, m, args.steps, torch)
        if sampler:
            clocks = sampler.stop()
        norms = m.residual_norms()
        esz = 8 if dtype == "f64" else 4
        res[dtype] = {"ms_per_step": ms / args.steps, "teff_gbs": A * esz / (ms / args.steps / 1e3) / 1e9,
                      "path": m.path, "setup_s": setup, "finite": bool(norms[11] == 0.0)}
        m.close()
        torch.cuda.empty_cache()
    d0 = res.get("f64") or next(iter(res.values()))
    dt0 = "f64" if "f64" in res else next(iter(res))
    cfg = {"workload": f"3D immersed-boundary glacier {n}^3 cells on the unit cube: bed = seeded sum of 64 Gaussian "
                       "bumps (a~U(0,0.2), w~U(0.05,0.2), centres uniform), surface z = 0.6 + 0.05 sin(2 pi x), "
                       "level sets from the DEMs, volume fractions from the level sets, traction-free box, "
                       f"{rdesc}, one PT iteration per step", "grid": list(dims), "a_eff_arrays": 36,
           "l2": "inputs exceed L2 (126 MB): no flush needed"}
    line = _base_line(f"IB PT-Stokes T_eff GB/s ({n}^3, {dt0.upper()}, 36-pass convention)", d0["teff_gbs"], "GB/s",
                      args.steps, args.warmup, d0["ms_per_step"], dt0, cfg)
    tr = IB_TRAFFIC_BYTES_PER_CELL.get(dt0)
    traffic = tr * n * n * n if tr else None
    dram = traffic / (d0["ms_per_step"] / 1e3) / 1e9 if traffic else None
    line.update({"kernel_path": d0["path"],
                 "gpu_launches": 8 * args.steps,  # update_σ!, update_V! and six boundary launches per iteration
                 "roofline": {"bound": "hbm", "achieved": d0["teff_gbs"], "peak": peak, "unit": "GB/s",
                              "frac": d0["teff_gbs"] / peak, "peak_source": peak_kind,
                              "algorithmic_bytes": A * (8 if dt0 == "f64" else 4), "traffic": traffic,
                              "dram_gbs": dram, "dram_frac": dram / peak if dram else None,
                              "note": "achieved counts 36 passes over the whole box; dram_gbs is the measured "
                                      "traffic per iteration over its time"},
                 "per_dtype": res, "clocks": clocks})
    return line


def run_split(args):
    """The per-GPU cost of a domain split on the slab workload at n^3 (one rank's
    slab of a weak-scaling run), measured on one GPU for a split along x and along y:
    K iterations timed with CUDA events on the model's stream (a) plain, (b) each
    followed by the halo exchange of V and η (pack toward both neighbours, the
    messages moved by a device copy, unpack), (c) the same with the overlapped
    iteration (the split-face tiles first, the others on the model's second stream
    while the halo moves).  The slab's own periodic images are its neighbours here
    (a one-rank ring), so every kernel of a multi-rank iteration runs; the transfer
    between GPUs is the only part replaced, by a copy in HBM, and its NVLink time is
    estimated from the message size at the measured 770 GB/s per direction.
    value = the x split with the plain exchange (the default of a split run; x is
    the fastest dimension, so its layers are the strided ones)."""
    import torch
    fi = load_fastice()
    n = (args.n,) * 3
    A = a_eff_elements(n)
    m = make_model(fi, n, "f64", 0)
    stream = torch.cuda.ExternalStream(m.stream_ptr)

    def timed(step, K):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m.synchronize()
        e0.record(stream)
        for _ in range(K):
            step()
        m.synchronize()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / K

    K = args.steps
    W = max(args.warmup, 3)
    plain = lambda: m.advance(1)
    for _ in range(W):
        plain()
    ms_plain = timed(plain, K)
    per_dim = {}
    for dim, name in ((0, "x"), (1, "y")):
        nb = [m.halo_bytes(dim, side, "iteration") for side in (0, 1)]
        send = [torch.empty(b, dtype=torch.uint8, device="cuda") for b in nb]
        recv = [torch.empty(b, dtype=torch.uint8, device="cuda") for b in nb[::-1]]

        def exchange():
            for side in (0, 1):
                m.halo_pack(dim, side, send[side].data_ptr(), "iteration")
            with torch.cuda.stream(stream):
                recv[1].copy_(send[0])  # toward low, received on the high side
                recv[0].copy_(send[1])
            m.halo_unpack(dim, 1, recv[1].data_ptr(), "iteration")
            m.halo_unpack(dim, 0, recv[0].data_ptr(), "iteration")

        res = {}
        for case, step in (("exchange", lambda: (m.advance(1), exchange())),
                           ("overlapped", lambda: (m.advance_begin(dim), m.advance_end(), exchange()))):
            for _ in range(W):
                step()
            res[case] = timed(step, K)
        per_dim[name] = {"ms_with_exchange": res["exchange"], "ms_overlapped": res["overlapped"],
                         "teff_gbs_overlapped": A * 8 / (res["overlapped"] / 1e3) / 1e9,
                         "message_bytes_per_side": nb, "nvlink_ms_at_770_gbs": sum(nb) / 770e9 * 1e3}
        del send, recv
    norms = m.residual_norms()
    m.close()
    line = _base_line("split slab: ms per iteration with the halo exchange (one rank's share, 1 GPU)",
                      per_dim["x"]["ms_with_exchange"], "ms", K, W, per_dim["x"]["ms_with_exchange"], "f64",
                      {"workload": f"3D tilted ice slab {n[0]}^3 (one rank's slab), split along x (and along y), halo "
                                   "of V and eta exchanged after every iteration with its two neighbours (here its own "
                                   "periodic images; the transfer by a device copy)", "grid": list(n)},
                      hib=False)
    line.update({"ms_plain": ms_plain, "teff_gbs_plain": A * 8 / (ms_plain / 1e3) / 1e9, "split": per_dim,
                 "finite": bool(norms[11] == 0.0),
                 "gpu_launches": 5 * K,
                 "gpu_launches_per_iteration": "plain: 1 sweep; exchange: + 2 packs and 2 unpacks (the 2 copies are "
                                               "torch's); overlapped: the sweep in two launches"})
    return line


def run_heat(args):
    """Heat diffusion (src/Models/Diffusion/Heat/ restated): the implicit step of the
    driver scripts_future_API/heat_wip.jl (Value sides south/north, Flux 0 elsewhere,
    λ/(ρCp) = 1, Δt = 1, a Gaussian initial temperature) at n^3 cells; one step = one
    PT iteration (one fused sweep).  value = T_eff over the 9 array passes of an
    iteration (T and q(3) read and written, T_o read)."""
    import torch
    fi = load_fastice()
    from fastice_b200 import heat
    n = args.n
    dims = (n, n, n)
    grid = fi.UniformGrid(origin=(-0.5, -0.5, 0.0), extent=(1.0, 1.0, 1.0), dims=dims)
    sides = {"west": heat.Flux(0.0), "east": heat.Flux(0.0), "south": heat.Value(-0.1), "north": heat.Value(0.3),
             "bottom": heat.Flux(0.0), "top": heat.Flux(0.0)}
    dtype = args.dtypes.split(",")[0]
    m = heat.HeatDiffusionModel(grid=grid, boundary_conditions=sides, physics={"λ_ρCp": 1.0},
                                iter_params=heat.heat_iter_params(grid, 1.0, 1.0), dtype=dtype)
    zc = (np.arange(n) + 0.5) / n
    xc = -0.5 + zc
    Z, Y, X = np.meshgrid(zc, xc, xc, indexing="ij")
    T0 = np.exp(-(X / 0.1) ** 2 - (Y / 0.1) ** 2 - ((Z - 0.5) / 0.1) ** 2)
    m.set_field("T", T0)
    m.set_field("T_o", T0)
    for q in ("qx", "qy", "qz"):
        m.set_field(q, 0.0)
    m.apply_bcs()
    m.advance(args.warmup, 1.0)
    m.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.15)
    stream = torch.cuda.ExternalStream(m.stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.advance(args.steps, 1.0)
    e1.record(stream)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    ck = clocks.stop()
    m.close()
    esz = 8 if dtype == "f64" else 4
    cells = n ** 3
    a_eff = esz * (2 * cells + cells + 2 * 3 * (n + 1) * n * n)
    teff = a_eff * args.steps / sec / 1e9
    peak, peak_kind = measured_peak_hbm()
    cfg = {"workload": f"heat diffusion {n}^3 cells, implicit step dt = 1 of heat_wip.jl (Value -0.1 / 0.3 on "
                       "south / north, Flux 0 elsewhere, Gaussian initial temperature), one PT iteration per step",
           "grid": list(dims), "a_eff_arrays": 9, "l2": "inputs exceed L2 (126 MB): no flush needed"}
    line = _base_line(f"heat PT T_eff GB/s ({n}^3, {dtype.upper()})", teff, "GB/s", args.steps, args.warmup,
                      1e3 * sec / args.steps, dtype, cfg)
    line.update({"gpu_launches": args.steps, "clocks": ck,
                 "roofline": {"bound": "hbm", "achieved": teff, "peak": peak, "unit": "GB/s", "frac": teff / peak,
                              "peak_source": peak_kind, "algorithmic_bytes": a_eff}})
    return line


def run_shapes(args):
    """Every launch shape of the fused sweep on the slab workload at n^3: 3 warm-up
    iterations, then `steps` iterations timed with CUDA events on the model's stream,
    per precision; one JSON line with ms per iteration and T_eff per shape."""
    import torch
    fi = load_fastice()
    n = (args.n,) * 3
    A = a_eff_elements(n)
    out = {}
    for dtype in [d for d in args.dtypes.split(",") if d in ("f64", "f32")]:
        m = make_model(fi, n, dtype, 0)
        res = {}
        for v in range(m.lib.fi_fused_variant_count()):
            try:
                m.set_variant(v)
            except fi.FastIceError as e:
                if e.status == 6:  # not offered in this precision
                    continue
                raise
            m.advance(3)
            ms = time_advance(fi, m, args.steps, torch) / args.steps
            res[m.lib.fi_fused_variant_name(v).decode()] = {"ms_per_iter": ms,
                                                           "teff_gbs": A * (8 if dtype == "f64" else 4) / ms / 1e6}
        m.close()
        torch.cuda.empty_cache()
        out[dtype] = res
    print(json.dumps({"workload": f"launch shapes of the fused sweep, slab {n[0]}^3", "steps": args.steps,
                      "shapes": out}))


def run_ibbatch(args):
    """3D immersed-boundary glaciers of uneven sizes (seeded beds, n^3 with n drawn
    uniformly from --sizes, 48 to 160 by default) advanced together by shared launches (BatchedIB3D:
    eight launches per iteration of all members, iteration pairs replayed as a CUDA
    graph) against the same models advanced one at a time (each model's own
    graph-replayed iterations, synchronised before the next model).  One step = one
    PT iteration of every member; value = member iterations per second of the
    batch, wall time around the advance and a synchronize, after warm-up."""
    fi = load_fastice()
    from fastice_b200 import scenarios
    dtype = args.dtypes.split(",")[0]
    count = args.instances if args.instances != 256 else 12
    rng = np.random.default_rng(7)
    lo, hi = (int(v) for v in args.sizes.split(","))
    sizes = [int(v) for v in rng.integers(lo, hi + 1, count)]
    models = [scenarios.bed_model(q, n, dtype=dtype)[0] for q, n in enumerate(sizes)]
    esz = 8 if dtype == "f64" else 4
    teff_bytes = sum(36 * n ** 3 * esz for n in sizes)  # the reference's 36-pass convention, whole boxes
    K, W = args.steps, max(args.warmup, 3)
    res = {}
    # one at a time (first, so that both arms start from the same state age)
    for m in models:
        m.advance(W)
        m.synchronize()
    t0 = time.perf_counter()
    for m in models:
        m.advance(K)
        m.synchronize()
    res["one_at_a_time_s"] = time.perf_counter() - t0
    b = fi.BatchedIB3D(models)
    b.advance(W)
    b.synchronize()
    t0 = time.perf_counter()
    b.advance(K)
    b.synchronize()
    res["batched_s"] = time.perf_counter() - t0
    b.close()
    for m in models:
        m.close()
    v = count * K / res["batched_s"]
    line = _base_line(f"batched 3D immersed-boundary iterations/s ({count} glaciers, {dtype.upper()})", v,
                      "member iterations/s", K, W, 1e3 * res["batched_s"] / K, dtype,
                      {"workload": f"{count} immersed-boundary glaciers (seeded 64-bump beds, seeds 0..{count - 1}) "
                                   f"of n^3 cells, n = {sizes}, linear viscosity, advanced together by shared "
                                   "launches; one step = one PT iteration of every member",
                       "members": count, "sizes": sizes, "timing": "wall clock around advance + synchronize"})
    line.update({"one_at_a_time": {"member_iterations_per_s": count * K / res["one_at_a_time_s"],
                                   "seconds": res["one_at_a_time_s"]},
                 "speedup_vs_one_at_a_time": res["one_at_a_time_s"] / res["batched_s"],
                 "teff_gbs_36_pass": teff_bytes * K / res["batched_s"] / 1e9,
                 "gpu_launches": f"{8 * K} (eight per iteration of all members; graph-replayed pairs)"})
    return line


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=511)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the glacier sweep, the mixed-precision glacier "
                                                            "solve and the heat sweep in the default line")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle comparison and manufactured-solution "
                                                            "errors (profiling runs)")
    ap.add_argument("--cpu-baseline-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help=argparse.SUPPRESS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape (profiling runs)")
    ap.add_argument("--variant", type=int, default=None, help="fused launch shape index (implies --no-autotune)")
    ap.add_argument("--dtypes", default="f64,f32", help="precisions to time, FP64 first")
    ap.add_argument("--workload", choices=("slab", "batched", "serving", "mixed", "glacier", "heat", "shapes", "ibbatch",
                                           "split"),
                    default="slab",
                    help="slab: the headline T_eff line; batched / serving / mixed / glacier / heat / shapes / "
                         "ibbatch / split: the batched 2D solves, the continuous-batching server, the mixed-precision "
                         "solve, the immersed-boundary glacier sweep, the heat sweep, the fused sweep's launch "
                         "shapes, the shared launches of 3D glaciers and one rank's share of a split slab (halo "
                         "exchange along x and y), one JSON line each")
    ap.add_argument("--instances", type=int, default=256,
                    help="batched: number of 2D instances; ibbatch: number of glaciers (default 12)")
    ap.add_argument("--sizes", default="48,160", help="ibbatch: smallest,largest cells per side of the glaciers")
    ap.add_argument("--tol", type=float, default=None, help="batched / serving / mixed: stop tolerance")
    ap.add_argument("--scale", type=float, default=0.25, help="serving: linear size scale of the request stream")
    ap.add_argument("--duration", type=float, default=2.0, help="serving: seconds of Poisson arrivals")
    ap.add_argument("--shared3d", action="store_true",
                    help="serving: 3D requests advance by shared launches instead of each on its own stream")
    ap.add_argument("--rounds", type=int, default=0, help="batched: stop after this many check rounds (profiling)")
    ap.add_argument("--storage", choices=("f32", "f64"), default="f32",
                    help="batched: FP32 sweeps in an FP64 defect correction (f32) or plain FP64 sweeps")
    ap.add_argument("--smooth", type=int, default=0, help="batched: log-space smoothing passes of the viscosity")
    ap.add_argument("--window", type=int, default=20000, help="batched: stall window in sweeps")
    ap.add_argument("--alone", type=int, default=16, help="batched: members timed one at a time")
    ap.add_argument("--errcheck", type=int, default=4, help="batched: members compared with a plain FP64 solve")
    ap.add_argument("--scenario", choices=("mms", "glacier"), default="mms",
                    help="mixed: the 3D manufactured solution or the immersed-boundary glacier")
    ap.add_argument("--rheology", choices=("linear", "glen", "glen_relaxed"), default="linear",
                    help="glacier workloads: linear viscosity 1 (the reference's glacier driver) or Glen's law "
                         "n=3, A=1, regularised at strain rate 1e-6 (glen_relaxed: relaxed in log scale at rate "
                         "0.1), with the slab's PT steps (r 0.7, re 8 pi)")
    args = ap.parse_args()
    if args.cpu_baseline_only:
        its, el, threads = _cpu_baseline_inproc((args.n,) * 3, args.cpu_seconds, args.warmup)
        print(json.dumps({"iterations": its, "seconds": el, "threads": threads}))
        return
    if args.workload != "slab":
        line = {"batched": run_batched, "serving": run_serving, "mixed": run_mixed,
                "glacier": run_glacier, "heat": run_heat, "shapes": run_shapes,
                "ibbatch": run_ibbatch, "split": run_split}[args.workload](args)
        if line is not None:
            print(json.dumps(line))
        return
    n = (args.n, args.n, args.n)
    ws, rank, local = dist_setup()
    metric = "PT-Stokes T_eff GB/s (511^3, FP64)"
    cfg = {"workload": f"3D tilted ice slab {n[0]}x{n[1]}x{n[2]} cells, Glen n=3 regularised, slip bed, free top, "
                       "periodic x/y, one PT iteration per step",
           "grid": list(n), "extent": [1.0, 1.0, 0.25], "alpha_deg": 10.0, "a_eff_arrays": 22,
           "l2": "inputs (11.8 GB FP64) exceed L2 (126 MB): no flush needed", "parallelism": f"replicas x{ws}"}

    if args.impl == "reference":
        if rank != 0:
            return
        its, el, cores = cpu_baseline(n, seconds=min(60.0, max(10.0, 0.5 * args.steps)), warm=min(args.warmup, 1))
        v = a_eff_elements(n) * 8 * its / el / 1e9
        line = {"metric": metric, "value": v, "unit": "GB/s", "n_gpus": args.gpus, "steps": its,
                "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * el / its, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "impl": "reference",
                "cpu_baseline": {"value": v, "unit": "GB/s", "cores": cores, "kind": "port",
                                 "sample": f"{its} whole PT iterations at {n[0]}^3 (C restatement of the reference "
                                           "CPU path, OpenMP threads pinned one per core, OMP_PROC_BIND=close; the "
                                           "Julia reference cannot run: no Julia toolchain)"},
                "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    fi = load_fastice()
    A = a_eff_elements(n)
    res = {}
    clocks = None
    for dtype in [d for d in args.dtypes.split(",") if d in ("f64", "f32")]:
        m = make_model(fi, n, dtype, local)
        tuned = None
        if args.variant is not None and m.path == "fused":
            m.set_variant(args.variant)
        elif m.path == "fused" and not args.no_autotune:
            # the autotuner times every launch shape on the model itself (3 iterations each);
            # those iterations are part of the warm-up
            best, per = m.autotune(iters=3)
            tuned = {"variant": best, "ms_per_iter": per}
        m.advance(args.warmup)
        m.synchronize()
        sampler = ClockSampler(local) if dtype == args.dtypes.split(",")[0] else None
        if sampler:
            sampler.start()
            time.sleep(0.15)
        if pg:
            pg.barrier()
        ms = time_advance(fi, m, args.steps, torch)
        if pg:
            pg.barrier()
        if sampler:
            clocks = sampler.stop()
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        if pg:
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_max = float(t.item())
        norms = m.residual_norms()
        res[dtype] = {"ms_total": ms_max, "ms_per_step": ms_max / args.steps, "path": m.path,
                      "finite": bool(norms[11] == 0.0), "tuned": tuned}
        m.close()
        torch.cuda.empty_cache()

    esz = {"f64": 8, "f32": 4}
    peak, peak_kind = measured_peak_hbm()
    prim = "f64" if "f64" in res else next(iter(res))  # FP64 unless only FP32 was timed (profiling runs)
    if prim != "f64":
        metric = metric.replace("FP64", prim.upper())
    f64 = res[prim]
    value = ws * A * esz[prim] * args.steps / (f64["ms_total"] / 1e3) / 1e9
    achieved = A * esz[prim] / (f64["ms_per_step"] / 1e3) / 1e9
    tr = TRAFFIC_BYTES_PER_CELL[prim]
    line = {
        "metric": metric, "value": value, "unit": "GB/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": f64["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": prim, "data": "synthetic", "config": cfg, "kernel_path": f64["path"],
        "launch_shape": {dt: (None if res[dt]["tuned"] is None else
                              list(res[dt]["tuned"]["ms_per_iter"])[res[dt]["tuned"]["variant"]]) for dt in res},
        "gpu_launches": args.steps,
        "autotune_ms_per_iter": {dt: (res[dt]["tuned"]["ms_per_iter"] if res[dt]["tuned"] else None) for dt in res},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": (tr * n[0] * n[1] * n[2]) if tr else None,
                     "algorithmic_bytes": A * esz[prim]},
        "reference_convention_teff": 23 * 8 * n[0] * n[1] * n[2] / (f64["ms_per_step"] / 1e3) / 1e9,
        "clocks": clocks,
    }
    if "f32" in res and prim == "f64":
        line["fp32"] = {"value": ws * A * 4 * args.steps / (res["f32"]["ms_total"] / 1e3) / 1e9, "unit": "GB/s",
                        "ms_per_step": res["f32"]["ms_per_step"],
                        "frac": (A * 4 / (res["f32"]["ms_per_step"] / 1e3) / 1e9) / peak}
    if not args.no_e2e and prim == "f64":
        v64 = res["f64"]["tuned"]["variant"] if res["f64"]["tuned"] else None
        if pg:
            pg.barrier()
        dt, h2d, d2h, _ = e2e_run(fi, n, "f64", local, args.steps, torch, variant=v64)
        if pg:  # every rank's replica, timed as the slowest one
            t = torch.tensor([dt], dtype=torch.float64, device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            dt = float(t.item())
        line["e2e"] = {"value": ws * A * 8 * args.steps / dt / 1e9, "unit": "GB/s",
                       "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                       "includes": "pinned host->device upload of the state, K iterations through the C ABI, "
                                   "residual norms, device->host download of the state"}
    if rank == 0 and ws == 1 and not args.no_parity:
        variants = {dt: (res[dt]["tuned"]["variant"] if res[dt]["tuned"] else args.variant) for dt in res}
        par = oracle_parity(fi, n, local, variants)
        line["error_vs_oracle"] = par["f64"]["max_rel_diff"] if "f64" in par else None
        line["fp32_error_vs_oracle"] = par["f32"]["max_rel_diff"] if "f32" in par else None
        line["parity"] = dict(par, bar="FP64 <= 1e-10 relative (production build, FMA contraction)",
                              pinned="partially: the reference is Julia and cannot run here; the oracle restates "
                                     "its kernels (operators, interpolation and ghost rules of Chmy.jl adopted)")
        mm = mms_errors(fi)
        line["mms_error"] = mm["mms3d_127"]["l2_rel_error"]
        line["mms"] = mm
    if rank == 0 and ws == 1 and not args.no_extras:
        # the other workloads, measured in the same run (one sub-object each)
        import copy
        extras = {}
        ga = copy.copy(args)
        ga.n, ga.steps, ga.warmup, ga.dtypes, ga.rheology = 383, 20, 3, "f64,f32", "linear"
        extras["glacier_sweep"] = run_glacier(ga)
        ma = copy.copy(args)
        ma.n, ma.scenario, ma.rheology, ma.tol = 383, "glacier", "linear", 1e-8
        extras["mixed_glacier"] = run_mixed(ma)
        ha = copy.copy(args)
        ha.n, ha.steps, ha.warmup, ha.dtypes = 511, 20, 3, "f64"
        extras["heat"] = run_heat(ha)
        line["other_workloads"] = extras
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        its, el, cores = cpu_baseline(n, seconds=12.0)
        line["cpu_baseline"] = {"value": A * 8 * its / el / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
                                "sample": f"{its} whole PT iterations at {n[0]}^3 in FP64 (C restatement of the "
                                          "reference CPU path, OpenMP threads pinned one per core, "
                                          "OMP_PROC_BIND=close)"}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
