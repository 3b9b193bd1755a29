"""Host mirror of FastIce's Stokes models over the C ABI.

``IsothermalFullStokesModel`` mirrors src/Models/FullStokes/Isothermal/Isothermal.jl:22-125
and ``IsothermalImmersedBoundaryFullStokesModel`` mirrors
src/Models/ImmersedBoundaryFullStokes/Isothermal/Isothermal.jl:22-136.  The
library owns the device fields; the attribute tree ``model.stress.P``,
``model.stress.τ.xx``, ``model.velocity.V.x``, ``model.viscosity.η``,
``model.residual.r_P``, ``model.field_masks.na.ccc`` gives ``FieldRef`` handles
whose ``interior()`` / ``set(...)`` copy to and from host numpy arrays (numpy
order (z, y, x), i.e. x fastest as in Julia).

``advance_iteration(model, t, Δt)`` and ``compute_residuals(model)`` are the
reference's ``advance_iteration!`` / ``compute_residuals!``.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from types import SimpleNamespace
from typing import Optional

import numpy as np

from . import _lib as L
from .grids import UniformGrid
from .physics import (ArrayField, BoundaryCondition, FunctionField, IceRheology, Periodic, Relaxation, ValueField,
                      rheology_desc)

_DTYPES = {"f64": (L.FI_F64, np.float64), "f32": (L.FI_F32, np.float32)}
_HALO = {"iteration": L.FI_HALO_ITERATION, "state": L.FI_HALO_STATE}
_PATHS = {"auto": L.FI_PATH_AUTO, "reference": L.FI_PATH_REFERENCE, "fused": L.FI_PATH_FUSED}


class Arch:
    """``Arch(CUDABackend())``: one CUDA device."""

    def __init__(self, backend: str = "cuda", device: int = 0):
        if backend != "cuda":
            raise ValueError("libfastice_b200 runs on CUDA devices only (no CPU backend)")
        self.device = int(device)


class FieldRef:
    """Handle to one device field of a model."""

    def __init__(self, model: "_StokesBase", name: str):
        self.model = model
        self.name = name

    @property
    def location(self):
        return L.FIELD_LOC[self.name]

    def shape(self):
        g = self.model.grid
        loc = self.location
        return tuple(g.dims[d] + loc[d] for d in reversed(range(g.ndims)))

    def interior(self) -> np.ndarray:
        return self.model.get_field(self.name)

    def set(self, value) -> None:
        self.model.set_field(self.name, value)

    def __array__(self, dtype=None):
        a = self.interior()
        return a if dtype is None else a.astype(dtype)

    def __repr__(self):
        return f"FieldRef({self.name}, shape={self.shape()})"


def _ns(**kw):
    return SimpleNamespace(**kw)


def _bc_struct(bc) -> L.fi_bc:
    s = L.fi_bc()
    if not isinstance(bc, BoundaryCondition):
        raise TypeError("boundary conditions must be BoundaryCondition objects")
    s.kind = bc.kind.kind
    for i, c in enumerate(bc.components[:3]):
        s.c[i] = c
    return s


def _dtau(solver_params, nd):
    sp = solver_params or {}
    dt = sp.get("Δτ", sp.get("dtau"))
    if dt is None:
        raise ValueError("solver_params must contain Δτ = (Pr=..., τ=(xx=...,...), V=(x=...,...))")
    p = L.fi_pt_params()
    p.dt_P = float(dt["Pr"])
    tau = dt.get("τ", dt.get("tau"))
    V = dt["V"]
    for i, k in enumerate(("xx", "yy", "zz", "xy", "xz", "yz")):
        if k in tau:
            p.dt_tau[i] = float(tau[k])
    for i, k in enumerate(("x", "y", "z")[:nd]):
        p.dt_V[i] = float(V[k])
    return p


def effective_rheology(rheology: IceRheology, solver_params: dict, eta_rel: Optional[str] = None) -> IceRheology:
    """The rheology a model iterates with.  Drivers pass an under-relaxation rate
    ``η_rel`` in ``solver_params`` (stokes_manufactured_solution_free_slip_2D.jl:76,
    tm_stokes_mpi_wip.jl:71) that the reference's kernels never read; by default it
    is ignored here too, so results stay the reference's.  With ``eta_rel`` =
    'log', 'log10' or 'lin' the rate is honoured as its evident intent: the new
    viscosity relaxes from the current one toward the rheology's value,
    Relaxation(η, rheology, η_rel; scale) of Physics.jl:28-47."""
    rate = None
    if solver_params:
        rate = solver_params.get("η_rel", solver_params.get("eta_rel"))
    if eta_rel is None or rate is None:
        return rheology
    if eta_rel not in ("log", "log10", "lin"):
        raise ValueError("eta_rel must be None, 'log', 'log10' or 'lin'")
    if isinstance(rheology, Relaxation):
        raise ValueError("the rheology is a Relaxation already; η_rel would nest a second one")
    return Relaxation(rheology, float(rate), scale=None if eta_rel == "lin" else eta_rel)


class _StokesBase:
    immersed = False

    def __init__(self, *, grid: UniformGrid, boundary_conditions, gravity, rheology, solver_params, arch=None,
                 dtype: str = "f64", path: str = "auto", outer_width=None, level_sets=None, library: str = "fast",
                 eta_rel: Optional[str] = None):
        self.lib = L.load(library)
        rheology = effective_rheology(rheology, solver_params, eta_rel)
        self.grid = grid
        self.arch = arch or Arch()
        self.dtype = dtype
        self.np_dtype = _DTYPES[dtype][1]
        self.boundary_conditions = boundary_conditions
        self.gravity = gravity
        self.rheology = rheology
        self.solver_params = solver_params
        self.level_sets = level_sets
        self.outer_width = outer_width  # accepted for signature parity; the fused sweep has no inner/outer split
        nd = grid.ndims
        d = L.fi_model_desc()
        d.grid.nd = nd
        for k in range(nd):
            d.grid.n[k] = grid.dims[k]
            d.grid.origin[k] = grid.origin[k]
            d.grid.extent[k] = grid.extent[k]
        names = ("x", "y", "z")[:nd]
        for k, nm in enumerate(names):
            left, right = boundary_conditions[nm]
            d.bc[k][0] = _bc_struct(left)
            d.bc[k][1] = _bc_struct(right)
        field_inputs = {}
        for k, nm in enumerate(names):
            g = gravity.get(nm, 0.0) if isinstance(gravity, dict) else getattr(gravity, nm)
            if isinstance(g, (int, float)):
                d.gravity.kind[k], d.gravity.value[k] = L.FI_G_VALUE, float(g)
            elif isinstance(g, ValueField):
                d.gravity.kind[k], d.gravity.value[k] = L.FI_G_VALUE, g.value
            else:
                d.gravity.kind[k] = L.FI_G_FIELD
                field_inputs["g" + nm] = g
        d.rheology, rfields = rheology_desc(rheology)
        field_inputs.update(rfields)
        d.dtau = _dtau(solver_params, nd)
        d.dtype = _DTYPES[dtype][0]
        d.immersed = 1 if self.immersed else 0
        d.path = _PATHS[path]
        d.device = self.arch.device
        self._desc = d
        h = C.c_void_p()
        L.check(self.lib, self.lib.fi_model_create(C.byref(d), C.byref(h)))
        self._h = h
        for name, src in field_inputs.items():
            self._upload_input(name, src)
        self._build_tree()

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self.lib.fi_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- field access --------------------------------------------------------
    def _build_tree(self):
        f = lambda n: FieldRef(self, n)
        nd = self.grid.ndims
        if nd == 3:
            tau = _ns(xx=f("txx"), yy=f("tyy"), zz=f("tzz"), xy=f("txy"), xz=f("txz"), yz=f("tyz"))
            V = _ns(x=f("Vx"), y=f("Vy"), z=f("Vz"))
            rV = _ns(x=f("rVx"), y=f("rVy"), z=f("rVz"))
        else:
            tau = _ns(xx=f("txx"), yy=f("tyy"), xy=f("txy"))
            V = _ns(x=f("Vx"), y=f("Vy"))
            rV = _ns(x=f("rVx"), y=f("rVy"))
        self.stress = _ns(P=f("P"), Pr=f("P"), τ=tau, tau=tau)
        self.velocity = _ns(V=V)
        self.viscosity = _ns(η=f("eta"), η_next=f("eta_next"), eta=f("eta"), eta_next=f("eta_next"))
        self.residual = _ns(r_V=rV, r_P=f("rP"), r_Pr=f("rP"))
        if self.immersed:
            comps = ("ccc", "vvv", "vcc", "cvc", "ccv", "vvc", "vcv", "cvv")
            self.field_masks = _ns(na=_ns(**{c: f("na_" + c) for c in comps}),
                                   ns=_ns(**{c: f("ns_" + c) for c in comps}))

    def field_shape(self, name):
        loc = L.FIELD_LOC[name]
        return tuple(self.grid.dims[d] + loc[d] for d in reversed(range(self.grid.ndims)))

    def set_field(self, name: str, value) -> None:
        shape = self.field_shape(name)
        if np.isscalar(value):
            arr = np.full(shape, value, dtype=self.np_dtype)
        else:
            arr = np.ascontiguousarray(np.asarray(value, dtype=self.np_dtype))
            if arr.shape != shape:
                arr = np.ascontiguousarray(np.broadcast_to(arr, shape))
        L.check(self.lib, self.lib.fi_model_set_field(self._h, L.FIELD_ID[name], arr.ctypes.data, arr.nbytes))

    def get_field(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Interior of a field as a host array; ``out`` (contiguous, right shape and
        dtype, e.g. a pinned buffer) is filled in place when given."""
        arr = np.empty(self.field_shape(name), dtype=self.np_dtype) if out is None else out
        if arr.shape != self.field_shape(name) or arr.dtype != self.np_dtype or not arr.flags.c_contiguous:
            raise ValueError("out must be a contiguous array of the field's interior shape and the model's dtype")
        L.check(self.lib, self.lib.fi_model_get_field(self._h, L.FIELD_ID[name], arr.ctypes.data, arr.nbytes))
        return arr

    def set_params(self, rheology: IceRheology = None, solver_params: dict = None) -> None:
        """New rheology and/or PT steps for the next iterations (fi_model_set_params);
        the state is kept.  The rheology must read the same fields as the model's."""
        rheology = self.rheology if rheology is None else rheology
        solver_params = self.solver_params if solver_params is None else solver_params
        rdesc, rfields = rheology_desc(rheology)
        if rfields:
            raise ValueError("set_params takes rheologies without field inputs; upload fields with set_field")
        dt = _dtau(solver_params, self.grid.ndims)
        L.check(self.lib, self.lib.fi_model_set_params(self._h, C.byref(rdesc), C.byref(dt)))
        self.rheology, self.solver_params = rheology, solver_params

    def solve_continuation(self, stages, retries: int = 0, **solve_kw) -> dict:
        """A continuation driver: for each stage (rheology, solver_params, tol) set the
        parameters and solve to that stage's tolerance from the previous stage's state
        (e.g. a viscosity cap raised stage by stage for Glen's law).  A stage's
        solver_params is a dict, or a function attempt -> dict: a stage whose solve
        diverges (non-finite residual) is run again, up to ``retries`` times, from the
        state it started from (kept on the host) with the parameters of the next
        attempt.  Returns the last stage's report with the sweeps, outer steps and
        seconds of every stage and attempt summed."""
        from .writers import STATE_FIELDS_2D, STATE_FIELDS_3D
        names = STATE_FIELDS_3D if self.grid.ndims == 3 else STATE_FIELDS_2D
        total = {"iterations": 0, "outer": 0, "seconds": 0.0, "stages": []}
        rep = None
        for rheology, solver_params, tol in stages:
            saved = {f: self.get_field(f) for f in names} if retries > 0 else None
            for attempt in range(retries + 1):
                sp = solver_params(attempt) if callable(solver_params) else solver_params
                self.set_params(rheology, sp)
                t0 = time.perf_counter()
                try:
                    rep = self.solve(tol=tol, **solve_kw)
                except L.FastIceError as e:
                    if e.status != L.FI_ERR_DIVERGED or attempt == retries:
                        raise
                    total["seconds"] += time.perf_counter() - t0
                    total["stages"].append({"tol": tol, "attempt": attempt, "diverged": True})
                    for f in names:
                        self.set_field(f, saved[f])
                    self.copy_field("eta_next", "eta")
                    self.apply_bcs()
                    continue
                break
            total["iterations"] += rep["iterations"]
            total["outer"] += rep["outer"]
            total["seconds"] += rep["seconds"]
            total["stages"].append({"tol": tol, "attempt": attempt, "iterations": rep["iterations"],
                                    "measure": rep["measure"], "converged": rep["converged"]})
            if not rep["converged"]:
                break
        out = dict(rep)
        out.update(iterations=total["iterations"], outer=total["outer"], seconds=total["seconds"],
                   stages=total["stages"])
        return out

    def copy_field(self, dst: str, src: str) -> None:
        """set!(dst, src) on the device between two fields at the same location
        (e.g. η_next from η), ghosts included."""
        L.check(self.lib, self.lib.fi_model_copy_field(self._h, L.FIELD_ID[dst], L.FIELD_ID[src]))

    def _upload_input(self, name, src):
        if isinstance(src, FunctionField):
            full = src.sample(halo=True)
            sl = tuple(slice(1, s + 1) for s in self.field_shape(name))
            self.set_field(name, full[sl])
        elif isinstance(src, ArrayField):
            self.set_field(name, src.values)
        elif isinstance(src, np.ndarray):
            self.set_field(name, src)
        else:
            raise TypeError(f"cannot use {type(src).__name__} as the input field {name}")

    # -- reference operations ---------------------------------------------------
    def apply_bcs(self):
        L.check(self.lib, self.lib.fi_model_apply_bcs(self._h))

    def advance(self, niter: int = 1):
        L.check(self.lib, self.lib.fi_model_advance(self._h, int(niter)))

    def compute_residuals(self):
        L.check(self.lib, self.lib.fi_model_compute_residuals(self._h))

    def residual_norms(self) -> np.ndarray:
        out = (C.c_double * L.FI_NORMS_LEN)()
        L.check(self.lib, self.lib.fi_model_residual_norms(self._h, out))
        return np.array(out[:], dtype=np.float64)

    def compute_tau(self):
        L.check(self.lib, self.lib.fi_model_compute_tau(self._h))

    def synchronize(self):
        L.check(self.lib, self.lib.fi_model_synchronize(self._h))

    @property
    def path(self) -> str:
        v = C.c_int32()
        L.check(self.lib, self.lib.fi_model_path(self._h, C.byref(v)))
        return {L.FI_PATH_REFERENCE: "reference", L.FI_PATH_FUSED: "fused"}[v.value]

    def set_variant(self, variant: int) -> None:
        L.check(self.lib, self.lib.fi_model_set_variant(self._h, int(variant)))

    def autotune(self, iters: int = 3):
        """Time every fused-sweep variant (advancing the model) and keep the fastest;
        returns (best index, {variant name: ms per iteration})."""
        nv = self.lib.fi_fused_variant_count()
        ms = (C.c_double * nv)()
        best = C.c_int32()
        L.check(self.lib, self.lib.fi_model_autotune(self._h, int(iters), C.byref(best), ms))
        names = [self.lib.fi_fused_variant_name(v).decode() for v in range(nv)]
        return best.value, dict(zip(names, ms[:]))

    # -- an iteration in two halves around the halo exchange (fi_model_advance_begin / _end)
    def advance_begin(self, dim: int) -> None:
        L.check(self.lib, self.lib.fi_model_advance_begin(self._h, int(dim)))

    def advance_end(self) -> None:
        L.check(self.lib, self.lib.fi_model_advance_end(self._h))

    # -- subdomain halo layers (fi_model_halo_*: a slab of a domain split along x or y)
    def halo_bytes(self, dim: int, side: int, what: str = "iteration") -> int:
        """Bytes of the halo message packed toward ``side`` (0 = low, 1 = high
        neighbour) of the split dimension ``dim``; ``what`` is "iteration" (V, η)
        or "state" (P, τ, V, η)."""
        b = C.c_size_t()
        L.check(self.lib, self.lib.fi_model_halo_bytes(self._h, int(dim), int(side), _HALO[what], C.byref(b)))
        return b.value

    def halo_pack(self, dim: int, side: int, dst_ptr: int, what: str = "iteration") -> None:
        """Fill the device buffer at ``dst_ptr`` with the message for the neighbour on
        ``side`` (on the model's stream)."""
        L.check(self.lib, self.lib.fi_model_halo_pack(self._h, int(dim), int(side), _HALO[what], C.c_void_p(dst_ptr)))

    def halo_unpack(self, dim: int, side: int, src_ptr: int, what: str = "iteration") -> None:
        """Write the message received from the neighbour on ``side`` (device buffer at
        ``src_ptr``) into this model's ghost layers (on the model's stream)."""
        L.check(self.lib, self.lib.fi_model_halo_unpack(self._h, int(dim), int(side), _HALO[what], C.c_void_p(src_ptr)))

    @property
    def stream_ptr(self) -> int:
        s = C.c_void_p()
        L.check(self.lib, self.lib.fi_model_stream(self._h, C.byref(s)))
        return s.value or 0

    def device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        L.check(self.lib, self.lib.fi_model_device_ptr(self._h, L.FIELD_ID[name], C.byref(p)))
        return p.value or 0

    def layout(self):
        a, b, c = C.c_size_t(), C.c_size_t(), C.c_size_t()
        L.check(self.lib, self.lib.fi_model_layout(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def solve(self, *, max_iter: int, ncheck: int, tol: float, measure: str = "abs_inf", rho_g_inf: float = 1.0,
              length_z: float = 1.0, mode: str = "plain", inner_iter: int = 0, inner_reduction: float = 0.0):
        """Driver loop with a convergence check every ``ncheck`` iterations
        (tm_stokes_chmy.jl:283-305); returns a dict report.  ``mode="mixed"``
        (FP64 models): FP32 PT sweeps inside an FP64 defect correction."""
        o = L.fi_solve_opts()
        o.max_iter, o.ncheck, o.tol = int(max_iter), int(ncheck), float(tol)
        o.measure = {"abs_inf": L.FI_CONV_ABS_INF, "rel_slab": L.FI_CONV_REL_SLAB}[measure]
        o.rho_g_inf, o.length_z = float(rho_g_inf), float(length_z)
        o.mode = {"plain": L.FI_SOLVE_PLAIN, "mixed": L.FI_SOLVE_MIXED}[mode]
        o.inner_iter, o.inner_reduction = int(inner_iter), float(inner_reduction)
        r = L.fi_solve_report()
        st = self.lib.fi_model_solve(self._h, C.byref(o), C.byref(r))
        if st not in (L.FI_OK, L.FI_ERR_TIMEOUT):
            L.check(self.lib, st)
        return {"iterations": r.iterations, "outer": r.outer, "measure": r.measure, "norms": list(r.norms),
                "seconds": r.seconds, "converged": bool(r.converged)}


class IsothermalFullStokesModel(_StokesBase):
    """``IsothermalFullStokesModel(; arch, grid, boundary_conditions, gravity,
    rheology, solver_params, outer_width)`` (FullStokes/Isothermal/Isothermal.jl:60-89)."""

    immersed = False


class IsothermalImmersedBoundaryFullStokesModel(_StokesBase):
    """``IsothermalImmersedBoundaryFullStokesModel(; ..., level_sets)``
    (ImmersedBoundaryFullStokes/Isothermal/Isothermal.jl:63-98).  The volume
    fractions ``field_masks.na`` / ``field_masks.ns`` are filled with
    :func:`omega_from_psi` or set directly."""

    immersed = True

    def omega_from_psi(self, group: str, psi_halo: np.ndarray) -> None:
        """ω_from_ψ!(arch, launch, model.field_masks.<group>, ψ, grid) on the device."""
        psi = np.ascontiguousarray(psi_halo, dtype=np.float64)
        n = self.grid.dims
        if psi.shape != (n[2] + 3, n[1] + 3, n[0] + 3):
            raise ValueError("psi must be a vertex field in halo storage (n+3 per dim)")
        L.check(self.lib, self.lib.fi_model_volfrac_from_levelset(self._h, {"na": 0, "ns": 1}[group], psi.ctypes.data))


class BatchedIB3D:
    """Several 3D immersed-boundary models advanced by shared launches
    (fi_ib_batch_* in the C ABI): one iteration of every small member is eight
    launches whatever their number, and pairs of iterations replay as a CUDA graph;
    a member whose launch spans more than 2048 blocks advances on its own stream.
    Each member's iteration is the one ``advance`` runs for it alone."""

    def __init__(self, models=()):
        models = list(models)
        self.lib = models[0].lib if models else L.load()
        self.models = []
        arr = (C.c_void_p * max(1, len(models)))(*[m._h for m in models])
        h = C.c_void_p()
        L.check(self.lib, self.lib.fi_ib_batch_create(arr, len(models), C.byref(h)))
        self._h = h
        self.models = models

    def add(self, m) -> None:
        L.check(self.lib, self.lib.fi_ib_batch_add(self._h, m._h))
        self.models.append(m)

    def remove(self, m) -> None:
        L.check(self.lib, self.lib.fi_ib_batch_remove(self._h, m._h))
        self.models.remove(m)

    def advance(self, niter: int) -> None:
        L.check(self.lib, self.lib.fi_ib_batch_advance(self._h, int(niter)))

    def synchronize(self) -> None:
        L.check(self.lib, self.lib.fi_ib_batch_synchronize(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self.lib.fi_ib_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchedStokes2D:
    """Many independent 2D models solved together (fi_batch_* in the C ABI).

    One persistent launch per PT iteration covers the tiles of every instance
    still iterating; checks, retirement and work-list compaction run on the
    device, and the check-to-check step replays as a CUDA graph.  Each member
    follows advance_iteration! of its own model (linear rheology, viscosity held
    at the member's current η).  The members stay usable as models: their state
    and iteration counts are updated in place.
    """

    def __init__(self, models):
        models = list(models)
        if not models:
            raise ValueError("empty batch")
        self.lib = models[0].lib
        if any(m.lib is not self.lib for m in models):
            raise ValueError("all members must come from one library build")
        self.models = models
        arr = (C.c_void_p * len(models))(*[m._h for m in models])
        h = C.c_void_p()
        L.check(self.lib, self.lib.fi_batch_create(arr, len(models), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.fi_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, model) -> None:
        """Admit a member between steps; its solve starts at the next step."""
        if model.lib is not self.lib:
            raise ValueError("all members must come from one library build")
        L.check(self.lib, self.lib.fi_batch_add(self._h, model._h))
        self.models.append(model)

    def remove(self, model) -> None:
        L.check(self.lib, self.lib.fi_batch_remove(self._h, model._h))
        self.models.remove(model)

    def __len__(self) -> int:
        return int(self.lib.fi_batch_size(self._h))

    def advance(self, niter: int = 1) -> None:
        L.check(self.lib, self.lib.fi_batch_advance(self._h, int(niter)))

    @staticmethod
    def _opts(max_iter, ncheck, tol, use_graph, window):
        o = L.fi_batch_opts()
        o.max_iter, o.ncheck, o.tol = int(max_iter), int(ncheck), float(tol)
        o.use_graph, o.window = 1 if use_graph else 0, int(window)
        return o

    def _items(self, items):
        return [{"iterations": it.iterations, "status": L.FI_ITEM_STATUS[it.status], "measure": it.measure}
                for it in items]

    def step(self, *, max_iter: int, ncheck: int, tol: float, rounds: int = 1, use_graph: bool = True,
             window: int = 0):
        """Up to ``rounds`` check-to-check steps of the members still iterating (no
        restart).  Returns (items, n_active)."""
        o = self._opts(max_iter, ncheck, tol, use_graph, window)
        items = (L.fi_batch_item * max(len(self.models), 1))()
        na = C.c_int32()
        L.check(self.lib, self.lib.fi_batch_step(self._h, C.byref(o), int(rounds), items, C.byref(na)))
        return self._items(items[:len(self.models)]), na.value

    def measures(self) -> np.ndarray:
        out = np.zeros(len(self.models))
        L.check(self.lib, self.lib.fi_batch_measure(self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def set_variant(self, variant: int) -> None:
        L.check(self.lib, self.lib.fi_batch_set_variant(self._h, int(variant)))

    def autotune(self, iters: int = 10):
        nv = self.lib.fi_batch_variant_count()
        ms = (C.c_double * nv)()
        best = C.c_int32()
        L.check(self.lib, self.lib.fi_batch_autotune(self._h, int(iters), C.byref(best), ms))
        names = [self.lib.fi_batch_variant_name(v).decode() for v in range(nv)]
        return best.value, dict(zip(names, list(ms)))

    def solve(self, *, max_iter: int, ncheck: int, tol: float, use_graph: bool = True, window: int = 0,
              mode: str = "plain", inner_tol: float = 0.0):
        """Iterate every member until it converges (measure < tol), stalls, fails or
        reaches max_iter.  Returns (items, seconds); items[k] is a dict with
        iterations, status and measure of member k.  ``mode="mixed"`` (FP64
        members): FP32 batched sweeps inside a per-member FP64 defect correction
        (fi_batch_solve_mixed); ``window`` then also ends the FP32 stages at their
        rounding floor."""
        o = self._opts(max_iter, ncheck, tol, use_graph, window)
        items = (L.fi_batch_item * len(self.models))()
        sec = C.c_double()
        if mode == "mixed":
            L.check(self.lib, self.lib.fi_batch_solve_mixed(self._h, C.byref(o), float(inner_tol), items, C.byref(sec)))
        elif mode == "plain":
            L.check(self.lib, self.lib.fi_batch_solve(self._h, C.byref(o), items, C.byref(sec)))
        else:
            raise ValueError(mode)
        return self._items(items), sec.value


# -- free functions with the reference names ----------------------------------------
def advance_iteration(model: _StokesBase, t: float = 0.0, dt: float = 1.0) -> None:
    """``advance_iteration!(model, t, Δt)`` (t and Δt are unused, as in the reference)."""
    model.advance(1)


def compute_residuals(model: _StokesBase) -> None:
    """``compute_residuals!(model)``: fills ``model.residual``."""
    model.compute_residuals()


def set_(field: FieldRef, value) -> None:
    """``set!(field, value)``."""
    field.set(value)


def interior(field: FieldRef) -> np.ndarray:
    """``Array(interior(field))``."""
    return field.interior()


def pt_params(grid: UniformGrid, r: float = 0.7, re_mech: float = 8 * math.pi, vdtau_factor: float = 1.1,
              use_center_spacing: bool = True, eta_rel: Optional[float] = None) -> dict:
    """Pseudo-transient steps as the drivers compute them
    (stokes_manufactured_solution_free_slip_2D.jl:67-77; tm_stokes_chmy.jl:48-54 uses
    re_mech=2π and factor 1.5): returns solver_params with Δτ."""
    nd = grid.ndims
    ltau = min(grid.extent) / re_mech
    vdtau = min(grid.spacing()) / math.sqrt(nd * vdtau_factor)
    theta = ltau * (r + 4 / 3) / vdtau
    dt_r = 1.0 / (theta + 1.0)
    nudt = vdtau * ltau
    taus = ("xx", "yy", "zz", "xy", "xz", "yz") if nd == 3 else ("xx", "yy", "xy")
    sp = {"Δτ": {"Pr": r / theta, "τ": {k: dt_r for k in taus}, "V": {k: nudt for k in ("x", "y", "z")[:nd]}}}
    if eta_rel is not None:
        sp["η_rel"] = float(eta_rel)  # read only by models created with eta_rel=... (see effective_rheology)
    return sp
