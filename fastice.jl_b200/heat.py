"""Heat diffusion (src/Models/Diffusion/Heat/): ``HeatDiffusionModel`` and
``advance_iteration!`` over the C ABI (fi_heat_*).

The reference module does not run as written (Heat.jl:35,43 call the
``KernelLaunch`` module as a constructor and read a ``model.fields`` that does not
exist; kernels.jl:3 expects the spacing where Heat.jl:53 passes the grid); this is
its evident intent: per PT iteration the flux relaxes toward -λ/(ρCp) ∇T and the
temperature toward the implicit step (T - T_o)/Δt = -∇·q, with
``BoundaryCondition{Value}`` (temperature on a side) and ``BoundaryCondition{Flux}``
(flux through a side).  Pseudo-time steps come from ``heat_iter_params``, the
driver's formulas (scripts_future_API/heat_wip.jl:35-45).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Mapping

import numpy as np

from . import _lib as L
from .grids import UniformGrid

_DT = {"f64": (L.FI_F64, np.float64), "f32": (L.FI_F32, np.float32)}
SIDES = (("west", "east"), ("south", "north"), ("bottom", "top"))


class Value:
    """``BoundaryCondition{Value}(v)``: temperature v on the side."""

    def __init__(self, v: float = 0.0):
        self.v = float(v)


class Flux:
    """``BoundaryCondition{Flux}(v)``: normal flux v through the side."""

    def __init__(self, v: float = 0.0):
        self.v = float(v)


def heat_iter_params(grid: UniformGrid, lambda_rhocp: float, dt: float) -> dict:
    """The driver's pseudo-transient steps (heat_wip.jl:35-45)."""
    cfl = 0.99 / math.sqrt(grid.ndims)
    lmax, dmin = max(grid.extent), min(grid.spacing())
    re = math.pi + math.sqrt(math.pi ** 2 + lmax ** 2 / lambda_rhocp / dt)
    theta = lmax / re / cfl / dmin
    beta = (re * lambda_rhocp) / (cfl * dmin * lmax)
    return {"Δτ": {"T": 1.0 / (dt + beta), "q": 1.0 / (1.0 + theta)}}


class HeatDiffusionModel:
    """``HeatDiffusionModel(; grid, boundary_conditions, physics, iter_params)``:
    boundary_conditions maps west/east/south/north/bottom/top to Value or Flux;
    physics is ``{"λ_ρCp": value}`` (or the driver's ``{"properties": value}``);
    iter_params is ``{"Δτ": {"T": ..., "q": ...}}``."""

    def __init__(self, *, grid: UniformGrid, boundary_conditions: Mapping, physics: Mapping, iter_params: Mapping,
                 dtype: str = "f64", device: int = 0, library: str = "fast"):
        if grid.ndims != 3:
            raise ValueError("the heat model is 3D")
        self.lib = L.load(library)
        self.grid, self.dtype = grid, dtype
        self._np = _DT[dtype][1]
        d = L.fi_heat_desc()
        d.grid.nd = 3
        for k in range(3):
            d.grid.n[k] = grid.dims[k]
            d.grid.origin[k] = grid.origin[k]
            d.grid.extent[k] = grid.extent[k]
            for s, side in enumerate(SIDES[k]):
                bc = boundary_conditions.get(side, Flux(0.0))
                d.kind[k][s] = L.FI_HEAT_VALUE if isinstance(bc, Value) else L.FI_HEAT_FLUX
                d.value[k][s] = bc.v
        lam = physics.get("λ_ρCp", physics.get("properties"))
        d.lambda_rhocp = float(lam)
        d.dtau_T = float(iter_params["Δτ"]["T"])
        d.dtau_q = float(iter_params["Δτ"]["q"])
        d.dtype = _DT[dtype][0]
        d.device = int(device)
        h = C.c_void_p()
        L.check(self.lib, self.lib.fi_heat_create(C.byref(d), C.byref(h)))
        self._h = h

    def field_shape(self, name: str):
        n = list(self.grid.dims)
        if name in ("qx", "qy", "qz"):
            n["xyz".index(name[1])] += 1
        return tuple(reversed(n))

    def set_field(self, name: str, values) -> None:
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(values, dtype=self._np), self.field_shape(name)))
        L.check(self.lib, self.lib.fi_heat_set_field(self._h, L.FI_HEAT_FIELDS[name], a.ctypes.data, a.nbytes))

    def get_field(self, name: str) -> np.ndarray:
        a = np.empty(self.field_shape(name), dtype=self._np)
        L.check(self.lib, self.lib.fi_heat_get_field(self._h, L.FI_HEAT_FIELDS[name], a.ctypes.data, a.nbytes))
        return a

    def apply_bcs(self) -> None:
        L.check(self.lib, self.lib.fi_heat_apply_bcs(self._h))

    def advance(self, niter: int, dt: float) -> None:
        L.check(self.lib, self.lib.fi_heat_advance(self._h, int(niter), float(dt)))

    @property
    def stream_ptr(self) -> int:
        s = C.c_void_p()
        L.check(self.lib, self.lib.fi_heat_stream(self._h, C.byref(s)))
        return s.value or 0

    def synchronize(self) -> None:
        L.check(self.lib, self.lib.fi_heat_synchronize(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.fi_heat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def advance_iteration(model: HeatDiffusionModel, t: float, dt: float) -> None:
    """``advance_iteration!(model, t, Δt)`` (Heat.jl:45-61)."""
    model.advance(1, dt)


__all__ = ["Value", "Flux", "HeatDiffusionModel", "advance_iteration", "heat_iter_params"]
