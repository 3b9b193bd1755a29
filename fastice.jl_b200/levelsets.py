"""Level sets and volume fractions (src/LevelSets/LevelSets.jl:3-4) on the device.

``compute_levelset_from_dem(grid, dem_grid2d, dem)`` mirrors
``compute_levelset_from_dem!(arch, launch, Ψ, dem, dem_grid2D, grid, R)``
(compute_levelsets.jl:21-25), ``invert`` applies ``invert_levelset!``
(:32-35), and ``omega_from_psi`` mirrors ``ω_from_ψ!``
(volume_fractions_kernels.jl:101-110).  Arrays use the uniform halo box
(n+3 per dim), numpy order (z, y, x).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib as L
from .grids import UniformGrid
from .physics import FunctionField

MASK_COMPONENTS_3D = ("ccc", "vvv", "vcc", "cvc", "ccv", "vvc", "vcv", "cvv")
MASK_COMPONENTS_2D = ("cc", "vv", "vc", "cv")


def _grid_struct(g: UniformGrid) -> L.fi_grid:
    s = L.fi_grid()
    s.nd = g.ndims
    for k in range(g.ndims):
        s.n[k] = g.dims[k]
        s.origin[k] = g.origin[k]
        s.extent[k] = g.extent[k]
    return s


def dem_halo(dem, dem_grid: UniformGrid) -> np.ndarray:
    """DEM vertex values in halo storage ((m1+3), (m0+3)) valid up to index m+2.
    A FunctionField is sampled on the extended vertex coordinates."""
    if isinstance(dem, FunctionField):
        return dem.sample(halo=True)
    a = np.asarray(dem, dtype=np.float64)
    if a.shape != (dem_grid.dims[1] + 3, dem_grid.dims[0] + 3):
        raise ValueError("dem array must be in 2D vertex halo storage")
    return np.ascontiguousarray(a)


def compute_levelset_from_dem(grid: UniformGrid, dem_grid: UniformGrid, dem, R=None, invert: bool = False,
                              device: int = 0, library: str = "fast") -> np.ndarray:
    lib = L.load(library)
    d = dem_halo(dem, dem_grid)
    psi = np.zeros((grid.dims[2] + 3, grid.dims[1] + 3, grid.dims[0] + 3), np.float64)
    Rp = None
    if R is not None:
        Ra = np.ascontiguousarray(np.asarray(R, dtype=np.float64).reshape(9))
        Rp = Ra.ctypes.data
    g3, g2 = _grid_struct(grid), _grid_struct(dem_grid)
    L.check(lib, lib.fi_levelset_from_dem(C.byref(g3), C.byref(g2), d.ctypes.data, Rp, int(invert), psi.ctypes.data,
                                          int(device)))
    return psi


def omega_from_psi(grid: UniformGrid, psi: np.ndarray, device: int = 0, library: str = "fast") -> dict:
    lib = L.load(library)
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    comps = MASK_COMPONENTS_3D if grid.ndims == 3 else MASK_COMPONENTS_2D
    out = {c: np.zeros_like(psi) for c in comps}
    ptrs = (C.c_void_p * 8)(*([out[c].ctypes.data for c in comps] + [None] * (8 - len(comps))))
    g = _grid_struct(grid)
    L.check(lib, lib.fi_volfrac(C.byref(g), psi.ctypes.data, ptrs, int(device)))
    return out
