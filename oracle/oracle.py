"""CPU oracle driver (TEST INFRASTRUCTURE ONLY).

Python side of the plain-C restatement of the FastIce pseudo-transient Stokes
path in ``oracle/*.c``.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` use this module, and only as the checker: the
product library never imports it.

Parity status: partially pinned -- grid geometry is pinned to the reference's
``test/test_chmy_grids.jl``; the Chmy.jl operator / boundary-condition rules are
"parity unpinned" (Chmy.jl 0.1 is not vendored) and follow the contract written
in ``oracle/fi_oracle.h``.

A problem is described by :class:`Spec`, a plain dataclass with the same
meaning as the reference's model constructor arguments
(``src/Models/FullStokes/Isothermal/Isothermal.jl:60-66``).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfi_oracle.so")

BC_SLIP, BC_TRACTION, BC_VELOCITY, BC_PERIODIC = 0, 1, 2, 3
RHEO_LINEAR, RHEO_POWER = 0, 1
RELAX_NONE, RELAX_LIN, RELAX_LOG, RELAX_LOG10 = 0, 1, 2, 3
G_VALUE, G_ARRAY = 0, 1
NORMS_LEN = 12

FIELDS_3D = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta", "eta_next")
FIELDS_2D = ("P", "txx", "tyy", "txy", "Vx", "Vy", "eta", "eta_next")
# location (Center=0 / Vertex=1) per dim, FullStokes Isothermal.jl:36-56
LOCS = {
    "P": (0, 0, 0), "txx": (0, 0, 0), "tyy": (0, 0, 0), "tzz": (0, 0, 0),
    "txy": (1, 1, 0), "txz": (1, 0, 1), "tyz": (0, 1, 1),
    "Vx": (1, 0, 0), "Vy": (0, 1, 0), "Vz": (0, 0, 1),
    "eta": (0, 0, 0), "eta_next": (0, 0, 0),
    "rP": (0, 0, 0), "rVx": (1, 0, 0), "rVy": (0, 1, 0), "rVz": (0, 0, 1),
    "gx": (1, 0, 0), "gy": (0, 1, 0), "gz": (0, 0, 1),
}
MASK_COMPONENTS = ("ccc", "vvv", "vcc", "cvc", "ccv", "vvc", "vcv", "cvv")
MASK_LOCS = {
    "ccc": (0, 0, 0), "vvv": (1, 1, 1), "vcc": (1, 0, 0), "cvc": (0, 1, 0),
    "ccv": (0, 0, 1), "vvc": (1, 1, 0), "vcv": (1, 0, 1), "cvv": (0, 1, 1),
}


class _Params(C.Structure):
    _fields_ = [
        ("nd", C.c_int), ("n", C.c_int * 3), ("inv_dx", C.c_double * 3),
        ("bc_kind", (C.c_int * 2) * 3), ("bc_val", ((C.c_double * 3) * 2) * 3),
        ("dt_P", C.c_double), ("dt_tau", C.c_double * 6), ("dt_V", C.c_double * 3),
        ("g_kind", C.c_int * 3), ("g_val", C.c_double * 3),
        ("rheo_inner", C.c_int), ("rheo_eta_val", C.c_double), ("rheo_A", C.c_double),
        ("rheo_n", C.c_int), ("rheo_has_reg", C.c_int), ("rheo_inv_eta_reg", C.c_double),
        ("rheo_relax", C.c_int), ("rheo_rate", C.c_double),
    ]


class _Fields(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in (
        "P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta", "eta_next",
        "rVx", "rVy", "rVz", "rP", "gx", "gy", "gz", "eta_lin", "A_field")] + [
        ("wna", C.c_void_p * 8), ("wns", C.c_void_p * 8)]


_lib = None


def build() -> None:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        for suf in ("_f64", "_f32"):
            for name in ("update_sigma", "update_V", "bc_stress", "bc_velocity", "compute_residuals",
                         "compute_tau", "ib_update_sigma", "ib_update_V", "ib_compute_residuals"):
                fn = getattr(L, f"fo_{name}{suf}")
                fn.argtypes = [C.POINTER(_Params), C.POINTER(_Fields)]
                fn.restype = None
            for name in ("advance", "ib_advance"):
                fn = getattr(L, f"fo_{name}{suf}")
                fn.argtypes = [C.POINTER(_Params), C.POINTER(_Fields), C.c_int]
                fn.restype = None
            for name in ("residual_norms", "ib_residual_norms"):
                fn = getattr(L, f"fo_{name}{suf}")
                fn.argtypes = [C.POINTER(_Params), C.POINTER(_Fields), C.POINTER(C.c_double)]
                fn.restype = None
            fn = getattr(L, f"fo_bc_eta{suf}")
            fn.argtypes = [C.POINTER(_Params), C.c_void_p]
            fn.restype = None
        L.fo_vol_box3.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.fo_vol_box3.restype = C.c_double
        L.fo_vol_box2.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.fo_vol_box2.restype = C.c_double
        L.fo_volfrac3d.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p, C.c_void_p * 8]
        L.fo_volfrac3d.restype = None
        L.fo_volfrac2d.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p, C.c_void_p * 4]
        L.fo_volfrac2d.restype = None
        L.fo_levelset_from_dem.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        L.fo_levelset_from_dem.restype = None
        L.fo_invert_levelset.argtypes = [C.POINTER(C.c_int), C.c_void_p]
        L.fo_invert_levelset.restype = None
        _lib = L
    return _lib


@dataclasses.dataclass
class Spec:
    """Plain description of one Stokes problem (grid, BCs, physics, PT steps).

    ``bcs[d] = ((kind, (c0, c1, c2)), (kind, (c0, c1, c2)))`` for the left and
    right side of dim ``d``; ``dt = (dt_P, dt_tau[6], dt_V[3])`` with tau in the
    order xx, yy, zz, xy, xz, yz.
    """
    nd: int
    n: Sequence[int]
    extent: Sequence[float]
    origin: Sequence[float]
    bcs: Sequence
    dt_P: float
    dt_tau: Sequence[float]
    dt_V: Sequence[float]
    g_val: Sequence[float] = (0.0, 0.0, 0.0)
    rheo_inner: int = RHEO_LINEAR
    rheo_eta_val: float = 1.0
    rheo_A: float = 1.0
    rheo_n: int = 3
    rheo_has_reg: int = 0
    rheo_inv_eta_reg: float = 0.0
    rheo_relax: int = RELAX_NONE
    rheo_rate: float = 0.0
    dtype: str = "f64"

    @property
    def dx(self):
        return tuple(self.extent[d] / self.n[d] for d in range(self.nd))

    @property
    def inv_dx(self):
        return tuple(1.0 / (self.extent[d] / self.n[d]) for d in range(self.nd))

    def storage_shape(self):
        """numpy shape (z, y, x) of the uniform halo storage."""
        return tuple(self.n[d] + 3 for d in reversed(range(self.nd)))


def _params(spec: Spec, g_kind) -> _Params:
    p = _Params()
    p.nd = spec.nd
    for d in range(3):
        p.n[d] = int(spec.n[d]) if d < spec.nd else 0
        p.inv_dx[d] = spec.inv_dx[d] if d < spec.nd else 0.0
    for d in range(spec.nd):
        for s in range(2):
            kind, vals = spec.bcs[d][s]
            p.bc_kind[d][s] = kind
            for c in range(3):
                p.bc_val[d][s][c] = float(vals[c]) if c < len(vals) else 0.0
    p.dt_P = spec.dt_P
    for i in range(6):
        p.dt_tau[i] = float(spec.dt_tau[i]) if i < len(spec.dt_tau) else 0.0
    for i in range(3):
        p.dt_V[i] = float(spec.dt_V[i]) if i < len(spec.dt_V) else 0.0
        p.g_kind[i] = g_kind[i]
        p.g_val[i] = float(spec.g_val[i]) if i < len(spec.g_val) else 0.0
    p.rheo_inner = spec.rheo_inner
    p.rheo_eta_val = spec.rheo_eta_val
    p.rheo_A = spec.rheo_A
    p.rheo_n = spec.rheo_n
    p.rheo_has_reg = spec.rheo_has_reg
    p.rheo_inv_eta_reg = spec.rheo_inv_eta_reg
    p.rheo_relax = spec.rheo_relax
    p.rheo_rate = spec.rheo_rate
    return p


def interior_slices(spec: Spec, loc):
    """numpy index of the interior of a field at ``loc`` inside halo storage."""
    return tuple(slice(1, spec.n[d] + loc[d] + 1) for d in reversed(range(spec.nd)))


class OracleStokes:
    """FullStokes (or immersed-boundary FullStokes) state on the CPU oracle."""

    def __init__(self, spec: Spec, gravity_arrays: Optional[dict] = None, eta_lin=None, A_field=None,
                 masks: Optional[dict] = None):
        self.spec = spec
        self.np_dtype = np.float64 if spec.dtype == "f64" else np.float32
        self.suf = "_" + spec.dtype
        shape = spec.storage_shape()
        names = FIELDS_3D if spec.nd == 3 else FIELDS_2D
        self.a = {k: np.zeros(shape, self.np_dtype) for k in names}
        for k in (("rP", "rVx", "rVy", "rVz") if spec.nd == 3 else ("rP", "rVx", "rVy")):
            self.a[k] = np.zeros(shape, self.np_dtype)
        g_kind = [G_VALUE, G_VALUE, G_VALUE]
        self.g = {}
        for c, key in enumerate(("gx", "gy", "gz")[: spec.nd]):
            if gravity_arrays and key in gravity_arrays:
                g_kind[c] = G_ARRAY
                self.g[key] = np.ascontiguousarray(gravity_arrays[key], dtype=self.np_dtype)
                assert self.g[key].shape == shape
        self.eta_lin = None if eta_lin is None else np.ascontiguousarray(eta_lin, dtype=self.np_dtype)
        self.A_field = None if A_field is None else np.ascontiguousarray(A_field, dtype=self.np_dtype)
        self.masks = None
        if masks is not None:
            self.masks = {grp: [np.ascontiguousarray(masks[grp][c], dtype=self.np_dtype) for c in MASK_COMPONENTS]
                          for grp in ("na", "ns")}
        self.p = _params(spec, g_kind)
        self.f = _Fields()
        self._bind()

    def _ptr(self, arr):
        return arr.ctypes.data_as(C.c_void_p) if arr is not None else None

    def _bind(self):
        f = self.f
        for k, v in self.a.items():
            setattr(f, k, self._ptr(v))
        for k, v in self.g.items():
            setattr(f, k, self._ptr(v))
        f.eta_lin = self._ptr(self.eta_lin)
        f.A_field = self._ptr(self.A_field)
        if self.masks is not None:
            for c in range(8):
                f.wna[c] = self._ptr(self.masks["na"][c])
                f.wns[c] = self._ptr(self.masks["ns"][c])

    def _sync_swap(self):
        # the C advance swaps eta/eta_next pointers; mirror that on the numpy side
        if self.f.eta == self.a["eta_next"].ctypes.data:
            self.a["eta"], self.a["eta_next"] = self.a["eta_next"], self.a["eta"]
            self._bind()

    # -- field access (interior, x fastest == numpy [z, y, x]) -------------
    def set_interior(self, name, values):
        loc = LOCS[name]
        self.a[name][interior_slices(self.spec, loc)] = values

    def interior(self, name):
        loc = LOCS[name]
        return self.a[name][interior_slices(self.spec, loc)].copy()

    def apply_initial_bcs(self):
        """Initial ghost fill used by the drivers after set! (stress, velocity, eta)."""
        L = lib()
        getattr(L, "fo_bc_stress" + self.suf)(C.byref(self.p), C.byref(self.f))
        getattr(L, "fo_bc_velocity" + self.suf)(C.byref(self.p), C.byref(self.f))
        getattr(L, "fo_bc_eta" + self.suf)(C.byref(self.p), self.f.eta)

    def advance(self, niter: int = 1):
        L = lib()
        fn = "fo_ib_advance" if self.masks is not None else "fo_advance"
        getattr(L, fn + self.suf)(C.byref(self.p), C.byref(self.f), int(niter))
        self._sync_swap()

    def residual_norms(self) -> np.ndarray:
        L = lib()
        out = (C.c_double * NORMS_LEN)()
        fn = "fo_ib_residual_norms" if self.masks is not None else "fo_residual_norms"
        getattr(L, fn + self.suf)(C.byref(self.p), C.byref(self.f), out)
        return np.array(out[:], dtype=np.float64)

    def compute_tau(self):
        getattr(lib(), "fo_compute_tau" + self.suf)(C.byref(self.p), C.byref(self.f))


# ----------------------------------------------------------------------------
# level sets / volume fractions
# ----------------------------------------------------------------------------
def vol_box3(psi8, d3) -> float:
    a = (C.c_double * 8)(*psi8)
    d = (C.c_double * 3)(*d3)
    return lib().fo_vol_box3(a, d)


def vol_box2(psi4, d2) -> float:
    a = (C.c_double * 4)(*psi4)
    d = (C.c_double * 2)(*d2)
    return lib().fo_vol_box2(a, d)


def volfrac3d(n, dx, psi):
    """omega_from_psi! 3D: returns dict of the 8 mask components (halo storage)."""
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    out = {c: np.zeros_like(psi) for c in MASK_COMPONENTS}
    ptrs = (C.c_void_p * 8)(*[out[c].ctypes.data for c in MASK_COMPONENTS])
    lib().fo_volfrac3d((C.c_int * 3)(*n), (C.c_double * 3)(*dx), psi.ctypes.data, ptrs)
    return out


def volfrac2d(n, dx, psi):
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    comps = ("cc", "vv", "vc", "cv")
    out = {c: np.zeros_like(psi) for c in comps}
    ptrs = (C.c_void_p * 4)(*[out[c].ctypes.data for c in comps])
    lib().fo_volfrac2d((C.c_int * 2)(*n), (C.c_double * 2)(*dx), psi.ctypes.data, ptrs)
    return out


def levelset_from_dem(n3, o3, dx3, n2, o2, dx2, dem, R=None, cutoff=None):
    """compute_levelset_from_dem! (compute_levelsets.jl:21-25): returns psi (halo storage)."""
    dem = np.ascontiguousarray(dem, dtype=np.float64)
    assert dem.shape == (n2[1] + 3, n2[0] + 3)
    psi = np.zeros((n3[2] + 3, n3[1] + 3, n3[0] + 3), np.float64)
    if cutoff is None:
        cutoff = 4.0 * max(dx3)
    Rp = None
    if R is not None:
        Rarr = np.ascontiguousarray(np.asarray(R, dtype=np.float64).reshape(9))
        Rp = Rarr.ctypes.data
    lib().fo_levelset_from_dem((C.c_int * 3)(*n3), (C.c_double * 3)(*o3), (C.c_double * 3)(*dx3),
                               (C.c_int * 2)(*n2), (C.c_double * 2)(*o2), (C.c_double * 2)(*dx2),
                               dem.ctypes.data, Rp, float(cutoff), psi.ctypes.data)
    return psi


def invert_levelset(n3, psi):
    lib().fo_invert_levelset((C.c_int * 3)(*n3), psi.ctypes.data)
    return psi


# ----------------------------------------------------------------------------
# heat diffusion (src/Models/Diffusion/Heat/), oracle/heat.c
# ----------------------------------------------------------------------------
class _FoHeat(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("dx", C.c_double * 3), ("kind", (C.c_int * 2) * 3),
                ("value", (C.c_double * 2) * 3), ("lam", C.c_double), ("dtau_T", C.c_double),
                ("dtau_q", C.c_double), ("dt", C.c_double)]


class OracleHeat:
    """Heat state on the CPU oracle: halo-storage arrays T, T_o, qx, qy, qz
    ((n2+3, n1+3, n0+3), x fastest); kinds 0 = Value, 1 = Flux per (dim, side)."""

    def __init__(self, n, extent, kinds, values, lam, dtau_T, dtau_q, dtype="f64"):
        self.n = tuple(int(v) for v in n)
        self.np_dtype = np.float64 if dtype == "f64" else np.float32
        self.suf = "_" + dtype
        p = _FoHeat()
        for k in range(3):
            p.n[k] = self.n[k]
            p.dx[k] = extent[k] / self.n[k]
            for s in range(2):
                p.kind[k][s] = int(kinds[k][s])
                p.value[k][s] = float(values[k][s])
        p.lam, p.dtau_T, p.dtau_q = float(lam), float(dtau_T), float(dtau_q)
        self.p = p
        shape = (self.n[2] + 3, self.n[1] + 3, self.n[0] + 3)
        self.a = {k: np.zeros(shape, self.np_dtype) for k in ("T", "T_o", "qx", "qy", "qz")}

    def _slices(self, name):
        ext = list(self.n)
        if name in ("qx", "qy", "qz"):
            ext["xyz".index(name[1])] += 1
        return tuple(slice(1, e + 1) for e in reversed(ext))

    def set_interior(self, name, values):
        self.a[name][self._slices(name)] = values

    def interior(self, name):
        return self.a[name][self._slices(name)].copy()

    def _ptr(self, k):
        return self.a[k].ctypes.data_as(C.c_void_p)

    def apply_bcs(self):
        L = lib()
        getattr(L, "fo_heat_bc_flux" + self.suf)(C.byref(self.p), self._ptr("qx"), self._ptr("qy"), self._ptr("qz"))
        getattr(L, "fo_heat_bc_value" + self.suf)(C.byref(self.p), self._ptr("T"))

    def advance(self, niter, dt):
        self.p.dt = float(dt)
        getattr(lib(), "fo_heat_advance" + self.suf)(C.byref(self.p), self._ptr("T"), self._ptr("T_o"),
                                                     self._ptr("qx"), self._ptr("qy"), self._ptr("qz"), int(niter))
