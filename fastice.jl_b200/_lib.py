"""ctypes binding of libfastice_b200 (include/fastice_b200.h).

The shared library is built in-tree (``make -C fastice.jl_b200``).  Loading fails
loudly when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAMES = {"fast": "libfastice_b200.so", "strict": "libfastice_b200_strict.so"}

FI_OK, FI_ERR_ARG, FI_ERR_OOM, FI_ERR_DIVERGED, FI_ERR_TIMEOUT, FI_ERR_CUDA, FI_ERR_UNSUPPORTED, FI_ERR_STATE = range(8)
FI_F64, FI_F32 = 0, 1
FI_BC_SLIP, FI_BC_TRACTION, FI_BC_VELOCITY, FI_BC_PERIODIC, FI_BC_HALO = 0, 1, 2, 3, 4
FI_RHEO_LINEAR, FI_RHEO_POWER = 0, 1
FI_RELAX_NONE, FI_RELAX_LIN, FI_RELAX_LOG, FI_RELAX_LOG10 = 0, 1, 2, 3
FI_G_VALUE, FI_G_FIELD = 0, 1
FI_PATH_AUTO, FI_PATH_REFERENCE, FI_PATH_FUSED = 0, 1, 2
FI_CONV_ABS_INF, FI_CONV_REL_SLAB = 0, 1
FI_SOLVE_PLAIN, FI_SOLVE_MIXED = 0, 1
FI_NORMS_LEN = 12
FI_HALO_ITERATION, FI_HALO_STATE = 0, 1
FI_HEAT_VALUE, FI_HEAT_FLUX = 0, 1
FI_HEAT_FIELDS = {"T": 0, "T_o": 1, "qx": 2, "qy": 3, "qz": 4}

FIELD_NAMES = (
    "P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta", "eta_next",
    "rP", "rVx", "rVy", "rVz", "gx", "gy", "gz", "eta_lin", "A",
    "na_ccc", "na_vvv", "na_vcc", "na_cvc", "na_ccv", "na_vvc", "na_vcv", "na_cvv",
    "ns_ccc", "ns_vvv", "ns_vcc", "ns_cvc", "ns_ccv", "ns_vvc", "ns_vcv", "ns_cvv",
)
FIELD_ID = {n: i for i, n in enumerate(FIELD_NAMES)}

# staggered locations (0 = Center, 1 = Vertex) per dim, matching the library
FIELD_LOC = {
    "P": (0, 0, 0), "txx": (0, 0, 0), "tyy": (0, 0, 0), "tzz": (0, 0, 0),
    "txy": (1, 1, 0), "txz": (1, 0, 1), "tyz": (0, 1, 1),
    "Vx": (1, 0, 0), "Vy": (0, 1, 0), "Vz": (0, 0, 1), "eta": (0, 0, 0), "eta_next": (0, 0, 0),
    "rP": (0, 0, 0), "rVx": (1, 0, 0), "rVy": (0, 1, 0), "rVz": (0, 0, 1),
    "gx": (1, 0, 0), "gy": (0, 1, 0), "gz": (0, 0, 1), "eta_lin": (0, 0, 0), "A": (0, 0, 0),
}
for _g in ("na", "ns"):
    for _c, _l in zip(("ccc", "vvv", "vcc", "cvc", "ccv", "vvc", "vcv", "cvv"),
                      ((0, 0, 0), (1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1))):
        FIELD_LOC[f"{_g}_{_c}"] = _l


class fi_bc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("c", C.c_double * 3)]


class fi_grid(C.Structure):
    _fields_ = [("nd", C.c_int32), ("n", C.c_int32 * 3), ("origin", C.c_double * 3), ("extent", C.c_double * 3)]


class fi_rheology(C.Structure):
    _fields_ = [("inner", C.c_int32), ("eta_is_field", C.c_int32), ("eta", C.c_double),
                ("A_is_field", C.c_int32), ("A", C.c_double), ("n", C.c_int32), ("has_reg", C.c_int32),
                ("eta_reg", C.c_double), ("relax", C.c_int32), ("rate", C.c_double)]


class fi_gravity(C.Structure):
    _fields_ = [("kind", C.c_int32 * 3), ("value", C.c_double * 3)]


class fi_pt_params(C.Structure):
    _fields_ = [("dt_P", C.c_double), ("dt_tau", C.c_double * 6), ("dt_V", C.c_double * 3)]


class fi_model_desc(C.Structure):
    _fields_ = [("grid", fi_grid), ("bc", (fi_bc * 2) * 3), ("gravity", fi_gravity), ("rheology", fi_rheology),
                ("dtau", fi_pt_params), ("dtype", C.c_int32), ("immersed", C.c_int32), ("path", C.c_int32),
                ("device", C.c_int32)]


class fi_solve_opts(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("ncheck", C.c_int32), ("tol", C.c_double), ("measure", C.c_int32),
                ("rho_g_inf", C.c_double), ("length_z", C.c_double), ("mode", C.c_int32),
                ("inner_iter", C.c_int32), ("inner_reduction", C.c_double)]


class fi_solve_report(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("outer", C.c_int32), ("measure", C.c_double),
                ("norms", C.c_double * FI_NORMS_LEN), ("seconds", C.c_double), ("converged", C.c_int32)]


class fi_state_view(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz")] + [
        ("g", C.c_void_p * 3), ("na", C.c_void_p * 8), ("ns", C.c_void_p * 8), ("pitch", C.c_size_t)]


class fi_batch_opts(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("ncheck", C.c_int32), ("tol", C.c_double), ("use_graph", C.c_int32),
                ("window", C.c_int32)]


class fi_batch_item(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32), ("measure", C.c_double)]


FI_ITEM_STATUS = {0: "active", 1: "converged", 2: "stalled", 3: "diverged", 4: "max_iter"}


class FastIceError(RuntimeError):
    """Raised for a non-FI_OK status; ``status`` holds the fi_status code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"fastice_b200 status {status}: {msg}")
        self.status = status


class fi_heat_desc(C.Structure):
    _fields_ = [("grid", fi_grid), ("kind", (C.c_int32 * 2) * 3), ("value", (C.c_double * 2) * 3),
                ("lambda_rhocp", C.c_double), ("dtau_T", C.c_double), ("dtau_q", C.c_double),
                ("dtype", C.c_int32), ("device", C.c_int32)]


# (name, restype, argtypes) of every exported entry point declared in include/fastice_b200.h
SIGNATURES = [
    ("fi_last_error", C.c_char_p, []),
    ("fi_abi_version", C.c_int, []),
    ("fi_model_create", C.c_int, [C.POINTER(fi_model_desc), C.POINTER(C.c_void_p)]),
    ("fi_model_destroy", C.c_int, [C.c_void_p]),
    ("fi_model_set_field", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t]),
    ("fi_model_get_field", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t]),
    ("fi_model_copy_field", C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    ("fi_model_set_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fi_model_field_size", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_size_t)]),
    ("fi_model_apply_bcs", C.c_int, [C.c_void_p]),
    ("fi_model_advance", C.c_int, [C.c_void_p, C.c_int32]),
    ("fi_model_compute_residuals", C.c_int, [C.c_void_p]),
    ("fi_model_residual_norms", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("fi_model_compute_tau", C.c_int, [C.c_void_p]),
    ("fi_model_solve", C.c_int, [C.c_void_p, C.POINTER(fi_solve_opts), C.POINTER(fi_solve_report)]),
    ("fi_model_device_ptr", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    ("fi_model_layout", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("fi_model_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("fi_model_synchronize", C.c_int, [C.c_void_p]),
    ("fi_model_path", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("fi_model_volfrac_from_levelset", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    ("fi_levelset_from_dem", C.c_int, [C.POINTER(fi_grid), C.POINTER(fi_grid), C.c_void_p, C.c_void_p, C.c_int32,
                                       C.c_void_p, C.c_int32]),
    ("fi_volfrac", C.c_int, [C.POINTER(fi_grid), C.c_void_p, C.POINTER(C.c_void_p), C.c_int32]),
    ("fi_fused_variant_count", C.c_int, []),
    ("fi_fused_variant_name", C.c_char_p, [C.c_int32]),
    ("fi_model_set_variant", C.c_int, [C.c_void_p, C.c_int32]),
    ("fi_model_autotune", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    ("fi_residual_norms_noalloc", C.c_int, [C.POINTER(fi_model_desc), C.POINTER(fi_state_view), C.c_void_p,
                                            C.c_void_p]),
    ("fi_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]),
    ("fi_batch_destroy", C.c_int, [C.c_void_p]),
    ("fi_batch_add", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fi_batch_remove", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fi_batch_size", C.c_int32, [C.c_void_p]),
    ("fi_batch_step", C.c_int, [C.c_void_p, C.POINTER(fi_batch_opts), C.c_int32, C.POINTER(fi_batch_item),
                                C.POINTER(C.c_int32)]),
    ("fi_batch_advance", C.c_int, [C.c_void_p, C.c_int32]),
    ("fi_batch_solve", C.c_int, [C.c_void_p, C.POINTER(fi_batch_opts), C.POINTER(fi_batch_item),
                                 C.POINTER(C.c_double)]),
    ("fi_batch_measure", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("fi_batch_solve_mixed", C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.POINTER(C.c_double)]),
    ("fi_ib_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]),
    ("fi_ib_batch_destroy", C.c_int, [C.c_void_p]),
    ("fi_ib_batch_add", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fi_ib_batch_remove", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fi_ib_batch_size", C.c_int32, [C.c_void_p]),
    ("fi_ib_batch_advance", C.c_int, [C.c_void_p, C.c_int32]),
    ("fi_ib_batch_synchronize", C.c_int, [C.c_void_p]),
    ("fi_batch_variant_count", C.c_int, []),
    ("fi_batch_variant_name", C.c_char_p, [C.c_int32]),
    ("fi_batch_set_variant", C.c_int, [C.c_void_p, C.c_int32]),
    ("fi_batch_autotune", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    ("fi_heat_create", C.c_int, [C.POINTER(fi_heat_desc), C.POINTER(C.c_void_p)]),
    ("fi_heat_destroy", C.c_int, [C.c_void_p]),
    ("fi_heat_field_size", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_size_t)]),
    ("fi_heat_set_field", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t]),
    ("fi_heat_get_field", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t]),
    ("fi_heat_apply_bcs", C.c_int, [C.c_void_p]),
    ("fi_heat_advance", C.c_int, [C.c_void_p, C.c_int32, C.c_double]),
    ("fi_heat_synchronize", C.c_int, [C.c_void_p]),
    ("fi_heat_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("fi_model_halo_bytes", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_size_t)]),
    ("fi_model_halo_pack", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    ("fi_model_halo_unpack", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    ("fi_model_advance_begin", C.c_int, [C.c_void_p, C.c_int32]),
    ("fi_model_advance_end", C.c_int, [C.c_void_p]),
    ("fi_halo_plan", C.c_int, [C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                               C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)]),
]

_libs = {}


def lib_path(flavor: str = "fast") -> str:
    return os.path.join(HERE, LIB_NAMES[flavor])


def load(flavor: str = "fast"):
    """Load the CUDA library (``fast`` or the no-FMA ``strict`` build)."""
    if flavor in _libs:
        return _libs[flavor]
    path = lib_path(flavor)
    if not os.path.exists(path):
        raise ImportError(f"libfastice_b200 is not built ({path} missing); run `make -C {HERE}` "
                          "-- there is no CPU fallback")
    L = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _libs[flavor] = L
    return L


def check(L, status: int):
    if status != FI_OK:
        raise FastIceError(status, L.fi_last_error().decode(errors="replace"))
