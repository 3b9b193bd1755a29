"""fi_residual_norms_noalloc: the residual-norm entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc -- a program whose device
memory is owned by another runtime's allocator, services that forbid allocation
after start-up.  Its partial sums
live in a static device array, so it must give the same norms as the model's own
entry point (fi_model_residual_norms), which keeps its partials in a buffer the
model allocated.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import Pair

SLIP = ("slip", (0.0, 0.0, 0.0))
TRAC = ("traction", (0.0, 0.0, 0.0))
NOSL = ("velocity", (0.0, 0.0, 0.0))
PER = ("periodic", ())

STATE = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz")


MASKS = ("ccc", "vvv", "vcc", "cvc", "ccv", "vvc", "vcv", "cvv")


def state_view(fi, model):
    """fi_state_view of the model's current device state (gravity fields and
    immersed-boundary masks included where the model has them)."""
    L = fi._lib
    v = L.fi_state_view()
    nd = model.grid.ndims
    for name in STATE:
        if nd == 2 and name in ("tzz", "txz", "tyz", "Vz"):
            continue
        setattr(v, name, model.device_ptr(name))
    for c, name in enumerate(("gx", "gy", "gz")[:nd]):
        if model._desc.gravity.kind[c] == L.FI_G_FIELD:
            v.g[c] = model.device_ptr(name)
    if model._desc.immersed:
        for c, comp in enumerate(MASKS):
            v.na[c] = model.device_ptr("na_" + comp)
            v.ns[c] = model.device_ptr("ns_" + comp)
    v.pitch = model.layout()[0]
    return v


def noalloc_norms(fi, model, out_dev, stream):
    lib = model.lib
    v = state_view(fi, model)
    fi._lib.check(lib, lib.fi_residual_norms_noalloc(C.byref(model._desc), C.byref(v), C.c_void_p(out_dev.data_ptr()),
                                                     C.c_void_p(stream)))


def compare(a, b):
    # the same kernel over the same block count as the model's entry point: the
    # same bits in every slot (the L2 sums are added in the same order)
    np.testing.assert_array_equal(a, b)


def _sphere_psi(n, dx, c, r):
    """Signed distance to a sphere at the vertices, halo storage (numpy (z, y, x))."""
    ax = [(np.arange(n[d] + 3) - 1) * dx[d] for d in range(3)]
    Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r


def _immersed_pair(seed):
    n, ext = (24, 20, 22), (1.0, 0.8, 0.9)
    dx = tuple(e / c for e, c in zip(ext, n))
    psi_ns = -_sphere_psi(n, dx, (0.5, 0.4, -0.3), 0.75)
    psi_na = _sphere_psi(n, dx, (0.5, 0.4, 0.45), 0.7)
    bcs = ((TRAC, TRAC), (TRAC, TRAC), (TRAC, TRAC))
    return Pair(n, bcs, seed=seed, path="reference", origin=(0.0, 0.0, 0.0), extent=ext,
                immersed_psi={"na": psi_na, "ns": psi_ns})


class _Gravity:
    """The 3D manufactured solution: gravity given as fields (FI_G_FIELD)."""

    def __init__(self, fi):
        self.grid, self.model = fi.scenarios.mms3d_model(20)

    def close(self):
        self.model.close()


CASES = [
    ("3d-fused-f64", (40, 17, 70), ((PER, PER), (PER, PER), (SLIP, TRAC)), "f64"),
    ("3d-fused-f32", (33, 20, 24), ((SLIP, SLIP), (SLIP, SLIP), (NOSL, TRAC)), "f32"),
    ("2d-f64", (45, 31), ((SLIP, SLIP), (NOSL, TRAC)), "f64"),
    ("3d-immersed-f64", None, None, "f64"),
    ("3d-gravity-field-f64", None, None, "f64"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,bcs,dtype", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_model_norms_twice(fi, name, n, bcs, dtype):
    import torch
    if name == "3d-immersed-f64":
        p = _immersed_pair(21)
    elif name == "3d-gravity-field-f64":
        p = _Gravity(fi)
    else:
        p = Pair(n, bcs, dtype=dtype, seed=21)
    m = p.model
    out = torch.empty(fi._lib.FI_NORMS_LEN, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row: the shared scratch keeps the last call's contents
        m.advance(3)
        m.synchronize()
        expect = m.residual_norms()
        out.fill_(-1.0)
        noalloc_norms(fi, m, out, stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        compare(got, expect)
        assert got[11] == 0.0
    p.close()


def test_noalloc_rejects_incomplete_views(fi):
    # argument checks come before any device work: runs without a GPU
    L = fi._lib
    lib = fi.load_library()
    d = L.fi_model_desc()
    d.grid.nd = 3
    for k in range(3):
        d.grid.n[k] = 600
        d.grid.extent[k] = 1.0
    d.dtype = L.FI_F64
    v = L.fi_state_view()
    for name in STATE[:-1]:
        setattr(v, name, 0x1000)  # never dereferenced: Vz is missing
    v.pitch = 640
    assert lib.fi_residual_norms_noalloc(C.byref(d), C.byref(v), C.c_void_p(0x2000), None) == L.FI_ERR_ARG
    assert b"missing state field" in lib.fi_last_error()
    v.Vz = 0x1000
    v.pitch = 500  # smaller than n0 + 3
    assert lib.fi_residual_norms_noalloc(C.byref(d), C.byref(v), C.c_void_p(0x2000), None) == L.FI_ERR_ARG
    assert b"pitch" in lib.fi_last_error()
    v.pitch = 640
    d.immersed = 1  # masks missing
    assert lib.fi_residual_norms_noalloc(C.byref(d), C.byref(v), C.c_void_p(0x2000), None) == L.FI_ERR_ARG
    assert b"mask" in lib.fi_last_error()
