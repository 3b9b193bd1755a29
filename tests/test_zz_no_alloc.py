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


def state_view(fi, model):
    """fi_state_view of the model's current device state."""
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
    v.pitch = model.layout()[0]
    return v


def noalloc_norms(fi, model, out_dev, stream):
    lib = model.lib
    v = state_view(fi, model)
    fi._lib.check(lib, lib.fi_residual_norms_noalloc(C.byref(model._desc), C.byref(v), C.c_void_p(out_dev.data_ptr()),
                                                     C.c_void_p(stream)))


def compare(a, b):
    # max-norms and max|V| are order independent; the L2 sums are added in a different block order
    np.testing.assert_array_equal(a[[0, 1, 2, 3, 8, 9, 10, 11]], b[[0, 1, 2, 3, 8, 9, 10, 11]])
    np.testing.assert_allclose(a[4:8], b[4:8], rtol=1e-12, atol=0.0)


CASES = [
    ("3d-fused-f64", (40, 17, 70), ((PER, PER), (PER, PER), (SLIP, TRAC)), "f64"),
    ("3d-fused-f32", (33, 20, 24), ((SLIP, SLIP), (SLIP, SLIP), (NOSL, TRAC)), "f32"),
    ("2d-f64", (45, 31), ((SLIP, SLIP), (NOSL, TRAC)), "f64"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,bcs,dtype", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_model_norms_twice(fi, name, n, bcs, dtype):
    import torch
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


def test_noalloc_rejects_grids_beyond_its_scratch(fi):
    # checked before any device work: runs without a GPU
    L = fi._lib
    lib = fi.load_library()
    d = L.fi_model_desc()
    d.grid.nd = 3
    for k in range(3):
        d.grid.n[k] = 600
        d.grid.extent[k] = 1.0
    d.dtype = L.FI_F64
    v = L.fi_state_view()
    for name in STATE:
        setattr(v, name, 0x1000)  # never dereferenced: the size check comes first
    v.pitch = 640
    st = lib.fi_residual_norms_noalloc(C.byref(d), C.byref(v), C.c_void_p(0x2000), None)
    assert st == L.FI_ERR_ARG
    assert b"too large" in lib.fi_last_error()
