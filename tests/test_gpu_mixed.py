"""Mixed-precision refinement (FP32 PT sweeps inside an FP64 defect correction)
reaches the FP64 tolerance and agrees with the plain FP64 solve, on the 3D
manufactured solution of stokes_manufactured_solution_free_slip_3D.jl."""
import math

import numpy as np
import pytest

from conftest import load_fastice
from helpers import mms3d_error, mms3d_model

pytestmark = pytest.mark.gpu


def test_mixed_reaches_fp64_tolerance_and_matches_plain():
    fi = load_fastice()
    n = 24
    kw = dict(max_iter=200 * n, ncheck=n, tol=1e-8)
    grid, plain = mms3d_model(fi, n)
    rp = plain.solve(**kw)
    _, mixed = mms3d_model(fi, n)
    rm = mixed.solve(mode="mixed", **kw)
    assert rp["converged"] and rm["converged"], (rp, rm)
    assert rm["measure"] < 1e-8 and rm["outer"] >= 1
    for name in ("Vx", "Vy", "Vz", "txx", "txy"):
        a, b = mixed.get_field(name), plain.get_field(name)
        rel = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert rel < 1e-7, (name, rel)
    # the exact pressure is zero and the free-slip box fixes it only up to a
    # constant: compare the mean-free parts on the deviatoric stress scale
    a, b = mixed.get_field("P"), plain.get_field("P")
    scale = np.max(np.abs(plain.get_field("txx")))
    assert np.max(np.abs((a - a.mean()) - (b - b.mean()))) < 1e-7 * scale
    # both carry the same discretisation error against the manufactured solution
    ep, em = mms3d_error(fi, grid, plain), mms3d_error(fi, grid, mixed)
    assert abs(ep - em) < 1e-6 * ep and ep < 1e-2
    plain.close()
    mixed.close()


def test_fp32_alone_stalls_above_fp64_tolerance():
    fi = load_fastice()
    n = 24
    _, m = mms3d_model(fi, n, dtype="f32")
    r = m.solve(max_iter=100 * n, ncheck=n, tol=1e-8)
    assert not r["converged"] and r["measure"] > 1e-7
    m.close()


def test_mixed_rejects_fp32_model():
    fi = load_fastice()
    _, m = mms3d_model(fi, 12, dtype="f32")
    with pytest.raises(fi.FastIceError):
        m.solve(mode="mixed", max_iter=100, ncheck=10, tol=1e-8)
    m.close()


def test_mixed_glacier_matches_fp64_solve():
    # the immersed-boundary glacier (seeded 64-bump bed, sinusoidal surface):
    # FP32 correction sweeps on volume fractions rounded so that every emptiness
    # test agrees with FP64, masked stress projection, FP64 residuals
    from fastice_b200 import scenarios
    fi = load_fastice()
    n = 24
    kw = dict(max_iter=400 * n, ncheck=n, tol=1e-8, measure="rel_slab", rho_g_inf=1.0, length_z=0.6)
    plain, _ = scenarios.bed_model(0, n)
    rp = plain.solve(**kw)
    mixed, _ = scenarios.bed_model(0, n)
    # a first, short mixed solve ends inside the FP32 full-problem phase; the
    # second solve (from the reset state) must still force its corrections with
    # the FP64 residual, not with the full problem's body force
    mixed.solve(mode="mixed", **dict(kw, max_iter=2 * n, tol=1e-30))
    for f in ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz"):
        mixed.set_field(f, 0.0)
    mixed.set_field("eta", 1.0)
    mixed.set_field("eta_next", 1.0)
    mixed.apply_bcs()
    rm = mixed.solve(mode="mixed", **kw)
    assert rp["converged"] and rm["converged"], (rp, rm)
    assert rm["measure"] < 1e-8 and rm["outer"] >= 1
    vmax = max(np.max(np.abs(plain.get_field(c))) for c in ("Vx", "Vy", "Vz"))
    for name in ("Vx", "Vy", "Vz"):
        d = np.max(np.abs(mixed.get_field(name) - plain.get_field(name))) / vmax
        assert d < 1e-6, (name, d)
    plain.close()
    mixed.close()


def test_glen_glacier_continuation_plain_and_mixed():
    # Glen's law on the glacier by continuation (linear, then the viscosity cap raised
    # 10 -> 100 -> 1000 -> 5000): both the plain FP64 and the mixed-precision solve
    # reach the relative residual 1e-8 and agree
    fi = load_fastice()
    from fastice_b200 import scenarios
    n = 47
    out = {}
    for mode in ("plain", "mixed"):
        m, _ = scenarios.bed_model(0, n, rheology=fi.glen_regularised())
        m.set_field("eta", 1.0)
        m.set_field("eta_next", 1.0)
        m.apply_bcs()
        stages = scenarios.glacier_glen_stages(m.grid, tol=1e-8)
        r = m.solve_continuation(stages, mode=mode, max_iter=2000 * n, ncheck=n, measure="rel_slab", rho_g_inf=1.0,
                                 length_z=0.6)
        assert r["converged"] and r["measure"] < 1e-8, (mode, r)
        assert len(r["stages"]) == 5
        out[mode] = [m.get_field(c) for c in ("Vx", "Vy", "Vz")]
        eta = m.get_field("eta")
        assert eta.max() <= 5000.0 and eta.min() > 0.0
        m.close()
    vmax = max(np.max(np.abs(v)) for v in out["plain"])
    dv = max(np.max(np.abs(a - b)) for a, b in zip(out["mixed"], out["plain"]))
    assert dv <= 1e-6 * vmax, dv / vmax
