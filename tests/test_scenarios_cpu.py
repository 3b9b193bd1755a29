"""The seeded synthetic inputs the benchmarks and GPU tests use (no GPU needed):
the pure-shear inclusion instances of the batched and serving workloads and the
64-bump glacier bed, checked against the distributions they are specified with."""
import math

import numpy as np
import pytest

from conftest import load_fastice


def scen():
    return load_fastice().scenarios


def test_inclusion_params_follow_their_distributions():
    s = scen()
    sizes = set()
    for seed in range(256):
        p = s.inclusion_params(seed)
        nx, ny = p["n"]
        assert 63 <= nx <= 511 and 63 <= ny <= 511
        sizes.add((nx, ny))
        assert 1 <= len(p["circles"]) <= 16
        for cx, cy, r, eta in p["circles"]:
            assert 0.0 <= cx < 1.0 and 0.0 <= cy < 1.0
            assert 0.02 <= r < 0.15
            assert 1e-4 * (1 - 1e-12) <= eta <= 1e4 * (1 + 1e-12)
        assert s.inclusion_params(seed) == p  # seeded: the same instance every time
    # x and y sizes are drawn independently
    assert any(nx != ny for nx, ny in sizes)
    assert len(sizes) > 200


def test_inclusion_viscosity_marks_each_circle():
    s = scen()
    n = (64, 48)
    eta = s.inclusion_viscosity(n, [(0.5, 0.5, 0.2, 10.0), (0.25, 0.25, 0.05, 0.1)])
    assert eta.shape == (48, 64)
    xc = (np.arange(64) + 0.5) / 64
    yc = (np.arange(48) + 0.5) / 48
    Y, X = np.meshgrid(yc, xc, indexing="ij")
    in1 = (X - 0.5) ** 2 + (Y - 0.5) ** 2 <= 0.04
    in2 = (X - 0.25) ** 2 + (Y - 0.25) ** 2 <= 0.0025
    assert np.all(eta[in2] == 0.1)  # the later circle is drawn over the earlier one
    assert np.all(eta[in1 & ~in2] == 10.0)
    assert np.all(eta[~in1 & ~in2] == 1.0)


def test_smooth_log_keeps_constants_and_bounds():
    s = scen()
    flat = np.full((20, 30), 7.0)
    np.testing.assert_allclose(s.smooth_log(flat, 4), flat, rtol=1e-14)
    eta = s.inclusion_viscosity((40, 40), [(0.5, 0.5, 0.25, 1e4)])
    sm = s.smooth_log(eta, 4)
    assert sm.min() >= 1.0 * (1 - 1e-12) and sm.max() <= 1e4 * (1 + 1e-12)
    assert s.stiffness_ratio(sm) < s.stiffness_ratio(eta)
    assert s.stiffness_ratio(flat) == 1.0


def test_bed_params_follow_their_distributions():
    s = scen()
    p = s.bed_params(0, 383)
    assert p["a"].shape == (64,) and p["w"].shape == (64,) and p["c"].shape == (64, 2)
    assert np.all((p["a"] >= 0.0) & (p["a"] < 0.2))
    assert np.all((p["w"] >= 0.05) & (p["w"] < 0.2))
    assert np.all((p["c"] >= 0.0) & (p["c"] < 1.0))
    q = s.bed_params(0, 383)
    for k in ("a", "w", "c"):
        np.testing.assert_array_equal(p[k], q[k])
    assert not np.array_equal(s.bed_params(1, 383)["a"], p["a"])


def test_bed_height_is_a_sum_of_gaussian_bumps():
    s = scen()
    prm = {"a": np.array([0.15]), "w": np.array([0.1]), "c": np.array([[0.3, 0.6]])}
    assert math.isclose(float(s.bed_height(prm, 0.3, 0.6)), 0.15, rel_tol=1e-15)
    assert math.isclose(float(s.bed_height(prm, 0.4, 0.6)), 0.15 / math.e, rel_tol=1e-14)
    two = {"a": np.array([0.1, 0.05]), "w": np.array([0.1, 0.2]), "c": np.array([[0.2, 0.2], [0.7, 0.7]])}
    x = np.linspace(0, 1, 11)
    X, Y = np.meshgrid(x, x, indexing="ij")
    one_a = {k: v[:1] for k, v in two.items()}
    one_b = {k: v[1:] for k, v in two.items()}
    np.testing.assert_allclose(s.bed_height(two, X, Y), s.bed_height(one_a, X, Y) + s.bed_height(one_b, X, Y),
                               rtol=1e-15)


def test_eta_rel_is_ignored_unless_asked_for():
    # drivers pass η_rel in solver_params; the reference's kernels never read it
    fi = load_fastice()
    from fastice_b200 import models
    g = fi.UniformGrid(origin=(0.0, 0.0), extent=(1.0, 1.0), dims=(8, 8))
    sp = fi.pt_params(g, eta_rel=0.1)
    assert sp["η_rel"] == 0.1
    glen = fi.glen_regularised()
    assert models.effective_rheology(glen, sp) is glen
    r = models.effective_rheology(glen, sp, "log")
    assert isinstance(r, fi.Relaxation) and r.rate == 0.1 and r.scale == "log" and r.target is glen
    assert models.effective_rheology(glen, sp, "lin").scale is None
    assert models.effective_rheology(glen, fi.pt_params(g), "log") is glen  # no rate given: nothing to honour
    with pytest.raises(ValueError):
        models.effective_rheology(fi.Relaxation(glen, 0.2), sp, "log")
