"""GPU parity for the 2D manufactured solution (128^2 unit square), the immersed-boundary
model, and the level-set / volume-fraction set-up kernels, against the oracle."""
import math

import numpy as np
import pytest

from conftest import load_fastice, load_oracle
from helpers import Pair, mms2d_exact, mms2d_gravity

pytestmark = pytest.mark.gpu


def mms2d_model(fi, n, library="fast", dtype="f64"):
    grid = fi.UniformGrid(origin=(0.0, 0.0), extent=(1.0, 1.0), dims=(n, n))
    slip = fi.SBC(0.0, 0.0)
    m = fi.IsothermalFullStokesModel(grid=grid, boundary_conditions={"x": (slip, slip), "y": (slip, slip)},
                                     gravity=mms2d_gravity(fi, grid), rheology=fi.LinearViscousRheology(1.0),
                                     solver_params=fi.pt_params(grid), dtype=dtype, library=library)
    m.set_field("eta", 1.0)
    m.set_field("eta_next", 1.0)
    m.apply_bcs()
    return grid, m


def mms2d_oracle(fi, O, grid, gravity):
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


def test_mms2d_128_bit_level_after_1000_iterations():
    # 128^2 unit square, free slip, manufactured forcing; strict build vs oracle, bit for bit
    fi, O = load_fastice(), load_oracle()
    grid, m = mms2d_model(fi, 128, library="strict")
    o = mms2d_oracle(fi, O, grid, mms2d_gravity(fi, grid))
    m.advance(1000)
    o.advance(1000)
    for name in ("P", "txx", "tyy", "txy", "Vx", "Vy"):
        a, b = m.get_field(name), o.interior(name)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name
    m.close()


def test_mms2d_converges_second_order():
    # the 2D manufactured solution solved to ||R||inf < 1e-8 on the GPU; L2 error vs the analytic field converges at O(h^2)
    fi = load_fastice()
    errs = []
    for n in (32, 64, 128):
        grid, m = mms2d_model(fi, n)
        rep = m.solve(max_iter=200 * n, ncheck=n, tol=1e-8)
        assert rep["converged"], rep
        ex, ey = mms2d_exact(grid)
        vx, vy = m.get_field("Vx"), m.get_field("Vy")
        err = math.sqrt((np.sum((vx - ex) ** 2) + np.sum((vy - ey) ** 2)) / (np.sum(ex ** 2) + np.sum(ey ** 2)))
        errs.append(err)
        m.close()
    orders = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(1.9 < o < 2.1 for o in orders), (errs, orders)


def _sphere_psi(n, dx, center, radius, noise=0.0, seed=0):
    rng = np.random.default_rng(seed)
    sh = (n[2] + 3, n[1] + 3, n[0] + 3)
    k, j, i = np.meshgrid(np.arange(sh[0]), np.arange(sh[1]), np.arange(sh[2]), indexing="ij")
    x, y, z = (i - 1) * dx[0], (j - 1) * dx[1], (k - 1) * dx[2]
    psi = np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2) - radius
    return psi + noise * rng.standard_normal(sh)


@pytest.mark.parametrize("library", ["strict", "fast"])
def test_volfrac3d_vs_oracle(library):
    fi, O = load_fastice(), load_oracle()
    n, ext = (21, 17, 13), (1.0, 0.8, 0.6)
    dx = tuple(e / c for e, c in zip(ext, n))
    psi = _sphere_psi(n, dx, (0.5, 0.4, 0.3), 0.27, noise=0.01)
    grid = fi.UniformGrid(origin=(0, 0, 0), extent=ext, dims=n)
    got = fi.omega_from_psi(grid, psi, library=library)
    exp = O.volfrac3d(n, dx, psi)
    for c in exp:
        sl = (slice(1, n[2] + 2), slice(1, n[1] + 2), slice(1, n[0] + 2))
        a, b = got[c][sl], exp[c][sl]
        if library == "strict":
            assert np.array_equal(a, b), c
        else:
            assert np.max(np.abs(a - b)) < 1e-12, c
    # the cut-cell fractions are fractions
    assert all(np.all((got[c] >= -1e-12) & (got[c] <= 1 + 1e-12)) for c in got)


def test_volfrac2d_vs_oracle():
    fi, O = load_fastice(), load_oracle()
    n, ext = (40, 27), (1.0, 0.7)
    dx = (ext[0] / n[0], ext[1] / n[1])
    j, i = np.meshgrid(np.arange(n[1] + 3), np.arange(n[0] + 3), indexing="ij")
    psi = np.sqrt(((i - 1) * dx[0] - 0.45) ** 2 + ((j - 1) * dx[1] - 0.3) ** 2) - 0.2
    grid = fi.UniformGrid(origin=(0, 0), extent=ext, dims=n)
    got = fi.omega_from_psi(grid, psi, library="strict")
    exp = O.volfrac2d(n, dx, psi)
    for c in exp:
        sl = (slice(1, n[1] + 2), slice(1, n[0] + 2))
        assert np.array_equal(got[c][sl], exp[c][sl]), c


@pytest.mark.parametrize("invert", [False, True])
def test_levelset_from_dem_vs_oracle(invert):
    fi, O = load_fastice(), load_oracle()
    n3, ext3, o3 = (24, 20, 16), (1.0, 1.0, 0.6), (0.0, 0.0, 0.0)
    n2, ext2, o2 = (40, 40), (1.2, 1.2), (-0.1, -0.1)
    g3 = fi.UniformGrid(origin=o3, extent=ext3, dims=n3)
    g2 = fi.UniformGrid(origin=o2, extent=ext2, dims=n2)
    bed = fi.FunctionField(lambda x, y: 0.2 + 0.08 * np.sin(6 * x) * np.cos(5 * y), g2, fi.Vertex())
    got = fi.compute_levelset_from_dem(g3, g2, bed, invert=invert, library="strict")
    dx3 = tuple(e / c for e, c in zip(ext3, n3))
    dx2 = tuple(e / c for e, c in zip(ext2, n2))
    exp = O.levelset_from_dem(n3, o3, dx3, n2, o2, dx2, bed.sample())
    if invert:
        exp = O.invert_levelset(n3, exp)
    assert np.array_equal(got, exp)


def test_immersed_boundary_bitwise_strict():
    fi, O = load_fastice(), load_oracle()
    n = (20, 14, 18)
    ext = (1.0 + 0.0, 1.25, 1.5)
    dx = tuple(e / c for e, c in zip(ext, n))
    # ns: solid below a sphere-shaped bed bump (psi < 0 inside), na: ice inside a box-like blob
    psi_ns = -_sphere_psi(n, dx, (0.5, 0.6, -0.3), 0.75)
    psi_na = _sphere_psi(n, dx, (0.5, 0.6, 0.5), 0.8)
    trac = ("traction", (0.0, 0.0, 0.0))
    bcs = ((trac, trac), (trac, trac), (trac, trac))
    p = Pair(n, bcs, path="reference", library="strict", seed=31, origin=(0.0, 0.0, 0.0), extent=ext,
             immersed_psi={"na": psi_na, "ns": psi_ns})
    p.advance(4)
    bad = p.bitwise_equal()
    a = p.model.residual_norms()
    b = p.oracle.residual_norms()
    p.close()
    assert not bad, bad
    np.testing.assert_array_equal(a[[0, 1, 2, 3]], b[[0, 1, 2, 3]])


def test_immersed_boundary_activity_follows_new_volume_fractions():
    # the kernels read per-index activity bytes computed from the volume
    # fractions; recomputing the fractions between iterations (ω_from_ψ! on a
    # moved bed) must be seen by the next iteration, bit for bit with the oracle
    fi, O = load_fastice(), load_oracle()
    n = (20, 14, 18)
    ext = (1.0, 1.25, 1.5)
    dx = tuple(e / c for e, c in zip(ext, n))
    psi_ns = -_sphere_psi(n, dx, (0.5, 0.6, -0.3), 0.75)
    psi_na = _sphere_psi(n, dx, (0.5, 0.6, 0.5), 0.8)
    trac = ("traction", (0.0, 0.0, 0.0))
    bcs = ((trac, trac), (trac, trac), (trac, trac))
    p = Pair(n, bcs, path="reference", library="strict", seed=32, origin=(0.0, 0.0, 0.0), extent=ext,
             immersed_psi={"na": psi_na, "ns": psi_ns})
    p.advance(2)
    moved = -_sphere_psi(n, dx, (0.45, 0.55, -0.2), 0.8)
    p.model.omega_from_psi("ns", moved)
    new = O.volfrac3d(n, dx, moved)
    for k, c in enumerate(O.MASK_COMPONENTS):
        p.oracle.masks["ns"][k][...] = new[c]
    p.advance(3)
    bad = p.bitwise_equal()
    a = p.model.residual_norms()
    b = p.oracle.residual_norms()
    p.close()
    assert not bad, bad
    np.testing.assert_array_equal(a[[0, 1, 2, 3]], b[[0, 1, 2, 3]])


# power laws regularised at η = 1, so that the time steps of a unit viscosity stay stable
@pytest.mark.parametrize("rheo", [{"kind": "linear", "eta": 1.0}, {"kind": "glen", "eta_reg": 1.0},
                                  {"kind": "relax_glen", "eta_reg": 1.0}],
                         ids=["linear", "glen", "relaxed_glen"])
def test_immersed_boundary_zero_stores_skipped_after_full_iterations(rheo):
    # after two full iterations the immersed-boundary updates stop rewriting the
    # zeros of inactive strict-interior points and run only the listed blocks;
    # state written from outside (here random values everywhere, inactive points
    # included) must be zeroed again, boundary values (non-zero velocities and
    # tractions) must not leak into skipped points, and the viscosity next to the
    # ice (power law) or everywhere (relaxation) must keep moving -- bit for bit
    # with the oracle, across single iterations and replayed iteration pairs
    fi, O = load_fastice(), load_oracle()
    n = (20, 14, 18)
    ext = (1.0, 1.25, 1.5)
    dx = tuple(e / c for e, c in zip(ext, n))
    psi_ns = -_sphere_psi(n, dx, (0.5, 0.6, -0.3), 0.75)
    psi_na = _sphere_psi(n, dx, (0.5, 0.6, 0.5), 0.8)
    bcs = ((("velocity", (0.1, -0.2, 0.05)), ("traction", (0.3, 0.0, -0.1))),
           (("slip", (0.0, 0.2, 0.0)), ("traction", (0.0, 0.0, 0.0))),
           (("velocity", (0.0, 0.1, 0.0)), ("traction", (0.0, 0.2, 0.1))))
    p = Pair(n, bcs, rheo=rheo, path="reference", library="strict", seed=33, origin=(0.0, 0.0, 0.0), extent=ext,
             immersed_psi={"na": psi_na, "ns": psi_ns})
    p.advance(11)
    bad = p.bitwise_equal()
    assert not bad, bad
    rng = np.random.default_rng(5)
    for name in ("P", "txy", "Vz", "eta"):
        vals = rng.standard_normal(p.model.field_shape(name))
        if name == "eta":
            vals = 0.5 + np.abs(vals)
        p.model.set_field(name, vals)
        p.oracle.set_interior(name, vals)
    p.advance(1)
    p.advance(9)
    bad = p.bitwise_equal()
    finite = all(np.isfinite(p.oracle.interior(name)).all() for name in p.state)
    a = p.model.residual_norms()
    b = p.oracle.residual_norms()
    p.close()
    assert finite
    assert not bad, bad
    np.testing.assert_array_equal(a[[0, 1, 2, 3]], b[[0, 1, 2, 3]])


def test_immersed_boundary_f32_two_points_per_thread():
    # FP32 threads of the immersed-boundary sweeps own two points 32 apart in x.
    # A row of 71 vertex positions fills one 64-wide block and part of a second,
    # so threads with both points in the row and threads whose second point lies
    # past the row's end both occur; bit for bit with the oracle in FP32, through
    # full iterations and the steady state (zeros not stored, block list)
    fi, O = load_fastice(), load_oracle()
    n = (70, 12, 14)
    ext = (1.0, 0.5, 0.6)
    dx = tuple(e / c for e, c in zip(ext, n))
    psi_ns = -_sphere_psi(n, dx, (0.5, 0.25, -0.2), 0.45)
    psi_na = _sphere_psi(n, dx, (0.5, 0.25, 0.3), 0.45)
    trac = ("traction", (0.0, 0.0, 0.0))
    bcs = ((("velocity", (0.1, 0.0, 0.0)), trac), (trac, trac), (("slip", (0.0, 0.0, 0.0)), trac))
    p = Pair(n, bcs, path="reference", library="strict", dtype="f32", seed=34, origin=(0.0, 0.0, 0.0), extent=ext,
             immersed_psi={"na": psi_na, "ns": psi_ns})
    # (an FP32 model rounds its FP64 volume fractions once, as the oracle does)
    p.advance(3)
    bad = p.bitwise_equal()
    assert not bad, bad
    p.advance(10)
    bad = p.bitwise_equal()
    finite = all(np.isfinite(p.oracle.interior(name)).all() for name in p.state)
    a = p.model.residual_norms()
    b = p.oracle.residual_norms()
    p.close()
    assert finite
    assert not bad, bad
    np.testing.assert_array_equal(a[[0, 1, 2, 3]], b[[0, 1, 2, 3]])


def test_model_omega_from_psi_matches_standalone():
    fi = load_fastice()
    n, ext = (16, 12, 10), (1.0, 0.75, 0.6)
    dx = tuple(e / c for e, c in zip(ext, n))
    psi = _sphere_psi(n, dx, (0.5, 0.4, 0.3), 0.3)
    grid = fi.UniformGrid(origin=(0, 0, 0), extent=ext, dims=n)
    slip = fi.SBC(0.0, 0.0, 0.0)
    m = fi.IsothermalImmersedBoundaryFullStokesModel(
        grid=grid, boundary_conditions={"x": (slip, slip), "y": (slip, slip), "z": (slip, slip)},
        gravity={"x": 0.0, "y": 0.0, "z": 1.0}, rheology=fi.LinearViscousRheology(1.0),
        solver_params=fi.pt_params(grid), dtype="f64")
    m.omega_from_psi("na", psi)
    ref = fi.omega_from_psi(grid, psi)
    for c in ("ccc", "vcc", "cvv"):
        np.testing.assert_array_equal(m.get_field("na_" + c), ref[c][tuple(slice(1, s + 1) for s in m.field_shape("na_" + c))])
    m.close()


def test_checkpoint_resumes_the_solve_bit_for_bit(tmp_path):
    # run, checkpoint, run on; a fresh model loaded from the checkpoint runs the
    # same iterations to the same bits (the dumps hold the interiors; the ghosts
    # follow from them through the boundary conditions)
    fi = load_fastice()
    per = ("periodic", ())
    bcs = ((per, per), (per, per), (("slip", (0.0, 0.0, 0.0)), ("traction", (0.0, 0.0, 0.0))))
    a = Pair((40, 24, 20), bcs, path="fused", library="strict", seed=21, rheo={"kind": "glen"})
    a.model.advance(5)
    fi.writers.save_checkpoint(a.model, str(tmp_path / "ck"))
    a.model.advance(7)
    b = Pair((40, 24, 20), bcs, path="fused", library="strict", seed=99, rheo={"kind": "glen"})
    fi.writers.load_checkpoint(b.model, str(tmp_path / "ck"))
    b.model.advance(7)
    for name in ("P", "txx", "txz", "Vx", "Vz", "eta"):
        x, y = a.model.get_field(name), b.model.get_field(name)
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), name
    a.close()
    b.close()
