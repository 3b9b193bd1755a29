"""GPU parity: the CUDA library (through the C ABI) against the CPU oracle on the
same seeded inputs.

Tolerances: the no-FMA build (libfastice_b200_strict.so) must match the oracle
bit for bit; the production build (FMA contraction) must match within 1e-10
relative in FP64 (the bar stated for the FP64 path) and 1e-4 relative in FP32,
after a fixed number of iterations.
"""
import numpy as np
import pytest

from helpers import Pair

pytestmark = pytest.mark.gpu

SLIP = ("slip", (0.0, 0.0, 0.0))
TRAC = ("traction", (0.0, 0.0, 0.0))
NOSL = ("velocity", (0.0, 0.0, 0.0))
PER = ("periodic", ())

BC3 = {
    "free_slip_box": ((SLIP, SLIP), (SLIP, SLIP), (SLIP, SLIP)),
    "slab_periodic": ((PER, PER), (PER, PER), (SLIP, TRAC)),
    "noslip_bed_free_top": ((SLIP, SLIP), (SLIP, SLIP), (NOSL, TRAC)),
    "noslip_box": ((NOSL, NOSL), (NOSL, NOSL), (NOSL, NOSL)),
    "mixed_values": ((("traction", (0.1, -0.2, 0.05)), ("traction", (0.0, 0.3, 0.0))), (PER, PER),
                     (("velocity", (0.2, -0.1, 0.0)), ("slip", (0.05, -0.05, 0.0)))),
    "shear_walls": ((("slip", (0.0, 0.0, 0.0)), ("slip", (-0.4, 0.0, 0.0))), (NOSL, ("velocity", (0.3, 0.0, 0.1))),
                    (TRAC, ("slip", (0.0, 0.2, 0.0)))),
    # nonzero wall velocities on every side: ghosts at edges where a later dim's
    # node assignment overrides an earlier dim's mirror image feed unfixed stresses
    "velocity_box": ((("velocity", (0.1, 0.2, 0.3)), ("velocity", (-0.1, 0.05, 0.2))),
                     (("velocity", (0.3, -0.2, 0.1)), ("velocity", (0.0, 0.4, -0.1))),
                     (("velocity", (0.2, 0.1, -0.3)), ("velocity", (0.1, -0.1, 0.25)))),
}
SIZES3 = [(13, 7, 9), (33, 9, 10), (40, 17, 70)]


@pytest.mark.parametrize("bc", list(BC3))
@pytest.mark.parametrize("path", ["reference", "fused"])
def test_3d_bitwise_strict(bc, path):
    p = Pair((13, 7, 9), BC3[bc], path=path, library="strict", seed=1)
    assert p.model.path == path
    p.advance(4)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad


@pytest.mark.parametrize("n", SIZES3)
@pytest.mark.parametrize("path", ["reference", "fused"])
def test_3d_sizes_bitwise_strict(n, path):
    p = Pair(n, BC3["slab_periodic"], path=path, library="strict", seed=2, rheo={"kind": "glen"})
    p.advance(3)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad


@pytest.mark.parametrize("bc", ["slab_periodic", "noslip_bed_free_top", "mixed_values"])
@pytest.mark.parametrize("path", ["reference", "fused"])
def test_3d_fp64_fast_within_1e10(bc, path):
    # a random state with the linear rheology converges; the reference PT scheme
    # diverges from a random state under Glen's law (see test_3d_glen_from_rest)
    p = Pair((33, 9, 10), BC3[bc], path=path, seed=3, rheo={"kind": "linear", "eta": 1.3})
    p.advance(50)
    err = p.compare()
    p.close()
    assert max(err.values()) <= 1e-10, err


@pytest.mark.parametrize("path", ["reference", "fused"])
@pytest.mark.parametrize("dtype,tol", [("f64", 1e-10), ("f32", 1e-4)])
def test_3d_glen_from_rest(path, dtype, tol):
    # the slab set-up of the benchmark: zero initial state, eta at the regularisation cap
    p = Pair((33, 17, 20), BC3["slab_periodic"], path=path, dtype=dtype, seed=3, rheo={"kind": "glen"},
             gravity=(-0.17, 0.0, 0.98), random_state=False)
    p.model.set_field("eta", 5000.0)
    p.model.set_field("eta_next", 5000.0)
    p.oracle.set_interior("eta", 5000.0)
    p.oracle.set_interior("eta_next", 5000.0)
    p.model.apply_bcs()
    p.oracle.apply_initial_bcs()
    p.advance(100)
    err = p.compare()
    p.close()
    assert max(err.values()) <= tol, err


@pytest.mark.parametrize("path", ["reference", "fused"])
def test_3d_fp32_strict_bitwise(path):
    p = Pair((33, 9, 10), BC3["noslip_bed_free_top"], path=path, dtype="f32", library="strict", seed=4)
    p.advance(4)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad


@pytest.mark.parametrize("path", ["reference", "fused"])
def test_3d_fp32_fast(path):
    p = Pair((33, 9, 10), BC3["slab_periodic"], path=path, dtype="f32", seed=5, rheo={"kind": "linear", "eta": 0.8})
    p.advance(20)
    err = p.compare()
    p.close()
    assert max(err.values()) <= 1e-4, err


@pytest.mark.parametrize("rheo", [{"kind": "linear", "eta": 2.0}, {"kind": "glen"},
                                  {"kind": "relax_glen", "rate": 0.3, "scale": None}])
def test_3d_rheologies_fused(rheo):
    p = Pair((33, 9, 10), BC3["free_slip_box"], path="fused", library="strict", seed=6, rheo=rheo)
    p.advance(3)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad


@pytest.mark.parametrize("scale", ["log", "log10"])
def test_3d_relaxation_log_scales(scale):
    # log/exp of the device math library differ from glibc in the last bits
    p = Pair((13, 7, 9), BC3["free_slip_box"], path="fused", seed=7,
             rheo={"kind": "relax_glen", "rate": 0.25, "scale": scale})
    p.advance(10)
    err = p.compare()
    p.close()
    assert max(err.values()) <= 1e-10, err


def _fused_variant_count():
    from conftest import load_fastice
    return load_fastice().load_library("strict").fi_fused_variant_count()


@pytest.mark.parametrize("variant", range(_fused_variant_count()))
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("bc,n", [("mixed_values", (150, 37, 70)), ("slab_periodic", (150, 37, 70)),
                                  ("noslip_box", (70, 37, 150))])
def test_every_fused_variant_bitwise(variant, dtype, bc, n):
    # each launch shape the autotuner may pick: tiles, z-blocks and clusters cut across
    # the grid; 150 x-positions leave interior columns for 64-wide tiles (the trimmed
    # boxes), and odd tile counts leave padded CTAs in clustered grids
    p = Pair(n, BC3[bc], path="fused", library="strict", dtype=dtype, seed=13)
    try:
        p.model.set_variant(variant)
    except Exception as e:
        p.close()
        if getattr(e, "status", None) == 6:  # FI_ERR_UNSUPPORTED: shape not offered in this precision
            pytest.skip(str(e))
        raise
    p.advance(3)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad


def test_fused_equals_reference_path():
    a = Pair((40, 17, 70), BC3["noslip_bed_free_top"], path="fused", seed=8, rheo={"kind": "glen"})
    b = Pair((40, 17, 70), BC3["noslip_bed_free_top"], path="reference", seed=8, rheo={"kind": "glen"})
    a.model.advance(7)
    b.model.advance(7)
    for name in a.state:
        x, y = a.model.get_field(name), b.model.get_field(name)
        assert np.max(np.abs(x - y)) <= 1e-12 * max(np.max(np.abs(y)), 1e-300), name
    a.close()
    b.close()


BC2 = {
    "free_slip": ((SLIP, SLIP), (SLIP, SLIP)),
    "mixed": ((("traction", (0.1, 0.0)), ("velocity", (0.2, -0.1))), (PER, PER)),
    "noslip_free_top": ((SLIP, SLIP), (NOSL, TRAC)),
}


@pytest.mark.parametrize("bc", list(BC2))
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_2d_bitwise_strict(bc, dtype):
    p = Pair((21, 13), BC2[bc], library="strict", dtype=dtype, seed=9, gravity=(0.3, -0.7, 0.0),
             rheo={"kind": "glen", "eta_reg": 10.0})
    p.advance(6)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad


@pytest.mark.parametrize("path", ["reference", "fused"])
@pytest.mark.parametrize("bc", ["noslip_bed_free_top", "slab_periodic", "mixed_values"])
def test_residual_norms(path, bc):
    p = Pair((33, 9, 10), BC3[bc], path=path, library="strict", seed=10)
    p.advance(5)
    a = p.model.residual_norms()
    b = p.oracle.residual_norms()
    p.close()
    # inf-norms and max|V| are order independent: bitwise; L2 sums differ in order
    np.testing.assert_array_equal(a[[0, 1, 2, 3, 8, 9, 10]], b[[0, 1, 2, 3, 8, 9, 10]])
    np.testing.assert_allclose(a[4:8], b[4:8], rtol=1e-12)
    assert a[11] == 0.0


def test_compute_residuals_fields():
    p = Pair((13, 7, 9), BC3["noslip_bed_free_top"], path="fused", library="strict", seed=11)
    p.advance(3)
    p.model.compute_residuals()
    p.oracle.residual_norms()  # fills the oracle residual arrays
    for name in ("rP", "rVx", "rVy", "rVz"):
        np.testing.assert_array_equal(p.model.get_field(name), p.oracle.interior(name))
    p.close()


def test_nonfinite_residual_flag():
    p = Pair((13, 7, 9), BC3["free_slip_box"], path="fused", seed=12)
    vx = p.model.get_field("Vx")
    vx[3, 3, 3] = np.nan
    p.model.set_field("Vx", vx)
    norms = p.model.residual_norms()
    p.close()
    assert norms[11] == 1.0


def test_eta_rel_honoured_as_log_relaxation():
    # a model told to honour the drivers' η_rel iterates exactly as one given
    # Relaxation(η, rheology, η_rel; scale=log) explicitly
    from conftest import load_fastice
    fi = load_fastice()
    grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=(1.0, 1.0, 0.25), dims=(33, 17, 20))
    bcs = {"x": (fi.PBC(), fi.PBC()), "y": (fi.PBC(), fi.PBC()), "z": (fi.SBC(0.0, 0.0, 0.0), fi.TBC(0.0, 0.0, 0.0))}
    glen = fi.glen_regularised()
    sp = fi.pt_params(grid, eta_rel=0.1)
    g = {"x": -0.17, "y": 0.0, "z": 0.98}
    a = fi.IsothermalFullStokesModel(grid=grid, boundary_conditions=bcs, gravity=g, rheology=glen, solver_params=sp,
                                     eta_rel="log")
    b = fi.IsothermalFullStokesModel(grid=grid, boundary_conditions=bcs, gravity=g,
                                     rheology=fi.Relaxation(glen, 0.1, scale="log"), solver_params=fi.pt_params(grid))
    c = fi.IsothermalFullStokesModel(grid=grid, boundary_conditions=bcs, gravity=g, rheology=glen, solver_params=sp)
    for m in (a, b, c):
        m.set_field("eta", 50.0)
        m.set_field("eta_next", 50.0)
        m.apply_bcs()
        m.advance(20)
    for name in ("P", "Vx", "eta"):
        assert np.array_equal(a.get_field(name), b.get_field(name)), name
    # by default η_rel is ignored, as in the reference
    assert not np.array_equal(a.get_field("eta"), c.get_field("eta"))
    for m in (a, b, c):
        m.close()
