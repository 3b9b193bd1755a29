"""GPU parity at the benchmark's scales: the fused sweep on the tilted-slab
workload at 255^3 and the immersed-boundary iteration on the seeded glacier at
191^3, against the CPU oracle after a fixed number of iterations from the
workloads' own initial states (zero state, the regularised viscosity cap for the
slab, unit viscosity for the glacier).

Tolerances as everywhere else: the no-FMA build matches the oracle bit for bit;
the production build within 1e-10 relative in FP64 and 1e-4 in FP32.
"""
import math

import numpy as np
import pytest

from conftest import load_fastice, load_oracle
from helpers import Pair

pytestmark = pytest.mark.gpu

PER = ("periodic", ())
SLAB_BCS = ((PER, PER), (PER, PER), (("slip", (0.0, 0.0, 0.0)), ("traction", (0.0, 0.0, 0.0))))
ALPHA = math.radians(10.0)
SLAB_GRAVITY = (-math.sin(ALPHA), 0.0, math.cos(ALPHA))


def _variant_index(lib, name):
    for v in range(lib.fi_fused_variant_count()):
        if lib.fi_fused_variant_name(v).decode() == name:
            return v
    raise KeyError(name)


def slab_pair(n, dtype, library, variant_name=None):
    p = Pair((n, n, n), SLAB_BCS, path="fused", library=library, dtype=dtype, rheo={"kind": "glen"},
             gravity=SLAB_GRAVITY, extent=(1.0, 1.0, 0.25), origin=(0.0, 0.0, 0.0), random_state=False)
    p.model.set_field("eta", 5000.0)
    p.model.set_field("eta_next", 5000.0)
    p.oracle.set_interior("eta", 5000.0)
    p.oracle.set_interior("eta_next", 5000.0)
    p.model.apply_bcs()
    p.oracle.apply_initial_bcs()
    if variant_name is not None:
        p.model.set_variant(_variant_index(p.model.lib, variant_name))
    return p


@pytest.mark.parametrize("variant", ["tile32x8_zb32", "tile32x8_zb32_trim_cl1x4"])
@pytest.mark.parametrize("library", ["fast", "strict"])
def test_slab_255_fp64(variant, library):
    p = slab_pair(255, "f64", library, variant)
    p.advance(3)
    if library == "strict":
        bad = p.bitwise_equal()
        p.close()
        assert not bad, bad
    else:
        err = p.compare()
        p.close()
        assert max(err.values()) <= 1e-10, err


@pytest.mark.parametrize("variant", ["tile32x8_zb32", "tile64x8_zb32_trim", "tile32x8_zb32_cl2x2"])
def test_slab_255_fp32_strict(variant):
    p = slab_pair(255, "f32", "strict", variant)
    p.advance(3)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad


def glacier_pair(n, dtype, library):
    """The glacier workload (seeded 64-bump bed, sinusoidal surface, traction-free
    box, ρg = (0, 0, 1), unit linear viscosity, the glacier driver's PT steps) on
    both sides from the same level sets; each side computes its own volume fractions."""
    fi = load_fastice()
    O = load_oracle()
    grid, psi_na, psi_ns, _ = fi.scenarios.bed_levelsets(0, n, library=library)
    # the oracle's DEM level set agrees with the device's bit for bit
    dem_grid, bed, surf, _ = fi.scenarios.bed_dems(0, n)
    dx = grid.spacing()
    exp = O.levelset_from_dem((n, n, n), grid.origin, dx, dem_grid.dims, dem_grid.origin, dem_grid.spacing(), surf)
    if library == "strict":
        assert np.array_equal(exp, psi_na)
    else:  # FMA contraction in the distance arithmetic
        assert np.max(np.abs(exp - psi_na)) <= 1e-12 * np.max(np.abs(exp))
    trac = ("traction", (0.0, 0.0, 0.0))
    return Pair((n, n, n), ((trac, trac), (trac, trac), (trac, trac)), path="reference", library=library, dtype=dtype,
                rheo={"kind": "linear", "eta": 1.0}, gravity=(0.0, 0.0, 1.0), extent=(1.0, 1.0, 1.0),
                origin=(0.0, 0.0, 0.0), random_state=False, immersed_psi={"na": psi_na, "ns": psi_ns},
                pt=(0.9, 5 * math.pi, 1.1))


@pytest.mark.parametrize("library", ["fast", "strict"])
def test_glacier_191_fp64(library):
    # three iterations: two full ones, then one that skips the stored zeros and runs the block list
    p = glacier_pair(191, "f64", library)
    p.advance(3)
    if library == "strict":
        bad = p.bitwise_equal()
        a, b = p.model.residual_norms(), p.oracle.residual_norms()
        p.close()
        assert not bad, bad
        np.testing.assert_array_equal(a[[0, 1, 2, 3]], b[[0, 1, 2, 3]])
    else:
        err = p.compare()
        p.close()
        assert max(err.values()) <= 1e-10, err


def test_glacier_191_fp32_strict():
    p = glacier_pair(191, "f32", "strict")
    p.advance(3)
    bad = p.bitwise_equal()
    p.close()
    assert not bad, bad
