"""Heat diffusion (src/Models/Diffusion/Heat/, restated): the library's fused heat
sweep against the CPU oracle bit for bit (no-FMA build), and the steady state
between two Value sides (a linear profile, exact for the discrete operator)."""
import numpy as np
import pytest

from conftest import load_fastice, load_oracle

pytestmark = pytest.mark.gpu

FIELDS = ("T", "qx", "qy", "qz")


def _bits(a):
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def _pair(fi, O, n, ext, bcs, dtype, seed, dt=0.7):
    from fastice_b200 import heat
    grid = fi.UniformGrid(origin=(-0.5, -0.5, 0.0), extent=ext, dims=n)
    lam = 1.3
    ip = heat.heat_iter_params(grid, lam, dt)
    sides = {s: bc for pair, bcp in zip(heat.SIDES, bcs) for s, bc in zip(pair, bcp)}
    m = heat.HeatDiffusionModel(grid=grid, boundary_conditions=sides, physics={"λ_ρCp": lam}, iter_params=ip,
                                dtype=dtype, library="strict")
    kinds = [[0 if isinstance(b, heat.Value) else 1 for b in bcp] for bcp in bcs]
    vals = [[b.v for b in bcp] for bcp in bcs]
    o = O.OracleHeat(n, ext, kinds, vals, lam, ip["Δτ"]["T"], ip["Δτ"]["q"], dtype=dtype)
    rng = np.random.default_rng(seed)
    npd = np.float64 if dtype == "f64" else np.float32
    for name in ("T", "T_o", "qx", "qy", "qz"):
        v = rng.standard_normal(m.field_shape(name)).astype(npd)
        m.set_field(name, v)
        o.set_interior(name, v)
    m.apply_bcs()
    o.apply_bcs()
    return m, o


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("case", [0, 1, 2])
def test_heat_sweep_bitwise_vs_oracle(dtype, case):
    fi, O = load_fastice(), load_oracle()
    from fastice_b200.heat import Flux, Value
    bcs = [((Flux(0.0), Flux(0.0)), (Value(-0.1), Value(0.3)), (Flux(0.0), Flux(0.0))),
           ((Value(0.2), Flux(0.5)), (Flux(-0.25), Value(0.0)), (Value(1.0), Flux(0.1))),
           ((Value(0.0), Value(0.0)), (Value(0.0), Value(0.0)), (Value(0.0), Value(0.0)))][case]
    n = [(19, 13, 11), (40, 9, 17), (33, 33, 8)][case]
    m, o = _pair(fi, O, n, (1.0, 0.8, 1.1), bcs, dtype, seed=case)
    m.advance(20, 0.7)
    o.advance(20, 0.7)
    bad = [(f, int(np.sum(m.get_field(f) != o.interior(f)))) for f in FIELDS
           if not np.array_equal(_bits(m.get_field(f)), _bits(o.interior(f)))]
    m.close()
    assert not bad, bad


def test_heat_steady_state_between_two_value_sides():
    fi = load_fastice()
    from fastice_b200 import heat
    # the linear profile between south (-0.1) and north (0.3) with insulated other
    # sides is steady: an implicit step from it (T_o) returns it, and the PT
    # iteration (the driver's Δt = 1 and pseudo-time steps) must reach it from T = 0
    n = (16, 32, 12)
    grid = fi.UniformGrid(origin=(-0.5, -0.5, 0.0), extent=(1.0, 1.0, 1.0), dims=n)
    dt = 1.0
    sides = {"west": heat.Flux(0.0), "east": heat.Flux(0.0), "south": heat.Value(-0.1), "north": heat.Value(0.3),
             "bottom": heat.Flux(0.0), "top": heat.Flux(0.0)}
    m = heat.HeatDiffusionModel(grid=grid, boundary_conditions=sides, physics={"properties": 1.0},
                                iter_params=heat.heat_iter_params(grid, 1.0, dt))
    yc = -0.5 + (np.arange(n[1]) + 0.5) / n[1]
    exact = np.broadcast_to((-0.1 + 0.4 * (yc + 0.5))[None, :, None], m.field_shape("T"))
    m.set_field("T", 0.0)
    m.set_field("T_o", exact)
    for q in ("qx", "qy", "qz"):
        m.set_field(q, 0.0)
    m.apply_bcs()
    m.advance(3000, dt)
    err = np.max(np.abs(m.get_field("T") - exact))
    m.close()
    assert err < 1e-8, err
