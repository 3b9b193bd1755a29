"""Pins of the CPU oracle and the host grid mirror (no GPU).

The reference's only tests touching the discretisation are the Chmy grid
geometry checks of test/test_chmy_grids.jl; their expected values are restated
here and checked against the host UniformGrid and the oracle's coordinate
convention.  The operators are further anchored by the O(h^2) convergence of
the manufactured solutions of scripts_future_API/stokes_manufactured_solution_free_slip_2D.jl
and _3D.jl, and the cut-cell volumes by closed-form known answers.
"""
import math

import numpy as np
import pytest


# ---- test/test_chmy_grids.jl:17-160 (origin=(-1,-2), extent=(2,4), dims=(5,20)) -------
@pytest.fixture
def chmy_grid(fi):
    return fi.UniformGrid(origin=(-1, -2), extent=(2, 4), dims=(5, 20))


def test_flip(fi):
    assert fi.flip(fi.Center()) == fi.Vertex()
    assert fi.flip(fi.Vertex()) == fi.Center()


def test_sizes(fi, chmy_grid):
    g, C, V = chmy_grid, fi.Center(), fi.Vertex()
    assert g.size(C) == (5, 20)
    assert g.size(V) == (6, 21)
    assert g.size((C, V)) == (5, 21)
    assert g.size((V, C)) == (6, 20)
    assert g.size(C) == g.size((C, C)) and g.size(V) == g.size((V, V))


def test_bounds_extent_origin(fi, chmy_grid):
    g, C, V = chmy_grid, fi.Center(), fi.Vertex()
    assert np.allclose(g.bounds(V, 0), (-1.0, 1.0)) and np.allclose(g.bounds(V, 1), (-2.0, 2.0))
    assert np.allclose(g.bounds(C, 0), (-0.8, 0.8)) and np.allclose(g.bounds(C, 1), (-1.9, 1.9))
    assert math.isclose(g.grid_extent(V, 0), 2.0) and math.isclose(g.grid_extent(V, 1), 4.0)
    assert math.isclose(g.grid_extent(C, 0), 1.6) and math.isclose(g.grid_extent(C, 1), 3.8)
    assert math.isclose(g.grid_origin(V, 0), -1) and math.isclose(g.grid_origin(C, 0), -0.8)
    assert math.isclose(g.grid_origin(C, 1), -1.9)


def test_spacing_and_inverse(fi, chmy_grid):
    g = chmy_grid
    assert np.allclose(g.spacing(), (0.4, 0.2))
    assert np.allclose(g.inv_spacing(), (2.5, 5.0))


def test_coords(fi, chmy_grid):
    g, C, V = chmy_grid, fi.Center(), fi.Vertex()
    assert math.isclose(g.coord(V, 0, 1), -1.0) and math.isclose(g.coord(V, 1, 1), -2.0)
    assert math.isclose(g.coord(V, 0, 6), 1.0) and math.isclose(g.coord(V, 1, 21), 2.0)
    assert math.isclose(g.coord(C, 0, 1), -0.8) and math.isclose(g.coord(C, 1, 1), -1.9)
    assert math.isclose(g.coord(C, 0, 5), 0.8) and math.isclose(g.coord(C, 1, 20), 1.9)
    xs = g.coords(V, 0, halo=True)  # storage index 0 is the ghost left of vertex 1
    assert math.isclose(xs[1], -1.0) and math.isclose(xs[0], -1.4)


# ---- 2D manufactured solution on the unit square ------------------------------------------
def _mms2d_oracle(orc, n, max_iter_factor=60):
    ext, org = (1.0, 1.0), (0.0, 0.0)
    dx = ext[0] / n
    r, re = 0.7, 8 * math.pi
    lt = min(ext) / re
    vdt = dx / math.sqrt(2 * 1.1)
    th = lt * (r + 4 / 3) / vdt
    dtr, nud = 1.0 / (th + 1.0), vdt * lt
    slip = (orc.BC_SLIP, (0, 0, 0))
    spec = orc.Spec(nd=2, n=(n, n), extent=ext, origin=org, bcs=((slip, slip), (slip, slip)), dt_P=r / th,
                    dt_tau=(dtr, dtr, 0, dtr, 0, 0), dt_V=(nud, nud, 0))
    sh = spec.storage_shape()
    iy, ix = np.meshgrid(np.arange(sh[0]), np.arange(sh[1]), indexing="ij")
    xv, xc = org[0] + (ix - 1) * dx, org[0] + (ix - 0.5) * dx
    yv, yc = org[1] + (iy - 1) * dx, org[1] + (iy - 0.5) * dx
    gx = -2 * math.pi ** 2 * np.sin(math.pi * xv) * np.cos(math.pi * yc)
    gy = 2 * math.pi ** 2 * np.cos(math.pi * xc) * np.sin(math.pi * yv)
    m = orc.OracleStokes(spec, gravity_arrays={"gx": gx, "gy": gy})
    m.a["eta"][:] = 1.0
    m.a["eta_next"][:] = 1.0
    m.apply_initial_bcs()
    it = 0
    while it < max_iter_factor * n:
        m.advance(n)
        it += n
        nr = m.residual_norms()
        if max(nr[:3]) < 1e-8:
            break
    ex = (np.sin(math.pi * xv) * np.cos(math.pi * yc))[1:n + 1, 1:n + 2]
    ey = (-np.cos(math.pi * xc) * np.sin(math.pi * yv))[1:n + 2, 1:n + 1]
    Vx, Vy = m.interior("Vx"), m.interior("Vy")
    err = math.sqrt((np.sum((Vx - ex) ** 2) + np.sum((Vy - ey) ** 2)) / (np.sum(ex ** 2) + np.sum(ey ** 2)))
    return err, it, max(nr[:3])


def test_oracle_mms2d_second_order(orc):
    errs = []
    for n in (16, 32, 64):
        err, it, res = _mms2d_oracle(orc, n)
        assert res < 1e-8, (n, it, res)
        errs.append(err)
    orders = [math.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    assert all(1.9 < o < 2.1 for o in orders), orders


# ---- 3D manufactured solution on [-1,1]^3 (stokes_manufactured_solution_free_slip_3D.jl:25-48) ----
def _mf(a, b):
    return np.cos(math.pi * a) * (b ** 2 - 1) ** 2 - np.cos(math.pi * b) * (a ** 2 - 1) ** 2


def _mp(a, b):
    return np.cos(math.pi * b) * (1 - 3 * a ** 2) * 2 - np.cos(math.pi * a) * (1 - 3 * b ** 2) * 2


def _mms3d_oracle(fi, orc, n, max_iter_factor=80):
    ext, org = (2.0, 2.0, 2.0), (-1.0, -1.0, -1.0)
    dx = ext[0] / n
    dt = fi.pt_params(fi.UniformGrid(origin=org, extent=ext, dims=(n, n, n)))["Δτ"]
    taus = ("xx", "yy", "zz", "xy", "xz", "yz")
    slip = (orc.BC_SLIP, (0, 0, 0))
    spec = orc.Spec(nd=3, n=(n, n, n), extent=ext, origin=org, bcs=((slip, slip),) * 3, dt_P=dt["Pr"],
                    dt_tau=tuple(dt["τ"][k] for k in taus), dt_V=tuple(dt["V"][k] for k in "xyz"))
    sh = spec.storage_shape()
    k, j, i = np.meshgrid(np.arange(sh[0]), np.arange(sh[1]), np.arange(sh[2]), indexing="ij")
    v = lambda q: org[0] + (q - 1) * dx  # noqa: E731  (vertex coordinate of index q)
    c = lambda q: org[0] + (q - 0.5) * dx  # noqa: E731  (centre coordinate of index q)
    gx = -2 * np.sin(math.pi * v(i)) * (_mf(c(j), c(k)) * math.pi ** 2 - _mp(c(j), c(k)))
    gy = -2 * np.sin(math.pi * v(j)) * (_mf(c(k), c(i)) * math.pi ** 2 - _mp(c(k), c(i)))
    gz = -2 * np.sin(math.pi * v(k)) * (_mf(c(i), c(j)) * math.pi ** 2 - _mp(c(i), c(j)))
    m = orc.OracleStokes(spec, gravity_arrays={"gx": gx, "gy": gy, "gz": gz})
    m.a["eta"][:] = 1.0
    m.a["eta_next"][:] = 1.0
    m.apply_initial_bcs()
    it = 0
    while it < max_iter_factor * n:
        m.advance(n)
        it += n
        nr = m.residual_norms()
        if max(nr[:4]) < 1e-8:
            break
    ex = (np.sin(math.pi * v(i)) * _mf(c(j), c(k)))[1:n + 1, 1:n + 1, 1:n + 2]
    ey = (np.sin(math.pi * v(j)) * _mf(c(k), c(i)))[1:n + 1, 1:n + 2, 1:n + 1]
    ez = (np.sin(math.pi * v(k)) * _mf(c(i), c(j)))[1:n + 2, 1:n + 1, 1:n + 1]
    num = sum(np.sum((m.interior(f) - e) ** 2) for f, e in (("Vx", ex), ("Vy", ey), ("Vz", ez)))
    den = sum(np.sum(e ** 2) for e in (ex, ey, ez))
    return math.sqrt(num / den), it, max(nr[:4])


def test_oracle_mms3d_second_order(fi, orc):
    errs = []
    for n in (8, 16, 32):
        err, it, res = _mms3d_oracle(fi, orc, n)
        assert res < 1e-8, (n, it, res)
        errs.append(err)
    orders = [math.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    assert 1.8 < orders[-1] < 2.2, (errs, orders)


# ---- hydrostatic column: sign of the pressure gradient against ρg, traction ghost of P --------
def test_oracle_hydrostatic_column_is_steady(fi, orc):
    # V = 0, τ = 0 and P = ρg_z (z_top - z) under a traction-free top: the residual
    # r_V = -∇P + ∇·τ - ρg (kernels_3d.jl:66-75) vanishes, the top's Dirichlet ghost
    # of P (boundary_conditions.jl:51-76) continues the line, and PT iterations leave
    # the state where it is
    n, ext, org = (6, 5, 12), (1.0, 0.8, 0.6), (0.0, 0.0, 0.0)
    dt = fi.pt_params(fi.UniformGrid(origin=org, extent=ext, dims=n))["Δτ"]
    taus = ("xx", "yy", "zz", "xy", "xz", "yz")
    per = (orc.BC_PERIODIC, (0, 0, 0))
    bcs = ((per, per), (per, per), ((orc.BC_SLIP, (0, 0, 0)), (orc.BC_TRACTION, (0, 0, 0))))
    spec = orc.Spec(nd=3, n=n, extent=ext, origin=org, bcs=bcs, dt_P=dt["Pr"], dt_tau=tuple(dt["τ"][k] for k in taus),
                    dt_V=tuple(dt["V"][k] for k in "xyz"), g_val=(0.0, 0.0, 1.0))
    m = orc.OracleStokes(spec)
    dz = ext[2] / n[2]
    zc = org[2] + (np.arange(n[2]) + 0.5) * dz
    P = np.broadcast_to((ext[2] - zc)[:, None, None], (n[2], n[1], n[0])).copy()
    m.set_interior("P", P)
    m.a["eta"][:] = 1.0
    m.a["eta_next"][:] = 1.0
    m.apply_initial_bcs()
    nr = m.residual_norms()
    assert max(nr[:4]) < 1e-12, nr[:4]
    m.advance(50)
    for f in ("Vx", "Vy", "Vz"):
        assert np.max(np.abs(m.interior(f))) < 1e-12, f
    np.testing.assert_allclose(m.interior("P"), P, rtol=0, atol=1e-12)


# ---- the immersed-boundary restatement with every volume fraction 1 is the plain model ----------
@pytest.mark.parametrize("rheo", ["linear", "glen"])
def test_oracle_immersed_boundary_with_full_fractions_is_the_plain_model(fi, orc, rheo):
    # ω = 1 everywhere: every masked derivative (IB kernels_3d.jl:3-74) reduces to the
    # plain one (kernels_3d.jl:3-40), every point is active, and the division by
    # the face fraction is by 1, so the two restatements agree bit for bit
    n, ext, org = (9, 7, 8), (1.0, 0.9, 0.8), (0.0, 0.0, 0.0)
    dt = fi.pt_params(fi.UniformGrid(origin=org, extent=ext, dims=n))["Δτ"]
    taus = ("xx", "yy", "zz", "xy", "xz", "yz")
    bcs = (((orc.BC_VELOCITY, (0.1, -0.2, 0.0)), (orc.BC_TRACTION, (0.0, 0.1, 0.0))),
           ((orc.BC_SLIP, (0.0, 0.0, 0.0)), (orc.BC_SLIP, (0.0, 0.05, 0.0))),
           ((orc.BC_SLIP, (0.0, 0.0, 0.0)), (orc.BC_TRACTION, (0.0, 0.0, 0.0))))
    kw = dict(rheo_inner=orc.RHEO_POWER, rheo_has_reg=1, rheo_inv_eta_reg=1.0) if rheo == "glen" else {}
    spec = orc.Spec(nd=3, n=n, extent=ext, origin=org, bcs=bcs, dt_P=dt["Pr"], dt_tau=tuple(dt["τ"][k] for k in taus),
                    dt_V=tuple(dt["V"][k] for k in "xyz"), g_val=(0.2, -0.1, 1.0), **kw)
    ones = {c: np.ones(spec.storage_shape()) for c in orc.MASK_COMPONENTS}
    plain = orc.OracleStokes(spec)
    ib = orc.OracleStokes(spec, masks={"na": ones, "ns": ones})
    rng = np.random.default_rng(11)
    names = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta")
    for name in names:
        shape = plain.interior(name).shape
        vals = 0.5 + rng.random(shape) if name == "eta" else 0.1 * rng.standard_normal(shape)
        for m in (plain, ib):
            m.set_interior(name, vals)
            if name == "eta":
                m.set_interior("eta_next", vals)
    for m in (plain, ib):
        m.apply_initial_bcs()
        m.advance(20)
    for name in names:
        a, b = plain.interior(name), ib.interior(name)
        assert np.isfinite(a).all(), name
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


# ---- rheologies at a known stress invariant (src/Physics.jl:7-53) ----------------------------
@pytest.mark.parametrize("case", ["linear", "power", "power_capped", "relax_lin", "relax_log", "relax_log10"])
def test_oracle_rheology_at_a_known_stress(fi, orc, case):
    # a uniform τxx = a with every other field zero on a periodic box: one iteration
    # relaxes it to a(1 - Δτ.τxx) (update_σ!, kernels_3d.jl:3-25), leaves V at rest,
    # and sets η_next = rheology(τII) with τII = |a (1 - Δτ.τxx)| / √2 at every cell
    # (update_V!, kernels_3d.jl:27-40); the swap makes it η.  Expected values from
    # Physics.jl's formulas: linear η, 0.5 / (A τII^(n-1)), the cap 1 / (1/η + 1/η_reg),
    # the relaxation η_old (1-r) + target r in linear, log or log10 scale.
    n, ext, org = (6, 5, 4), (1.0, 0.8, 0.6), (0.0, 0.0, 0.0)
    dt = fi.pt_params(fi.UniformGrid(origin=org, extent=ext, dims=n))["Δτ"]
    taus = ("xx", "yy", "zz", "xy", "xz", "yz")
    per = (orc.BC_PERIODIC, (0, 0, 0))
    A, nexp, eta_reg, rate, eta0, a = 2.0, 3, 50.0, 0.3, 7.0, 0.8
    kw = {"linear": dict(rheo_inner=orc.RHEO_LINEAR, rheo_eta_val=3.5),
          "power": dict(rheo_inner=orc.RHEO_POWER, rheo_A=A, rheo_n=nexp),
          "power_capped": dict(rheo_inner=orc.RHEO_POWER, rheo_A=A, rheo_n=nexp, rheo_has_reg=1,
                               rheo_inv_eta_reg=1.0 / eta_reg)}
    for scale, code in (("lin", orc.RELAX_LIN), ("log", orc.RELAX_LOG), ("log10", orc.RELAX_LOG10)):
        kw["relax_" + scale] = dict(rheo_inner=orc.RHEO_POWER, rheo_A=A, rheo_n=nexp, rheo_relax=code, rheo_rate=rate)
    spec = orc.Spec(nd=3, n=n, extent=ext, origin=org, bcs=((per, per), (per, per), (per, per)), dt_P=dt["Pr"],
                    dt_tau=tuple(dt["τ"][k] for k in taus), dt_V=tuple(dt["V"][k] for k in "xyz"),
                    g_val=(0.0, 0.0, 0.0), **kw[case])
    m = orc.OracleStokes(spec)
    m.set_interior("txx", np.full(m.interior("txx").shape, a))
    m.a["eta"][:] = eta0
    m.a["eta_next"][:] = eta0
    m.apply_initial_bcs()
    m.advance(1)
    tII = abs(a * (1.0 - dt["τ"]["xx"])) / math.sqrt(2.0)
    power = 0.5 / (A * tII ** (nexp - 1))
    expected = {"linear": 3.5, "power": power, "power_capped": 1.0 / (1.0 / power + 1.0 / eta_reg),
                "relax_lin": eta0 * (1 - rate) + power * rate,
                "relax_log": math.exp(math.log(eta0) * (1 - rate) + math.log(power) * rate),
                "relax_log10": 10.0 ** (math.log10(eta0) * (1 - rate) + math.log10(power) * rate)}[case]
    eta = m.interior("eta")
    np.testing.assert_allclose(eta, expected, rtol=1e-13, atol=0)
    for f in ("Vx", "Vy", "Vz", "P"):
        assert np.max(np.abs(m.interior(f))) == 0.0, f


# ---- simple shear: the staggered shear strain rate and its stress (kernels_3d.jl:3-25) ---------
def test_oracle_simple_shear_stress(fi, orc):
    # Vx = γ z between a bottom at rest and a top moving at γ L (Velocity conditions
    # continue the line into the ghosts), η uniform: ε̇xz = ½(∂z Vx + ∂x Vz) = γ/2 at
    # every interior (V, C, V) point and ∇·V = 0, so one iteration from rest sets
    # τxz = Δτ.τxz · 2η · γ/2 and leaves P and the other stresses at zero.
    n, ext, org = (6, 5, 8), (1.0, 0.8, 0.6), (0.0, 0.0, 0.0)
    dt = fi.pt_params(fi.UniformGrid(origin=org, extent=ext, dims=n))["Δτ"]
    taus = ("xx", "yy", "zz", "xy", "xz", "yz")
    per = (orc.BC_PERIODIC, (0, 0, 0))
    gamma, eta0, L = 0.4, 2.5, ext[2]
    bcs = ((per, per), (per, per), ((orc.BC_VELOCITY, (0.0, 0.0, 0.0)), (orc.BC_VELOCITY, (gamma * L, 0.0, 0.0))))
    spec = orc.Spec(nd=3, n=n, extent=ext, origin=org, bcs=bcs, dt_P=dt["Pr"], dt_tau=tuple(dt["τ"][k] for k in taus),
                    dt_V=tuple(dt["V"][k] for k in "xyz"), g_val=(0.0, 0.0, 0.0), rheo_eta_val=eta0)
    m = orc.OracleStokes(spec)
    dz = L / n[2]
    zc = org[2] + (np.arange(n[2]) + 0.5) * dz
    vx = m.interior("Vx")
    m.set_interior("Vx", np.broadcast_to((gamma * zc)[:, None, None], vx.shape).copy())
    m.a["eta"][:] = eta0
    m.a["eta_next"][:] = eta0
    m.apply_initial_bcs()
    m.advance(1)
    txz = m.interior("txz")  # (z vertices 1..n+1, y centres, x vertices 1..n+1)
    np.testing.assert_allclose(txz[1:-1], dt["τ"]["xz"] * 2.0 * eta0 * 0.5 * gamma, rtol=1e-13, atol=0)
    for f in ("P", "txx", "tyy", "tzz", "txy", "tyz"):
        assert np.max(np.abs(m.interior(f))) <= 1e-15, f


# ---- cut-cell volumes (volume_fractions.jl) -------------------------------------------------
def test_vol_box_full_and_empty(orc):
    d = (0.3, 0.2, 0.5)
    assert orc.vol_box3([-1.0] * 8, d) == pytest.approx(0.03, rel=1e-14)
    assert orc.vol_box3([1.0] * 8, d) == 0.0
    assert orc.vol_box2([-1.0] * 4, (0.3, 0.2)) == pytest.approx(0.06, rel=1e-14)
    assert orc.vol_box2([1.0] * 4, (0.3, 0.2)) == 0.0


@pytest.mark.parametrize("h", [0.1, 0.37, 0.5, 0.83])
def test_vol_box_planar_cut(orc, h):
    # psi = z - h*dz: the fraction below the plane is exactly h
    d = (0.3, 0.2, 0.5)
    psi = [((m >> 2) & 1) * d[2] - h * d[2] for m in range(8)]
    assert orc.vol_box3(psi, d) / (d[0] * d[1] * d[2]) == pytest.approx(h, rel=1e-12)
    psi2 = [((m >> 1) & 1) * 0.2 - h * 0.2 for m in range(4)]
    assert orc.vol_box2(psi2, (0.3, 0.2)) / 0.06 == pytest.approx(h, rel=1e-12)


def test_vol_box_oblique_plane(orc):
    # plane x + y + z = s through a unit cube: exact volume of the corner region
    d = (1.0, 1.0, 1.0)
    for s in (0.4, 0.9, 1.5, 2.2):
        psi = [(m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) - s for m in range(8)]
        v = orc.vol_box3(psi, d)

        def corner(t):
            return max(t, 0.0) ** 3 / 6.0
        exact = corner(s) - 3 * corner(s - 1) + 3 * corner(s - 2) - corner(s - 3)
        assert v == pytest.approx(exact, rel=1e-12, abs=1e-15)


def test_volfrac3d_planar_field(orc):
    n, dx = (6, 5, 8), (0.2, 0.25, 0.125)
    sh = (n[2] + 3, n[1] + 3, n[0] + 3)
    k = np.arange(sh[0])[:, None, None]
    z = (k - 1) * dx[2]
    h = 0.43
    psi = np.broadcast_to(z - h, sh).astype(np.float64).copy()
    w = orc.volfrac3d(n, dx, psi)
    # cell-centred fraction of the cell spanning z in [(k-1)dz, k dz]
    for kk in range(1, n[2] + 1):
        lo, hi = (kk - 1) * dx[2], kk * dx[2]
        exact = min(max((h - lo) / dx[2], 0.0), 1.0)
        assert np.allclose(w["ccc"][kk, 1:n[1] + 1, 1:n[0] + 1], exact, rtol=1e-12, atol=1e-14)


def test_levelset_flat_dem(orc):
    # a flat DEM at height h: the signed distance is z - h inside the window
    n3, o3, dx3 = (6, 6, 6), (0.0, 0.0, 0.0), (1 / 6, 1 / 6, 1 / 6)
    n2, o2, dx2 = (12, 12), (-0.5, -0.5), (2 / 12, 2 / 12)
    h = 0.41
    dem = np.full((n2[1] + 3, n2[0] + 3), h)
    psi = orc.levelset_from_dem(n3, o3, dx3, n2, o2, dx2, dem)
    k = np.arange(n3[2] + 3)
    z = o3[2] + (k - 1) * dx3[2]
    inner = psi[1:n3[2] + 2, 1:n3[1] + 2, 1:n3[0] + 2]
    expect = np.broadcast_to((z[1:n3[2] + 2] - h)[:, None, None], inner.shape)
    assert np.allclose(inner, expect, atol=1e-13)
    inv = orc.invert_levelset(n3, psi.copy())
    assert np.allclose(inv[1:-1, 1:-1, 1:-1], -psi[1:-1, 1:-1, 1:-1])
