"""Seeded problem set-ups of the benchmark workloads, in the pattern of the
reference's driver scripts (scripts_future_API/*.jl): each builds a model
through the public API and returns it with a description of what was drawn.

* ``inclusion_model`` -- 2D pure shear of a matrix with circular inclusions of
  contrasting viscosity between free-slip walls (the wall-velocity pattern of
  scripts_future_API/tm_stokes_wip.jl:41-52: normal velocity -ε̇·x on the x walls,
  +ε̇·y on the y walls, zero shear stress).
* ``bed_model`` -- 3D gravity-driven ice over a seeded bed of Gaussian bumps
  (the DEM -> level set -> volume fraction set-up of
  scripts_future_API/test_volume_fractions.jl:93-100, with the bed level set
  restated analytically as height above the bed).

Random draws use numpy's PCG64 generator seeded per instance.
"""
from __future__ import annotations

import math

import numpy as np

from .grids import UniformGrid
from .models import IsothermalFullStokesModel, pt_params
from .physics import ArrayField, LinearViscousRheology, SBC

INCLUSION_N_RANGE = (63, 511)


def inclusion_params(seed: int, n=None, n_range=INCLUSION_N_RANGE, sigma: float = 3.0, max_contrast: float = 1e4):
    """Draw one inclusion instance: cells per side (independent in x and y),
    1-16 circles of radius U(0.02, 0.15) centred U([0,1]^2), inclusion viscosity
    exp(N(0, sigma)) clipped to [1/max_contrast, max_contrast] (background 1)."""
    rng = np.random.default_rng(seed)
    if n is None:
        n = (int(rng.integers(n_range[0], n_range[1] + 1)), int(rng.integers(n_range[0], n_range[1] + 1)))
    k = int(rng.integers(1, 17))
    circles = []
    lim = math.log(max_contrast)
    for _ in range(k):
        r = float(rng.uniform(0.02, 0.15))
        cx, cy = (float(v) for v in rng.uniform(0.0, 1.0, 2))
        eta = float(math.exp(min(max(rng.normal(0.0, sigma), -lim), lim)))
        circles.append((cx, cy, r, eta))
    return {"n": tuple(n), "circles": circles}


def inclusion_viscosity(n, circles) -> np.ndarray:
    """Cell-centre viscosity (numpy order (y, x)) on [0,1]^2: 1 in the matrix, the
    circle's value inside a circle (later circles over earlier ones)."""
    xc = (np.arange(n[0]) + 0.5) / n[0]
    yc = (np.arange(n[1]) + 0.5) / n[1]
    Y, X = np.meshgrid(yc, xc, indexing="ij")
    eta = np.ones((n[1], n[0]))
    for cx, cy, r, e in circles:
        eta[(X - cx) ** 2 + (Y - cy) ** 2 <= r * r] = e
    return eta


def smooth_log(eta: np.ndarray, passes: int) -> np.ndarray:
    """``passes`` five-point averages of log η (edge-replicated borders): spreads a
    viscosity jump over a few cells, as PT codes do before iterating sharp
    inclusions."""
    lg = np.log(eta)
    for _ in range(passes):
        p = np.pad(lg, 1, mode="edge")
        lg = 0.2 * (p[1:-1, 1:-1] + p[:-2, 1:-1] + p[2:, 1:-1] + p[1:-1, :-2] + p[1:-1, 2:])
    return np.exp(lg)


def stiffness_ratio(eta: np.ndarray) -> float:
    """Largest ratio, over the velocity points, of the viscosities entering a
    velocity update's stencil (the two cells, and the four-cell vertex averages
    the shear stresses use) to the face average the update divides by.  The PT
    velocity step of kernels_2d.jl:20-29 scales with the inverse face average, so
    the step has to shrink by this ratio for the update to stay stable."""
    p = np.pad(eta, 1, mode="edge")
    exy = 0.25 * (p[:-1, :-1] + p[:-1, 1:] + p[1:, :-1] + p[1:, 1:])
    fx = 0.5 * (p[1:-1, :-1] + p[1:-1, 1:])
    mx = np.maximum(np.maximum(exy[:-1, :], exy[1:, :]), np.maximum(p[1:-1, :-1], p[1:-1, 1:]))
    fy = 0.5 * (p[:-1, 1:-1] + p[1:, 1:-1])
    my = np.maximum(np.maximum(exy[:, :-1], exy[:, 1:]), np.maximum(p[:-1, 1:-1], p[1:, 1:-1]))
    return float(max((mx / fx).max(), (my / fy).max(), 1.0))


def inclusion_model(seed: int, n=None, dtype: str = "f32", library: str = "fast", path: str = "auto",
                    strain_rate: float = 1.0, smooth: int = 4, vdtau_factor=None, **draw):
    """Build the pure-shear inclusion model of ``seed``: returns (model, params).
    The viscosity (smoothed by ``smooth`` log-space passes) is the linear
    rheology's field; η is set to it (with its Neumann ghosts), as drivers do
    before iterating.  The PT steps are the drivers' (pt_params) with the
    velocity-step factor raised by the field's stiffness ratio unless
    ``vdtau_factor`` is given."""
    prm = inclusion_params(seed, n=n, **draw)
    n = prm["n"]
    grid = UniformGrid(origin=(0.0, 0.0), extent=(1.0, 1.0), dims=n)
    e = float(strain_rate)
    bcs = {"x": (SBC(-e * 0.0, 0.0), SBC(-e * 1.0, 0.0)), "y": (SBC(0.0, e * 0.0), SBC(0.0, e * 1.0))}
    eta = smooth_log(inclusion_viscosity(n, prm["circles"]), smooth)
    ratio = stiffness_ratio(eta)
    factor = vdtau_factor if vdtau_factor is not None else 1.1 * ratio
    prm.update(smooth=smooth, stiffness_ratio=ratio, vdtau_factor=factor)
    m = IsothermalFullStokesModel(grid=grid, boundary_conditions=bcs, gravity={"x": 0.0, "y": 0.0},
                                  rheology=LinearViscousRheology(ArrayField(eta)),
                                  solver_params=pt_params(grid, vdtau_factor=factor),
                                  dtype=dtype, library=library, path=path)
    m.set_field("eta", eta)
    m.set_field("eta_next", eta)
    m.apply_bcs()
    return m, prm


def bed_model(seed: int, n: int, dtype: str = "f64", library: str = "fast", rheology=None, dem_cells=None,
              pt=(0.9, 5 * math.pi, 1.1)):
    """Build the immersed-boundary glacier of ``seed`` on the unit cube with n^3
    cells: returns (model, params).  Bed and surface DEMs live on a 2D vertex grid
    slightly wider than the cube; ψ.na comes from the surface DEM, ψ.ns from the
    bed DEM inverted, and the volume fractions from ω_from_ψ!
    (scripts_future_API/test_volume_fractions.jl:86-100).  Traction-free box
    sides, ρg = (0, 0, 1), linear viscosity 1 unless ``rheology`` is given, and
    that driver's PT steps (``pt`` = (r, re, factor) = (0.9, 5π, 1.1)) unless given."""
    from .models import IsothermalImmersedBoundaryFullStokesModel
    from .physics import TBC
    grid, psi_na, psi_ns, prm = bed_levelsets(seed, n, library=library, dem_cells=dem_cells)
    free = TBC(0.0, 0.0, 0.0)
    r, re_mech, factor = pt
    sp = pt_params(grid, r=r, re_mech=re_mech, vdtau_factor=factor)
    m = IsothermalImmersedBoundaryFullStokesModel(
        grid=grid, boundary_conditions={"x": (free, free), "y": (free, free), "z": (free, free)},
        gravity={"x": 0.0, "y": 0.0, "z": 1.0}, rheology=rheology or LinearViscousRheology(1.0),
        solver_params=sp, dtype=dtype, library=library)
    m.omega_from_psi("ns", psi_ns)
    m.omega_from_psi("na", psi_na)
    m.set_field("eta", 1.0)
    m.set_field("eta_next", 1.0)
    m.apply_bcs()
    prm.update(thickness=0.6)
    return m, prm


def bed_dems(seed: int, n: int, dem_cells=None):
    """The glacier's DEMs on their 2D vertex grid (halo storage): returns
    (dem_grid, bed heights, surface heights, params)."""
    prm = bed_params(seed, n)
    m2 = dem_cells or n + 1
    dem_grid = UniformGrid(origin=(-0.05, -0.05), extent=(1.1, 1.1), dims=(m2, m2))
    # vertex coordinates of the DEM grid in halo storage (index 0 is one spacing outside)
    h = 1.1 / m2
    xv = -0.05 + (np.arange(m2 + 3) - 1) * h
    Y, X = np.meshgrid(xv, xv, indexing="ij")
    return dem_grid, bed_height(prm, X, Y), 0.6 + 0.05 * np.sin(2.0 * math.pi * X), prm


def bed_levelsets(seed: int, n: int, library: str = "fast", dem_cells=None):
    """Level sets of the glacier of ``seed`` on the unit cube with n^3 cells, from
    its DEMs on the device: returns (grid, ψ.na from the surface, ψ.ns from the bed
    inverted, params)."""
    from .levelsets import compute_levelset_from_dem
    grid = UniformGrid(origin=(0.0, 0.0, 0.0), extent=(1.0, 1.0, 1.0), dims=(n, n, n))
    dem_grid, bed, surf, prm = bed_dems(seed, n, dem_cells)
    psi_na = compute_levelset_from_dem(grid, dem_grid, surf, library=library)
    psi_ns = compute_levelset_from_dem(grid, dem_grid, bed, invert=True, library=library)
    return grid, psi_na, psi_ns, prm


def glacier_glen_stages(grid, tol: float = 1e-8, stage_tol: float = 1e-6, n: int = 3, A: float = 1.0,
                        cap: float = 5000.0):
    """Continuation stages for Glen's law on the glacier (stages for
    ``solve_continuation``): the linear solution with the glacier driver's PT steps,
    then the regularised power law with its viscosity cap raised 10 -> 100 -> 1000 ->
    ``cap`` (5000: the Glen viscosity at the strain rate 1e-6), each stage to
    ``stage_tol`` and the last to ``tol``; from the cap of 1000 on, the velocity PT
    step factor is 4.4 instead of 1.1, without which those stages diverge (measured at
    127^3).  The solver parameters are functions of the attempt: a retried stage
    doubles the factor (at 383^3 the cap of 5000 diverges with 4.4 and converges with
    8.8).  The reference's PT iteration started from rest with the cap of 5000
    diverges on this geometry."""
    from .physics import PowerLawRheology, ViscoplasticRegularisation
    r, re = 0.9, 5 * math.pi

    def sp(f):
        return lambda attempt: pt_params(grid, r=r, re_mech=re, vdtau_factor=f * 2.0 ** attempt)

    caps = [c for c in (10.0, 100.0, 1000.0) if c < cap] + [cap]
    stages = [(LinearViscousRheology(1.0), sp(1.1), stage_tol)]
    for c in caps:
        stages.append((ViscoplasticRegularisation(PowerLawRheology(A, n), c), sp(1.1 if c < 1000.0 else 4.4),
                       tol if c == caps[-1] else stage_tol))
    return stages


def bed_params(seed: int, n: int, bumps: int = 64):
    """Seeded bed of ``bumps`` Gaussian bumps a·exp(-|x-c|^2/w^2), a~U(0,0.2),
    w~U(0.05,0.2), c~U([0,1]^2), and the surface z = 0.6 + 0.05 sin(2πx)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 0.2, bumps)
    w = rng.uniform(0.05, 0.2, bumps)
    c = rng.uniform(0.0, 1.0, (bumps, 2))
    return {"n": n, "a": a, "w": w, "c": c}


def bed_height(prm, x, y):
    h = np.zeros(np.broadcast(x, y).shape)
    for a, w, (cx, cy) in zip(prm["a"], prm["w"], prm["c"]):
        h = h + a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (w * w))
    return h


# ---- 2D manufactured solution on the unit square (the 128^2 plain-method case):
# forcing of scripts_future_API/stokes_manufactured_solution_free_slip_2D.jl:31-32
def mms2d_gravity(grid, eta: float = 1.0):
    """Body force of the 2D free-slip manufactured solution vx = sin πx cos πy,
    vy = -cos πx sin πy, P = 0 (η = 1), at the velocity locations."""
    from .physics import FunctionField
    from .grids import Center, Vertex

    def gx(x, y):
        return -2 * eta * math.pi ** 2 * np.sin(math.pi * x) * np.cos(math.pi * y)

    def gy(x, y):
        return 2 * eta * math.pi ** 2 * np.cos(math.pi * x) * np.sin(math.pi * y)
    return {"x": FunctionField(gx, grid, (Vertex(), Center())), "y": FunctionField(gy, grid, (Center(), Vertex()))}


def mms2d_exact(grid):
    """Exact vx, vy at their staggered interior locations (numpy (y, x) order)."""
    from .grids import Center, Vertex
    xv, xc = grid.coords(Vertex(), 0), grid.coords(Center(), 0)
    yv, yc = grid.coords(Vertex(), 1), grid.coords(Center(), 1)
    vx = np.sin(math.pi * xv)[None, :] * np.cos(math.pi * yc)[:, None]
    vy = -np.cos(math.pi * xc)[None, :] * np.sin(math.pi * yv)[:, None]
    return vx, vy


def mms2d_model(n: int, dtype: str = "f64", library: str = "fast"):
    """The 2D manufactured-solution model on the unit square with n^2 cells (η = 1,
    free slip on every side, zero initial state): returns (grid, model, gravity)."""
    grid = UniformGrid(origin=(0.0, 0.0), extent=(1.0, 1.0), dims=(n, n))
    slip = SBC(0.0, 0.0)
    gravity = mms2d_gravity(grid)
    m = IsothermalFullStokesModel(grid=grid, boundary_conditions={"x": (slip, slip), "y": (slip, slip)},
                                  gravity=gravity, rheology=LinearViscousRheology(1.0),
                                  solver_params=pt_params(grid), dtype=dtype, library=library)
    m.set_field("eta", 1.0)
    m.set_field("eta_next", 1.0)
    m.apply_bcs()
    return grid, m, gravity


def mms2d_error(grid, m) -> float:
    """Relative L2 error of the model's velocity against the 2D manufactured solution."""
    ex, ey = mms2d_exact(grid)
    vx, vy = m.get_field("Vx").astype(np.float64), m.get_field("Vy").astype(np.float64)
    return math.sqrt((np.sum((vx - ex) ** 2) + np.sum((vy - ey) ** 2)) / (np.sum(ex ** 2) + np.sum(ey ** 2)))


# ---- 3D manufactured solution (scripts_future_API/stokes_manufactured_solution_free_slip_3D.jl:25-48)
def _mf(a, b):
    return np.cos(math.pi * a) * (b ** 2 - 1) ** 2 - np.cos(math.pi * b) * (a ** 2 - 1) ** 2


def _mp(a, b):
    return np.cos(math.pi * b) * (1 - 3 * a ** 2) * 2 - np.cos(math.pi * a) * (1 - 3 * b ** 2) * 2


def mms3d_gravity(grid, eta: float = 1.0):
    """Body force of the 3D free-slip manufactured solution on [-1, 1]^3 (the
    driver's ρg, evaluated at each velocity component's location)."""
    from .physics import FunctionField
    from .grids import Center, Vertex
    V, Cc = Vertex(), Center()
    return {"x": FunctionField(lambda x, y, z: -2 * eta * np.sin(math.pi * x) * (_mf(y, z) * math.pi ** 2 - _mp(y, z)),
                               grid, (V, Cc, Cc)),
            "y": FunctionField(lambda x, y, z: -2 * eta * np.sin(math.pi * y) * (_mf(z, x) * math.pi ** 2 - _mp(z, x)),
                               grid, (Cc, V, Cc)),
            "z": FunctionField(lambda x, y, z: -2 * eta * np.sin(math.pi * z) * (_mf(x, y) * math.pi ** 2 - _mp(x, y)),
                               grid, (Cc, Cc, V))}


def mms3d_exact(grid):
    """Exact vx, vy, vz at their staggered interior locations (numpy (z, y, x) order)."""
    from .grids import Center, Vertex
    V, Cc = Vertex(), Center()
    out = []
    for comp, locs in (("x", (V, Cc, Cc)), ("y", (Cc, V, Cc)), ("z", (Cc, Cc, V))):
        x, y, z = (grid.coords(locs[d], d) for d in range(3))
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        if comp == "x":
            out.append(np.sin(math.pi * X) * _mf(Y, Z))
        elif comp == "y":
            out.append(np.sin(math.pi * Y) * _mf(Z, X))
        else:
            out.append(np.sin(math.pi * Z) * _mf(X, Y))
    return out


def mms3d_model(n: int, dtype: str = "f64", library: str = "fast"):
    """The 3D manufactured-solution model (η = 1, free slip on every side, zero
    initial state) at n^3 cells: returns (grid, model)."""
    grid = UniformGrid(origin=(-1.0, -1.0, -1.0), extent=(2.0, 2.0, 2.0), dims=(n, n, n))
    slip = SBC(0.0, 0.0, 0.0)
    m = IsothermalFullStokesModel(grid=grid, boundary_conditions={"x": (slip, slip), "y": (slip, slip),
                                                                 "z": (slip, slip)},
                                  gravity=mms3d_gravity(grid), rheology=LinearViscousRheology(1.0),
                                  solver_params=pt_params(grid), dtype=dtype, library=library)
    m.set_field("eta", 1.0)
    m.set_field("eta_next", 1.0)
    m.apply_bcs()
    return grid, m


def mms3d_error(grid, m) -> float:
    """Relative L2 error of the model's velocity against the manufactured solution."""
    ex = mms3d_exact(grid)
    num = sum(np.sum((m.get_field(f).astype(np.float64) - e) ** 2) for f, e in zip(("Vx", "Vy", "Vz"), ex))
    den = sum(np.sum(e ** 2) for e in ex)
    return math.sqrt(num / den)


__all__ = ["mms2d_gravity", "mms2d_exact", "mms2d_model", "mms2d_error", "mms3d_gravity", "mms3d_exact", "mms3d_model", "mms3d_error", "inclusion_params", "inclusion_viscosity", "inclusion_model", "smooth_log", "stiffness_ratio",
           "bed_model", "bed_params", "bed_height", "bed_dems", "bed_levelsets", "glacier_glen_stages",
           "INCLUSION_N_RANGE"]
