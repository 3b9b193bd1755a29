"""Shared problem builders for the parity tests: one description, two
realisations -- the library model (through the public API / C ABI) and the CPU
oracle -- with the same seeded initial state."""
from __future__ import annotations

import math

import numpy as np

from conftest import load_fastice, load_oracle

STATE_3D = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta")
STATE_2D = ("P", "txx", "tyy", "txy", "Vx", "Vy", "eta")

KIND = {"slip": 0, "traction": 1, "velocity": 2, "periodic": 3, "halo": 4}


def make_bcs(fi, spec_bcs, nd):
    """spec_bcs: tuple per dim of ((kind, comps), (kind, comps))."""
    ctor = {"slip": fi.SBC, "traction": fi.TBC, "velocity": fi.VBC}
    out = {}
    for d, nm in enumerate(("x", "y", "z")[:nd]):
        pair = []
        for kind, comps in spec_bcs[d]:
            if kind == "periodic":
                pair.append(fi.PBC())
            elif kind == "halo":
                pair.append(fi.HBC())
            else:
                pair.append(ctor[kind](*comps))
        out[nm] = tuple(pair)
    return out


def rheology_objects(fi, rheo):
    kind = rheo["kind"]
    if kind == "linear":
        return fi.LinearViscousRheology(rheo.get("eta", 1.0))
    if kind == "glen":
        return fi.ViscoplasticRegularisation(fi.PowerLawRheology(rheo.get("A", 1.0), rheo.get("n", 3)),
                                             rheo.get("eta_reg", 5000.0))
    if kind == "power":
        return fi.PowerLawRheology(rheo.get("A", 1.0), rheo.get("n", 3))
    if kind == "relax_glen":
        return fi.Relaxation(fi.ViscoplasticRegularisation(fi.PowerLawRheology(1.0, 3), rheo.get("eta_reg", 50.0)),
                             rheo.get("rate", 0.3), scale=rheo.get("scale"))
    raise ValueError(kind)


def oracle_rheo_kwargs(O, rheo):
    kind = rheo["kind"]
    if kind == "linear":
        return dict(rheo_inner=O.RHEO_LINEAR, rheo_eta_val=float(rheo.get("eta", 1.0)))
    if kind in ("glen", "power", "relax_glen"):
        kw = dict(rheo_inner=O.RHEO_POWER, rheo_A=float(rheo.get("A", 1.0)), rheo_n=int(rheo.get("n", 3)))
        if kind in ("glen", "relax_glen"):
            eta_reg = float(rheo.get("eta_reg", 5000.0 if kind == "glen" else 50.0))
            kw.update(rheo_has_reg=1, rheo_inv_eta_reg=1.0 / eta_reg)
        if kind == "relax_glen":
            kw.update(rheo_relax={None: O.RELAX_LIN, "log": O.RELAX_LOG, "log10": O.RELAX_LOG10}[rheo.get("scale")],
                      rheo_rate=float(rheo.get("rate", 0.3)))
        return kw
    raise ValueError(kind)


class Pair:
    """Library model + oracle model for the same problem and initial state."""

    def __init__(self, n, bcs, rheo=None, gravity=(0.3, -0.2, 1.0), dtype="f64", path="auto", seed=0,
                 extent=None, origin=None, library="fast", random_state=True, immersed_psi=None, pt=None):
        fi = load_fastice()
        O = load_oracle()
        nd = len(n)
        self.nd = nd
        rheo = rheo or {"kind": "linear", "eta": 1.0}
        extent = extent or tuple(1.0 + 0.25 * d for d in range(nd))
        origin = origin or tuple(-0.1 * d for d in range(nd))
        grid = fi.UniformGrid(origin=origin, extent=extent, dims=n)
        sp = fi.pt_params(grid) if pt is None else fi.pt_params(grid, r=pt[0], re_mech=pt[1], vdtau_factor=pt[2])
        dt = sp["Δτ"]
        g = {nm: float(gravity[d]) for d, nm in enumerate(("x", "y", "z")[:nd])}
        cls = fi.IsothermalImmersedBoundaryFullStokesModel if immersed_psi is not None else fi.IsothermalFullStokesModel
        self.model = cls(grid=grid, boundary_conditions=make_bcs(fi, bcs, nd), gravity=g,
                         rheology=rheology_objects(fi, rheo), solver_params=sp, dtype=dtype, path=path,
                         library=library)
        taus = ("xx", "yy", "zz", "xy", "xz", "yz")
        spec_bcs = tuple(tuple((KIND[k], tuple(c) + (0.0,) * (3 - len(c))) for k, c in bcs[d]) for d in range(nd))
        self.spec = O.Spec(nd=nd, n=n, extent=extent, origin=origin, bcs=spec_bcs, dt_P=dt["Pr"],
                           dt_tau=tuple(dt["τ"].get(k, 0.0) for k in taus),
                           dt_V=tuple(dt["V"].get(k, 0.0) for k in ("x", "y", "z")),
                           g_val=tuple(float(v) for v in gravity), dtype=dtype, **oracle_rheo_kwargs(O, rheo))
        masks = None
        if immersed_psi is not None:
            # ω_from_ψ! on both sides: the model computes its masks on the device, the
            # oracle with its own volume-fraction restatement
            dxs = tuple(extent[d] / n[d] for d in range(nd))
            masks = {grp: O.volfrac3d(n, dxs, immersed_psi[grp]) for grp in ("na", "ns")}
            for grp in ("na", "ns"):
                self.model.omega_from_psi(grp, immersed_psi[grp])
        self.oracle = O.OracleStokes(self.spec, masks=masks)
        self.state = STATE_3D if nd == 3 else STATE_2D
        npd = np.float64 if dtype == "f64" else np.float32
        rng = np.random.default_rng(seed)
        for name in self.state:
            shape = self.model.field_shape(name)
            if name == "eta":
                vals = (0.5 + rng.random(shape)).astype(npd) if random_state else np.ones(shape, npd)
            else:
                vals = (0.1 * rng.standard_normal(shape)).astype(npd) if random_state else np.zeros(shape, npd)
            self.model.set_field(name, vals)
            self.oracle.set_interior(name, vals)
        # eta_next starts equal to eta, as the drivers do (tm_stokes_chmy.jl:277-278)
        eta = self.model.get_field("eta")
        self.model.set_field("eta_next", eta)
        self.oracle.set_interior("eta_next", eta)
        self.model.apply_bcs()
        self.oracle.apply_initial_bcs()

    def advance(self, n):
        self.model.advance(n)
        self.oracle.advance(n)

    def compare(self, rtol=0.0, fields=None):
        """max relative difference per field (interior), relative to the field's max |value|."""
        out = {}
        for name in fields or self.state:
            a = self.model.get_field(name).astype(np.float64)
            b = self.oracle.interior(name).astype(np.float64)
            scale = max(np.max(np.abs(b)), 1e-300)
            out[name] = float(np.max(np.abs(a - b)) / scale)
        return out

    def bitwise_equal(self, fields=None):
        bad = []
        for name in fields or self.state:
            a = self.model.get_field(name)
            b = self.oracle.interior(name)
            if not np.array_equal(a.view(np.uint64 if a.dtype == np.float64 else np.uint32),
                                  b.view(np.uint64 if b.dtype == np.float64 else np.uint32)):
                diff = np.argwhere(a != b)
                bad.append((name, len(diff), diff[:3].tolist()))
        return bad

    def close(self):
        self.model.close()


def mms2d_gravity(fi, grid, eta=1.0):
    """Forcing of the free-slip manufactured solution on the unit square
    (stokes_manufactured_solution_free_slip_2D.jl:31-32), as FunctionFields."""
    def gx(x, y):
        return -2 * eta * math.pi ** 2 * np.sin(math.pi * x) * np.cos(math.pi * y)

    def gy(x, y):
        return 2 * eta * math.pi ** 2 * np.cos(math.pi * x) * np.sin(math.pi * y)
    return {"x": fi.FunctionField(gx, grid, (fi.Vertex(), fi.Center())),
            "y": fi.FunctionField(gy, grid, (fi.Center(), fi.Vertex()))}


def mms2d_exact(grid):
    """Exact vx, vy at their staggered interior locations (numpy (y, x) order)."""
    xv = grid.coords(load_fastice().Vertex(), 0)
    xc = grid.coords(load_fastice().Center(), 0)
    yv = grid.coords(load_fastice().Vertex(), 1)
    yc = grid.coords(load_fastice().Center(), 1)
    vx = np.sin(math.pi * xv)[None, :] * np.cos(math.pi * yc)[:, None]
    vy = -np.cos(math.pi * xc)[None, :] * np.sin(math.pi * yv)[:, None]
    return vx, vy


# ---- 3D manufactured solution: the package's builders (fastice_b200.scenarios)
def mms3d_gravity(fi, grid, eta=1.0):
    return fi.scenarios.mms3d_gravity(grid, eta)


def mms3d_exact(fi, grid):
    return fi.scenarios.mms3d_exact(grid)


def mms3d_model(fi, n, dtype="f64", library="fast"):
    return fi.scenarios.mms3d_model(n, dtype=dtype, library=library)


def mms3d_error(fi, grid, m):
    return fi.scenarios.mms3d_error(grid, m)
