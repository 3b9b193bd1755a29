"""Rheologies, field-valued inputs and boundary conditions, mirroring
``src/Physics.jl``, ``src/Models/FullStokes/Isothermal/boundary_conditions.jl``
and the Chmy field types the reference drivers pass (``ValueField``,
``ZeroField``, ``ConstantField``, ``OneField``, ``FunctionField``).
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib as L
from .grids import Center, UniformGrid, Vertex, _locs


# ---------------------------------------------------------------------------
# field-valued inputs
# ---------------------------------------------------------------------------
class ValueField:
    """Chmy ``ValueField(v)``: the same value everywhere."""

    def __init__(self, value: float):
        self.value = float(value)


class ConstantField(ValueField):
    """Chmy ``ConstantField(v)``."""


class ZeroField(ValueField):
    """Chmy ``ZeroField{T}()``."""

    def __init__(self):
        super().__init__(0.0)


class OneField(ValueField):
    """Chmy ``OneField{T}()``."""

    def __init__(self):
        super().__init__(1.0)


class FunctionField:
    """Chmy ``FunctionField(f, grid, loc; parameters)``: ``f(x, y[, z], params...)``
    evaluated at the coordinates of ``loc``.  Sampled on the host into the
    uniform halo box (ghost coordinates extrapolate the grid)."""

    def __init__(self, func: Callable, grid: UniformGrid, loc, parameters=None):
        self.func = func
        self.grid = grid
        self.loc = _locs(loc, grid.ndims)
        if parameters is None:
            self.parameters = ()
        elif isinstance(parameters, tuple):
            self.parameters = parameters
        else:
            self.parameters = (parameters,)

    def sample(self, halo: bool = True) -> np.ndarray:
        """numpy array (z, y, x) over the halo box (or the interior if not halo)."""
        g = self.grid
        axes = [g.coords(self.loc[d], d, halo=halo) for d in range(g.ndims)]
        mesh = np.meshgrid(*axes, indexing="ij")  # (x, y, z) ordering
        try:
            vals = np.asarray(self.func(*mesh, *self.parameters), dtype=np.float64)
        except TypeError:  # scalar-only function (e.g. math.sin): evaluate point by point
            vals = np.vectorize(lambda *xs: float(self.func(*xs, *self.parameters)), otypes=[np.float64])(*mesh)
        vals = np.broadcast_to(vals, mesh[0].shape)
        return np.ascontiguousarray(np.transpose(vals))  # -> (z, y, x)


class ArrayField:
    """Values given directly as an interior numpy array (x fastest, numpy order (z, y, x))."""

    def __init__(self, values: np.ndarray):
        self.values = np.asarray(values, dtype=np.float64)


# ---------------------------------------------------------------------------
# rheology (src/Physics.jl)
# ---------------------------------------------------------------------------
class IceRheology:
    pass


class LinearViscousRheology(IceRheology):
    """``LinearViscousRheology(η)``: η a number, a ValueField, a FunctionField or
    an ArrayField (Physics.jl:7-11)."""

    def __init__(self, eta):
        self.eta = eta


class PowerLawRheology(IceRheology):
    """``PowerLawRheology(A, n)``: η = 0.5 / (A τII^(n-1)) (Physics.jl:13-18, Glen, stress form)."""

    def __init__(self, A, n: int):
        if int(n) != n:
            raise ValueError("the power-law exponent must be an integer (Physics.jl keeps n an Int)")
        self.A = A
        self.n = int(n)


class ViscoplasticRegularisation(IceRheology):
    """``ViscoplasticRegularisation(viscosity, η_reg)``: η = 1/(1/η_v + 1/η_reg) (Physics.jl:20-26)."""

    def __init__(self, viscosity: IceRheology, eta_reg: float):
        if isinstance(viscosity, (ViscoplasticRegularisation, Relaxation)):
            raise ValueError("the regularised viscosity must be a linear or power-law rheology")
        self.viscosity = viscosity
        self.eta_reg = float(eta_reg)
        self.inv_eta_reg = 1.0 / self.eta_reg


class Relaxation(IceRheology):
    """``Relaxation(field, target, rate; scale=None|'log'|'log10')`` (Physics.jl:28-47).
    The relaxed field is the model's current viscosity η."""

    def __init__(self, target: IceRheology, rate: float, scale: Optional[str] = None):
        if scale not in (None, "log", "log10"):
            raise ValueError("only None, 'log' and 'log10' are supported for the relaxation scale")
        if isinstance(target, Relaxation):
            raise ValueError("nested relaxation is not supported")
        self.target = target
        self.rate = float(rate)
        self.scale = scale


def glen_regularised(A: float = 1.0, n: int = 3, strain_rate_0: float = 1e-6) -> ViscoplasticRegularisation:
    """Glen's law with a strain-rate regularisation expressed through the
    reference's own types: the viscosity is capped at the Glen value at
    ε̇II = ε̇0, η_reg = ½ A^(-1/n) ε̇0^((1-n)/n) (5000 for A=1, n=3, ε̇0=1e-6)."""
    eta_reg = 0.5 * A ** (-1.0 / n) * strain_rate_0 ** ((1.0 - n) / n)
    return ViscoplasticRegularisation(PowerLawRheology(A, n), eta_reg)


def rheology_desc(r: IceRheology):
    """Return (fi_rheology, dict of field arrays to upload)."""
    d = L.fi_rheology()
    fields = {}
    if isinstance(r, Relaxation):
        d.relax = {None: L.FI_RELAX_LIN, "log": L.FI_RELAX_LOG, "log10": L.FI_RELAX_LOG10}[r.scale]
        d.rate = r.rate
        r = r.target
    if isinstance(r, ViscoplasticRegularisation):
        d.has_reg = 1
        d.eta_reg = r.eta_reg
        r = r.viscosity
    if isinstance(r, LinearViscousRheology):
        d.inner = L.FI_RHEO_LINEAR
        if isinstance(r.eta, (int, float)):
            d.eta = float(r.eta)
        elif isinstance(r.eta, ValueField):
            d.eta = r.eta.value
        else:
            d.eta_is_field = 1
            fields["eta_lin"] = r.eta
    elif isinstance(r, PowerLawRheology):
        d.inner = L.FI_RHEO_POWER
        d.n = r.n
        if isinstance(r.A, (int, float)):
            d.A = float(r.A)
        elif isinstance(r.A, ValueField):
            d.A = r.A.value
        else:
            d.A_is_field = 1
            fields["A"] = r.A
    else:
        raise TypeError(f"unsupported rheology {type(r).__name__}")
    return d, fields


# ---------------------------------------------------------------------------
# boundary conditions (boundary_conditions.jl:1-13)
# ---------------------------------------------------------------------------
class Traction:
    kind = L.FI_BC_TRACTION


class Velocity:
    kind = L.FI_BC_VELOCITY


class Slip:
    kind = L.FI_BC_SLIP


class Periodic:
    """Extension: periodic dimension (both sides must be Periodic)."""
    kind = L.FI_BC_PERIODIC


class Halo:
    """The side of a subdomain whose ghost layer comes from its neighbour (the
    reference's distributed boundary, exchanged by Chmy.Distributed): x or y of a 3D
    FullStokes subdomain; the other side of that dimension may be physical."""
    kind = L.FI_BC_HALO


class BoundaryCondition:
    """``BoundaryCondition{Kind}(components...)``; e.g. ``BoundaryCondition(Slip, 0.0, 0.0, 0.0)``."""

    def __init__(self, kind, *components: float):
        if kind not in (Traction, Velocity, Slip, Periodic, Halo):
            raise TypeError("kind must be Traction, Velocity, Slip, Periodic or Halo")
        self.kind = kind
        self.components = tuple(float(c) for c in components)

    def __repr__(self):
        return f"BoundaryCondition{{{self.kind.__name__}}}{self.components}"


def SBC(*c):
    return BoundaryCondition(Slip, *c)


def TBC(*c):
    return BoundaryCondition(Traction, *c)


def VBC(*c):
    return BoundaryCondition(Velocity, *c)


def PBC():
    return BoundaryCondition(Periodic)


def HBC():
    return BoundaryCondition(Halo)
