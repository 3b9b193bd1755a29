"""Uniform staggered grid with Chmy.jl's conventions (``UniformGrid``).

Conventions pinned by the reference's own ``test/test_chmy_grids.jl:30-160``:
``n`` cells per dim, Center size ``n`` and Vertex size ``n+1``, spacing
``extent/n``, vertex ``i`` (1-based) at ``origin + (i-1)*Δ`` and centre ``i`` at
``origin + (i-1/2)*Δ``.
"""
from __future__ import annotations

from typing import Sequence, Tuple


class Center:
    """Cell-centre location (Chmy ``Center()``)."""

    def __repr__(self):
        return "Center()"

    def __eq__(self, other):
        return isinstance(other, Center)

    def __hash__(self):
        return 0


class Vertex:
    """Cell-vertex location (Chmy ``Vertex()``)."""

    def __repr__(self):
        return "Vertex()"

    def __eq__(self, other):
        return isinstance(other, Vertex)

    def __hash__(self):
        return 1


def flip(loc):
    """``flip(Center()) == Vertex()`` and vice versa (test_chmy_grids.jl:9-10)."""
    return Vertex() if isinstance(loc, Center) else Center()


def _locs(loc, nd):
    if isinstance(loc, (Center, Vertex)):
        return (loc,) * nd
    return tuple(loc)


class UniformGrid:
    """``UniformGrid(arch; origin, extent, dims)``."""

    def __init__(self, origin: Sequence[float], extent: Sequence[float], dims: Sequence[int], arch=None):
        if not (len(origin) == len(extent) == len(dims)):
            raise ValueError("origin, extent and dims must have the same length")
        if len(dims) not in (2, 3):
            raise ValueError("only 2D and 3D grids are supported")
        self.origin = tuple(float(v) for v in origin)
        self.extent = tuple(float(v) for v in extent)
        self.dims = tuple(int(v) for v in dims)
        self.arch = arch

    @property
    def ndims(self) -> int:
        return len(self.dims)

    def size(self, loc=None) -> Tuple[int, ...]:
        """``size(grid, loc)``: n per Center dim, n+1 per Vertex dim."""
        if loc is None:
            loc = Center()
        locs = _locs(loc, self.ndims)
        return tuple(n + (1 if isinstance(l, Vertex) else 0) for n, l in zip(self.dims, locs))

    def spacing(self, loc=None, dim=None, *I):
        """``spacing(grid, loc, dim, i)``: uniform Δ = extent/n (tuple if dim is None)."""
        sp = tuple(e / n for e, n in zip(self.extent, self.dims))
        return sp if dim is None else sp[dim]

    def inv_spacing(self, loc=None, dim=None, *I):
        """``inv_spacing`` = ``iΔ``: 1/Δ."""
        isp = tuple(1.0 / s for s in self.spacing())
        return isp if dim is None else isp[dim]

    def coord(self, loc, dim: int, i: int) -> float:
        """1-based coordinate of index ``i`` along ``dim`` at ``loc`` (Vertex or Center)."""
        d = self.spacing()[dim]
        if isinstance(loc, Vertex):
            return self.origin[dim] + (i - 1) * d
        return self.origin[dim] + (i - 1) * d + 0.5 * d

    def bounds(self, loc, dim: int):
        n = self.size(loc)[dim] if isinstance(loc, (Center, Vertex)) else self.size(loc)[dim]
        l = _locs(loc, self.ndims)[dim]
        return (self.coord(l, dim, 1), self.coord(l, dim, n))

    def grid_origin(self, loc, dim: int) -> float:
        return self.coord(_locs(loc, self.ndims)[dim], dim, 1)

    def grid_extent(self, loc, dim: int) -> float:
        lo, hi = self.bounds(_locs(loc, self.ndims)[dim], dim)
        return hi - lo

    def coords(self, loc, dim: int, halo: bool = False):
        """numpy vector of coordinates along ``dim`` at ``loc``; with ``halo`` it
        covers storage indices 0..n+2 (uniform halo box)."""
        import numpy as np
        l = _locs(loc, self.ndims)[dim]
        d = self.spacing()[dim]
        if halo:
            idx = np.arange(self.dims[dim] + 3, dtype=np.float64)
        else:
            idx = np.arange(1, self.size(loc)[dim] + 1, dtype=np.float64)
        base = self.origin[dim] + (idx - 1) * d
        return base if isinstance(l, Vertex) else base + 0.5 * d

    def __repr__(self):
        return f"UniformGrid(origin={self.origin}, extent={self.extent}, dims={self.dims})"
