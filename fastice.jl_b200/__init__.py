"""fastice_b200: B200-native pseudo-transient Stokes solver with FastIce.jl's API.

The compute path is libfastice_b200 (hand-written sm_100a CUDA, C ABI in
include/fastice_b200.h); this package is the host-side mirror of the
reference's model / boundary-condition / level-set API over that ABI.
"""
from . import _lib
from ._lib import FastIceError
from .grids import Center, UniformGrid, Vertex, flip
from .levelsets import compute_levelset_from_dem, omega_from_psi
from .models import (Arch, BatchedIB3D, BatchedStokes2D, FieldRef, IsothermalFullStokesModel, IsothermalImmersedBoundaryFullStokesModel,
                     advance_iteration, compute_residuals, interior, pt_params, set_)
from .physics import (ArrayField, BoundaryCondition, ConstantField, FunctionField, Halo, HBC, LinearViscousRheology,
                      OneField, PBC, Periodic, PowerLawRheology, Relaxation, SBC, Slip, TBC, Traction, VBC, ValueField, Velocity,
                      ViscoplasticRegularisation, ZeroField, glen_regularised)
from . import scenarios  # noqa: E402  (seeded problem set-ups over the names above)
from . import writers  # noqa: E402
from . import heat  # noqa: E402
from .heat import HeatDiffusionModel  # noqa: E402
from .writers import write_h5, write_xdmf  # noqa: E402

__all__ = [
    "FastIceError", "BatchedIB3D", "BatchedStokes2D", "Center", "Vertex", "UniformGrid", "flip", "compute_levelset_from_dem", "omega_from_psi", "Arch",
    "FieldRef", "IsothermalFullStokesModel", "IsothermalImmersedBoundaryFullStokesModel", "advance_iteration",
    "compute_residuals", "interior", "pt_params", "set_", "ArrayField", "BoundaryCondition", "ConstantField", "Halo", "HBC",
    "FunctionField", "LinearViscousRheology", "OneField", "PBC", "Periodic", "PowerLawRheology", "Relaxation", "SBC",
    "Slip", "TBC", "Traction", "VBC", "ValueField", "Velocity", "ViscoplasticRegularisation", "ZeroField",
    "glen_regularised", "load_library", "scenarios", "writers", "write_h5", "write_xdmf", "heat", "HeatDiffusionModel",
]


def load_library(flavor: str = "fast"):
    """Load libfastice_b200 (raises ImportError when it has not been built)."""
    return _lib.load(flavor)
