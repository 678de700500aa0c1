"""B200-native lattice-Boltzmann step of the 2D differentially heated cavity.

Drop-in for the step of bbrangeo/cfd_cavity (``uniform::solver::CavitySolver``,
``src/uniform/solver.rs``): CUDA kernels for sm_100a behind the C ABI of
``include/cavity.h``; this package is its Python host mirror.
"""
from ._lib import CavError, load  # noqa: F401
from .batch import CavityBatch, sweep_configs  # noqa: F401
from .octree import OctreeSolver  # noqa: F401
from .solver import DELTA_T, T_COLD, T_HOT, CavitySolver, TimeAverager  # noqa: F401

__all__ = ["CavitySolver", "CavityBatch", "OctreeSolver", "TimeAverager", "CavError", "load", "sweep_configs",
           "T_HOT", "T_COLD", "DELTA_T"]
