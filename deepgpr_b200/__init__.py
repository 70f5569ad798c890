"""deepgpr_b200 -- B200-native differentiable Maxwell FDTD (the DeepGPR compute path).

Public API (same names and contracts as the reference package ``DeepGPR``):

* :func:`compute` -- forward solve with the exact discrete adjoint behind autograd;
* :func:`checkpoint_initial_field` -- zero states for segmented runs;
* :func:`max_stable_time_step` -- CFL limit;
* :func:`ricker` -- Ricker wavelet.

The solver runs only in ``deepgpr_b200/lib/libdeepgpr_b200.so`` (CUDA, sm_100a).
"""

from .config import SPEED_OF_LIGHT, VACUUM_PERMEABILITY, VACUUM_PERMITTIVITY
from .errors import (
    CFLConditionError,
    DeepGPRError,
    NativeLibraryError,
    NativeLibraryNotFoundError,
    NonFiniteTensorError,
)
from .grid import max_stable_time_step, normalize_grid_spacing
from .solver import FDTDFunction, SolverConfig, checkpoint_initial_field, compute
from .wavelets import ricker

__all__ = [
    "CFLConditionError",
    "DeepGPRError",
    "FDTDFunction",
    "NativeLibraryError",
    "NativeLibraryNotFoundError",
    "NonFiniteTensorError",
    "SPEED_OF_LIGHT",
    "SolverConfig",
    "VACUUM_PERMEABILITY",
    "VACUUM_PERMITTIVITY",
    "checkpoint_initial_field",
    "compute",
    "max_stable_time_step",
    "normalize_grid_spacing",
    "ricker",
]
