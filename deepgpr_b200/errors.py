"""Exception types, matching the reference's hierarchy (src/DeepGPR/utils/exceptions.py).

Each error also derives from the built-in type callers already catch.
"""


class DeepGPRError(Exception):
    """Base class of this package's errors."""


class NativeLibraryError(DeepGPRError, RuntimeError):
    """The CUDA library is missing, stale, or a native call failed."""


class NativeLibraryNotFoundError(NativeLibraryError, FileNotFoundError):
    """libdeepgpr_b200.so was not built or cannot be loaded."""


class CFLConditionError(DeepGPRError, ValueError):
    """The time step violates the CFL limit of the staggered scheme."""


class NonFiniteTensorError(DeepGPRError, FloatingPointError):
    """A solver input or output contains NaN or Inf."""
