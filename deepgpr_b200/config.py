"""Constants of the FDTD path: physics, stencil, CPML and the native option word.

The values are those of the reference package (src/DeepGPR/config/constants.py,
src/DeepGPR/lib/deepgpr.h:21-33) so that coefficients, CFL limits and the
packed ``storage_type`` argument are identical.  FP8 histories (storage kind 4)
and FP64 histories (kind 5) are additions of this library.
"""

from __future__ import annotations

SPEED_OF_LIGHT = 299792458.0
VACUUM_PERMEABILITY = 1.25663706212e-06
VACUUM_PERMITTIVITY = 8.8541878128e-12
PEC_CONDUCTIVITY_THRESHOLD = 100.0
MIN_RELATIVE_PERMITTIVITY = 1.0

SUPPORTED_FDTD_ORDERS = (2, 4, 8)
SUPPORTED_GRADIENT_MODES = (2, 3)
FIELD_COMPONENTS = (0, 1, 2)

# Sum of |taps| of each staggered stencil (scales the CFL limit).
STENCIL_TAP_SUMS = {
    2: 1.0,
    4: 9.0 / 8.0 + 1.0 / 24.0,
    8: 1225.0 / 1024.0 + 245.0 / 3072.0 + 49.0 / 5120.0 + 5.0 / 7168.0,
}

# CPML: single-pole CFS profile, quartic sigma, kappa = 1, alpha = 0.
CPML_SIGMA_ORDER = 4
CPML_SIGMA_MAX_FACTOR = 0.8
CPML_FACES = ("x0", "xm", "y0", "ym", "z0", "zm")

# Native option word (storage_type).
STORAGE_FLOAT32 = 0
STORAGE_FLOAT16 = 1
STORAGE_BFLOAT16 = 2
STORAGE_INT8 = 3          # INT8 codes with one FP32 scale per 32-cell tile (this library's layout)
STORAGE_FP8_E4M3 = 4      # FP8 E4M3 with one FP32 scale per 256-cell tile
STORAGE_FLOAT64 = 5       # exact histories of the FP64 runs
STORAGE_KIND_MASK = 0x0F
RHS_FROM_E = 1 << 4
PHYSICAL_HISTORY = 1 << 5
SOLVER_TM2D = 1 << 6
HISTORY_DISABLED = 1 << 26

NATIVE_ABI_VERSION = 6
MAX_SHOTS_PER_CALL = 65535
INT32_MAX = 2**31 - 1

# Indices (within the 24 CPML arrays) that couple only Ex, Ey and Hz in 2D.
TM2D_INACTIVE_PHI = (0, 3, 4, 7, 8, 11, 12, 15)
TM2D_INACTIVE_STATES = (0, 1, 5) + tuple(6 + i for i in TM2D_INACTIVE_PHI)

DEFAULT_PML_THICKNESS = 10
DEFAULT_FDTD_ORDER = 2
DEFAULT_GRADIENT_MODE = 2
DEFAULT_SOURCE_COMPONENT = 2
DEFAULT_RECEIVER_COMPONENT = 2
DEFAULT_SAMPLING_INTERVAL = 1

STATE_COUNT = 30
STATE_NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz") + tuple(
    f"{face}{field}Phi{index}" for face in CPML_FACES for field in ("E", "H") for index in (1, 2)
)
