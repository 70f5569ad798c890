"""Grid spacing, CPML thickness and the CFL limit.

Semantics follow src/DeepGPR/preprocessing/grid.py:17-116 and
src/DeepGPR/preprocessing/stability.py:20-114.
"""

from __future__ import annotations

import math
import numbers
from typing import Any, Optional, Sequence, Tuple

import torch

from .config import INT32_MAX, SPEED_OF_LIGHT, STENCIL_TAP_SUMS, SUPPORTED_FDTD_ORDERS
from .errors import CFLConditionError

Spacing = Tuple[float, float, float]


def positive_finite(name: str, value: Any) -> float:
    """Return ``value`` as a finite positive float or raise ``ValueError``."""
    if isinstance(value, bool):
        raise TypeError(f"{name} must be a finite positive scalar.")
    if torch.is_tensor(value):
        if value.numel() != 1:
            raise ValueError(f"{name} must be a scalar.")
        value = value.detach().item()
    try:
        out = float(value)
    except (TypeError, ValueError) as exc:
        raise TypeError(f"{name} must be a finite positive scalar.") from exc
    if not math.isfinite(out) or out <= 0.0:
        raise ValueError(f"{name} must be a finite positive scalar.")
    return out


def normalize_grid_spacing(value: Any) -> Spacing:
    """``dx`` as ``(dx, dy, dz)``: a scalar, a 3-sequence, or a 1/3-element tensor."""
    if torch.is_tensor(value):
        if value.numel() == 1:
            items = [value.detach().item()] * 3
        elif value.numel() == 3:
            items = value.detach().cpu().reshape(-1).tolist()
        else:
            raise ValueError("dx tensor must contain either one or three values.")
    elif isinstance(value, numbers.Real) and not isinstance(value, bool):
        items = [value] * 3
    elif isinstance(value, (list, tuple)):
        if len(value) != 3:
            raise ValueError("dx list or tuple must contain exactly three values.")
        items = list(value)
    else:
        raise TypeError("dx must be a positive scalar or a three-value list, tuple, or tensor.")
    try:
        spacing = tuple(float(v) for v in items)
    except (TypeError, ValueError) as exc:
        raise TypeError("dx, dy, and dz must be finite positive scalars.") from exc
    if any(not math.isfinite(v) or v <= 0.0 for v in spacing):
        raise ValueError("dx, dy, and dz must be finite positive scalars.")
    return spacing  # type: ignore[return-value]


def normalize_pml_thickness(p: Any, nz: int) -> Tuple[int, ...]:
    """Six face thicknesses ``[x0, xm, y0, ym, z0, zm]`` from an int, 4 or 6 values.

    An integer applies to every active face (z faces are zero in 2D, ``nz == 1``).
    """
    if isinstance(p, bool):
        raise TypeError("PML thickness must contain integer values, not bool.")
    if isinstance(p, numbers.Integral):
        v = int(p)
        values = [v, v, v, v, 0, 0] if nz == 1 else [v] * 6
    elif isinstance(p, (list, tuple)) or torch.is_tensor(p):
        if torch.is_tensor(p):
            if p.ndim != 1:
                raise ValueError("PML thickness tensor must be one-dimensional.")
            items = p.detach().cpu().tolist()
        else:
            items = list(p)
        if len(items) == 4:
            values = [*items, 0, 0]
        elif len(items) == 6:
            values = items
        else:
            raise ValueError(f"Unsupported PML length: {len(items)}. Must be 4 or 6.")
    else:
        raise TypeError(f"Unsupported PML thickness type: {type(p)}")
    out = []
    for v in values:
        if isinstance(v, bool):
            raise TypeError("PML thickness must contain integer values, not bool.")
        try:
            f = float(v)
        except (TypeError, ValueError, OverflowError) as exc:
            raise TypeError("PML thickness must contain finite integer values.") from exc
        if not math.isfinite(f) or not f.is_integer():
            raise ValueError("PML thickness must contain finite integer values.")
        iv = int(f)
        if iv < 0 or iv > INT32_MAX:
            raise ValueError("PML thickness values must fit in non-negative int32.")
        out.append(iv)
    return tuple(out)


def max_stable_time_step(
    dx: Any, nx: int, ny: int, nz: int, *, fdtd_order: int = 2, min_er_mr: Optional[float] = None
) -> float:
    """Largest stable ``dt``: ``sqrt(min eps_r mu_r) / (c * S_order * sqrt(sum 1/d^2))``.

    Only axes with more than one cell contribute (src/DeepGPR/preprocessing/stability.py:20-68).
    """
    spacing = normalize_grid_spacing(dx)
    if fdtd_order not in SUPPORTED_FDTD_ORDERS:
        raise ValueError("fdtd_order must be one of 2, 4, or 8.")
    inv2 = sum(1.0 / (d * d) for n, d in zip((nx, ny, nz), spacing) if n > 1)
    if inv2 == 0.0:
        raise ValueError("At least one model dimension must contain more than one cell.")
    factor = 1.0
    if min_er_mr is not None:
        v = float(min_er_mr)
        if not math.isfinite(v) or v <= 0.0:
            raise ValueError("epsilon_r * mu_r must be finite and positive for the CFL check.")
        factor = math.sqrt(v)
    return factor / (SPEED_OF_LIGHT * STENCIL_TAP_SUMS[fdtd_order] * math.sqrt(inv2))


def check_cfl(dx: Any, dt: Any, nx: int, ny: int, nz: int, *, fdtd_order: int, min_er_mr: float) -> None:
    """Raise :class:`CFLConditionError` when ``dt`` exceeds the stable limit."""
    step = positive_finite("dt", dt)
    limit = max_stable_time_step(dx, nx, ny, nz, fdtd_order=fdtd_order, min_er_mr=min_er_mr)
    if step > limit:
        raise CFLConditionError(f"Does not meet CFL conditions: dt={step:.3e} > dt_max={limit:.3e}")


def extended_shape(shape: Sequence[int], pml: Sequence[int]) -> Tuple[int, int, int]:
    """Solver-grid shape of a physical model with CPML faces ``pml``."""
    return tuple(int(n) + int(pml[2 * a]) + int(pml[2 * a + 1]) for a, n in enumerate(shape))  # type: ignore


def physical_shape(shape: Sequence[int], pml: Sequence[int]) -> Tuple[int, int, int]:
    """Inverse of :func:`extended_shape`."""
    return tuple(int(n) - int(pml[2 * a]) - int(pml[2 * a + 1]) for a, n in enumerate(shape))  # type: ignore
