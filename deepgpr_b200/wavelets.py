"""Ricker source wavelet: ``(1 - 2 (pi f (t - t0))^2) exp(-(pi f (t - t0))^2)``.

Same formula as src/DeepGPR/preprocessing/wavelets.py:46-68 with the peak at
``t0 = 1/f`` by default.
"""

from __future__ import annotations

import math
from typing import Optional

import torch


def ricker(freq: float, nt: int, dt: float, peak_time: Optional[float] = None,
           dtype: torch.dtype = torch.float32) -> torch.Tensor:
    """Ricker wavelet of ``nt`` samples, returned as ``(nt,)``."""
    t0 = 1.0 / freq if peak_time is None else float(peak_time)
    t = torch.arange(nt, dtype=torch.float64) * dt - t0
    arg = (math.pi * freq * t) ** 2
    return ((1.0 - 2.0 * arg) * torch.exp(-arg)).to(dtype)
