"""Wavefield-history options, the native ``storage_type`` word and buffer layouts.

History layout (as src/DeepGPR/solver/storage.py:359-369): ``E_saved`` is
``(nt_saved, nstep, hx, hy, hz)`` for gradient mode 2 (Ez only) and
``(3, nt_saved, nstep, hx, hy, hz)`` for mode 3.  The box ``(hx, hy, hz)`` is
the extended grid or, with ``"physical"``, the physical model only
(storage.py:161-195).

One-byte histories keep one byte per value followed, after 256-byte
alignment, by one FP32 scale per (component, saved step, shot, tile); a tile
is 32 cells of one row (32 z columns of an (x, y) row in 3D, 32 y columns of
an x row on the 2D TM path), and they always keep the E and R pair:

* ``wavefield_compression="fp8"`` (kind 4): E4M3 codes, value ``code * scale``
  with ``scale = absmax(tile) / 448`` -- about 4 significant bits for every
  value of the tile;
* ``wavefield_compression="int8"`` (kind 3, the reference's option name):
  signed integer codes in [-127, 127] rounded to nearest, value
  ``code * scale`` with ``scale = absmax(tile) / 127`` -- a uniform grid, so the
  tile's largest values, which dominate the imaging sums, keep 8 bits.  The
  reference's INT8 history uses its own block shape and packing
  (src/DeepGPR/solver/storage.py:372-414); this one shares the FP8 layout, so
  the reference's Python does not hand its INT8 layout to this library
  (``deepgpr_supports_int8_wavefield`` is 0) while this package's own
  ``compute`` accepts the option.
"""

from __future__ import annotations

from typing import Any, NamedTuple, Optional, Sequence, Tuple

import torch

from .config import (
    HISTORY_DISABLED,
    PHYSICAL_HISTORY,
    RHS_FROM_E,
    SOLVER_TM2D,
    STORAGE_BFLOAT16,
    STORAGE_FLOAT16,
    STORAGE_FLOAT32,
    STORAGE_FLOAT64,
    STORAGE_FP8_E4M3,
    STORAGE_INT8,
)

TILE_Z, TILE_Y, TILE_2D = 32, 1, 32

DTYPE_ALIASES = {
    "float32": torch.float32, "fp32": torch.float32, "float": torch.float32,
    "float16": torch.float16, "fp16": torch.float16, "half": torch.float16,
    "bfloat16": torch.bfloat16, "bf16": torch.bfloat16,
}
KIND_OF_DTYPE = {torch.float32: STORAGE_FLOAT32, torch.float16: STORAGE_FLOAT16, torch.bfloat16: STORAGE_BFLOAT16}


class StorageConfig(NamedTuple):
    """Resolved history storage: element dtype (or FP8) and native kind code."""

    dtype: torch.dtype
    compression: str   # "none" or "fp8"
    kind: int


def normalize_storage_dtype(value: Any) -> torch.dtype:
    if isinstance(value, str):
        value = DTYPE_ALIASES.get(value.lower())
    if value not in KIND_OF_DTYPE:
        raise ValueError("wavefield_storage_dtype must be float32, float16, or bfloat16.")
    return value


def normalize_compression(value: Any) -> str:
    if value is None:
        return "none"
    if not isinstance(value, str):
        raise TypeError("wavefield_compression must be 'none', 'fp8', 'int8', or 'zfp'.")
    value = value.lower()
    if value not in ("none", "fp8", "int8", "zfp"):
        raise ValueError("wavefield_compression must be 'none', 'fp8', 'int8', or 'zfp'.")
    if value == "zfp":
        raise NotImplementedError("wavefield_compression='zfp' has no block decoder in this library; use 'int8'.")
    return value


ONE_BYTE = ("fp8", "int8")   # compressions stored as one byte per value plus tile scales


def normalize_choice(name: str, value: Any, choices: Sequence[str]) -> str:
    msg = f"{name} must be one of {', '.join(repr(c) for c in choices)}."
    if not isinstance(value, str):
        raise TypeError(msg)
    value = value.lower()
    if value not in choices:
        raise ValueError(msg)
    return value


def history_box(
    nx: int, ny: int, nz: int, pml: Sequence[int], region: str
) -> Tuple[Tuple[int, int, int], Tuple[int, int, int]]:
    """Origin and extent of the saved cells (extended grid or physical model)."""
    if region != "physical":
        return (0, 0, 0), (nx, ny, nz)
    origin = (int(pml[0]), int(pml[2]), int(pml[4]))
    extent = (nx - pml[0] - pml[1], ny - pml[2] - pml[3], nz - pml[4] - pml[5])
    return origin, tuple(int(v) for v in extent)  # type: ignore[return-value]


def saved_time_steps(nt: int, interval: int) -> int:
    return (nt + interval - 1) // interval


def saved_history_shape(mode: int, nt_saved: int, nstep: int, hx: int, hy: int, hz: int) -> Tuple[int, ...]:
    if mode == 3:
        return (3, nt_saved, nstep, hx, hy, hz)
    return (nt_saved, nstep, hx, hy, hz)


def fp8_tiles(field_shape: Tuple[int, int, int], tm2d: bool) -> int:
    """Scale tiles per (component, saved step, shot) for a field grid ``(NX, NY, NZ)``."""
    NX, NY, NZ = field_shape
    if tm2d:
        return NX * ((NY + TILE_2D - 1) // TILE_2D)
    return NX * ((NY + TILE_Y - 1) // TILE_Y) * ((NZ + TILE_Z - 1) // TILE_Z)


def fp8_tile_of(i: torch.Tensor, j: torch.Tensor, k: torch.Tensor, field_shape: Tuple[int, int, int],
                tm2d: bool) -> torch.Tensor:
    NX, NY, NZ = field_shape
    if tm2d:
        return i * ((NY + TILE_2D - 1) // TILE_2D) + j // TILE_2D
    nyt, nzt = (NY + TILE_Y - 1) // TILE_Y, (NZ + TILE_Z - 1) // TILE_Z
    return (i * nyt + j // TILE_Y) * nzt + k // TILE_Z


def fp8_history_bytes(ncomp: int, nt_saved: int, nstep: int, box_cells: int, field_shape: Tuple[int, int, int],
                      tm2d: bool) -> int:
    """Bytes of one FP8 history buffer: aligned payload plus the tile scales."""
    values = ncomp * nt_saved * nstep * box_cells
    return (values + 255) // 256 * 256 + ncomp * nt_saved * nstep * fp8_tiles(field_shape, tm2d) * 4


def encode_storage_type(
    config: StorageConfig, save_history: bool, rhs_from_e: bool = False, physical: bool = False, tm2d: bool = False
) -> int:
    """Pack the native option word (src/DeepGPR/solver/storage.py:322-356)."""
    word = config.kind
    if not save_history:
        word |= HISTORY_DISABLED
    else:
        if rhs_from_e:
            word |= RHS_FROM_E
        if physical:
            word |= PHYSICAL_HISTORY
    if tm2d:
        word |= SOLVER_TM2D
    return word


def resolve_rhs_reconstruction(requested: str, interval: int, stores_history: bool, lossless: bool) -> bool:
    """E-only history (R^n rebuilt from E^n, E^(n+1)) decision (storage.py:210-262)."""
    if requested == "stored":
        return False
    if requested == "reconstructed":
        if interval != 1:
            raise ValueError(
                "wavefield_rhs_history='reconstructed' requires model_gradient_sampling_interval=1 "
                "(R^n is rebuilt from E^n and E^(n+1))."
            )
        return bool(stores_history)
    return interval == 1 and lossless and stores_history


def storage_config(dtype: torch.dtype, compression: str, precision: torch.dtype) -> StorageConfig:
    if precision == torch.float64:
        return StorageConfig(torch.float64, "none", STORAGE_FLOAT64)
    if compression == "fp8":
        return StorageConfig(torch.uint8, "fp8", STORAGE_FP8_E4M3)
    if compression == "int8":
        return StorageConfig(torch.uint8, "int8", STORAGE_INT8)
    return StorageConfig(dtype, "none", KIND_OF_DTYPE[dtype])


def allocate_history(
    config: StorageConfig, shape: Tuple[int, ...], field_shape: Tuple[int, int, int], tm2d: bool, device: Any,
    pinned: bool
) -> torch.Tensor:
    """One history buffer (``E_saved`` or ``R_saved``) for ``shape``."""
    if config.compression in ONE_BYTE:
        ncomp = shape[0] if len(shape) == 6 else 1
        nt_saved, nstep = shape[-5], shape[-4]
        box = shape[-3] * shape[-2] * shape[-1]
        nbytes = fp8_history_bytes(ncomp, nt_saved, nstep, box, field_shape, tm2d)
        return torch.empty(nbytes, dtype=torch.uint8, device=device)
    if pinned:
        return torch.empty(shape, dtype=config.dtype, device="cpu", pin_memory=True)
    return torch.empty(shape, dtype=config.dtype, device=device)


def decode_fp8_history(
    packed: torch.Tensor, shape: Sequence[int], field_shape: Tuple[int, int, int], origin: Tuple[int, int, int],
    tm2d: bool = False, compression: str = "fp8",
) -> torch.Tensor:
    """Decode a one-byte (FP8 or INT8) history into float32 of ``shape`` (diagnostics; not used by backward).

    ``field_shape`` is ``(NX, NY, NZ)`` of the field grid and ``origin`` the
    history box origin.
    """
    shape = tuple(int(v) for v in shape)
    full = shape if len(shape) == 6 else (1,) + shape
    ncomp, nt_saved, nstep, hx, hy, hz = full
    values = ncomp * nt_saved * nstep * hx * hy * hz
    codes = packed[:values].view(torch.float8_e4m3fn if compression == "fp8" else torch.int8)
    payload = codes.to(torch.float32).reshape(full)
    tiles = fp8_tiles(field_shape, tm2d)
    offset = (values + 255) // 256 * 256
    scales = packed[offset : offset + ncomp * nt_saved * nstep * tiles * 4].view(torch.float32)
    scales = scales.reshape(ncomp, nt_saved, nstep, tiles)
    dev = packed.device
    ii = torch.arange(hx, device=dev).view(hx, 1, 1) + origin[0]
    jj = torch.arange(hy, device=dev).view(1, hy, 1) + origin[1]
    kk = torch.arange(hz, device=dev).view(1, 1, hz) + origin[2]
    tile = fp8_tile_of(ii, jj, kk, field_shape, tm2d).expand(hx, hy, hz)
    out = payload * scales[:, :, :, tile.reshape(-1)].reshape(ncomp, nt_saved, nstep, hx, hy, hz)
    return out if len(shape) == 6 else out[0]


def optional_tensor(t: Optional[torch.Tensor], device: Any, dtype: torch.dtype) -> torch.Tensor:
    return t if t is not None else torch.empty(0, device=device, dtype=dtype)
