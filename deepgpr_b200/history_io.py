"""Forward wavefield history files (``save_forward_wavefield_path``).

Same file scheme as the reference (``postprocessing/io.py:17-95``,
``solver/modeling.py:640-663``): ``<directory>/forward_wavefield_<HH-MM>.pt``,
``_01``, ``_02`` ... appended when the name is taken (exclusive creation, so
processes saving into one directory in the same minute do not overwrite each
other).  A full-grid FP32/FP16/BF16 history is saved as the bare ``E_saved``
tensor (on the CPU); a physical-region history, and an FP8 history, as a
dictionary ``{"wavefield": tensor, **metadata}``.  The FP8 metadata carries
what ``load_forward_wavefield`` needs to decode the payload and its tile
scales back to float32.
"""

from __future__ import annotations

from datetime import datetime
from pathlib import Path
from typing import Any, Dict, Optional

import torch

FORWARD_WAVEFIELD_PREFIX = "forward_wavefield"
FORWARD_WAVEFIELD_TIME_FORMAT = "%H-%M"

__all__ = ["normalize_forward_wavefield_directory", "save_forward_wavefield", "load_forward_wavefield"]


def normalize_forward_wavefield_directory(value: Any) -> Optional[Path]:
    """``None`` or a directory path (created on save); an existing non-directory is an error."""
    if value is None:
        return None
    try:
        directory = Path(value).expanduser()
    except TypeError as exc:
        raise TypeError("save_forward_wavefield_path must be a string, path-like object, or None.") from exc
    if directory.exists() and not directory.is_dir():
        raise NotADirectoryError(f"save_forward_wavefield_path is not a directory: {directory}")
    return directory


def _reserve(directory: Path, label: str) -> Path:
    candidate = directory / f"{FORWARD_WAVEFIELD_PREFIX}_{label}.pt"
    n = 1
    while True:
        try:
            with open(candidate, "xb"):
                return candidate
        except FileExistsError:
            candidate = directory / f"{FORWARD_WAVEFIELD_PREFIX}_{label}_{n:02d}.pt"
            n += 1


def save_forward_wavefield(wavefield: torch.Tensor, directory: Path, run_time: datetime,
                           metadata: Optional[Dict[str, Any]] = None) -> Path:
    """Write a detached CPU copy of ``E_saved`` (with ``metadata``, as a dictionary)
    and return the resolved path."""
    directory.mkdir(parents=True, exist_ok=True)
    path = _reserve(directory, run_time.strftime(FORWARD_WAVEFIELD_TIME_FORMAT))
    cpu = wavefield.detach().to(device="cpu")
    payload: Any = {"wavefield": cpu, **metadata} if metadata is not None else cpu
    try:
        torch.save(payload, path)
    except BaseException:
        path.unlink(missing_ok=True)
        raise
    return path.resolve()


def load_forward_wavefield(path: Any) -> torch.Tensor:
    """Read a history file: the stored tensor, FP8 histories decoded to float32
    of their ``uncompressed_shape``."""
    payload = torch.load(Path(path), map_location="cpu", weights_only=True)
    if torch.is_tensor(payload):
        return payload
    wavefield = payload["wavefield"]
    if payload.get("compression") in ("fp8", "int8"):
        from .storage import decode_fp8_history

        return decode_fp8_history(wavefield, payload["uncompressed_shape"], tuple(payload["field_shape"]),
                                  tuple(payload["history_origin"]), bool(payload["tm2d"]), payload["compression"])
    return wavefield
