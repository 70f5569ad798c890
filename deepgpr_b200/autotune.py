"""Launch-shape autotuner: picks the schedule of a solve by timing short probe solves.

The kernels' launch shapes follow built-in heuristics (``fdtd_api.cu``:
``tm_plan`` for the 2D TM rectangles, ``k3_layout`` / ``k3t_layout`` for the
3D x chunks).  The autotuner measures alternatives on the problem itself and
keeps the fastest, per problem signature (grid, shots, order, gradient mode,
history format, precision):

* 2D TM: interior row chunks (``tm_chunks``), frame rows per warp chunk
  (``tm_frame_rows``), time steps per captured graph (``chunk``);
* 3D: x chunks of the streamed kernels (``k3_xchunks``), the forward kernel
  family (FP32: 2 wide, 0 z-streamed, 1 TMA-staged), time steps per graph.

The knobs change how the work is split, never what is computed, so results
are the same for every choice.  A probe is a forward solve without history
over ``2 * chunk`` steps on copies of the input states; each candidate runs
once to warm up and twice timed (CUDA events on the current stream), and the
search goes coordinate by coordinate.  Choices are kept in memory and in a
JSON file (``DEEPGPR_B200_TUNE_CACHE``, default
``~/.cache/deepgpr_b200/tuning.json``) so a signature is tuned once.
"""

from __future__ import annotations

import dataclasses
import json
import os
import threading
from pathlib import Path
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import torch

from . import native
from .storage import encode_storage_type

DEFAULT = {"tm_chunks": 0, "tm_frame_rows": 0, "k3_xchunks": 0, "tma": -1, "chunk": 32}


def signature(cfg) -> str:
    """Key of a tuned choice: everything that shapes the launches."""
    return (f"{'tm2d' if cfg.tm2d else '3d'}|{cfg.nx}x{cfg.ny}x{cfg.nz}|pml{','.join(map(str, cfg.pml))}|"
            f"shots{cfg.nstep}|o{cfg.fdtd_order}|m{cfg.mode}|k{cfg.storage.kind}|{str(cfg.dtype).split('.')[-1]}")


def search_space(cfg) -> List[Tuple[str, Sequence[int]]]:
    """Coordinates searched in turn (the first value of each is the default)."""
    if cfg.tm2d:
        return [("tm_chunks", (0, 1, 2, 4, 8)), ("tm_frame_rows", (0, 4, 8, 32)), ("chunk", (32, 16, 64))]
    space: List[Tuple[str, Sequence[int]]] = [("k3_xchunks", (0, 4, 8, 12, 16, 24))]
    if cfg.dtype == torch.float32:
        space.append(("tma", (2, 0, 1)))
    space.append(("chunk", (32, 16, 64)))
    return space


def tuning_tuple(choice: Dict[str, int]) -> Tuple[int, int, int, int]:
    return (int(choice["tm_chunks"]), int(choice["tm_frame_rows"]), int(choice["k3_xchunks"]), int(choice["tma"]))


def coordinate_search(space: List[Tuple[str, Sequence[int]]], cost: Callable[[Dict[str, int]], float],
                      start: Optional[Dict[str, int]] = None) -> Tuple[Dict[str, int], Dict[str, float]]:
    """Minimise ``cost`` one coordinate at a time; returns the choice and every measured cost."""
    best = dict(DEFAULT if start is None else start)
    seen: Dict[str, float] = {}

    def run(c: Dict[str, int]) -> float:
        key = json.dumps(c, sort_keys=True)
        if key not in seen:
            seen[key] = cost(c)
        return seen[key]

    best_cost = run(best)
    for name, values in space:
        for v in values:
            cand = dict(best, **{name: v})
            c = run(cand)
            if c < best_cost:
                best, best_cost = cand, c
    return best, seen


class Autotuner:
    """Keeps tuned choices per signature (memory + JSON file)."""

    def __init__(self, path: Optional[os.PathLike] = None):
        default = Path.home() / ".cache" / "deepgpr_b200" / "tuning.json"
        self.path = Path(path or os.environ.get("DEEPGPR_B200_TUNE_CACHE", default))
        self.lock = threading.Lock()
        self.table: Dict[str, Dict[str, int]] = {}
        try:
            self.table = {k: dict(DEFAULT, **v) for k, v in json.loads(self.path.read_text()).items()}
        except (OSError, ValueError):
            self.table = {}

    def lookup(self, cfg) -> Optional[Dict[str, int]]:
        with self.lock:
            return self.table.get(signature(cfg))

    def store(self, cfg, choice: Dict[str, int]) -> None:
        with self.lock:
            self.table[signature(cfg)] = dict(choice)
            try:
                self.path.parent.mkdir(parents=True, exist_ok=True)
                tmp = self.path.with_suffix(".tmp")
                tmp.write_text(json.dumps(self.table, indent=1, sort_keys=True))
                os.replace(tmp, self.path)
            except OSError:
                pass   # the in-memory table still serves this process

    def choose(self, cfg, tensors, states: Sequence[torch.Tensor], waveform: torch.Tensor) -> Dict[str, int]:
        """The kept choice for cfg's signature, tuned now if there is none."""
        got = self.lookup(cfg)
        if got is not None:
            return got
        choice, _ = coordinate_search(search_space(cfg), lambda c: probe_ms(cfg, tensors, states, waveform, c))
        self.store(cfg, choice)
        return choice


def probe_ms(cfg, tensors, states: Sequence[torch.Tensor], waveform: torch.Tensor, choice: Dict[str, int]) -> float:
    """Milliseconds per time step of a history-free forward probe with launch choice ``choice``."""
    from .solver import forward_arguments

    steps = min(cfg.nt, 2 * int(choice["chunk"]))
    pcfg = dataclasses.replace(cfg, nt=steps)
    dev = cfg.device
    empty = torch.empty(0, device=dev, dtype=cfg.storage.dtype)
    stype = encode_storage_type(cfg.storage, False, False, cfg.region == "physical", cfg.tm2d)
    wave = waveform.detach()[:, :steps].contiguous()
    stream = torch.cuda.current_stream(dev)
    times = []
    for rep in range(3):
        probe_states = [t.detach().clone() for t in states]
        rx = torch.empty((cfg.nstep, steps, cfg.nrx), device=dev, dtype=cfg.dtype)
        args = forward_arguments(pcfg, tensors, probe_states, empty, empty, rx, wave, stype, False)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        native.invoke(cfg.entry[0], args, fdtd_order=cfg.fdtd_order, stream=stream, acc64=cfg.acc64,
                      chunk=int(choice["chunk"]), tuning=tuning_tuple(choice))
        b.record(stream)
        b.synchronize()
        if rep:   # the first run warms up (graph instantiation, caches)
            times.append(a.elapsed_time(b) / max(1, steps))
    return min(times)


_TUNER: Optional[Autotuner] = None


def default_tuner() -> Autotuner:
    global _TUNER
    if _TUNER is None:
        _TUNER = Autotuner()
    return _TUNER
