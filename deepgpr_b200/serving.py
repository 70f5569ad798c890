"""Serving loop: continuous batching of forward and gradient solves on one GPU.

A ``SolveServer`` accepts requests -- 2D or 3D forward solves and L2-misfit
gradient solves of any grid size, nt, shot count and order -- as they arrive,
and admits them in arrival order as soon as a slot and enough device memory are
free.  Admission is by HBM footprint: ``footprint_bytes`` estimates every
device buffer a request holds while it runs (fields and CPML state, material
and coefficient arrays, the solver's working copies, histories, adjoint state
and scratch); a request whose footprint alone exceeds the budget is rejected
when it is submitted.

Run a serving process with ``PYTORCH_CUDA_ALLOC_CONF=backend:cudaMallocAsync``:
then the buffers of all requests (PyTorch's and the solver's scratch) come
from one stream-ordered pool shared by every slot and stay mapped between
requests.  PyTorch's default caching allocator keeps one cache per stream, so
slots cannot reuse each other's freed buffers and a size-varied stream of
requests keeps allocating (and synchronising the device).

Each slot is a host thread with its own CUDA stream; inside the native library
every host thread has its own work and side streams.  The kernels of all
admitted requests therefore run concurrently on the GPU, and every solve's time
loop is replayed from CUDA graphs captured per 32-step chunk.  Gradient solves
call the native forward and adjoint directly from the slot's thread
(``solver.misfit_gradient``), so they do not queue behind PyTorch's single
per-device autograd thread.  They keep the exact FP32 E-only histories by
default (``history="fp32"``).  ``history="bf16"`` keeps BF16 E and R (the
same bytes as FP32 E alone; on 3D gradient requests of 96^3-160^3 cells,
1-4 shots and 80-150 steps the eps_r gradient within 1e-3 of an FP64 solve,
sigma within about 2e-3); ``history="int8"`` stores one-byte INT8 codes with
per-tile scales and
``"fp8"`` E4M3 codes on the same tiles, which halve the history footprint at
a gradient error of about 0.5-2 % on those requests (0.1-0.5 % on small
test problems).

The result of a request does not depend on what else is running: the kernels
are deterministic and no arithmetic is shared between requests.

``run_plain`` is the comparison path: the same requests, one after another,
through ``compute`` (and ``loss.backward()`` for gradients) on the caller's
thread -- plain per-request launches.
"""

from __future__ import annotations

import collections
import math
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass
from typing import Any, Callable, Deque, Dict, List, Optional, Sequence, Tuple

import torch

from .grid import extended_shape, normalize_pml_thickness

__all__ = ["SolveRequest", "SolveResult", "SolveServer", "footprint_bytes", "run_plain", "percentile"]


@dataclass
class SolveRequest:
    """One forward or gradient solve.

    ``kind`` is ``"forward"`` (returns the receiver data) or ``"gradient"``
    (returns the L2 misfit against ``observed`` and its gradients with respect
    to ``eps_r`` and ``sigma``).  Tensors may live on the host or the device;
    the server copies them to its device.  The remaining fields are
    ``compute``'s arguments of the same names.
    """

    kind: str
    eps_r: torch.Tensor
    sigma: torch.Tensor
    source_amplitudes: torch.Tensor
    source_location: torch.Tensor
    receiver_location: torch.Tensor
    dx: Any
    dt: float
    pmlthick: Any = 10
    fdtd_order: int = 4
    mode: int = 2
    observed: Optional[torch.Tensor] = None
    tag: Any = None


@dataclass
class SolveResult:
    """Outputs of a request (on the host) and its timing."""

    tag: Any
    kind: str
    receivers: Optional[torch.Tensor] = None
    loss: Optional[float] = None
    grad_eps_r: Optional[torch.Tensor] = None
    grad_sigma: Optional[torch.Tensor] = None
    submitted: float = 0.0
    started: float = 0.0
    finished: float = 0.0
    footprint: int = 0

    @property
    def latency(self) -> float:
        """Seconds from submission to the result on the host."""
        return self.finished - self.submitted


def _field_cells(ext: Sequence[int]) -> int:
    return (ext[0] + 1) * (ext[1] + 1) * (ext[2] + 1)


HISTORY_FORMATS = ("fp8", "int8", "bf16", "fp32")


def history_options(history: str) -> Dict[str, Any]:
    """``compute`` keywords of a served history format."""
    if history in ("fp8", "int8"):
        return {"wavefield_compression": history}
    if history == "bf16":
        return {"wavefield_compression": "none", "wavefield_storage_dtype": torch.bfloat16}
    if history == "fp32":
        return {"wavefield_compression": "none"}
    raise ValueError(f"unknown history format {history!r}")


def footprint_bytes(req: SolveRequest, history: str = "fp32") -> int:
    """Upper estimate of the device memory a request holds while it runs.

    Counts, in FP32 unless stated: the 6 field and 24 CPML state arrays (and
    their adjoint copies for a gradient), 3 padded material and 6 coefficient
    arrays, the solver's working copy of the fields and 5 coefficients (z
    pitch rounded up to 32), receivers (observed data and residual for a
    gradient), the histories (INT8 / FP8: E and R, one byte each plus one scale
    per 32 values; BF16: E and R, two bytes each; FP32: E only, plus the last
    E^(n+1) frame), the CPML weight
    scratch and the FP64 gradient accumulators, plus 25 % and 64 MiB of
    margin for the allocators' rounding and the point tables.
    """
    eps = req.eps_r
    phys = tuple(eps.shape) + (1,) * (3 - eps.dim())
    pml = normalize_pml_thickness(req.pmlthick, phys[2])
    ext = extended_shape(phys, pml)
    shots = int(req.source_location.shape[0])
    w = req.source_amplitudes
    nt = int(w.shape[0] if w.dim() == 1 else w.shape[1])
    nrx = int(req.receiver_location.shape[1])
    fc = _field_cells(ext)
    nxp, nyp, nzp = ext[0] + 1, ext[1] + 1, (ext[2] + 1 + 31) // 32 * 32
    work = (6 * shots + 5) * nxp * nyp * nzp * 4
    faces = max(nyp * nzp, nxp * nzp, nxp * nyp)
    psi = 24 * shots * (max(pml) + 1) * faces * 4
    fields = 6 * shots * fc * 4
    model = (3 + 6) * fc * 4
    rx = shots * nt * nrx * 4
    total = fields + psi + model + work + rx
    if req.kind == "gradient":
        ncomp = 3 if req.mode == 3 else 1
        box = ext[0] * ext[1] * ext[2]
        if history in ("fp8", "int8"):
            frames = 2 * (nt + 1) * ncomp * shots * box
            hist = frames + frames // 32 * 4
        elif history == "bf16":
            hist = 2 * (nt + 1) * ncomp * shots * box * 2
        else:
            hist = (nt + 1) * ncomp * shots * box * 4
        total += hist + fields + psi + work + 2 * rx + psi + 2 * box * 8 + 2 * box * 4
    return int(total * 1.25) + (64 << 20)


def percentile(values: Sequence[float], q: float) -> float:
    """Nearest-rank percentile (q in [0, 100])."""
    if not values:
        return float("nan")
    v = sorted(values)
    k = max(0, min(len(v) - 1, int(math.ceil(q / 100.0 * len(v))) - 1))
    return v[k]


def _solve(req: SolveRequest, device: torch.device, history: str, stream: torch.cuda.Stream) -> SolveResult:
    """Run one request on the calling thread and the given stream; outputs on the host."""
    import deepgpr_b200 as dg
    from deepgpr_b200.solver import misfit_gradient

    res = SolveResult(tag=req.tag, kind=req.kind)
    with torch.cuda.device(device), torch.cuda.stream(stream):
        dev = lambda t: t.to(device, non_blocking=True)  # noqa: E731
        kw = dict(dx=req.dx, dt=req.dt, pmlthick=req.pmlthick, fdtd_order=req.fdtd_order, mode=req.mode,
                  source_amplitudes=dev(req.source_amplitudes), source_location=dev(req.source_location),
                  receiver_location=dev(req.receiver_location))
        if req.kind == "forward":
            with torch.no_grad():
                out = dg.compute(device, eps_r=dev(req.eps_r), sigma=dev(req.sigma), save_wavefield_history=False,
                                 **kw)
            res.receivers = out[-1].cpu()
        elif req.kind == "gradient":
            if req.observed is None:
                raise ValueError("a gradient request needs observed receiver data")
            loss, ge, gs, _ = misfit_gradient(device, dev(req.observed), eps_r=dev(req.eps_r),
                                              sigma=dev(req.sigma), **history_options(history), **kw)
            res.loss = float(loss.cpu())
            res.grad_eps_r = ge.cpu()
            res.grad_sigma = gs.cpu()
        else:
            raise ValueError(f"unknown request kind {req.kind!r}")
    return res


class SolveServer:
    """Continuous-batching request loop on one GPU.

    ``slots`` requests run at a time (one host thread and CUDA stream each);
    requests wait in arrival order until a slot is free and their footprint
    fits in ``memory_budget`` bytes (default: 80 % of the device memory that is
    free or cached unused by PyTorch at start).  ``submit`` returns a ``concurrent.futures.Future`` of a
    ``SolveResult``.  ``run`` (a callable ``(request, slot) -> SolveResult``)
    replaces the GPU solve, for tests of the admission logic.
    """

    def __init__(self, device: Any = None, slots: int = 8, memory_budget: Optional[int] = None,
                 history: str = "fp32", run: Optional[Callable[[SolveRequest, int], SolveResult]] = None,
                 footprint: Optional[Callable[[SolveRequest], int]] = None):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        if history not in HISTORY_FORMATS:
            raise ValueError("history must be 'fp8', 'int8', 'bf16' or 'fp32'")
        self.history = history
        if device is not None:
            self.device = torch.device(device)
        elif run is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        else:
            self.device = torch.device("cpu")
        if memory_budget is None:
            if run is not None or self.device.type != "cuda":
                raise ValueError("memory_budget is required without a CUDA device")
            # free device memory plus what PyTorch's caching allocator holds unused
            free, _ = torch.cuda.mem_get_info(self.device)
            cached = torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
            memory_budget = int(0.8 * (free + cached))
        self.budget = int(memory_budget)
        if run is None:
            # keep freed device memory mapped between requests (released at close).
            # With PyTorch's cudaMallocAsync backend every buffer of every slot comes
            # from the same stream-ordered pool, so the whole budget is retained there;
            # with the caching allocator (per-stream caches) only the solver's
            # scratch is, a quarter of the budget, so that PyTorch still finds memory.
            from . import native

            shared_pool = torch.cuda.get_allocator_backend() == "cudaMallocAsync"
            with torch.cuda.device(self.device):
                native.set_scratch_retention(self.budget if shared_pool else self.budget // 4)
        self._footprint = footprint or (lambda r: footprint_bytes(r, history))
        self._run = run
        self._cond = threading.Condition()
        self._queue: Deque[Tuple[SolveRequest, Future, float, int]] = collections.deque()
        self._reserved = 0
        self._running = 0
        self._closed = False
        self.peak_reserved = 0
        self.peak_running = 0
        self.completed: List[SolveResult] = []
        self.admitted: List[Any] = []   # request tags in admission order
        self._streams: List[Optional[torch.cuda.Stream]] = []
        self._threads = []
        for slot in range(slots):
            self._streams.append(torch.cuda.Stream(self.device) if run is None else None)
            t = threading.Thread(target=self._worker, args=(slot,), name=f"solve-slot-{slot}", daemon=True)
            t.start()
            self._threads.append(t)

    def submit(self, req: SolveRequest) -> Future:
        """Queue a request; its future resolves to a ``SolveResult`` (or raises)."""
        fut: Future = Future()
        fp = int(self._footprint(req))
        if fp > self.budget:
            fut.set_exception(MemoryError(
                f"request {req.tag!r} needs ~{fp / 2**30:.2f} GiB of device memory, more than the server's "
                f"budget of {self.budget / 2**30:.2f} GiB"))
            return fut
        with self._cond:
            if self._closed:
                raise RuntimeError("the server is closed")
            self._queue.append((req, fut, time.perf_counter(), fp))
            self._cond.notify_all()
        return fut

    def _admit(self) -> Optional[Tuple[SolveRequest, Future, float, int]]:
        with self._cond:
            while True:
                if self._queue:
                    fp = self._queue[0][3]
                    if self._reserved + fp <= self.budget:
                        item = self._queue.popleft()
                        self.admitted.append(item[0].tag)
                        self._reserved += fp
                        self._running += 1
                        self.peak_reserved = max(self.peak_reserved, self._reserved)
                        self.peak_running = max(self.peak_running, self._running)
                        self._cond.notify_all()
                        return item
                elif self._closed:
                    return None
                self._cond.wait()

    def _worker(self, slot: int) -> None:
        while True:
            item = self._admit()
            if item is None:
                return
            req, fut, submitted, fp = item
            started = time.perf_counter()
            try:
                if self._run is not None:
                    res = self._run(req, slot)
                else:
                    res = _solve(req, self.device, self.history, self._streams[slot])
                res.submitted, res.started, res.finished, res.footprint = submitted, started, time.perf_counter(), fp
            except BaseException as exc:  # the request fails, the slot goes on
                with self._cond:
                    self._reserved -= fp
                    self._running -= 1
                    self._cond.notify_all()
                fut.set_exception(exc)
                continue
            with self._cond:
                self._reserved -= fp
                self._running -= 1
                self.completed.append(res)
                self._cond.notify_all()
            fut.set_result(res)

    def close(self, wait: bool = True) -> None:
        """Stop accepting requests; queued requests still run."""
        with self._cond:
            self._closed = True
            self._cond.notify_all()
        if wait:
            for t in self._threads:
                t.join()
            if self._run is None:
                from . import native

                with torch.cuda.device(self.device):
                    torch.cuda.synchronize()
                    native.set_scratch_retention(0)

    def __enter__(self) -> "SolveServer":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def stats(self, results: Optional[Sequence[SolveResult]] = None) -> Dict[str, Any]:
        """solves/s over the span of the results, p50/p99 latency, peak concurrency."""
        res = list(self.completed if results is None else results)
        if not res:
            return {"solves": 0}
        span = max(r.finished for r in res) - min(r.submitted for r in res)
        lat = [r.latency for r in res]
        return {"solves": len(res), "solves_per_s": len(res) / span if span > 0 else float("inf"),
                "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
                "peak_running": self.peak_running, "peak_reserved_bytes": self.peak_reserved,
                "budget_bytes": self.budget}


def run_plain(requests: Sequence[SolveRequest], device: Any, arrivals: Optional[Sequence[float]] = None,
              history: str = "fp32") -> List[SolveResult]:
    """The requests one after another through ``compute`` (plus ``loss.backward()``
    for gradients) on this thread: plain per-request launches.  ``arrivals``
    (seconds from the start) delay a request until its arrival time."""
    import deepgpr_b200 as dg

    device = torch.device(device)
    out = []
    t0 = time.perf_counter()
    for n, req in enumerate(requests):
        if arrivals is not None:
            wait = arrivals[n] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        submitted = t0 + (arrivals[n] if arrivals is not None else 0.0)
        res = SolveResult(tag=req.tag, kind=req.kind, submitted=submitted, started=time.perf_counter())
        dev = lambda t: t.to(device)  # noqa: E731
        kw = dict(dx=req.dx, dt=req.dt, pmlthick=req.pmlthick, fdtd_order=req.fdtd_order, mode=req.mode,
                  source_amplitudes=dev(req.source_amplitudes), source_location=dev(req.source_location),
                  receiver_location=dev(req.receiver_location))
        if req.kind == "forward":
            with torch.no_grad():
                res.receivers = dg.compute(device, eps_r=dev(req.eps_r), sigma=dev(req.sigma),
                                           save_wavefield_history=False, **kw)[-1].cpu()
        else:
            eps = dev(req.eps_r).requires_grad_(True)
            sig = dev(req.sigma).requires_grad_(True)
            rx = dg.compute(device, eps_r=eps, sigma=sig, **history_options(history), **kw)[-1]
            loss = 0.5 * ((rx - dev(req.observed)) ** 2).sum()
            loss.backward()
            res.loss = float(loss.detach().cpu())
            res.grad_eps_r = eps.grad.cpu()
            res.grad_sigma = sig.grad.cpu()
        res.finished = time.perf_counter()
        out.append(res)
    return out
