"""Segment checkpointing with recompute: gradients whose wavefield history exceeds HBM.

The reference leaves this to its users: they split ``nt`` into segments, pass
each segment's final 30 states (fields and CPML arrays, zeroed by
``checkpoint_initial_field``) to the next ``compute`` call and let autograd chain
them (src/DeepGPR/solver/fields.py:63-143, docs/API.md:344-359,
tests/test_external_pml.py:145-191).  That still keeps every segment's history
alive until the backward pass.  Here the same segmentation runs inside one
autograd node, with recompute:

* forward: the time loop runs in segments of ``S`` steps *without* history;
  the 30 states at each segment start are kept on the device (a checkpoint);
* backward: for the segments in reverse order, the segment's checkpoint is
  restored, the segment is solved again *with* its history, and the native
  adjoint of that segment runs at once; its history is then released.  The
  adjoint states (lambda of the 30 states) are handed from one segment to the
  one before it, exactly as the single-call adjoint carries them between its
  time steps.

Peak device memory is one segment's history plus the checkpoints instead of
the whole history.  When even the checkpoints of all shots do not fit, the
shots are processed in batches in the backward pass: each batch first re-runs
its forward to build its own checkpoints (one more forward pass).  Shots are
independent; they meet only in the sums of the material and source gradients.

Receivers and final states are bit-for-bit those of the single-call solve
(the same kernels on the same values), and so are the adjoint states; the
material gradients differ only in where the FP64 accumulation of each
segment is rounded into the FP32 output.
"""

from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import torch

from . import native
from .config import STATE_COUNT, TM2D_INACTIVE_STATES
from .storage import allocate_history, encode_storage_type, fp8_history_bytes, saved_history_shape


@dataclasses.dataclass(frozen=True)
class SegmentPlan:
    """How a checkpointed gradient runs: shots per batch and time steps per segment."""

    shot_batch: int
    segment_steps: int
    nsegments: int
    peak_bytes: int
    forward_passes: int   # forward solves per gradient: 2, or 3 when the shots run in batches


def state_bytes_per_shot(states: Sequence[torch.Tensor], nshot: int) -> int:
    return sum(t.numel() * t.element_size() for t in states) // max(1, nshot)


def history_bytes_per_step(cfg, nshot: int = 1) -> int:
    """Device bytes of the history of one saved step of ``nshot`` shots (E, and R unless rebuilt from E)."""
    shape = saved_history_shape(cfg.mode, 1, nshot, *cfg.history_cells)
    if cfg.storage.compression in ("fp8", "int8"):
        ncomp = shape[0] if len(shape) == 6 else 1
        per = fp8_history_bytes(ncomp, 1, nshot, math.prod(shape[-3:]), cfg.field_shape, cfg.tm2d)
    else:
        per = math.prod(shape) * torch.empty(0, dtype=cfg.storage.dtype).element_size()
    return per if cfg.reconstruct_rhs else 2 * per


def plan_segments(cfg, state_bytes: int, budget_bytes: int, segment_steps: Optional[int] = None,
                  shot_batch: Optional[int] = None) -> SegmentPlan:
    """Largest shot batch, then the longest segment, whose peak memory fits ``budget_bytes``.

    Peak memory of a batch of B shots with segments of S steps: the
    checkpoints (B states per segment), one segment's history, and about
    four more states per shot of the batch (the live fields, the adjoint
    states and the solver's working copies), on top of the states and
    adjoint states of all shots and the gradient accumulators.  S is a
    multiple of the history sampling interval, so every segment saves the
    same steps the single call would.
    """
    nt, nshot, interval = cfg.nt, cfg.nstep, cfg.interval
    hist = history_bytes_per_step(cfg)
    fixed = 3 * nshot * state_bytes + 4 * 8 * cfg.nx * cfg.ny * cfg.nz

    def peak(b: int, s: int) -> int:
        nseg = -(-nt // s)
        saved = -(-s // interval) + 1
        return b * (state_bytes * (nseg + 4) + hist * saved) + fixed

    batches = [shot_batch] if shot_batch else sorted({max(1, nshot // d) for d in range(1, nshot + 1)}, reverse=True)
    for b in batches:
        if segment_steps:
            cands = [segment_steps]
        else:
            cands = sorted({min(nt, interval * k) for k in range(1, -(-nt // interval) + 1)}, reverse=True)
        for s in cands:
            if s % interval and s != nt:
                continue
            if peak(b, s) <= budget_bytes or (segment_steps and shot_batch):
                nseg = -(-nt // s)
                return SegmentPlan(b, s, nseg, peak(b, s), 2 if b >= nshot else 3)
    raise MemoryError(f"no checkpoint plan fits {budget_bytes / 2**30:.1f} GiB: one shot with one-step segments "
                      f"needs {peak(1, interval) / 2**30:.1f} GiB")


def allocate_history_bytes(config, shape, field_shape, tm2d) -> int:
    """Bytes of a one-byte history of ``shape`` (payload and tile scales)."""
    ncomp = shape[0] if len(shape) == 6 else 1
    return fp8_history_bytes(ncomp, shape[-5], shape[-4], math.prod(shape[-3:]), field_shape, tm2d)


def _slice_states(states: Sequence[torch.Tensor], b0: int, b1: int) -> List[torch.Tensor]:
    return [t[b0:b1].clone() if t.numel() else t.clone() for t in states]


def _batch_tensors(tensors, b0: int, b1: int):
    return dataclasses.replace(tensors, source_location=tensors.source_location[b0:b1].contiguous(),
                               receiver_location=tensors.receiver_location[b0:b1].contiguous())


class CheckpointedFDTDFunction(torch.autograd.Function):
    """``apply(cfg, tensors, plan, eps_r, sigma, source_amplitudes, *30 states)``.

    Returns the 30 states (advanced in place), an empty ``E_saved`` (no full
    history exists) and the receivers ``(nstep, nt, nrx)``.
    """

    @staticmethod
    def forward(ctx, cfg, tensors, plan: SegmentPlan, eps_r, sigma, source_amplitudes, *states):  # type: ignore[override]
        from .solver import forward_arguments

        if len(states) != STATE_COUNT:
            raise ValueError(f"Expected {STATE_COUNT} state tensors, got {len(states)}.")
        ctx.set_materialize_grads(False)
        dev = cfg.device
        wave = source_amplitudes.detach().contiguous()
        receivers = torch.empty((cfg.nstep, cfg.nt, cfg.nrx), device=dev, dtype=cfg.dtype)
        empty = torch.empty(0, device=dev, dtype=cfg.storage.dtype)
        stype = encode_storage_type(cfg.storage, False, False, cfg.region == "physical", cfg.tm2d)
        keep = plan.shot_batch >= cfg.nstep
        checkpoints: List[List[torch.Tensor]] = []
        initial = [t.detach().clone() for t in states] if not keep else None
        for t0 in range(0, cfg.nt, plan.segment_steps):
            t1 = min(cfg.nt, t0 + plan.segment_steps)
            if keep:
                checkpoints.append([t.detach().clone() for t in states])
            seg = dataclasses.replace(cfg, nt=t1 - t0)
            rx = torch.empty((cfg.nstep, t1 - t0, cfg.nrx), device=dev, dtype=cfg.dtype)
            args = forward_arguments(seg, tensors, states, empty, empty, rx, wave[:, t0:t1].contiguous(), stype,
                                     False)
            native.invoke(cfg.entry[0], args, fdtd_order=cfg.fdtd_order, stream=torch.cuda.current_stream(dev),
                          acc64=cfg.acc64, chunk=cfg.chunk, tuning=cfg.tuning)
            receivers[:, t0:t1] = rx
        ctx.cfg, ctx.tensors, ctx.plan = cfg, tensors, plan
        ctx.wave = wave
        ctx.checkpoints = checkpoints
        ctx.initial = initial
        ctx.want = (bool(source_amplitudes.requires_grad), bool(eps_r.requires_grad), bool(sigma.requires_grad))
        ctx.source_shape = tuple(source_amplitudes.shape)
        ctx.state_shapes = tuple(s.shape for s in states)
        ctx.mark_non_differentiable(empty)
        return (*states, empty, receivers)

    @staticmethod
    def backward(ctx, *grads):  # type: ignore[override]
        from .solver import backward_arguments, forward_arguments

        cfg, tensors, plan = ctx.cfg, ctx.tensors, ctx.plan
        if ctx.wave is None:
            raise RuntimeError("The checkpoints were already released by a previous backward pass; "
                               "re-run compute before calling backward again.")
        dev, dtype = cfg.device, cfg.dtype
        want_src, want_eps, want_sig = ctx.want
        want_model = want_eps or want_sig
        lambdas = [torch.zeros(shape, device=dev, dtype=dtype) if g is None else g.clone(memory_format=torch.contiguous_format)
                   for g, shape in zip(grads[:STATE_COUNT], ctx.state_shapes)]
        data_grad = grads[STATE_COUNT + 1]
        data_grad = (torch.zeros((cfg.nstep, cfg.nt, cfg.nrx), device=dev, dtype=dtype) if data_grad is None
                     else data_grad.to(dtype).contiguous())
        ext = (cfg.nx, cfg.ny, cfg.nz)
        grad_eps = torch.zeros(ext, device=dev, dtype=dtype) if want_eps else torch.empty(0, device=dev, dtype=dtype)
        grad_sig = torch.zeros(ext, device=dev, dtype=dtype) if want_sig else torch.empty(0, device=dev, dtype=dtype)
        grad_src = (torch.zeros(ctx.source_shape, device=dev, dtype=dtype) if want_src
                    else torch.empty(0, device=dev, dtype=dtype))
        stream = torch.cuda.current_stream(dev)
        physical = cfg.region == "physical"
        save_model = want_model
        rhs_from_e = bool(cfg.reconstruct_rhs and save_model)
        st_hist = encode_storage_type(cfg.storage, save_model, rhs_from_e, physical, cfg.tm2d)
        st_none = encode_storage_type(cfg.storage, False, False, physical, cfg.tm2d)
        empty = torch.empty(0, device=dev, dtype=cfg.storage.dtype)
        bounds = [(t0, min(cfg.nt, t0 + plan.segment_steps)) for t0 in range(0, cfg.nt, plan.segment_steps)]
        wave = ctx.wave

        for b0 in range(0, cfg.nstep, plan.shot_batch):
            b1 = min(cfg.nstep, b0 + plan.shot_batch)
            nb = b1 - b0
            bt = _batch_tensors(tensors, b0, b1)
            if ctx.checkpoints:
                ckpts = ctx.checkpoints
            else:
                # this batch's checkpoints: its forward again, without history
                ckpts = []
                cur = _slice_states(ctx.initial, b0, b1)
                for t0, t1 in bounds:
                    ckpts.append([t.clone() for t in cur])
                    seg = dataclasses.replace(cfg, nt=t1 - t0, nstep=nb)
                    rx = torch.empty((nb, t1 - t0, cfg.nrx), device=dev, dtype=dtype)
                    args = forward_arguments(seg, bt, cur, empty, empty, rx, wave[:, t0:t1].contiguous(), st_none,
                                             False)
                    native.invoke(cfg.entry[0], args, fdtd_order=cfg.fdtd_order, stream=stream, acc64=cfg.acc64,
                                  chunk=cfg.chunk, tuning=cfg.tuning)
                del cur
            lam = [t[b0:b1].clone() if t.numel() else t for t in lambdas] if plan.shot_batch < cfg.nstep else lambdas
            # one E and one R buffer of the longest segment, reused by every segment of the batch (views of
            # their leading bytes): fresh buffers per segment would fragment the allocator's cache
            e_buf = r_buf = None
            if save_model:
                nts_max = -(-plan.segment_steps // cfg.interval)
                shape = saved_history_shape(cfg.mode, nts_max, nb, *cfg.history_cells)
                e_buf = allocate_history(cfg.storage, shape, cfg.field_shape, cfg.tm2d, dev, False).reshape(-1)
                rshape = saved_history_shape(cfg.mode, 1, nb, *cfg.history_cells) if rhs_from_e else shape
                r_buf = allocate_history(cfg.storage, rshape, cfg.field_shape, cfg.tm2d, dev, False).reshape(-1)

            def history_view(buf, shape):
                if cfg.storage.compression in ("fp8", "int8"):
                    n = allocate_history_bytes(cfg.storage, shape, cfg.field_shape, cfg.tm2d)
                    return buf[:n]
                return buf[:math.prod(shape)].view(shape)

            for k in range(len(bounds) - 1, -1, -1):
                t0, t1 = bounds[k]
                seg = dataclasses.replace(cfg, nt=t1 - t0, nstep=nb)
                cur = ckpts[k]   # consumed: the solve advances it in place
                ckpts[k] = None
                e_saved, r_saved = empty, empty
                if save_model:
                    nts = -(-(t1 - t0) // cfg.interval)
                    shape = saved_history_shape(cfg.mode, nts, nb, *cfg.history_cells)
                    e_saved = history_view(e_buf, shape)
                    rshape = saved_history_shape(cfg.mode, 1, nb, *cfg.history_cells) if rhs_from_e else shape
                    r_saved = history_view(r_buf, rshape)
                rx = torch.empty((nb, t1 - t0, cfg.nrx), device=dev, dtype=dtype)
                ws = wave[:, t0:t1].contiguous()
                fargs = forward_arguments(seg, bt, cur, e_saved, r_saved, rx, ws, st_hist if save_model else st_none,
                                          save_model)
                native.invoke(cfg.entry[0], fargs, fdtd_order=cfg.fdtd_order, stream=stream, acc64=cfg.acc64,
                              chunk=cfg.chunk, tuning=cfg.tuning)
                del cur, rx
                gsrc = torch.zeros((ctx.source_shape[0], t1 - t0), device=dev, dtype=dtype) if want_src else empty.to(dtype)
                dg = data_grad[b0:b1, t0:t1].contiguous()
                bargs = backward_arguments(seg, bt, lam, e_saved, r_saved, dg, gsrc, grad_eps, grad_sig, ctx.want,
                                           st_hist if save_model else st_none)
                native.invoke(cfg.entry[1], bargs, fdtd_order=cfg.fdtd_order, stream=stream, acc64=cfg.acc64,
                              chunk=cfg.chunk, tuning=cfg.tuning)
                del e_saved, r_saved, fargs, bargs
                if want_src:
                    grad_src.view(grad_src.shape[0], -1)[:, t0:t1] += gsrc
            del e_buf, r_buf
            if lam is not lambdas:
                for full, part in zip(lambdas, lam):
                    if full.numel():
                        full[b0:b1] = part
        ctx.checkpoints = None
        ctx.initial = None
        ctx.wave = None
        if cfg.tm2d:
            for i in TM2D_INACTIVE_STATES:
                lambdas[i].zero_()
        state_needs = ctx.needs_input_grad[6 : 6 + STATE_COUNT]
        return (
            None, None, None,
            grad_eps if want_eps else None,
            grad_sig if want_sig else None,
            grad_src if want_src else None,
            *(g if need else None for g, need in zip(lambdas, state_needs)),
        )
