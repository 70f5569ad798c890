"""Shot-parallel multi-GPU gradients (one process per GPU).

Shots are independent through the forward and adjoint solves; they meet only
in the sums over shots of the eps_r / sigma gradient (the imaging condition,
src/DeepGPR/lib/deepgpr_cpu.c:1690-1736) and of the source-waveform gradient
(deepgpr_cpu.c:1524-1533).  So a gradient evaluation shards the shots over
the ranks, each rank solves its share on its own GPU, and one all-reduce (sum)
of the model gradients per evaluation is the only exchange (NCCL over
NVLink on GPUs; any torch.distributed backend works).
"""

from __future__ import annotations

from typing import Iterable, Optional, Tuple

import torch


def shard_shots(nshot: int, world: int, rank: int) -> slice:
    """Contiguous, balanced share of ``range(nshot)`` for ``rank`` (may be empty)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(nshot, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def allreduce_gradients(grads: Iterable[Optional[torch.Tensor]], group=None) -> None:
    """Sum gradients over the ranks in place (one all-reduce per tensor)."""
    import torch.distributed as dist

    for g in grads:
        if g is not None:
            dist.all_reduce(g, op=dist.ReduceOp.SUM, group=group)


def shard_acquisition(source_location: torch.Tensor, receiver_location: torch.Tensor, world: int,
                      rank: int) -> Tuple[torch.Tensor, torch.Tensor, slice]:
    """This rank's source and receiver geometry."""
    sl = shard_shots(source_location.shape[0], world, rank)
    return source_location[sl], receiver_location[sl], sl


class RankFailure(RuntimeError):
    """A rank of the shot-parallel group failed, left, or did not answer in time."""


class ShotGroup:
    """Shot-parallel gradient steps with a host-side liveness check.

    Before each step's all-reduce every rank checks in on a gloo side group
    (``monitored_barrier``): a rank that raised, exited or left between steps
    makes the others raise :class:`RankFailure` within ``timeout_s`` on the
    host, before they launch the collective, instead of waiting in it.  The
    process group itself should also carry a short timeout
    (``init_process_group(timeout=...)``) so that a rank lost *inside* a
    collective ends that collective with an error.  Ranks leave only between
    steps, with no kernel or collective in flight.
    """

    def __init__(self, timeout_s: float = 30.0, group=None):
        import datetime

        import torch.distributed as dist

        self.timeout = datetime.timedelta(seconds=float(timeout_s))
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        backend = dist.get_backend(group)
        # monitored_barrier is a gloo operation: NCCL groups get a gloo twin for it
        self.monitor = group if backend == "gloo" else dist.new_group(backend="gloo", timeout=self.timeout)

    def check_in(self, step: int) -> None:
        """Raise RankFailure unless every rank reaches this point of step ``step``."""
        import torch.distributed as dist

        if self.world == 1:
            return
        try:
            dist.monitored_barrier(group=self.monitor, timeout=self.timeout, wait_all_ranks=True)
        except RuntimeError as exc:   # gloo reports a missing or dead peer as RuntimeError
            raise RankFailure(f"shot-parallel step {step}: a rank failed or left ({exc})") from exc

    def reduce(self, step: int, grads: Iterable[Optional[torch.Tensor]]) -> None:
        """Liveness check, then the one all-reduce (sum) of the step's gradients."""
        grads = list(grads)
        self.check_in(step)
        allreduce_gradients(grads, group=self.group)
