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
