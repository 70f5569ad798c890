"""Shot-parallel gradient over 2 gloo ranks on CPU equals the single-process gradient.

The solver inside each rank is the CPU oracle (this tests the sharding and the
all-reduce, which are host logic); the GPU path uses the same functions with
NCCL.
"""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(shots):
    sys.path.insert(0, str(ROOT / "tests"))
    from helpers import problem_2d

    p = problem_2d(nt=40, order=4)
    p.source_location = torch.tensor([[[10, 4 + 5 * s, 0]] for s in range(shots)], dtype=torch.int32)
    p.receiver_location = torch.tensor([[[10, 30, 0], [5, 7, 0]]] * shots, dtype=torch.int32)
    return p


def _worker(rank, world, port, shots, out_path):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from deepgpr_b200.shots import allreduce_gradients, shard_acquisition
    from oracle import driver

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = _problem(shots)
        p.source_location, p.receiver_location, _ = shard_acquisition(p.source_location, p.receiver_location, world,
                                                                      rank)
        res = driver.run(p, "oracle")
        ge, gs = res["grad_eps"].clone(), res["grad_sigma"].clone()
        allreduce_gradients([ge, gs])
        if rank == 0:
            torch.save({"grad_eps": ge, "grad_sigma": gs}, out_path)
    finally:
        dist.destroy_process_group()


def test_shard_shots_is_a_partition():
    from deepgpr_b200.shots import shard_shots

    for n in (1, 5, 32, 33):
        for w in (1, 2, 3, 8):
            idx = [i for r in range(w) for i in range(n)[shard_shots(n, w, r)]]
            assert idx == list(range(n))


def test_two_rank_gradient_equals_single_process(tmp_path):
    from oracle import driver

    driver.build("oracle")
    shots = 4
    out = tmp_path / "g.pt"
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, shots, str(out))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = torch.load(out)
    full = driver.run(_problem(shots), "oracle")
    for key in ("grad_eps", "grad_sigma"):
        rel = (got[key] - full[key]).norm() / full[key].norm()
        assert rel < 1e-5, (key, float(rel))
