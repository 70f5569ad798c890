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


# ---------------------------------------------------------------------------
# Failure detection: a rank raises or leaves between steps; the survivors get
# an error within a bounded time on the host instead of waiting forever.
# ---------------------------------------------------------------------------

def _fault_worker(rank, world, port, behaviour, out_path, pg_timeout_s, check_timeout_s):
    import datetime
    import json
    import time as _time

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from deepgpr_b200.shots import RankFailure, ShotGroup

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=pg_timeout_s))
    group = ShotGroup(timeout_s=check_timeout_s)
    result = {"rank": rank, "steps": 0, "error": None, "elapsed": None}
    g = torch.ones(8)
    try:
        for step in range(3):
            if rank == 1 and step == 1:
                if behaviour == "raise":
                    raise ValueError("planted failure between steps")
                if behaviour == "leave":
                    os._exit(0)          # leaves without a word, between steps
                if behaviour == "stall":
                    _time.sleep(pg_timeout_s + check_timeout_s + 5)
                    os._exit(0)
            t0 = _time.monotonic()
            if behaviour == "stall":
                # no liveness check: the collective itself must end by the group's timeout
                try:
                    dist.all_reduce(g)
                except RuntimeError as exc:
                    raise RankFailure(str(exc)) from exc
            else:
                group.reduce(step, [g])
            result["steps"] = step + 1
    except RankFailure as exc:
        result["error"] = "RankFailure"
        result["message"] = str(exc)[:300]
        result["elapsed"] = _time.monotonic() - t0
    except ValueError:
        os._exit(3)
    with open(out_path + f".{rank}", "w") as f:
        json.dump(result, f)
    os._exit(0)   # no teardown collective with a dead peer


def _run_fault(tmp_path, behaviour, pg_timeout_s=6.0, check_timeout_s=3.0):
    import json
    import time as _time

    port = _free_port()
    ctx = mp.get_context("spawn")
    out = str(tmp_path / "res")
    procs = [ctx.Process(target=_fault_worker, args=(r, 2, port, behaviour, out, pg_timeout_s, check_timeout_s))
             for r in range(2)]
    t0 = _time.monotonic()
    for p in procs:
        p.start()
    deadline = t0 + 120
    for p in procs:
        p.join(timeout=max(1.0, deadline - _time.monotonic()))
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a surviving rank hung"
    res = json.loads((tmp_path / "res.0").read_text())
    return res, procs


@pytest.mark.parametrize("behaviour", ["raise", "leave"])
def test_survivor_detects_a_failed_rank_between_steps(tmp_path, behaviour):
    res, procs = _run_fault(tmp_path, behaviour)
    assert res["steps"] == 1, res                 # step 0 completed on both ranks
    assert res["error"] == "RankFailure", res
    assert res["elapsed"] < 30.0, res              # bounded by the check's timeout, not a hang
    assert procs[1].exitcode == (3 if behaviour == "raise" else 0)


def test_short_group_timeout_ends_a_collective_with_a_stalled_peer(tmp_path):
    res, _ = _run_fault(tmp_path, "stall", pg_timeout_s=4.0)
    assert res["error"] == "RankFailure", res
    assert res["elapsed"] < 30.0, res
