"""Multi-GPU host logic on CPU: two gloo ranks in spawned processes.

The path runs replicas (one process per GPU, each with its own ensemble
members; src/azeban.cpp:131-152 splits samples across MPI sub-communicators
the same way), so what crosses ranks is bookkeeping: the split of members by
cost, the max over ranks of a timed region, and the whole-job rate.
"""

import datetime
import os
import socket

import pytest

from azeban_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist

    from azeban_b200 import replicas as rp
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = rp.partition_by_cost(costs, world)[rank]
        local = float(sum(costs[i] for i in mine))
        slowest = rp.max_over_ranks(local)
        total = rp.sum_over_ranks(local)
        rp.barrier()
        rate = rp.aggregate_rate(len(mine), world, slowest)
        q.put((rank, mine, local, slowest, total, rate))
    finally:
        dist.destroy_process_group()


def test_partition_by_cost_covers_and_balances():
    costs = [5.0, 1.0, 1.0, 8.0, 3.0, 3.0, 2.0, 9.0, 0.5]
    for world in (1, 2, 3, 4):
        parts = replicas.partition_by_cost(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert replicas.partition_by_cost([], 2) == [[], []]
    with pytest.raises(ValueError):
        replicas.partition_by_cost([1.0], 0)


def test_reductions_without_process_group():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.sum_over_ranks(2.0) == 2.0
    replicas.barrier()
    assert replicas.aggregate_rate(40, 1, 100.0) == pytest.approx(400.0)
    with pytest.raises(ValueError):
        replicas.aggregate_rate(1, 1, 0.0)


def test_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    world = 2
    # a mixed ensemble: member costs proportional to bytes per step of 2-D
    # 128^2, 256^2 and 512^2 solves
    costs = [1.0] * 6 + [4.0] * 4 + [16.0] * 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    out = sorted(q.get() for _ in range(world))
    members = sorted(i for r in out for i in r[1])
    assert members == list(range(len(costs)))
    locals_ = [r[2] for r in out]
    for r in out:
        assert r[3] == max(locals_)          # max over ranks
        assert r[4] == pytest.approx(sum(costs))  # sum over ranks
    assert max(locals_) - min(locals_) <= max(costs)
    # whole-job rate: every rank's members over the slowest rank's time
    assert out[0][5] == pytest.approx(world * len(out[0][1]) / (max(locals_) / 1e3))


def test_bench_launches_one_rank_per_gpu_dry_run():
    """bench.py --gpus 2 without a launcher starts two ranks itself
    (torch.distributed.run, rendezvous on 127.0.0.1); --dry-run does the rank
    bookkeeping on gloo without a GPU."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    res = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--dry-run"],
                         capture_output=True, text=True, timeout=300, env=env, cwd=root)
    assert res.returncode == 0, res.stderr[-2000:]
    line = [ln for ln in res.stdout.splitlines() if ln.startswith("{")][-1]
    out = json.loads(line)
    assert out["n_gpus"] == 2 and out["ranks_seen"] == 2 and out["max_over_ranks"] == 2.0
    assert sorted(sum(out["members"], [])) == list(range(8))
