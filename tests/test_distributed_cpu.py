"""CPU: the multi-GPU plumbing with two gloo ranks (no GPU)."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.dirname(here), os.path.join(os.path.dirname(here), "vfs-python_b200")]
    import datetime
    import torch.distributed as dist
    from vfs_b200.distributed import shard, pair_cost, max_over_ranks, sum_gradients
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [480, 640, 800, 1024] * 8
        costs = [pair_cost(s, s, 4, 2.0, 10, 50) for s in sizes]
        mine = shard(costs, world, rank)
        t = max_over_ranks(1.5 + rank)
        g = sum_gradients({"Lambda": 1.0 + rank, "alpha0": 2.0 * rank})
        q.put((rank, mine, t, g))
    finally:
        dist.destroy_process_group()


def test_shard_is_a_balanced_partition():
    from vfs_b200.distributed import shard, pair_cost
    costs = [pair_cost(s, s, 4, 2.0, 10, 50) for s in [480, 640, 800, 1024] * 8]
    parts = [shard(costs, 3, r) for r in range(3)]
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.1


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, g0), (r1, m1, t1, g1) = out
    assert sorted(m0 + m1) == list(range(32)) and not set(m0) & set(m1)
    assert t0 == t1 == 2.5
    assert g0 == g1 == {"Lambda": 3.0, "alpha0": 2.0}


def test_bench_launches_two_ranks_dry_run():
    """`bench.py --gpus 2` starts two ranks through torch.distributed.run; in a
    dry run (gloo, no GPU) rank 0 prints one line with n_gpus 2, disjoint
    cost-balanced shards covering the batch, and the summed theta gradient."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--dry-run"],
                       capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["n_gpus"] == 2 and line["dry_run"]
    a, b = line["shards"]
    assert sorted(a + b) == list(range(32)) and not set(a) & set(b)
    c0, c1 = line["shard_costs"]
    assert max(c0, c1) / min(c0, c1) < 1.05
    assert line["max_over_ranks"] == 2.0
    assert line["theta_grad_sum"] == [3.0, 2.0, 1.0, -1.0, 6.0]
