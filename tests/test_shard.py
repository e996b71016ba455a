"""Sharding of independent disks over ranks (CPU, gloo, world_size 2)."""
import os
import socket

import pytest


def test_lpt_shards_cover_and_balance():
    from fargo3d_b200 import config_batched
    from fargo3d_b200.shard import lpt_shards
    cfgs = config_batched(64, seed=3)
    costs = [c.active_cells for c in cfgs]
    for world in (1, 2, 3, 8):
        sh = lpt_shards(costs, world)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(cfgs)))
        loads = [sum(costs[i] for i in s) for s in sh]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(costs) / world + max(costs)
    assert lpt_shards(costs, 2) == lpt_shards(costs, 2)   # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    from fargo3d_b200 import config_batched
    from fargo3d_b200.shard import max_over_ranks, shard_disks, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    cfgs = config_batched(64, seed=5)
    mine = shard_disks(cfgs, rank, world)
    cells = sum(c.active_cells for c in mine)
    total = sum_over_ranks(cells)
    tmax = max_over_ranks(1.0 + rank)       # stand-in per-rank time
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, [c.seed for c in mine], cells, total, tmax))


def test_shards_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    from fargo3d_b200 import config_batched
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds = sorted(s for r in res for s in r[1])
    assert seeds == sorted(c.seed for c in config_batched(64, seed=5))   # every disk once
    assert not set(res[0][1]) & set(res[1][1])
    total = sum(r[2] for r in res)
    assert all(r[3] == total for r in res)                               # SUM seen by both
    assert all(r[4] == 2.0 for r in res)                                 # MAX over ranks


def test_bench_gpus_2_shards_one_global_list():
    """`bench.py --gpus 2` starts two ranks itself (torch.distributed.run on
    127.0.0.1), each takes its LPT share of one global list of 128 disks, and
    rank 0 reports n_gpus = 2 (--plan: the rank set-up without GPU work)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--plan"],
                         capture_output=True, text=True, timeout=300, env=env, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("{")][-1]
    plan = json.loads(line)
    assert plan["n_gpus"] == 2 and len(plan["ranks"]) == 2
    seeds = sorted(s for r in plan["ranks"] for s in r["seeds"])
    assert seeds == list(range(128))
    from fargo3d_b200 import config_batched
    total = sum(c.active_cells for c in config_batched(128, seed=0))
    loads = [r["cells"] for r in plan["ranks"]]
    assert sum(loads) == total
    assert max(loads) <= total / 2 + max(c.active_cells for c in config_batched(128, seed=0))
