"""Multi-rank frame sharding (the N>1 path of bench.py) on CPU with gloo,
world size 2: each rank evaluates its frame block with the CPU oracle, the
per-rank chi-square totals are all-reduced, and the total must equal the
single-process evaluation of all frames."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from shape_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    sys.path[:0] = [here, repo, os.path.join(repo, "shape-cuda-v1.2_b200", "python")]
    import torch.distributed as dist
    from datetime import timedelta
    import golden_cases as gc
    from oracle.bindings import Oracle
    from shape_b200 import shard as sh
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    orc = Oracle()
    model_fn, ds_fn, params = gc.DELDOP_CASES["small_long_orig"]
    m = model_fn()
    ds = ds_fn(lambda d, p: orc.eval_deldop(m, d, p)["fits"], params)
    sub, (lo, hi) = sh.shard_dataset(ds, rank, world)
    o = orc.eval_deldop(m, sub, params)
    local = {"chi2": sum(r["chi2"] for r in o["results"]), "chi2_deldop": 0.0, "chi2_lghtcrv": 0.0,
             "posbnd": 0, "badradar": 0}
    tot = sh.allreduce_summary(local, dist)
    if rank == 0:
        full = orc.eval_deldop(m, ds, params)
        out_q.put((tot["chi2"], sum(r["chi2"] for r in full["results"]), (lo, hi)))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_bounds_cover_and_balance():
    costs = [5, 1, 1, 1, 9, 2, 2, 3, 7, 1]
    for world in (1, 2, 3, 4):
        b = shard.shard_bounds(costs, world)
        assert b[0][0] == 0 and b[-1][1] == len(costs)
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        assert all(hi > lo for lo, hi in b)
        tot = [sum(costs[lo:hi]) for lo, hi in b]
        assert max(tot) <= sum(costs) / world + max(costs)


def test_two_rank_chi2_equals_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tot, full, _ = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert abs(tot - full) <= 1e-12 * abs(full)
