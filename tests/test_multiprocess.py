"""The multi-process path of the bench on CPU: two ranks over gloo (127.0.0.1).

One process per GPU runs the batched instances sharded by `sharding.lpt_partition` with no
data-path collective; only timings and counts are reduced (`bench.max_over_ranks`,
`bench.sum_over_ranks`).  These tests run that host logic with world size 2 on the gloo
backend: the shards are disjoint, cover every instance and are balanced, and the reductions
return the same value on every rank.
"""
import json
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    from brian2cuda_b200 import models
    from brian2cuda_b200.sharding import instance_cost, lpt_partition
    w, r, _ = bench.dist_setup(world, backend="gloo")
    sizes, _ = models.batch_sizes()
    mine = lpt_partition(instance_cost(sizes, 0.02), w)[r]
    res = {"rank": r, "world": w, "mine": mine,
           "max": bench.max_over_ranks(float(r + 1), w),
           "sum": bench.sum_over_ranks(float(len(mine)), w)}
    bench.barrier(w)
    import torch.distributed as dist
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump(res, f)


def test_lpt_partition_balances_and_covers():
    from brian2cuda_b200 import models
    from brian2cuda_b200.sharding import instance_cost, lpt_partition
    sizes, _ = models.batch_sizes()
    cost = instance_cost(sizes, 0.02)
    for k in (1, 2, 4, 8):
        parts = lpt_partition(cost, k)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = np.array([cost[p].sum() for p in parts])
        # longest processing time first: within 4/3 of the optimum, which is >= the mean
        assert loads.max() <= (4 / 3) * max(loads.mean(), cost.max()) + 1e-9
    assert lpt_partition(cost, 2) == lpt_partition(cost, 2)


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    a, b = set(res[0]["mine"]), set(res[1]["mine"])
    assert not (a & b) and len(a | b) == 256
    for r in res:
        assert r["world"] == 2 and r["max"] == 2.0 and r["sum"] == 256.0
