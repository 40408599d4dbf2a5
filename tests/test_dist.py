"""Multi-rank host logic on CPU: world size 2 over gloo (127.0.0.1).

A batch of independent factorizations shards with no data-path collective: every rank holds the
plan and factors its own block of ONE global batch (glu_public_b200.shard).  The only cross-rank
steps of the benchmark are the barrier around the timed region and the max over ranks of the
elapsed time.  These tests check that the ranks' shards together are the batch exactly once (for
one pattern and for the multi-pattern batch bin-packed by cost), that a rank's instance values are
the same rows of the batch whatever the rank count, and the timing collectives.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from glu_public_b200 import shard

# the multi-pattern batch: (pattern, instances, F_alg per instance)
MULTI = [("mna2000_s3", 1024, 4.92e7), ("mna50000_s4", 64, 7.65e11), ("grid512_s1", 4, 7.34e10)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    from glu_public_b200 import gen
    bench.barrier(world)
    elapsed = 10.0 + rank                          # rank 1 is the slower one
    m = bench.max_over_ranks(world, elapsed)
    first, count = bench.shard_of(8, world, rank)
    c = gen.mna_netlist(200, 3)
    vals = c.instance_values_indexed(first, count, bench.INST_SEED)
    shards = shard.plan_shards(MULTI, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, (first, count, [(s.name, s.first, s.count) for s in shards]))
    out[rank] = (m, first, count, vals, gathered)
    bench.barrier(world)
    dist.destroy_process_group()


def test_two_ranks_shard_one_batch_and_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0
    # one pattern: the two blocks are the global batch of 16, each instance exactly once
    idx = sorted(i for r in (0, 1) for i in range(res[r][1], res[r][1] + res[r][2]))
    assert idx == list(range(16))
    # a rank's values are those rows of the batch generated in one piece
    from glu_public_b200 import gen
    import bench
    full = gen.mna_netlist(200, 3).instance_values_indexed(0, 16, bench.INST_SEED)
    for r in (0, 1):
        assert np.array_equal(res[r][3], full[res[r][1]:res[r][1] + res[r][2]])
    # every rank saw the same multi-pattern assignment, covering every instance once
    assert res[0][4] == res[1][4]
    seen = {}
    for _, _, parts in res[0][4]:
        for name, first, count in parts:
            for i in range(first, first + count):
                seen[(name, i)] = seen.get((name, i), 0) + 1
    assert set(seen.values()) == {1}
    assert set(seen) == {(n, i) for n, cnt, _ in MULTI for i in range(cnt)}


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_plan_shards_covers_the_batch_and_balances_cost(world):
    cost = {n: f for n, _, f in MULTI}
    shards = shard.plan_shards(MULTI, world)
    assert len(shards) == world
    seen = set()
    for parts in shards:
        for s in parts:
            for i in range(s.first, s.first + s.count):
                assert (s.name, i) not in seen
                seen.add((s.name, i))
    assert seen == {(n, i) for n, cnt, _ in MULTI for i in range(cnt)}
    loads = [shard.shard_cost(p, cost) for p in shards]
    ideal = sum(cnt * f for _, cnt, f in MULTI) / world
    biggest = max(f for _, _, f in MULTI)
    # LPT over chunks: no rank exceeds the ideal share by more than one chunk of the costliest
    # pattern (a whole instance at least)
    chunk = max(biggest, ideal / 4)
    assert max(loads) <= ideal + chunk + 1e-6 * ideal


@pytest.mark.parametrize("total,world", [(0, 3), (5, 1), (7, 3), (512, 8), (3, 8)])
def test_instance_range_partitions(total, world):
    parts = [shard.instance_range(total, world, r) for r in range(world)]
    assert sum(c for _, c in parts) == total
    pos = 0
    for first, count in parts:
        assert first == pos and count >= 0
        pos += count
    assert max(c for _, c in parts) - min(c for _, c in parts) <= 1


def test_single_rank_needs_no_process_group():
    import bench
    bench.barrier(1)
    assert bench.max_over_ranks(1, 3.5) == 3.5
    with pytest.raises(ValueError):
        dist.get_backend()
