"""Multi-rank host logic of the benchmark on CPU: world size 2 over gloo (127.0.0.1).

The multi-GPU configuration runs independent replicas (each rank factors its own value sets, no
data-path collective); the only cross-rank steps are the barrier around the timed region and the
max over ranks of the elapsed time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


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
    bench.barrier(world)
    elapsed = 10.0 + rank                          # rank 1 is the slower one
    m = bench.max_over_ranks(world, elapsed)
    out[rank] = (m, bench.instance_seed(rank))
    bench.barrier(world)
    dist.destroy_process_group()


def test_two_ranks_time_is_max_over_ranks_and_seeds_differ():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0
    assert res[0][1] != res[1][1]


def test_single_rank_needs_no_process_group():
    import bench
    bench.barrier(1)
    assert bench.max_over_ranks(1, 3.5) == 3.5
    with pytest.raises(ValueError):
        dist.get_backend()
