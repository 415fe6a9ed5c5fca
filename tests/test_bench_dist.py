"""Multi-rank host logic of bench.py on CPU: world_size-2 gloo ranks agree on
the max-over-ranks timing (the N > 1 replicas path uses it with NCCL)."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    assert bench.dist_env() == (world, rank, rank)
    got = bench.max_over_ranks(10.0 + rank * 5.5, world)
    bench.barrier(world)
    out[rank] = got
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    assert out[0] == out[1] == pytest.approx(15.5)


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.25, 1) == 3.25
