"""The N>1 replica path (bench.py under torchrun) with world_size 2 on CPU:
barrier, max over ranks of the timed region, whole-job throughput."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world_size, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world_size), LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world_size,
                            timeout=datetime.timedelta(seconds=60))
    from mdff_b200 import replicas
    r, w, lr = replicas.world()
    assert (r, w, lr) == (rank, world_size, rank)
    replicas.barrier(w)
    # rank 1 is the slow replica: the job is bounded by it
    secs = 2.0 if rank == 1 else 1.0
    value, t = replicas.throughput(w, 10, secs)
    out[rank] = (value, t)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_world_size_2():
    port = 29500 + (os.getpid() % 2000)
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    for rank in (0, 1):
        value, t = out[rank]
        assert t == 2.0 and abs(value - 2 * 10 / 2.0) < 1e-12


def test_single_process_needs_no_group():
    from mdff_b200 import replicas
    assert replicas.max_over_ranks(1, 3.5) == 3.5
    assert replicas.throughput(1, 4, 2.0) == (2.0, 2.0)
