"""Multi-GPU bookkeeping for independent replicas (one process per GPU).

The engforce path does not shard: one B200 holds the whole system, and the
reference's MPI atom / k-point decomposition (mpi_mdff.f90:38-97) only exists to
spread one configuration over CPU ranks.  N GPUs therefore run N independent
replicas; the only collectives are a barrier and the max-over-ranks of the
timed region.  The same functions run on NCCL (GPU ranks) and gloo (CPU
tests).
"""
import os


def world():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def barrier(world_size):
    if world_size > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world_size, x):
    """Largest value of x over all ranks (the slowest replica bounds the job)."""
    if world_size <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(world_size, steps_per_rank, seconds_this_rank):
    """Whole-job steps/s: all ranks' steps over the slowest rank's time."""
    t = max_over_ranks(world_size, seconds_this_rank)
    return world_size * steps_per_rank / t, t
