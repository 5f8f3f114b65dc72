"""Replica bookkeeping for running the evaluation core on several GPUs of
one node.

Key switching needs every limb of a digit, so the library does not shard a
ciphertext across GPUs; ciphertext batches are split across ranks (one
process per GPU, keys replicated) and no collective runs on the data path.
The only collectives are the barrier around a timed region and the maximum
of the per-rank device times, through torch.distributed (NCCL on GPUs, gloo
for host-only runs)."""
import os
from datetime import timedelta


def env_rank():
    """(rank, world size, local rank) from the torchrun environment; a
    single process without it is rank 0 of 1."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_group(world, backend="nccl", timeout_s=120):
    """The process group of a multi-rank run (None for one rank).  A short
    timeout makes ranks that wait for a missing peer fail instead of
    hanging."""
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, value, device="cpu"):
    """The maximum of a per-rank figure (a device time in ms) over all ranks;
    every rank takes part and receives the result."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, units_per_rank, steps, ms):
    """Whole-job throughput of a weak-scaling run: every rank processes
    units_per_rank units per step, and the job's time is the slowest rank's
    (ms over `steps` steps)."""
    if ms <= 0:
        raise ValueError("job_throughput: non-positive time")
    return world * units_per_rank * steps / (ms / 1e3)


def rank_seed(base, rank):
    """Seed of a rank's synthetic inputs: replicas work on different data."""
    return base + 7919 * rank


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
