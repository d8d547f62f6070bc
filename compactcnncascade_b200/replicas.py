"""Host-side bookkeeping for running the detector as independent replicas, one process per GPU.

Frames are independent, so N GPUs simply split the frame stream: rank r takes its own disjoint
seeds / frames, nothing crosses GPUs on the data path, and the job's throughput is all ranks'
frames divided by the slowest rank's time.
"""


def rank_seeds(rank, count, stride=100_000):
    """Disjoint synthetic-frame seeds of one rank."""
    return [rank * stride + i for i in range(count)]


def shard(items, rank, world):
    """Round-robin share of a frame list for one rank."""
    return items[rank::world]


def job_throughput(frames_per_rank, seconds_per_rank):
    """Whole-job frames/s: every rank's frames over the slowest rank's time."""
    return sum(frames_per_rank) / max(seconds_per_rank)


def reduce_max(value, dist=None, device=None):
    """Max over ranks (identity without a process group)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])
