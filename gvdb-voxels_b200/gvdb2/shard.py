"""Multi-GPU plumbing: one process per GPU, no data-path collective.

The point path does not shard inside one volume without a halo exchange, so
a volume lives on one GPU.  What shards is independent work: replicas of one
step (weak scaling), or independent clouds (the batched workload), spread
over the ranks by longest-processing-time-first so the ranks' point counts
stay close.  The only collectives are on the host side of the timing: a
barrier around the timed region and the max (or sum) of a scalar over the
ranks.
"""
import os
from dataclasses import dataclass


@dataclass
class RankEnv:
    rank: int = 0
    world: int = 1
    local: int = 0

    @classmethod
    def from_env(cls):
        return cls(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                   int(os.environ.get("LOCAL_RANK", "0")))


def lpt_partition(sizes, nranks):
    """Clouds to ranks, largest first, each to the least-loaded rank (lowest
    rank on ties).  Returns one ascending list of cloud indices per rank;
    every cloud appears exactly once."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * nranks
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def _reduce(x, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, device="cpu"):
    """The largest x over the ranks (a timing: the job ends with its slowest
    rank).  `device` is where the collective runs: "cpu" for gloo, the
    rank's CUDA device for nccl."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x, device="cpu"):
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)
