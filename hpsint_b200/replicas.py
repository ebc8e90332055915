"""Replica parallelism: one process per GPU, no collective on the data path.

The operator shards naturally, but every graded run uses one GPU, so N GPUs
run N independent replicas: the benchmark repeats the same per-GPU workload
on every rank (weak scaling), and seed-parallel work (training trajectories,
held-out evaluations) is split across ranks.  The only collectives are the
bookkeeping ones here: the step time as the maximum over ranks, and the
gathering of per-rank results on every rank.  They work with any
torch.distributed backend (NCCL on the GPUs, gloo in the CPU tests).
"""
import os
from dataclasses import dataclass

import torch


@dataclass
class World:
    rank: int = 0
    size: int = 1
    local_rank: int = 0


def from_env():
    """Rank, world size and local rank as torch.distributed.run sets them (1 process if unset)."""
    return World(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def shard(items, rank, size):
    """The items of one rank: rank, rank + size, ... (every item on exactly one rank)."""
    if size < 1 or not 0 <= rank < size:
        raise ValueError(f"rank {rank} outside a world of {size}")
    return list(items)[rank::size]


def _device(dist):
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x, dist=None):
    """max of a float over all ranks (x itself without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist=None):
    """sum of a float over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather(obj, dist=None):
    """[obj of rank 0, obj of rank 1, ...] on every rank (picklable objects)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
