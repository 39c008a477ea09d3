"""Multi-GPU plumbing: one process per GPU, independent worlds per rank, no collective on the data path.

The field update of one world does not shard at the sizes it runs (a halo exchange per hydro step, an all-to-all per
FFT solve and an all-reduce per CG dot would make it latency-bound), so several GPUs advance different worlds:
replicas of the benchmark world, or the worlds of a batch split by cell count. torch.distributed carries only the
start barrier and the max-over-ranks of the timings.
"""
from __future__ import annotations

import datetime
import os


def partition(cells, world: int):
    """Longest-processing-time-first split of worlds (their cell counts) over `world` ranks: worlds sorted by size,
    each to the rank with the fewest cells so far (ties to the lowest rank). Returns each rank's world indices."""
    order = sorted(range(len(cells)), key=lambda i: (-cells[i], i))
    share = [[] for _ in range(world)]
    load = [0] * world
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        share[r].append(i)
        load[r] += cells[i]
    return share


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init(backend: str = "nccl", timeout_s: int = 300):
    """Initialises the default process group from the torchrun environment when WORLD_SIZE > 1; returns the module
    (torch.distributed) or None for a single process."""
    rank, world, _ = env_rank()
    if world <= 1:
        return None
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(dist, value: float, device=None) -> float:
    """The largest `value` over the ranks (the slowest rank's time)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
