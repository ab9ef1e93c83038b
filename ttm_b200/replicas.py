"""Multi-GPU helpers: one process per GPU (torch.distributed), no data-path collective.

A mode-q TTM partitions into independent slices C_k = A_k x B (k < outer): `shard_slices`
gives each rank a contiguous range of slices (the ranks share B and never exchange data).
`max_over_ranks` reduces a timing to its maximum over ranks, the figure a multi-GPU run
reports. bench.py runs one full replica of its workload per GPU (weak scaling) and times it
with these helpers.
"""
from __future__ import annotations


def shard_slices(outer: int, rank: int, world: int):
    """[begin, end) of the slices rank `rank` of `world` owns: contiguous, sizes differing by at most 1."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(outer, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over the ranks of the default process group (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None):
    import torch
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
    if device is not None and getattr(device, "type", "") == "cuda":
        torch.cuda.synchronize(device)
