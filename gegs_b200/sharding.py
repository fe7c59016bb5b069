"""History sharding over GPUs (one process per GPU, torch.distributed).

Histories are independent, so the only exchange is one sum of the int64
tallies at the end. The reference drives its GPUs serially from one host
thread and sums double tallies on the host (CUDA_EGS.cu:463-482, 1723-1735);
here every rank transports a contiguous range of the per-history RNG
counters, and because the tally is integer the summed result is the same bit
for bit for any number of ranks.
"""
from __future__ import annotations


def shard(hist_begin: int, hist_end: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced slice [a, b) of [hist_begin, hist_end) for `rank` of `world`.
    The first (n % world) ranks get one history more; empty slices are allowed."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    if hist_end < hist_begin:
        raise ValueError("hist_end < hist_begin")
    n = hist_end - hist_begin
    q, r = divmod(n, world)
    a = hist_begin + rank * q + min(rank, r)
    return a, a + q + (1 if rank < r else 0)


def allreduce_tally_(tally, group=None):
    """Sum an int64 tally tensor over the ranks of `group` in place (NCCL on GPUs,
    gloo on CPU). Integer addition is exact, so the order of ranks does not matter."""
    import torch
    import torch.distributed as dist
    if tally.dtype != torch.int64:
        raise TypeError("the tally is int64 (MeV * 2^30 per voxel)")
    dist.all_reduce(tally, op=dist.ReduceOp.SUM, group=group)
    return tally


def tally_tensor(engine, device):
    """Zero-copy torch view of an engine's device tally (int64, nvox)."""
    import torch

    class _Dev:
        def __init__(self, ptr, n):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i8", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Dev(engine.tally_device_ptr(), engine.nvox), device=device)
