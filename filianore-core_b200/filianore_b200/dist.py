"""Multi-GPU rendering, one process per GPU: every rank renders its own range of sample
indices of the same image (rank r renders samples [base + r * spp, base + (r + 1) * spp)
with the per-pixel PCG32 streams advanced to them), and the FP64 XYZ films are summed on
rank 0 with one reduce per frame. The sum equals a single render of world * spp samples.
Ray batches (trace calls) are independent per rank and need no collective."""
from __future__ import annotations


def rank_sample_offset(rank: int, spp: int, base: int = 0) -> int:
    """first sample index rendered by `rank` when every rank renders `spp` samples"""
    return base + rank * spp


def reduce_film(xyz, dst: int = 0):
    """sums the ranks' FP64 XYZ films (torch tensors) into rank `dst`"""
    import torch.distributed as dist
    dist.reduce(xyz, dst=dst, op=dist.ReduceOp.SUM)
    return xyz


def max_over_ranks(x: float, device=None) -> float:
    """the largest value of x over all ranks (step times are reported this way)"""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
