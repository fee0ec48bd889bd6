"""Multi-GPU replicas: one process per GPU, each serving its own tensors.

The compose / transform / factorisation path has no data exchange between
GPUs: every tensor (and every chain of the serving loop) is independent, so
N GPUs run N independent replicas (weak scaling).  The only collectives are
the timing ones: a barrier on both sides of the timed region and the maximum
of the ranks' device times, so the reported time is that of the slowest
replica.  These helpers are what ``bench.py`` uses under torchrun; they take
the process group's device (CUDA for NCCL, CPU for gloo), which lets the same
code run in multi-process CPU tests.
"""

from __future__ import annotations

from typing import List, Tuple


def replica_seeds(rank: int, count: int, base_a: int = 1, base_b: int = 5001) -> List[Tuple[int, int]]:
    """splitmix64 seeds of the (A, B) operands of a rank's ``count`` tensors; disjoint across ranks."""
    if count > 1000:
        raise ValueError("at most 1000 tensors per rank keep the seed ranges of the ranks disjoint")
    return [(base_a + i + 1000 * rank, base_b + i + 1000 * rank) for i in range(count)]


def max_over_ranks(value: float, device="cpu") -> float:
    """Maximum of ``value`` over the ranks of the default process group (the value itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
