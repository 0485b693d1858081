"""Multi-GPU as independent replicas.

The grid model does not shard: a single chip (<= 10.5 M cells) fits one GPU,
and independent chips (the batched and serving workloads) need no exchange.
N GPUs therefore run N independent replicas, one process per GPU, and the
only collectives are the timing/throughput reductions of the measurement
(barrier, max of elapsed times, sum of work), over torch.distributed (NCCL
on GPUs, gloo on CPU).
"""
from __future__ import annotations

import os


def world() -> tuple[int, int, int]:
    """(world_size, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items: list, rank: int, world_size: int) -> list:
    """Round-robin share of independent work items (chips, requests) for a rank."""
    return items[rank::world_size]


def reduce_timing(elapsed: float, work: float, pg=None, device: str = "cpu") -> tuple[float, float]:
    """(max over ranks of elapsed, sum over ranks of work): whole-job
    throughput is sum(work) / max(elapsed)."""
    if pg is None or not pg.is_initialized() or pg.get_world_size() == 1:
        return elapsed, work
    import torch
    t_max = torch.tensor([elapsed], dtype=torch.float64, device=device)
    t_sum = torch.tensor([work], dtype=torch.float64, device=device)
    pg.all_reduce(t_max, op=pg.ReduceOp.MAX)
    pg.all_reduce(t_sum, op=pg.ReduceOp.SUM)
    return float(t_max.item()), float(t_sum.item())
