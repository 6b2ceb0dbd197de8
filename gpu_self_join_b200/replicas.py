"""Whole-job numbers of replicated joins (one process per GPU, each joining
its own copy of the workload; the join has no exchange step, so ranks never
communicate on the data path).  The only collective is this reduction of the
measured numbers: the slowest rank's time and the sum of all ranks' pairs."""

from __future__ import annotations


def reduce_step(ms: float, pairs: float, device=None) -> tuple[float, float]:
    """(max over ranks of ms, sum over ranks of pairs); the inputs unchanged
    without an initialised process group of more than one rank."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms), float(pairs)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    p = torch.tensor([float(pairs)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(p, op=dist.ReduceOp.SUM)
    return float(t.item()), float(p.item())
