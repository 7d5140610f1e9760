"""Multi-GPU as independent replicas: one process per GPU, each baking its
own workload (texels are independent; there is no data-path collective).
The only cross-rank step is the timing reduction of a measured region:
the job's time is the slowest rank's, its work is the sum over ranks."""
from __future__ import annotations

import os
from typing import Optional, Tuple


def rank_info() -> Tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def job_rate(ms: float, units: int, dist=None, device: Optional[str] = None) -> Tuple[float, int, float]:
    """Whole-job (max ms over ranks, total units, units per second).  `dist`
    is torch.distributed with an initialised process group (NCCL: device
    "cuda", gloo: "cpu"), or None for one process.  Every rank must call it."""
    if dist is not None:
        import torch
        dev = device or ("cuda" if dist.get_backend() == "nccl" else "cpu")
        t = torch.tensor([float(ms)], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        u = torch.tensor([float(units)], device=dev, dtype=torch.float64)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
        ms, units = float(t.item()), int(u.item())
    return ms, units, units / (ms / 1e3) if ms > 0 else 0.0
