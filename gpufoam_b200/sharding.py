"""Multi-GPU sharding of the per-cell chemistry solve (one process per GPU).

Cells are independent, so a batch splits into contiguous cell ranges with no
data exchange; the one cross-cell quantity of a flow step is minDeltaT, the
minimum over all cells of the new chemistry time step before clamping
(gpuKernelEvaluator.cu:91-92 of the reference), which the ranks combine with
one all-reduce (NCCL over NVLink on GPUs, gloo on CPU).

Cells differ widely in cost (substep counts spread over ~10x), so ranges can
be balanced by the previous step's per-cell attempt counts (the kernel's
`counters`), which predict the next step's cost.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np


def shard_ranges(n_cells: int, world: int, weights: Optional[Sequence[float]] = None) -> List[Tuple[int, int]]:
    """[start, stop) cell range of every rank: contiguous, covering 0..n_cells
    in rank order. Without weights the ranges differ in size by at most one;
    with per-cell weights (e.g. last step's attempts) each range holds about
    1/world of the total weight."""
    if world < 1 or n_cells < 0:
        raise ValueError("world must be >= 1 and n_cells >= 0")
    if weights is None:
        base, extra = divmod(n_cells, world)
        out, start = [], 0
        for r in range(world):
            stop = start + base + (1 if r < extra else 0)
            out.append((start, stop))
            start = stop
        return out
    w = np.asarray(weights, dtype=np.float64)
    if w.shape != (n_cells,) or (w < 0).any():
        raise ValueError("weights must be n_cells non-negative numbers")
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, total * r / world, side="left")))
    cuts.append(n_cells)
    cuts = np.maximum.accumulate(np.clip(cuts, 0, n_cells))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def local_range(n_cells: int, rank: int, world: int, weights=None) -> Tuple[int, int]:
    return shard_ranges(n_cells, world, weights)[rank]


def global_min_delta_t(local_min: float, device=None, group=None) -> float:
    """min over ranks of the ranks' minDeltaT (the step's one exchange)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local_min)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())
