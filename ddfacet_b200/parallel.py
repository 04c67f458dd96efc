"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host-side exchange.

The hot path shards without a data-path collective in the two ways the facet machine allows:

* replicas -- each rank images its own visibility chunk (a time range) onto its own copy of all
  facet grids; ranks only agree on timing (``max_over_ranks``).  This is what ``bench.py --gpus N``
  runs (weak scaling).
* by facet -- each rank grids and degrids its share of the facets (``shard_facets``) over the
  same visibilities.  Gridding needs no exchange; the degridded predictions of all ranks are
  summed once per chunk (``reduce_predictions``), which the reference does by serialising the
  subtraction of every facet process into one shared array (degridder.h:236-263).

Everything here runs on CPU tensors with the gloo backend as well (tested that way).
"""
from __future__ import annotations

from typing import List

import torch
import torch.distributed as dist


def shard_facets(nfacets: int, rank: int, world: int) -> List[int]:
    """Contiguous, balanced facet indices of ``rank`` (sizes differ by at most one)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(nfacets, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def reduce_predictions(pred: torch.Tensor, group=None) -> torch.Tensor:
    """Sum over ranks of each rank's degridded prediction (in place) and return it."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        if pred.is_complex():
            dist.all_reduce(torch.view_as_real(pred), op=dist.ReduceOp.SUM, group=group)
        else:
            dist.all_reduce(pred, op=dist.ReduceOp.SUM, group=group)
    return pred


def max_over_ranks(value: float, device=None, group=None) -> float:
    """Largest value over ranks (timings are reported as the slowest rank's)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        return float(t.item())
    return float(value)
