"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host-side exchange.

The hot path shards without a data-path collective in the two ways the facet machine allows:

* replicas -- each rank images its own visibility chunk (a time range) onto its own copy of all
  facet grids; ranks only agree on timing (``max_over_ranks``).  This is what ``bench.py --gpus N``
  runs (weak scaling).
* by facet -- each rank grids and degrids its share of the facets (``shard_facets``) over the
  same visibilities.  Gridding needs no exchange; the degridded predictions of all ranks are
  summed once per chunk (``reduce_predictions``), which the reference does by serialising the
  subtraction of every facet process into one shared array (degridder.h:236-263).
  ``sharded_residual_step`` composes the two for one chunk.

Everything here runs on CPU tensors with the gloo backend as well (tested that way).
"""
from __future__ import annotations

import dataclasses
from typing import Callable, List, Optional, Sequence

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


def sharded_residual_step(vs, facets_model: Sequence, facets_grid: Sequence, pol, jones, rank: int, world: int,
                          group=None, batch_degrid=None, batch_grid=None, degrid: Optional[Callable] = None,
                          grid: Optional[Callable] = None) -> List[int]:
    """One major-cycle pass over a chunk with the facets sharded over ``world`` ranks that share the
    chunk's visibilities: this rank degrids its facets into a zero buffer (the library's degridder
    subtracts, so the buffer holds minus its facets' prediction), the buffers are summed over ranks
    (``reduce_predictions``), the sum is added to ``vs.vis`` (every rank then holds the same
    residual visibilities) and this rank grids the residuals onto its facets.  Returns the indices
    of this rank's facets.  ``degrid`` / ``grid`` default to the library's batched calls
    (``device.degrid`` / ``device.grid``)."""
    if degrid is None or grid is None:
        from . import device as D

        degrid = degrid or D.degrid
        grid = grid or D.grid
    mine = shard_facets(len(facets_model), rank, world)
    pred = torch.zeros_like(vs.vis)
    degrid(dataclasses.replace(vs, vis=pred), [facets_model[i] for i in mine], pol, jones, batch=batch_degrid)
    reduce_predictions(pred, group=group)
    vs.vis.add_(pred)
    grid(vs, [facets_grid[i] for i in mine], pol, jones, batch=batch_grid)
    return mine
