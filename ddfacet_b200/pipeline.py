"""Residual step over host-resident visibilities with the copies overlapped.

A major-cycle step on visibilities that live in host memory: every row chunk is copied to the GPU,
its facets' model predictions are subtracted (degrid), the residuals are gridded onto every facet,
and the residual visibilities are copied back -- what DDFacet does chunk by chunk through its
visibility server (ClassVisServer / ClassFacetMachine.putChunk / getChunk), here with the
host->device copy of chunk k+1 and the device->host copy of chunk k-1 running on their own
streams while the kernels work on chunk k.  Gridding is linear, so the facets' grids accumulate
over the chunks exactly as over the whole set.

Each chunk is a ``device.VisData`` over a row range of the device buffers, with a block map whose
row indices are relative to the chunk (the reference's chunks carry their own maps too), and the
matching slice of the per-row Jones maps.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence, Tuple

import torch

from . import device as D


@dataclasses.dataclass
class Chunk:
    rows: Tuple[int, int]               # [row0, row1) of the full set
    vs: D.VisData                       # views of the device buffers for these rows
    jones: Optional[D.JonesData] = None


def jones_rows(jones: Optional[D.JonesData], row0: int, row1: int) -> Optional[D.JonesData]:
    """The per-row Jones maps (time slots, antennas) restricted to a row range."""
    if jones is None:
        return None
    cut = lambda t: None if t is None else t[row0:row1]  # noqa: E731
    return dataclasses.replace(jones, kms_tmap=cut(jones.kms_tmap), beam_tmap=cut(jones.beam_tmap),
                               a0=cut(jones.a0), a1=cut(jones.a1))


class PipelinedStep:
    """Degrid-then-grid of every chunk with overlapped copies.

    ``run(host)`` takes pinned host tensors ``vis`` (complex64 [nrow][nchan][ncorr]), ``uvw``,
    ``flags``, ``weights`` and ``out`` (complex64, receives the residual visibilities) and
    returns when the copies are queued; the caller synchronises.  With ``batch_grid`` /
    ``batch_degrid`` the chunks go through the batched (queue-driven) calls."""

    def __init__(self, chunks: Sequence[Chunk], facets_grid: List[D.FacetGrid], facets_model: List[D.FacetGrid],
                 pol, device=None, batch_grid: Optional[D.Batch] = None, batch_degrid: Optional[D.Batch] = None):
        self.chunks = list(chunks)
        self.facets_grid = facets_grid
        self.facets_model = facets_model
        self.pol = pol
        self.batch_grid = batch_grid
        self.batch_degrid = batch_degrid
        dev = D._dev(device)
        self.h2d = torch.cuda.Stream(device=dev)
        self.d2h = torch.cuda.Stream(device=dev)

    def run(self, host: dict, stream: Optional[torch.cuda.Stream] = None):
        comp = stream or torch.cuda.current_stream()
        loaded, done = [], []
        with torch.cuda.stream(self.h2d):
            self.h2d.wait_stream(comp)  # the device buffers are free once earlier work is done
            for c in self.chunks:
                r0, r1 = c.rows
                c.vs.vis.copy_(host["vis"][r0:r1], non_blocking=True)
                c.vs.uvw.copy_(host["uvw"][r0:r1], non_blocking=True)
                c.vs.flags.copy_(host["flags"][r0:r1], non_blocking=True)
                c.vs.weights.copy_(host["weights"][r0:r1], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.h2d)
                loaded.append(ev)
        for c, ev in zip(self.chunks, loaded):
            comp.wait_event(ev)
            D.degrid(c.vs, self.facets_model, self.pol, c.jones, stream=comp, batch=self.batch_degrid)
            D.grid(c.vs, self.facets_grid, self.pol, c.jones, stream=comp, batch=self.batch_grid)
            e = torch.cuda.Event()
            e.record(comp)
            done.append(e)
        with torch.cuda.stream(self.d2h):
            for c, e in zip(self.chunks, done):
                self.d2h.wait_event(e)
                r0, r1 = c.rows
                host["out"][r0:r1].copy_(c.vs.vis, non_blocking=True)
        comp.wait_stream(self.d2h)
