"""Scheduling autotuner for the batched grid / degrid calls.

The batched calls (``device.grid`` / ``device.degrid`` with a ``device.Batch``) run one persistent
launch whose CTAs take work items from a queue; how fast they go depends on the workload: how many
facets a warp applies to a stripe before moving on (facets per pack: inputs re-read per pack
against the L2 working set of the pack's grids and CF tables), how many stripes one queue item
holds (queue traffic against load balance) and whether the gridder's warps sum a stripe into a
shared-memory tile before adding it to the grid (fewer grid additions against shared-memory round
trips; pays when a stripe's footprints overlap a lot).  ``tune`` times every candidate on a sample
of the workload's blocks (scratch grids and a scratch copy of the visibilities, so the caller's
data are untouched), keeps the fastest for each call, and caches the choice in a JSON file keyed
by the workload's shape and the GPU's name.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os
from typing import Dict, List, Optional, Sequence

import torch

from . import device as D

GRID_CANDIDATES: List[dict] = [dict(facets_per_pack=p, stripes_per_item=s, tiles=t)
                               for p in (8, 16, 32) for s in (0, 64) for t in (False, True)]
DEGRID_CANDIDATES: List[dict] = [dict(facets_per_pack=p, stripes_per_item=s) for p in (16, 32, 0) for s in (0, 64)]


def _cache_path() -> str:
    return os.environ.get("DDFG_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "ddfacet_b200",
                                                          "autotune.json"))


def workload_key(vs: D.VisData, facets: Sequence[D.FacetGrid], pol, jones: Optional[D.JonesData]) -> str:
    """Hash of what the best schedule depends on: grid sizes, facet count, block count (rounded to a
    power of two), channels, correlations, Stokes planes, single-visibility map, supports, Jones mode,
    FP64 accumulation, large-block list and the GPU."""
    sizes = sorted({tuple(f.grid.shape) for f in facets})
    nb = max(1, int(vs.nblocks))
    desc = dict(sizes=sizes, nfacets=len(facets), nblocks_log2=nb.bit_length(), nchan=int(vs.vis.shape[1]),
                ncorr=int(vs.vis.shape[2]), npol=int(pol.npol), single=int(vs.single_vis_blocks),
                sup=max(int(f.cf.max_support) for f in facets), jones=0 if jones is None else int(jones.mode),
                acc64=any(f.grid_acc is not None for f in facets), large=vs.large_blocks is not None,
                gpu=torch.cuda.get_device_name(vs.vis.device))
    return hashlib.sha1(json.dumps(desc, sort_keys=True, default=str).encode()).hexdigest()[:16]


def sample_blocks(vs: D.VisData, nblocks: int) -> D.VisData:
    """The first ``nblocks`` blocks of ``vs`` (block starts and sparsification cut; the large-block
    list is kept, the kernels skip its entries beyond the sample).  A contiguous prefix keeps the
    map's locality -- the CTAs of the full call work on neighbouring stripes at any moment, and
    their L2 reuse of grid lines is what the schedules trade against each other; a sample of
    stripes taken at a stride over the whole map loses it and ranks the schedules wrongly."""
    n = min(int(nblocks), vs.nblocks)
    sp = None if vs.sparsification is None else vs.sparsification[:n]
    return dataclasses.replace(vs, block_start=vs.block_start[:n], nblocks=n, sparsification=sp)


def _time(fn, reps: int = 2) -> float:
    fn()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _refine(table: Dict[str, list], name: str, best_ms: float, tol: float, call, dev) -> Optional[dict]:
    """Times the sample's near-best candidates of ``name`` once each on the full call (the
    kernels are loaded by then); records them as ``name + "_full"`` and returns the fastest, or
    None when there is no tie to break."""
    near = sorted([(ms, c) for c, ms in table[name] if ms <= best_ms * (1. + tol)], key=lambda x: x[0])[:3]
    if len(near) < 2:
        return None
    s = torch.cuda.current_stream()
    full = []
    for _, cand in near:
        b = D.Batch.create(dev, **cand)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        call(b)
        e1.record(s)
        torch.cuda.synchronize()
        full.append((cand, round(e0.elapsed_time(e1), 3)))
    table[name + "_full"] = full
    return min(full, key=lambda x: x[1])[0]


@dataclasses.dataclass
class Tuned:
    grid: D.Batch
    degrid: D.Batch
    grid_ms: float
    degrid_ms: float
    table: Dict[str, list]
    cached: bool = False

    def describe(self) -> dict:
        def short(c):
            return "fpp%d/spi%d%s" % (c.get("facets_per_pack", 0), c.get("stripes_per_item", 0),
                                      "/tiles" if c.get("tiles") else "")

        return {"grid": self.grid.describe(), "degrid": self.degrid.describe(), "cached": self.cached,
                "sample_grid_ms": round(self.grid_ms, 3), "sample_degrid_ms": round(self.degrid_ms, 3),
                "timed_ms": {k: {short(c): ms for c, ms in v} for k, v in self.table.items()}}


def tune(vs: D.VisData, facets_grid: Sequence[D.FacetGrid], facets_model: Sequence[D.FacetGrid], pol,
         jones: Optional[D.JonesData] = None, sample_fraction: float = 0.02, min_blocks: int = 1 << 21,
         use_cache: bool = True, grid_candidates=None, degrid_candidates=None, refine: bool = True,
         refine_tol: float = 0.03) -> Tuned:
    """Times every candidate schedule of the batched grid and degrid calls on a sample of ``vs``'s
    blocks; with ``refine``, the candidates within ``refine_tol`` of the sample's best (at most
    three) are then timed once on the full call, since a sample's cache behaviour cannot separate
    near ties (packs of 16 and 32 facets tie on a 2 % sample of the at-scale chunk and differ by
    4 % on the whole of it).  Returns the fastest of each (cached by ``workload_key``)."""
    dev = vs.vis.device
    key = workload_key(vs, facets_grid, pol, jones)
    path = _cache_path()
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                hit = json.load(f).get(key)
            if hit:
                return Tuned(D.Batch.create(dev, **hit["grid"]), D.Batch.create(dev, **hit["degrid"]), hit["grid_ms"],
                             hit["degrid_ms"], {}, cached=True)
        except (OSError, ValueError, TypeError):
            pass
    n = max(min_blocks, int(vs.nblocks * sample_fraction))
    sv = sample_blocks(vs, n)
    scratch = [dataclasses.replace(f, grid=torch.zeros_like(f.grid),
                                   grid_acc=None if f.grid_acc is None else torch.zeros_like(f.grid_acc),
                                   sumwt=None if f.sumwt is None else torch.zeros_like(f.sumwt),
                                   sumjones=None if f.sumjones is None else torch.zeros_like(f.sumjones),
                                   sumjones_chan=None if f.sumjones_chan is None else torch.zeros_like(f.sumjones_chan))
               for f in facets_grid]
    table: Dict[str, list] = {"grid": [], "degrid": []}
    best_g, best_gms = None, float("inf")
    cands = list(grid_candidates or GRID_CANDIDATES)
    if not vs.single_vis_blocks:  # warp tiles serve single-visibility maps only; the library ignores them otherwise
        cands = [c for c in cands if not c.get("tiles")]
    for cand in cands:
        b = D.Batch.create(dev, **cand)
        ms = _time(lambda: D.grid(sv, scratch, pol, jones, batch=b))
        table["grid"].append((cand, round(ms, 3)))
        if ms < best_gms:
            best_g, best_gms = cand, ms
    if refine and sv.nblocks < vs.nblocks:
        best_g = _refine(table, "grid", best_gms, refine_tol,
                         lambda b: D.grid(vs, scratch, pol, jones, batch=b), dev) or best_g
    del scratch
    sd = dataclasses.replace(sv, vis=vs.vis.clone())
    best_d, best_dms = None, float("inf")
    for cand in (degrid_candidates or DEGRID_CANDIDATES):
        b = D.Batch.create(dev, **cand)
        ms = _time(lambda: D.degrid(sd, list(facets_model), pol, jones, batch=b))
        table["degrid"].append((cand, round(ms, 3)))
        if ms < best_dms:
            best_d, best_dms = cand, ms
    if refine and sv.nblocks < vs.nblocks:
        full = dataclasses.replace(vs, vis=sd.vis)
        best_d = _refine(table, "degrid", best_dms, refine_tol,
                         lambda b: D.degrid(full, list(facets_model), pol, jones, batch=b), dev) or best_d
        del full
    del sd
    torch.cuda.empty_cache()
    if use_cache:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            data = {}
            if os.path.exists(path):
                with open(path) as f:
                    data = json.load(f)
            data[key] = {"grid": best_g, "degrid": best_d, "grid_ms": best_gms, "degrid_ms": best_dms}
            with open(path, "w") as f:
                json.dump(data, f, indent=1)
        except (OSError, ValueError):
            pass
    return Tuned(D.Batch.create(dev, **best_g), D.Batch.create(dev, **best_d), best_gms, best_dms, table)
