"""The pipelined residual step (ddfacet_b200.pipeline): time chunks with their own block maps and
Jones row maps, copies overlapped with the kernels, gives the same residual visibilities and
facet grids as one degrid + grid over the whole device-resident set (1e-5 relative: only the
order of the floating-point additions differs)."""
import numpy as np
import pytest
import torch

from ddfacet_b200 import configs, device as D, pipeline

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.to(torch.complex128)
    b = b.to(torch.complex128)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_pipelined_step_matches_whole_set():
    dev = torch.device("cuda", 0)
    w = configs.multifacet_dde(device=dev, scale=0.01, nfacets_side=2, nchan=16, nw=8, nsrc=20)
    vis0 = w.vs.vis.clone()
    for f in w.facets_grid:
        f.grid.zero_()
    D.degrid(w.vs, w.facets_model, w.pol, w.jones)
    D.grid(w.vs, w.facets_grid, w.pol, w.jones)
    want_vis = w.vs.vis.clone()
    want_grids = [f.grid.clone() for f in w.facets_grid]

    host = {"vis": vis0.cpu().pin_memory(), "uvw": w.vs.uvw.cpu().pin_memory(),
            "flags": w.vs.flags.cpu().pin_memory(), "weights": w.vs.weights.cpu().pin_memory()}
    host["out"] = torch.empty_like(host["vis"]).pin_memory()
    chunks = configs.row_chunks(w, 3)
    assert len(chunks) == 3 and chunks[0].rows[0] == 0 and chunks[-1].rows[1] == w.nrow
    step = pipeline.PipelinedStep(chunks, w.facets_grid, w.facets_model, w.pol, dev)
    for f in w.facets_grid:
        f.grid.zero_()
    w.vs.vis.zero_()
    step.run(host)
    torch.cuda.synchronize()
    got = host["out"].to(dev)
    assert _rel(vis0 - got, vis0 - want_vis) < 1e-5
    for f, g in zip(w.facets_grid, want_grids):
        assert _rel(f.grid, g) < 1e-5
