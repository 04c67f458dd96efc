"""A degrid-then-grid step captured in a CUDA graph (device.capture_graph) and replayed gives the
eager step's residual visibilities and grids (1e-6 relative: only the order of the atomic
additions differs)."""
import pytest
import torch

from ddfacet_b200 import configs, device as D

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.to(torch.complex128)
    b = b.to(torch.complex128)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_graph_replay_matches_eager():
    w = configs.multifacet_dde(device=torch.device("cuda", 0), scale=0.01, nfacets_side=2, nchan=16, nw=8, nsrc=20)
    vis0 = w.vs.vis.clone()

    def step():
        for f in w.facets_grid:
            f.grid.zero_()
        D.degrid(w.vs, w.facets_model, w.pol, w.jones)
        D.grid(w.vs, w.facets_grid, w.pol, w.jones)

    step()
    torch.cuda.synchronize()
    want_vis = w.vs.vis.clone()
    want = [f.grid.clone() for f in w.facets_grid]
    g = D.capture_graph(step)
    w.vs.vis.copy_(vis0)
    g.replay()
    torch.cuda.synchronize()
    assert _rel(vis0 - w.vs.vis, vis0 - want_vis) < 1e-6
    for f, x in zip(w.facets_grid, want):
        assert _rel(f.grid, x) < 1e-6
