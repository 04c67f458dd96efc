"""Per-facet GPU transforms and stitching against the NumPy restatement of the reference
(oracle/facets.py): GridToIm, FacetsToIm_Channel (+ facet norm), GiveModelTessel(ToGrid).
Tolerance: 1e-5 relative RMS (complex64 cuFFT against complex128 numpy)."""
import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def _fm(kind, nfs=3, npix=1200):
    from ddfacet_b200 import geometry
    from ddfacet_b200.facetmachine import FacetMachine

    freqs = np.linspace(1.3e9, 1.45e9, 8)
    tess = None
    if kind == "voronoi":  # five directions: uneven facets (ClassFacetMachineTessel)
        r = npix * 6.0 / 3600 * np.pi / 180 / 2
        rng = np.random.default_rng(4)
        tess = geometry.voronoi_facets(npix, 6.0, rng.uniform(-0.8 * r, 0.8 * r, 5), rng.uniform(-0.8 * r, 0.8 * r, 5),
                                       1.7)
        assert len({f.npix_padded for f in tess.facets}) > 1
    return FacetMachine(npix, 6.0, nfs, freqs, padding=1.7, nband=1, stokes_ids=(1,), corr_ids=(9, 10, 11, 12),
                        support=7, nw=3, wmax=2000.0, mixing_width=10.0, tessellation=tess)


@pytest.mark.parametrize("kind", ["regular", "voronoi"])
def test_grid_to_image_and_stitch(kind):
    from oracle import facets as OF

    fm = _fm(kind)
    rng = np.random.default_rng(0)
    grids = []
    for f in fm.facets:
        g = (rng.standard_normal(f.grid.grid.shape) + 1j * rng.standard_normal(f.grid.grid.shape)).astype(np.complex64)
        grids.append(g)
        f.grid.grid.copy_(torch.from_numpy(g))
        f.grid.sumwt.fill_(123.0)
    image = fm.facets_to_image().cpu().numpy()
    dirties = [OF.grid_to_im(g, fm.overs) for g in grids]
    for f, d in zip(fm.facets, dirties):
        got = f.grid.grid.cpu().numpy()  # transformed in place
        assert cases.rel_rms(got, d) < 1e-5
    want = OF.facets_to_im_channel(dirties, [f.sphe.cpu().numpy() for f in fm.facets],
                                   [f.invsphe.cpu().numpy() for f in fm.facets], [f.sw_host for f in fm.facets],
                                   [np.full((1, 1), 123.0) for _ in fm.facets], [f.geom.pix_central for f in fm.facets],
                                   fm.npix_out, fm.facet_norm_host)
    assert cases.rel_rms(image, want) < 1e-5


@pytest.mark.parametrize("kind", ["regular", "voronoi"])
def test_image_to_grid(kind):
    from oracle import facets as OF

    fm = _fm(kind)
    rng = np.random.default_rng(1)
    img = np.zeros((1, 1, fm.npix_out, fm.npix_out), np.float32)
    for _ in range(30):
        img[0, 0, rng.integers(0, fm.npix_out), rng.integers(0, fm.npix_out)] = rng.uniform(0.01, 1.0)
    fm.image_to_facets(torch.from_numpy(img))
    for f in fm.facets:
        want = OF.give_model_tessel(img, fm.facet_norm_host, f.sphe.cpu().numpy(), f.sw_host, *f.geom.pix_central,
                                    f.model.grid.shape[-1], fm.overs)
        got = f.model.grid.cpu().numpy()
        if np.abs(want).max() == 0:
            assert np.abs(got).max() == 0
        else:
            assert cases.rel_rms(got, want) < 1e-5
