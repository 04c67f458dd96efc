"""Errors of the whole GPU imaging path against the FP64 direct Fourier transform (oracle/dft.py),
stated rather than targeted: W-projection with a truncated (support 7), oversampled convolution
function and a taper correction differs from the exact transform at the 1e-4 (dirty image) to 1e-2
(prediction of point sources off the facet centre) level, as the reference's own CPU path does on
the same grids (printed beside it).

* degrid: point sources on pixel centres of the model image -> every facet's model grid
  (FacetMachine.image_to_facets) -> the batched degrid of all facets into zero visibilities,
  against the DFT prediction of the same sources (the degridder subtracts: its output is -V);
* grid: visibilities of the same sources from the FP64 DFT -> the batched grid of all facets ->
  the stitched, normalised dirty image, against the FP64 direct dirty image at the source pixels.

Image pixel (i, j) of the main image is at (l, m) = ((i - M//2) cell, (j - M//2) cell), the
reference's convention (facet centres sit at l0 / cell + M//2, ClassFacetMachine.py:414-548).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(nfs):
    import torch

    from ddfacet_b200 import device as D, synth
    from ddfacet_b200.facetmachine import FacetMachine

    obs = synth.make_observation(77, 20, 1500.0, 34.0, 40.0, 40 * 30.0 / 3600.0, 30.0, 8, 1.30e9, 1.45e9)
    wmax = float(np.abs(obs.uvw[:, 2]).max()) * 1.01
    fm = FacetMachine(512, 4.0, nfs, obs.freqs, padding=1.7, nband=1, stokes_ids=(1,), corr_ids=(9, 10, 11, 12),
                      support=7, nw=8, wmax=wmax, device=torch.device("cuda", 0))
    M = fm.npix_out
    cell = fm.tess.cell_rad
    rng = np.random.default_rng(3)
    pix = rng.integers(M // 2 - M // 3, M // 2 + M // 3, size=(6, 2))
    flux = rng.uniform(0.2, 1.0, 6)
    l = (pix[:, 0] - M // 2) * cell
    m = (pix[:, 1] - M // 2) * cell
    return obs, fm, pix, flux, l, m


@pytest.mark.parametrize("nfs", [1, 3])
def test_degrid_against_dft(nfs):
    import torch

    from ddfacet_b200 import bda, device as D
    from oracle import dft

    obs, fm, pix, flux, l, m = _setup(nfs)
    M = fm.npix_out
    img = np.zeros((1, 1, M, M), np.float32)
    img[0, 0, pix[:, 0], pix[:, 1]] = flux
    fm.image_to_facets(torch.from_numpy(img))
    vis = np.zeros((obs.nrow, obs.freqs.size, 4), np.complex64)
    vs = D.VisData.create(vis, obs.uvw, np.zeros(vis.shape, bool), np.ones(vis.shape[:2], np.float32), obs.freqs,
                          np.zeros(obs.freqs.size, np.int32), bda.plain_map(obs.A0, obs.A1, obs.freqs.size),
                          device=fm.device)
    D.degrid(vs, [f.model for f in fm.facets], fm.pol, batch=D.Batch.create(fm.device))
    got = -vs.vis.cpu().numpy()[:, :, 0].astype(np.complex128)
    want = dft.predict(obs.uvw, obs.freqs, l, m, flux)
    # the reference's own degridder on the same model grids, for comparison
    from oracle import ref

    bmap = bda.plain_map(obs.A0, obs.A1, obs.freqs.size)
    refv = np.zeros_like(vis)
    for f in fm.facets:
        wt = f.wterms
        ref.degrid(f.model.grid.cpu().numpy(), refv, obs.uvw, np.zeros(vis.shape, bool), wt.Wplanes, wt.WplanesConj,
                   np.array([wt.RefWave, wt.wmax, len(wt.Wplanes), fm.overs], np.float64), np.array(f.model.incr),
                   obs.freqs, np.array([wt.Cu, wt.Cv, f.geom.l0, f.geom.m0, f.geom.index], np.float64), bmap,
                   np.zeros(obs.freqs.size, np.int32), [9, 10, 11, 12], [1])
    refp = -refv[:, :, 0].astype(np.complex128)
    err = float(np.sqrt(np.mean(np.abs(got - want) ** 2) / np.mean(np.abs(want) ** 2)))
    eref = float(np.sqrt(np.mean(np.abs(refp - want) ** 2) / np.mean(np.abs(want) ** 2)))
    print(f"{nfs}x{nfs} facets: degrid vs FP64 DFT rel RMS: gpu {err:.2e}, reference {eref:.2e}")
    assert err < 5e-2 and err < 1.05 * eref + 1e-4


@pytest.mark.parametrize("nfs", [1, 3])
def test_grid_against_dft(nfs):
    import torch

    from ddfacet_b200 import bda, device as D
    from oracle import dft

    obs, fm, pix, flux, l, m = _setup(nfs)
    v = dft.predict(obs.uvw, obs.freqs, l, m, flux)
    vis = np.zeros((obs.nrow, obs.freqs.size, 4), np.complex64)
    vis[:, :, 0] = v
    vis[:, :, 3] = v
    w = np.ones(vis.shape[:2], np.float32)
    vs = D.VisData.create(vis, obs.uvw, np.zeros(vis.shape, bool), w, obs.freqs, np.zeros(obs.freqs.size, np.int32),
                          bda.plain_map(obs.A0, obs.A1, obs.freqs.size), device=fm.device)
    fm.reset_grids()
    D.grid(vs, [f.grid for f in fm.facets], fm.pol, batch=D.Batch.create(fm.device))
    image = fm.facets_to_image().cpu().numpy()[0, 0]
    got = image[pix[:, 0], pix[:, 1]].astype(np.float64)
    want = dft.dirty(obs.uvw, obs.freqs, v, w, l, m)
    err = float(np.sqrt(np.mean((got - want) ** 2) / np.mean(want ** 2)))
    print(f"{nfs}x{nfs} facets: dirty image at the sources vs FP64 direct dirty image rel RMS {err:.2e}")
    assert err < 2e-2
