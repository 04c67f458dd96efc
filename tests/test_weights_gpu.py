"""Imaging-weight kernels (ddfacet_b200.weights, ddfg_weights_*) against the reference's outputs
(tests/golden/weights_golden.npz) and the oracle: indices bit-exact; density grids to 1e-12
relative (float64 atomics change only the order of the additions); final weights to 1 float32
ulp; a larger case against the oracle."""
import os

import numpy as np
import pytest
import torch

from ddfacet_b200.weights import ImagingWeights
from oracle import weights as W

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(HERE, "golden", "weights_golden.npz")))


@pytest.mark.parametrize("nbands", [1, 2])
def test_against_reference(gold, nbands):
    iw = ImagingWeights(float(gold["uvmax"]), float(gold["cell_rad"]), int(gold["npix_image"]), mode="briggs",
                        robust=float(gold["robust"]), nbands=nbands, super_uniform=float(gold["super_uniform"]))
    assert (iw.xymax, iw.npixx, iw.npix) == (gold["xymax"], gold["npixx"], gold["npix"])
    _, index = iw._index(gold["uvw"], gold["freqs"], gold["weights_in"], gold["band_of_chan"])
    np.testing.assert_array_equal(index.cpu().numpy(), gold[f"index_{nbands}"])
    iw.accumulate(gold["uvw"], gold["freqs"], gold["weights_in"], gold["band_of_chan"])
    np.testing.assert_allclose(iw.grid.cpu().numpy(), gold[f"grid_{nbands}"], rtol=1e-12)
    iw.finish()
    np.testing.assert_allclose(iw.grid.cpu().numpy(), gold[f"grid_briggs_{nbands}"], rtol=1e-12)
    w = iw.apply(gold["uvw"], gold["freqs"], gold["weights_in"], gold["band_of_chan"])
    np.testing.assert_array_max_ulp(w.cpu().numpy(), gold[f"weights_briggs_{nbands}"], maxulp=1)


def test_uniform_multi_chunk_against_oracle():
    """Two chunks accumulated into one grid, uniform weighting, 1.3 M visibilities."""
    rng = np.random.default_rng(5)
    freqs = np.linspace(0.9e9, 1.67e9, 64)
    chunks = []
    for _ in range(2):
        uvw = rng.normal(0, 3000.0, (10000, 3))
        w = rng.uniform(0.1, 1.0, (10000, 64)).astype(np.float32)
        w[rng.uniform(size=w.shape) < 0.05] = 0
        chunks.append((uvw, w))
    uvmax = max(W.uvmax_wavelengths(u, np.zeros(len(u), bool), freqs) for u, _ in chunks)
    cell_rad, npix_image = 1.5 / 3600 * np.pi / 180, 4096
    iw = ImagingWeights(uvmax, cell_rad, npix_image, mode="uniform")
    for uvw, w in chunks:
        iw.accumulate(uvw, freqs, w)
    iw.finish()
    cell, xymax, npixx, _, npix = W.grid_geometry(uvmax, cell_rad, npix_image)
    grid = np.zeros((1, npix))
    idx = []
    for uvw, w in chunks:
        i = W.uv_to_index(uvw[:, :2].copy(), w, freqs, cell, npix, npixx, 1, xymax)
        idx.append(i)
        W.accumulate(grid, w, i)
    np.testing.assert_allclose(iw.grid.cpu().numpy(), grid, rtol=1e-12)
    for (uvw, w), i in zip(chunks, idx):
        got = iw.apply(uvw, freqs, w).cpu().numpy()
        np.testing.assert_array_max_ulp(got, W.finalize(w.copy(), i, grid), maxulp=1)


def test_natural_is_identity():
    w = np.random.default_rng(1).uniform(size=(100, 8)).astype(np.float32)
    iw = ImagingWeights(1000.0, 1e-5, 512, mode="natural")
    np.testing.assert_array_equal(iw.apply(np.zeros((100, 3)), np.ones(8), w).cpu().numpy(), w)
