"""The imaging-weight oracle (oracle/weights.py) against the reference's own outputs
(tests/golden/weights_golden.npz, made by tests/golden/make_golden.py from ClassVisServer's
_uv_to_index / _finalizeWeights_handler and the compiled pyAccumulateWeightsOntoGridNoSem):
indices bit-exact, density grids and Briggs grids to 1e-12 relative, weights to 1 float32 ulp."""
import os

import numpy as np
import pytest

from oracle import weights as W

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(HERE, "golden", "weights_golden.npz")))


def test_geometry(gold):
    uvmax = W.uvmax_wavelengths(gold["uvw"], np.zeros(len(gold["uvw"]), bool), gold["freqs"])
    assert uvmax == gold["uvmax"]
    cell, xymax, npixx, npixy, npix = W.grid_geometry(uvmax, float(gold["cell_rad"]), int(gold["npix_image"]),
                                                      float(gold["super_uniform"]))
    assert (cell, xymax, npixx, npix) == (gold["cell"], gold["xymax"], gold["npixx"], gold["npix"])


@pytest.mark.parametrize("nbands", [1, 2])
def test_weight_pipeline(gold, nbands):
    cell, xymax, npixx, npix = float(gold["cell"]), int(gold["xymax"]), int(gold["npixx"]), int(gold["npix"])
    w = gold["weights_in"].copy()
    uv = gold["uvw"][:, :2].copy()
    index = W.uv_to_index(uv, w, gold["freqs"], cell, npix, npixx, nbands, xymax, gold["band_of_chan"])
    np.testing.assert_array_equal(index, gold[f"index_{nbands}"])
    grid = W.accumulate(np.zeros((nbands, npix)), w, index)
    np.testing.assert_allclose(grid, gold[f"grid_{nbands}"], rtol=1e-12, atol=0)
    W.robust(grid, float(gold["robust"]))
    np.testing.assert_allclose(grid, gold[f"grid_briggs_{nbands}"], rtol=1e-12)
    out = W.finalize(w, W.uv_to_index(uv, w, gold["freqs"], cell, npix, npixx, nbands, xymax, gold["band_of_chan"]),
                     grid)
    np.testing.assert_array_max_ulp(out, gold[f"weights_briggs_{nbands}"], maxulp=1)
