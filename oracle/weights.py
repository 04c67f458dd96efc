"""NumPy restatement of DDFacet's imaging-weight computation -- TEST INFRASTRUCTURE ONLY.

Follows DDFacet/Data/ClassVisServer.py and DDFacet/Gridder/GridderSmearPols.cc:
  * uvmax_wavelengths   -- _loadWeights_handler, ClassVisServer.py:947-951
  * grid_geometry       -- _CalcWeights_serial, ClassVisServer.py:866-883
  * uv_to_index         -- _uv_to_index, ClassVisServer.py:981-1003
  * accumulate          -- pyAccumulateWeightsOntoGridNoSem, GridderSmearPols.cc:55-74
  * robust              -- the Briggs step of _CalcWeights_serial, ClassVisServer.py:897-904
  * finalize            -- _finalizeWeights_handler, ClassVisServer.py:1036-1043
The checker of the GPU kernels in ddfacet_b200/csrc/ddfg_weights.cu; never imported by the
product.  Pinned against the reference itself by tests/golden/weights_golden.npz.
"""
import math

import numpy as np

C_LIGHT = 299792458.0


def uvmax_wavelengths(uvw, rowflags, freqs):
    uv = uvw[:, :2]
    return abs(uv[~rowflags, :]).max() * np.max(freqs) / C_LIGHT


def grid_geometry(uvmax, cell_rad, npix_image, super_uniform=1.0):
    """(cell, xymax, npixx, npixy, npix) of the weight grid."""
    fov = cell_rad * npix_image
    cell = 1. / (super_uniform * fov)
    xymax = int(math.floor(uvmax / cell)) + 1
    npixx = xymax * 2 + 1
    npixy = xymax + 1
    return cell, xymax, npixx, npixy, npixx * npixy


def uv_to_index(uv, weights, freqs, cell, npix, npixx, nbands, xymax, band_of_chan=None):
    """Index of every (row, channel) into the [nbands][npix] weight grid; uv is flipped in place
    where v < 0, as the reference does."""
    uv[uv[:, 1] < 0] *= -1
    uvl = uv[..., np.newaxis] * freqs[np.newaxis, np.newaxis, :] / C_LIGHT
    uvl = np.floor(uvl / cell).astype(int)
    x = uvl[:, 0, :]
    y = uvl[:, 1, :]
    x += xymax
    index = np.zeros((uvl.shape[0], len(freqs)), np.int32)
    index[...] = y * npixx + x
    if nbands > 1:
        index += np.asarray(band_of_chan)[np.newaxis, :] * npix
    index[weights == 0] = 0
    return index


def accumulate(grid, weights, index):
    """grid[index] += weight for every non-zero weight, in order (float64 grid)."""
    g = grid.reshape(-1)
    w = weights.reshape(-1)
    i = index.reshape(-1)
    nz = np.flatnonzero(w != 0)
    np.add.at(g, i[nz].astype(np.int64), w[nz].astype(np.float64))  # in order, as the C loop
    return grid


def robust(grid, robust_param):
    """Briggs: per band, grid = 1 + grid * (5 * 10^-R)^2 / (sum g^2 / sum g)."""
    numerator_sqrt = 5.0 * 10 ** (-robust_param)
    for band in range(grid.shape[0]):
        g = grid[band, :]
        avg_w = (g ** 2).sum() / g.sum()
        s_sq = numerator_sqrt ** 2 / avg_w
        g[...] = 1 + g * s_sq
    return grid


def finalize(weights, index, grid):
    """weight /= grid[index] (float32 weights, float64 grid), indices past the grid read cell 0."""
    g = grid.reshape(-1)
    index = index.copy()
    index[index >= len(g)] = 0
    weights /= g[index]
    return weights
