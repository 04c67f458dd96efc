"""Facet geometry: FFT-friendly sizes and the regular facet tessellation (host, one-off).

* ``fft_fast_sizes`` / ``closest_fast_size`` -- sizes 3^a 5^b 7^c x {1, 11, 13} (odd) or with
  powers of 2 (even), restating ``GiveFFTFastSizes`` / ``GiveClosestFastSize``
  (DDFacet/ToolsDir/ModToolBox.py:273-302).
* ``estimate_npix``   -- ``EstimateNpix`` (ModToolBox.py:64-88): (non-padded, padded) odd sizes,
                          padded size at least ``min_size_fft`` = 513.
* ``regular_facets``  -- the NxN square tessellation of ``ClassFacetMachine.setFacetsLocs`` and
                          ``AppendFacet`` (ClassFacetMachine.py:321-548): facet centres (l0, m0),
                          facet and padded grid sizes, central pixel and pixel box in the main
                          image, nearest-solution index.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np


def fft_fast_sizes(odd=True, nlim=100000):
    sizes = np.array([1])
    for base, powers in [(2, [0] if odd else range(1, 20)), (3, range(15)), (5, range(15)), (7, range(15))]:
        sizes = (sizes[np.newaxis, :] * base ** np.array(powers)[:, np.newaxis]).ravel()
    sizes = sizes[np.newaxis, :] * np.array([1, 11, 13])[:, np.newaxis]
    return np.array(sorted(sizes[(sizes < nlim) & (sizes > 64)]))


_ODD = fft_fast_sizes(True, 200000)
_EVEN = fft_fast_sizes(False, 200000)


def closest_fast_size(n, odd=True):
    tab = _ODD if odd else _EVEN
    return int(tab[np.argmin(np.abs(n - tab))])


def estimate_npix(npix, padding=1.0, min_size_fft=513):
    npix = int(round(npix))
    npix = closest_fast_size(npix, odd=True)
    npix_opt = npix
    npix = npix * padding
    if npix < min_size_fft:
        npix = min_size_fft
    npix = int(round(npix))
    npix = closest_fast_size(npix, odd=True)
    return npix_opt, npix


@dataclass
class FacetGeom:
    index: int
    l0: float
    m0: float
    npix_facet: int
    npix_padded: int
    pix_central: tuple
    pix_extent: tuple       # (x0, x1, y0, y1) in the main image
    isol: int


@dataclass
class Tessellation:
    npix: int               # main image side
    npix_facet: int
    npix_padded: int
    cell_rad: float
    facets: List[FacetGeom]


def regular_facets(npix_image, nfacets_side, cell_arcsec, padding):
    cell_rad = cell_arcsec / 3600.0 * np.pi / 180.0
    npix_facet, _ = estimate_npix(float(npix_image) / nfacets_side, padding=1)
    npix = npix_facet * nfacets_side
    _, npix_padded = estimate_npix(npix_facet, padding=padding)
    radius_tot = cell_rad * npix * 0.5
    radius_facet = npix_facet * cell_rad * 0.5
    lc = radius_tot - radius_facet
    lf, mf = np.mgrid[-lc:lc:nfacets_side * 1j, -lc:lc:nfacets_side * 1j]
    lf = lf.flatten()
    mf = mf.flatten()
    out = []
    for i in range(lf.size):
        l0, m0 = float(lf[i]), float(mf[i])
        d = np.sqrt((l0 - lf) ** 2 + (m0 - mf) ** 2)
        isol = int(np.where(d == np.min(d))[0][0])
        xc = int(round(l0 / cell_rad + npix // 2))
        yc = int(round(m0 / cell_rad + npix // 2))
        out.append(FacetGeom(i, l0, m0, npix_facet, npix_padded, (xc, yc),
                             (xc - npix_facet // 2, xc + npix_facet // 2 + 1, yc - npix_facet // 2,
                              yc + npix_facet // 2 + 1), isol))
    return Tessellation(npix, npix_facet, npix_padded, cell_rad, out)
