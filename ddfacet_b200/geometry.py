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
from typing import List, Optional

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
    polygon: Optional[np.ndarray] = None   # [k][2] (l, m) vertices of a tessellation cell


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


# ------------------------------------------------------------------------------------------
# Voronoi tessellation (ClassFacetMachineTessel.setFacetsLocs, ClassFacetMachineTessel.py:65-866)
# ------------------------------------------------------------------------------------------
def _clip_halfplane(poly, a, b, c):
    """The part of a convex polygon with a x + b y <= c (one Sutherland-Hodgman step)."""
    out = []
    n = len(poly)
    for i in range(n):
        p, q = poly[i], poly[(i + 1) % n]
        fp = a * p[0] + b * p[1] - c
        fq = a * q[0] + b * q[1] - c
        if fp <= 0:
            out.append(p)
        if (fp < 0 < fq) or (fq < 0 < fp):
            t = fp / (fp - fq)
            out.append((p[0] + t * (q[0] - p[0]), p[1] + t * (q[1] - p[1])))
    return out


def voronoi_cells(l, m, radius):
    """The Voronoi cell of every direction (l[i], m[i]) inside the square [-radius, radius]^2:
    the square clipped by the perpendicular bisector of the direction and every other one.
    Directions whose cell is empty get None."""
    sq = [(-radius, -radius), (radius, -radius), (radius, radius), (-radius, radius)]
    cells = []
    for i in range(len(l)):
        poly = list(sq)
        for j in range(len(l)):
            if j == i or not poly:
                continue
            # |x - p_i|^2 <= |x - p_j|^2  <=>  2 (p_j - p_i) . x <= |p_j|^2 - |p_i|^2
            a = 2.0 * (l[j] - l[i])
            b = 2.0 * (m[j] - m[i])
            c = (l[j] ** 2 + m[j] ** 2) - (l[i] ** 2 + m[i] ** 2)
            poly = _clip_halfplane(poly, a, b, c)
        cells.append(np.array(poly) if len(poly) >= 3 else None)
    return cells


def polygon_centroid(poly):
    """Area centroid of a simple polygon."""
    x, y = poly[:, 0], poly[:, 1]
    xs, ys = np.roll(x, -1), np.roll(y, -1)
    cross = x * ys - xs * y
    area = cross.sum() / 2.0
    return float(((x + xs) * cross).sum() / (6.0 * area)), float(((y + ys) * cross).sum() / (6.0 * area))


def voronoi_facets(npix_image, cell_arcsec, l_dirs, m_dirs, padding, oversize=1.0):
    """Facets of a Voronoi tessellation around the given directions, sized by the reference's
    rules: the cell's bounding box inside the image about its centroid gives the diameter
    (ClassFacetMachineTessel.py:626-648, kept in float32 as there), the facets are ordered by
    decreasing diameter (:652-654), the centre and the diameter are rounded to whole cells
    (:766-775) and sized by EstimateNpix with and without padding (AppendFacet,
    ClassFacetMachine.py:321-399).  DiamMax subdivision and DiamMin merging (:344-587) are not
    applied (their defaults, 180 and 0 degrees, do neither)."""
    cell_rad = cell_arcsec / 3600.0 * np.pi / 180.0
    npix, _ = estimate_npix(float(npix_image), padding=1)
    radius = cell_rad * npix / 2
    l_dirs = np.asarray(l_dirs, np.float64)
    m_dirs = np.asarray(m_dirs, np.float64)
    cells = voronoi_cells(l_dirs, m_dirs, radius) if l_dirs.size > 1 else [
        np.array([(-radius, -radius), (radius, -radius), (radius, radius), (-radius, radius)])]
    polys = [c for c in cells if c is not None]
    lmd = np.zeros((len(polys), 4), np.float32)
    lmd[:, 3] = np.arange(len(polys))
    for i, poly in enumerate(polys):
        l0 = max(-radius, poly[:, 0].min())
        l1 = min(radius, poly[:, 0].max())
        m0 = max(-radius, poly[:, 1].min())
        m1 = min(radius, poly[:, 1].max())
        lc, mc = polygon_centroid(poly)
        dl = max(abs(l0 - lc), abs(l1 - lc))
        dm = max(abs(m0 - mc), abs(m1 - mc))
        lmd[i, 0], lmd[i, 1], lmd[i, 2] = lc, mc, 2 * max(dl, dm)
    lmd = lmd[np.argsort(lmd[:, 2])[::-1]]
    out = []
    npix_facets, npix_pads = [], []
    for k in range(lmd.shape[0]):
        x0 = round(float(lmd[k, 0]) / cell_rad)
        y0 = round(float(lmd[k, 1]) / cell_rad)
        l0, m0 = x0 * cell_rad, y0 * cell_rad
        diam = round(float(lmd[k, 2]) / cell_rad) * cell_rad * oversize
        nf, _ = estimate_npix(diam / cell_rad, padding=1)
        _, npad = estimate_npix(nf, padding=padding)
        d = np.sqrt((l0 - l_dirs) ** 2 + (m0 - m_dirs) ** 2)
        isol = int(np.where(d == np.min(d))[0][0])
        xc = int(round(l0 / cell_rad + npix // 2))
        yc = int(round(m0 / cell_rad + npix // 2))
        out.append(FacetGeom(k, l0, m0, nf, npad, (xc, yc), (xc - nf // 2, xc + nf // 2 + 1, yc - nf // 2,
                                                             yc + nf // 2 + 1), isol, polys[int(lmd[k, 3])]))
        npix_facets.append(nf)
        npix_pads.append(npad)
    return Tessellation(npix, max(npix_facets), max(npix_pads), cell_rad, out)
