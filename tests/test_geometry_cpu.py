"""Voronoi tessellation (geometry.voronoi_facets, restating ClassFacetMachineTessel's sizing):
the cells partition the image square and contain their own direction; facet sizes follow the
reference's rules (EstimateNpix: odd fast sizes, padded grids >= 513 -> 525); facets come in
order of decreasing cell diameter; the main image of 6000 pixels becomes 6075."""
import numpy as np

from ddfacet_b200 import geometry as G


def _area(poly):
    x, y = poly[:, 0], poly[:, 1]
    return 0.5 * abs(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


def test_cells_partition_the_square():
    rng = np.random.default_rng(0)
    r = 0.01
    l, m = rng.uniform(-r, r, 25), rng.uniform(-r, r, 25)
    cells = G.voronoi_cells(l, m, r)
    assert all(c is not None for c in cells)
    assert abs(sum(_area(c) for c in cells) - (2 * r) ** 2) < 1e-12 * (2 * r) ** 2
    for i, c in enumerate(cells):
        # the direction is inside its own convex cell
        lc, mc = G.polygon_centroid(c)
        n = len(c)
        s = []
        for k in range(n):
            e = c[(k + 1) % n] - c[k]
            q = np.array([l[i], m[i]]) - c[k]
            s.append(e[0] * q[1] - e[1] * q[0])
        assert all(v >= -1e-18 for v in s) or all(v <= 1e-18 for v in s)
        assert abs(lc) <= r and abs(mc) <= r


def test_facet_sizes_follow_reference_rules():
    rng = np.random.default_rng(1)
    cell = 1.0
    r = 6075 * cell / 3600 * np.pi / 180 / 2
    t = G.voronoi_facets(6000, cell, rng.uniform(-r, r, 25), rng.uniform(-r, r, 25), 1.7)
    assert t.npix == 6075
    fast = set(G.fft_fast_sizes(odd=True))
    for f in t.facets:
        assert f.npix_facet in fast and f.npix_padded in fast
        assert f.npix_padded >= 525 and f.npix_padded >= f.npix_facet
        assert f.npix_padded == G.estimate_npix(f.npix_facet, 1.7)[1]
    diams = [f.npix_facet for f in t.facets]
    assert diams == sorted(diams, reverse=True)
    assert t.npix_padded == max(f.npix_padded for f in t.facets)


def test_single_direction_is_the_whole_image():
    t = G.voronoi_facets(1000, 2.0, [0.0], [0.0], 1.7)
    assert len(t.facets) == 1
    f = t.facets[0]
    assert f.npix_facet == G.estimate_npix(t.npix * 1.0, 1)[0]
