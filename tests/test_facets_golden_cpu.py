"""The NumPy restatement of the per-facet transforms and the stitching (oracle/facets.py) and the
host-side facet-norm builder against the reference's own functions run on a regular 3 x 3 and an
uneven 4-facet tessellation (tests/golden/facets_golden.npz, made by tests/golden/make_golden.py
--only facets from ClassDDEGridMachine.GridToIm, ClassFacetMachine.BuildFacetNormImage /
FacetsToIm_Channel and ClassImToGrid.GiveModelTessel(ToGrid=True)).

The regular case holds a band with zero weight sum (stitched without normalisation) and a facet
whose padded box sees negative model components only: the reference's SumFlux is zero there and
GiveModelTessel returns the scaled model without the FFT (ClassImToGrid.py:249-256)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "facets_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _facets(g, name):
    n = len(g[f"{name}_sizes"])
    return [{k: g[f"{name}_f{i}_{k}"] for k in ("grid", "dirty", "sphe", "invsphe", "sw", "sumweights",
                                                 "sumjonesnorm", "model_grid", "sumflux")} for i in range(n)]


def _rel(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2)) / np.sqrt(np.mean(np.abs(b) ** 2)))


@pytest.mark.parametrize("name", ["reg", "vor"])
def test_grid_to_im(gold, name):
    from oracle import facets as OF

    for f in _facets(gold, name):
        # the reference transforms in complex64 storage; the restatement in complex128
        assert _rel(OF.grid_to_im(f["grid"], int(gold["overs"])), f["dirty"]) < 1e-6


@pytest.mark.parametrize("name", ["reg", "vor"])
def test_facet_norm(gold, name):
    from oracle import facets as OF
    from ddfacet_b200 import geometry
    from ddfacet_b200.facetmachine import FacetMachine

    m = int(gold[f"{name}_m"])
    fs = _facets(gold, name)
    cs, ns = gold[f"{name}_centres"], gold[f"{name}_sizes"]
    want = gold[f"{name}_facet_norm"]
    got = OF.facet_norm([f["sw"] for f in fs], [tuple(c) for c in cs], ns, m)
    np.testing.assert_array_equal(got, want)
    # the facet machine's own host builder, in the same facet order
    host = np.zeros((m, m), np.float32)
    for f, c, n in zip(fs, cs, ns):
        geom = geometry.FacetGeom(0, 0.0, 0.0, int(n), int(n), (int(c[0]), int(c[1])), (0, 0, 0, 0), 0)
        FacetMachine._add_norm(host, f["sw"], geom, int(n))
    np.testing.assert_array_equal(host, want)


@pytest.mark.parametrize("name", ["reg", "vor"])
def test_facets_to_im_channel(gold, name):
    from oracle import facets as OF

    m = int(gold[f"{name}_m"])
    fs = _facets(gold, name)
    img = OF.facets_to_im_channel([f["dirty"] for f in fs], [f["sphe"] for f in fs], [f["invsphe"] for f in fs],
                                  [f["sw"] for f in fs],
                                  [f["sumweights"] * np.sqrt(f["sumjonesnorm"])[:, None] for f in fs],
                                  [tuple(c) for c in gold[f"{name}_centres"]], m, gold[f"{name}_facet_norm"])
    want = gold[f"{name}_image"]
    np.testing.assert_allclose(img, want, rtol=0, atol=1e-6 * np.abs(want).max())


@pytest.mark.parametrize("name", ["reg", "vor"])
def test_give_model_tessel(gold, name):
    from oracle import facets as OF

    model, norm = gold[f"{name}_model"], gold[f"{name}_facet_norm"]
    quirk = 0
    for f, c, n in zip(_facets(gold, name), gold[f"{name}_centres"], gold[f"{name}_sizes"]):
        want = f["model_grid"]
        if float(f["sumflux"]) == 0.0 and np.abs(want).max() > 0:
            # no positive component: the reference leaves the facet model untransformed
            got = OF.give_model_tessel(model, norm, f["sphe"], f["sw"], int(c[0]), int(c[1]), int(n),
                                       int(gold["overs"]), transform=False)
            np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)
            quirk += 1
            continue
        got = OF.give_model_tessel(model, norm, f["sphe"], f["sw"], int(c[0]), int(c[1]), int(n), int(gold["overs"]))
        assert _rel(got, want) < 1e-6
    assert quirk == (1 if name == "reg" else 0)
