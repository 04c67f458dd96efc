"""CPU tests: the host restatements and the FP64 oracle pinned to fixtures the reference made
(tests/golden/make_golden.py), and the oracle's own checks.  No GPU needed."""
import os

import numpy as np
import pytest

import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name), allow_pickle=False)


def test_cf_tables_match_reference():
    from ddfacet_b200 import cf

    g = _load("cf_golden.npz")
    for i in range(2):
        w = cf.WTerms(Cell=3.0, Sup=7, Npix=129, Freqs=g["freqs"], wmax=3000.0, Nw=4, OverS=11,
                      lmShift=tuple(g[f"f{i}_lm"]))
        np.testing.assert_array_equal(np.array(w.Sups), g[f"f{i}_sups"])
        np.testing.assert_allclose([w.Cu, w.Cv], g[f"f{i}_cucv"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(w.ifzfCF, g[f"f{i}_ifzf"], rtol=1e-12, atol=1e-14)
        for k in range(4):
            a, b = g[f"f{i}_w{k}"], g[f"f{i}_wc{k}"]
            assert w.Wplanes[k].dtype == np.complex64 and w.Wplanes[k].shape == a.shape
            np.testing.assert_allclose(w.Wplanes[k], a, rtol=0, atol=1e-7 * np.abs(a).max())
            np.testing.assert_allclose(w.WplanesConj[k], b, rtol=0, atol=1e-7 * np.abs(b).max())


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("which", ["a", "b"])
def test_bda_maps_bit_exact(mode, which):
    from ddfacet_b200 import bda

    g = _load("bda_golden.npz")
    m = bda.smear_mapping(g["A0"], g["A1"], g["uvw"], g["freqs"], float(g["dfreq"]), float(g[f"dphi_{which}"]),
                          float(g["l"]), g["chan_map"], mode=mode)
    np.testing.assert_array_equal(m, g[f"map_mode{mode}_{which}"])


def test_plain_map_is_mode1_without_averaging():
    from ddfacet_b200 import bda

    g = _load("bda_golden.npz")
    a = bda.plain_map(g["A0"], g["A1"], g["freqs"].size)
    b = bda.smear_mapping(g["A0"], g["A1"], g["uvw"], g["freqs"], float(g["dfreq"]), 0.0, float(g["l"]),
                          np.zeros(g["freqs"].size, np.int32), mode=1)
    np.testing.assert_array_equal(a, b)


def test_bda_header_words():
    from ddfacet_b200 import bda

    h = bda._header((5 << 32) + 7)
    assert int(np.uint32(h[0].view(np.uint32))) == 7 and int(h[1]) == 5


def _golden_case():
    g = _load("grid_golden.npz")
    c = cases.Case()
    c.vis, c.uvw, c.flags, c.weights, c.freqs = g["vis"], g["uvw"], g["flags"], g["weights"], g["freqs"]
    c.chan_map, c.bda, c.incr, c.winfos = g["chan_map"], g["bda"], g["incr"], g["winfos"]
    c.facet_infos, c.lm = g["facet_infos"], tuple(g["lm"])
    nw = int(g["nw"])

    class WT:
        pass

    c.wt = WT()
    c.wt.Wplanes = [g[f"w{k}"] for k in range(nw)]
    c.wt.WplanesConj = [g[f"wc{k}"] for k in range(nw)]
    c.wt.RefWave, c.wt.wmax = c.winfos[0], c.winfos[1]
    c.wt.Cu, c.wt.Cv = c.facet_infos[0], c.facet_infos[1]
    c.nrow, c.nchan = c.vis.shape[:2]
    c.corr_ids, c.stokes_ids, c.nband, c.npol, c.npix = [9, 10, 11, 12], [1], 2 if c.chan_map.max() > 0 else 1, 1, \
        g["grid"].shape[-1]
    c.nband = g["grid"].shape[0]
    c.jones = {"kms": g["jones_kms"], "kms_tmap": g["jones_tmap"], "kms_cmap": g["jones_cmap"], "A0": g["A0"],
               "A1": g["A1"], "idir_kms": int(g["idir"]), "idir_beam": 0, "mode": 1, "interp_mode": 0,
               "apply_amp": 1, "apply_phase": 1, "scale": 0, "calib_err": 0.0}
    c.smear = None
    return c, g


def test_fp64_oracle_against_reference_golden():
    c, g = _golden_case()
    f = cases.run_fp64_grid(c)
    e = cases.rel_rms(g["grid"], f["grid"])
    assert e < 1e-6, e
    np.testing.assert_array_equal(g["grid"] != 0, f["grid"] != 0)
    np.testing.assert_allclose(f["sumwt"], g["sumwt"], rtol=1e-12)
    np.testing.assert_allclose(f["sumjones"], g["sumjones"], rtol=1e-9)
    np.testing.assert_allclose(f["sumjones_chan"], g["sumjones_chan"], rtol=1e-9)
    vf = cases.run_fp64_degrid(c, g["grid"], vis0=c.vis)
    # the model here is the dirty grid, whose taps cancel strongly: the reference's float products
    # then differ from the FP64 sums by a few 1e-5
    assert cases.rel_rms(c.vis - g["vis_degrid"], c.vis - vf) < 2e-4


def test_reference_module_reproduces_golden():
    from oracle import ref

    if not ref.available():
        pytest.skip("reference gridder not built here")
    c, g = _golden_case()
    r = cases.run_ref_grid(c)
    np.testing.assert_array_equal(r["grid"], g["grid"])
    np.testing.assert_array_equal(r["sumwt"], g["sumwt"])
    vr = cases.run_ref_degrid(c, g["grid"], vis0=c.vis)
    np.testing.assert_array_equal(vr, g["vis_degrid"])


def test_spatial_weight_smoothing_matches_reference():
    from ddfacet_b200.facetmachine import convolve_gaussian

    g = _load("sw_golden.npz")
    got = convolve_gaussian(g["mask"], (10, 10, 0), cell_rad=1.0)
    np.testing.assert_allclose(got, g["sw"], rtol=0, atol=1e-5 * np.abs(g["sw"]).max())


def test_fp64_oracle_rejects_unsupported_policy():
    c = cases.make_case(ncorr=2, corr_ids=[9, 12], stokes_ids=(3,), nw=2, ntimes=4, nant=4)
    with pytest.raises(ValueError):
        cases.run_fp64_grid(c)


def test_estimate_npix_and_regular_facets():
    from ddfacet_b200 import geometry as G

    assert G.estimate_npix(1024, 1.7) == (1029, 1755)
    assert G.estimate_npix(455, 1.7) == (455, 735)
    assert G.estimate_npix(909, 1.7) == (891, 1485)
    t = G.regular_facets(4096, 9, 1.5, 1.7)
    assert (t.npix, t.npix_facet, t.npix_padded, len(t.facets)) == (4095, 455, 735, 81)
    t = G.regular_facets(10000, 11, 1.0, 1.7)
    assert (t.npix, t.npix_facet, t.npix_padded) == (9801, 891, 1485)


def test_model_tessel_adjoint_dot_product():
    """give_model_tessel_adjoint is the adjoint of give_model_tessel for real images: Re <y, A x> =
    <A^H y, x> within the forward's float32 rounding (1e-5 relative), for facets inside, across
    and at the corner of the image, with taper cells below 1e-3."""
    from oracle import facets as OF

    rng = np.random.default_rng(0)
    n, m = 55, 120
    sphe = rng.uniform(0.0, 1.0, (n, n)).astype(np.float32)
    sphe[0, :] = 1e-4
    sw = rng.uniform(0.0, 1.0, (n, n)).astype(np.float32)
    norm = rng.uniform(0.5, 1.5, (m, m)).astype(np.float32)
    for xc, yc in [(60, 60), (10, 100), (115, 3)]:
        x = rng.standard_normal((1, 2, m, m)).astype(np.float32)
        y = rng.standard_normal((1, 2, n, n)) + 1j * rng.standard_normal((1, 2, n, n))
        ax = OF.give_model_tessel(x, norm, sphe, sw, xc, yc, n, 11)
        lhs = float(np.sum(np.conj(y) * ax).real)
        rhs = float(np.sum(OF.give_model_tessel_adjoint(y, norm, sphe, sw, xc, yc, m, 11) * x))
        assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
