"""The batched (cell-sorted) kernels against the reference gridder/degridder.

Same tolerances as the direct kernels: 1e-4 relative RMS vs the reference's complex64 path,
identical footprint, weight sums to 1e-9."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _cmp(c, dopsf=False, **kw):
    r = cases.run_ref_grid(c, dopsf=dopsf)
    g = cases.run_gpu_grid(c, dopsf=dopsf, sorted_=True, **kw)
    assert cases.rel_rms(g["grid"], r["grid"]) < TOL
    np.testing.assert_array_equal(g["grid"] != 0, r["grid"] != 0)
    np.testing.assert_allclose(g["sumwt"], r["sumwt"], rtol=1e-9)
    if c.jones:
        np.testing.assert_allclose(g["sumjones"], r["sumjones"], rtol=1e-5)
        np.testing.assert_allclose(g["sumjones_chan"], r["sumjones_chan"], rtol=1e-5)
    if dopsf:
        return
    model = r["grid"]
    vr = cases.run_ref_degrid(c, model, vis0=c.vis)
    vg = cases.run_gpu_degrid(c, model, vis0=c.vis, sorted_=True, chunk=kw.get("chunk", 256))
    assert cases.rel_rms(c.vis - vg, c.vis - vr) < TOL


def test_sorted_plain():
    _cmp(cases.make_case())


def test_sorted_uncompensated_small_chunks():
    _cmp(cases.make_case(), compensated=False, chunk=32)


def test_sorted_large_support_slots():
    # supports 9..15 exercise the 4- and 8-slot register footprints
    _cmp(cases.make_case(sup=9, nw=4, lm=(0.01, -0.01)))
    _cmp(cases.make_case(sup=15, nw=3))


def test_sorted_4corr_jones_bda_flags_bands():
    c = cases.make_case(ncorr=4, stokes_ids=(1, 2, 3, 4), nw=3, bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=16,
                        flag_frac=0.1, lm=(0.01, 0.005), nband=2)
    cases.add_jones(c, mode=1, beam=True)
    _cmp(c)


def test_sorted_jones_mode2_smearing():
    c = cases.make_case(ncorr=4, stokes_ids=(1,), nw=3, bda_mode=2, dphi=np.sqrt(6 * 0.05), nchan=8, lm=(0.006, 0.0))
    cases.add_jones(c, mode=2)
    c.smear = cases.smear_list(c)
    _cmp(c)


def test_sorted_psf():
    c = cases.make_case(ncorr=4, stokes_ids=(1,), nw=3)
    cases.add_jones(c, mode=1)
    _cmp(c, dopsf=True)


def test_sorted_multi_facet():
    from ddfacet_b200 import device as D
    cs = [cases.make_case(lm=lm, nw=3) for lm in [(0.0, 0.0), (0.01, 0.0), (0.0, -0.01), (0.008, 0.008)]]
    for c in cs[1:]:
        c.vis = cs[0].vis
    objs = [cases._gpu_objs(c) for c in cs]
    vs = objs[0][0]
    fgs = [o[1] for o in objs]
    plan = D.SortPlan.build(vs, fgs, chunk=300)
    D.grid_sorted(vs, fgs, D.make_pol([1], [1]), plan, facets_per_launch=3)
    for c, fg in zip(cs, fgs):
        r = cases.run_ref_grid(c)
        assert cases.rel_rms(fg.grid.cpu().numpy(), r["grid"]) < TOL
        np.testing.assert_allclose(fg.sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)
    # degrid all four in one call == sum of four single-facet predictions
    models = [cases.run_ref_grid(c)["grid"] for c in cs]
    vis0 = cs[0].vis
    want = vis0.copy()
    for c, m in zip(cs, models):
        want = want - (vis0 - cases.run_ref_degrid(c, m, vis0=vis0))
    objs = [cases._gpu_objs(c, model_grid=m, vis=vis0) for c, m in zip(cs, models)]
    plan = D.SortPlan.build(objs[0][0], [o[1] for o in objs], chunk=200)
    D.degrid_sorted(objs[0][0], [o[1] for o in objs], D.make_pol([1], [1]), plan, facets_per_launch=3)
    got = objs[0][0].vis.cpu().numpy()
    assert cases.rel_rms(vis0 - got, vis0 - want) < TOL
