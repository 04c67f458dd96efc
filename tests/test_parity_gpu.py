"""GPU kernels vs the reference's own CPU gridder/degridder on identical inputs.

Tolerances: grids and degridded visibilities within 1e-4 relative RMS of the reference's
complex64 path; the set of grid cells touched (which encodes every integer index: w plane,
location, oversampling phase, skipped blocks) identical; weight sums within 1e-9 relative.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _cmp_grid(c, **kw):
    r = cases.run_ref_grid(c, **kw)
    g = cases.run_gpu_grid(c, **kw)
    assert cases.rel_rms(g["grid"], r["grid"]) < TOL
    np.testing.assert_array_equal(g["grid"] != 0, r["grid"] != 0)
    np.testing.assert_allclose(g["sumwt"], r["sumwt"], rtol=1e-9)
    if c.jones:
        np.testing.assert_allclose(g["sumjones"], r["sumjones"], rtol=1e-5)
        np.testing.assert_allclose(g["sumjones_chan"], r["sumjones_chan"], rtol=1e-5)
    return r, g


def _cmp_degrid(c, model=None):
    if model is None:
        model = cases.run_ref_grid(c)["grid"]
    vr = cases.run_ref_degrid(c, model, vis0=c.vis)
    vg = cases.run_gpu_degrid(c, model, vis0=c.vis)
    # compare the predictions (vis0 - result) so the input visibilities do not dilute the error
    assert cases.rel_rms(c.vis - vg, c.vis - vr) < TOL
    return vr, vg


def test_grid_plain_stokes_i():
    _cmp_grid(cases.make_case())


def test_degrid_plain_stokes_i():
    _cmp_degrid(cases.make_case())


@pytest.mark.parametrize("stokes", [(1,), (1, 2), (1, 2, 3, 4), (2,), (3,), (4,), (1, 4), (2, 3), (1, 2, 3), (1, 3)])
def test_grid_linear_4corr(stokes):
    _cmp_grid(cases.make_case(ncorr=4, stokes_ids=stokes, nw=3))


@pytest.mark.parametrize("stokes", [(1,), (1, 2), (1, 3), (1, 4), (2, 3), (1, 2, 3), (1, 2, 3, 4)])
def test_grid_circular_4corr(stokes):
    _cmp_grid(cases.make_case(ncorr=4, corr_ids=[5, 6, 7, 8], stokes_ids=stokes, nw=3))


@pytest.mark.parametrize("corr,stokes", [([9, 12], (1,)), ([9, 12], (1, 2)), ([5, 8], (1,)), ([5, 8], (1, 4))])
def test_grid_2corr(corr, stokes):
    _cmp_grid(cases.make_case(ncorr=2, corr_ids=corr, stokes_ids=stokes, nw=3))


@pytest.mark.parametrize("corr,stokes", [
    ([9, 10, 11, 12], (1,)), ([9, 10, 11, 12], (2,)), ([9, 10, 11, 12], (3,)), ([9, 10, 11, 12], (4,)),
    ([9, 10, 11, 12], (1, 2, 3, 4)), ([5, 6, 7, 8], (1, 2, 3, 4)), ([9, 10, 11, 12], (1, 2)),
    ([5, 6, 7, 8], (1, 2)), ([9, 12], (1, 2)), ([9, 10, 11, 12], (1, 3)), ([5, 6, 7, 8], (1, 3)),
    ([5, 6, 7, 8], (1, 4)), ([9, 10, 11, 12], (1, 4)), ([5, 8], (1, 4)), ([9, 10, 11, 12], (2, 3)),
    ([9, 10, 11, 12], (1, 2, 3)), ([5, 6, 7, 8], (1, 2, 3)), ([5, 8], (1,)), ([1], (1,))])
def test_degrid_policies(corr, stokes):
    c = cases.make_case(ncorr=len(corr), corr_ids=corr, stokes_ids=stokes, nw=3)
    rng = np.random.default_rng(3)
    model = (rng.standard_normal((1, len(stokes), c.npix, c.npix)) +
             1j * rng.standard_normal((1, len(stokes), c.npix, c.npix))).astype(np.complex64)
    _cmp_degrid(c, model)


def test_grid_offset_facet_and_bands():
    c = cases.make_case(lm=(0.01, -0.007), nband=2, nchan=8)
    _cmp_grid(c)
    _cmp_degrid(c)


@pytest.mark.parametrize("mode", [1, 2])
def test_bda_blocks(mode):
    c = cases.make_case(bda_mode=mode, dphi=np.sqrt(6 * 0.05), nchan=16, flag_frac=0.1)
    _cmp_grid(c)
    _cmp_degrid(c)


def test_flags_and_sparsification():
    c = cases.make_case(flag_frac=0.3)
    _cmp_grid(c)
    nb = int(c.bda[0])
    sp = np.random.default_rng(0).uniform(size=nb) < 0.5
    r = cases.run_ref_grid(c, sparsification=sp)
    from ddfacet_b200 import device as D
    import torch
    vs, fg, jd = cases._gpu_objs(c)
    vs.sparsification = torch.from_numpy(sp.astype(np.uint8)).cuda()
    D.grid(vs, [fg], D.make_pol(c.corr_ids, c.stokes_ids), jd)
    assert cases.rel_rms(fg.grid.cpu().numpy(), r["grid"]) < TOL
    np.testing.assert_allclose(fg.sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)


@pytest.mark.parametrize("jmode,psf,scale", [(0, False, 0), (1, False, 0), (2, False, 0), (1, True, 0), (2, True, 0),
                                             (1, False, 1)])
def test_large_blocks(jmode, psf, scale):
    """Mode-1 maps whose short-baseline blocks hold hundreds of visibilities (one lane walks
    each): grid, touched cells, weight and Jones sums and prediction against the reference, with
    per-visibility, per-block and uv-dependent (DoScaleJones) Jones and in PSF mode."""
    c = cases.make_case(bda_mode=1, dphi=np.sqrt(6 * 1.0), nchan=16, ntimes=60, flag_frac=0.1, ncorr=4)
    nb = int(np.uint32(c.bda[0]))
    sz = c.bda[2:2 + nb].astype(np.int64)
    st = 2 + nb + np.concatenate([[0], np.cumsum(sz)[:-1]])
    nv = (sz - 2) * (c.bda[st + 1] - c.bda[st])
    assert (nv > 128).sum() >= 32 and nv.max() >= 900
    if jmode:
        cases.add_jones(c, mode=jmode, nt=3, nd=3, scale=scale, calib_err=0.05 if scale else 0.0)
    _cmp_grid(c, dopsf=psf)
    if not psf:
        _cmp_degrid(c)


@pytest.mark.parametrize("jmode,psf,sparse", [(0, False, True), (1, False, False), (2, False, False), (1, True, False),
                                              (2, True, True)])
def test_large_block_list(jmode, psf, sparse):
    """Blocks of more than 128 visibilities given a whole warp each (VisData.with_large_blocks,
    ddfg_vis large_blocks): grid, touched cells, weight and Jones sums and prediction against the
    reference, with a sparsification mask in some cases."""
    import torch

    from ddfacet_b200 import device as D

    c = cases.make_case(bda_mode=1, dphi=np.sqrt(6 * 1.0), nchan=16, ntimes=60, flag_frac=0.1, ncorr=4)
    if jmode:
        cases.add_jones(c, mode=jmode, nt=3, nd=3)
    nb = int(np.uint32(c.bda[0]))
    sp = (np.random.default_rng(2).uniform(size=nb) < 0.7) if sparse else None
    r = cases.run_ref_grid(c, dopsf=psf, sparsification=sp)
    pol = D.make_pol(c.corr_ids, c.stokes_ids)
    vs, fg, jd = cases._gpu_objs(c)
    if sparse:
        vs.sparsification = torch.from_numpy(sp.astype(np.uint8)).cuda()
    vs = vs.with_large_blocks(128)
    assert vs.large_blocks is not None and vs.large_blocks.numel() >= 32
    D.grid(vs, [fg], pol, jd, dopsf=psf)
    g = fg.grid.cpu().numpy()
    assert cases.rel_rms(g, r["grid"]) < TOL
    np.testing.assert_array_equal(g != 0, r["grid"] != 0)
    np.testing.assert_allclose(fg.sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)
    if jmode:
        np.testing.assert_allclose(fg.sumjones.cpu().numpy(), r["sumjones"], rtol=1e-5)
        np.testing.assert_allclose(fg.sumjones_chan.cpu().numpy(), r["sumjones_chan"], rtol=1e-5)
    if not psf:
        model = cases.run_ref_grid(c)["grid"]
        vr = cases.run_ref_degrid(c, model, vis0=c.vis)
        vs2, fm, jd2 = cases._gpu_objs(c, model_grid=model)
        vs2 = vs2.with_large_blocks(128)
        D.degrid(vs2, [fm], pol, jd2)
        assert cases.rel_rms(c.vis - vs2.vis.cpu().numpy(), c.vis - vr) < TOL


def test_large_block_list_needs_uv_independent_jones():
    from ddfacet_b200 import device as D

    c = cases.make_case(bda_mode=1, dphi=np.sqrt(6 * 1.0), nchan=16, ntimes=60, ncorr=4)
    cases.add_jones(c, mode=1, nt=3, nd=3, scale=1, calib_err=0.05)
    vs, fg, jd = cases._gpu_objs(c)
    with pytest.raises(ValueError, match="large-block list"):
        D.grid(vs.with_large_blocks(128), [fg], D.make_pol(c.corr_ids, c.stokes_ids), jd)


@pytest.mark.parametrize("jmode", [0, 1, 2])
def test_bda_blocks_in_uv_order(jmode):
    """The blocks of a mode-1 map visited in uv Z order (VisData.with_block_order): grid, weight
    sums and prediction against the reference run on the original map, with a sparsification
    mask that follows its blocks."""
    import torch

    from ddfacet_b200 import bda, device as D

    c = cases.make_case(bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=16, flag_frac=0.1, ncorr=4)
    if jmode:
        cases.add_jones(c, mode=jmode, nt=3, nd=3)
    nb = int(c.bda[0])
    sp = np.random.default_rng(1).uniform(size=nb) < 0.7
    r = cases.run_ref_grid(c, sparsification=sp)
    model = r["grid"]
    vr = cases.run_ref_degrid(c, model, vis0=c.vis)
    pol = D.make_pol(c.corr_ids, c.stokes_ids)
    vs, fg, jd = cases._gpu_objs(c)
    vs.sparsification = torch.from_numpy(sp.astype(np.uint8)).cuda()
    order = bda.uv_locality_order(vs.bda_map, vs.block_start, vs.uvw, vs.freqs, 200.0)
    assert not torch.equal(order, torch.arange(nb, device=order.device))
    vs2 = vs.with_block_order(order)
    D.grid(vs2, [fg], pol, jd)
    assert cases.rel_rms(fg.grid.cpu().numpy(), r["grid"]) < TOL
    np.testing.assert_array_equal(fg.grid.cpu().numpy() != 0, r["grid"] != 0)
    np.testing.assert_allclose(fg.sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)
    vs2.sparsification = None
    fm = cases._gpu_objs(c, model_grid=model)[1]
    D.degrid(vs2, [fm], pol, jd)
    assert cases.rel_rms(c.vis - vs2.vis.cpu().numpy(), c.vis - vr) < TOL


@pytest.mark.parametrize("jmode,beam,kms,interp", [(1, False, True, 0), (1, True, True, 0), (2, False, True, 0),
                                                   (2, True, True, 0), (1, True, False, 0), (1, False, True, 1)])
def test_jones(jmode, beam, kms, interp):
    c = cases.make_case(ncorr=4, stokes_ids=(1,), nw=3, bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=8)
    cases.add_jones(c, mode=jmode, beam=beam, kms=kms, interp_mode=interp)
    _cmp_grid(c)
    _cmp_degrid(c)


@pytest.mark.parametrize("amp,phase", [(0, 1), (1, 0)])
def test_jones_norm_modes(amp, phase):
    c = cases.make_case(ncorr=4, stokes_ids=(1,), nw=3)
    cases.add_jones(c, mode=1, apply_amp=amp, apply_phase=phase)
    _cmp_grid(c)
    _cmp_degrid(c)


def test_jones_psf():
    c = cases.make_case(ncorr=4, stokes_ids=(1,), nw=3, bda_mode=1, dphi=np.sqrt(6 * 0.05))
    cases.add_jones(c, mode=1, beam=True)
    _cmp_grid(c, dopsf=True)
    c2 = cases.make_case(ncorr=4, stokes_ids=(1,), nw=3, bda_mode=1, dphi=np.sqrt(6 * 0.05))
    cases.add_jones(c2, mode=2)
    _cmp_grid(c2, dopsf=True)
    _cmp_grid(cases.make_case(), dopsf=True)


def test_smearing():
    c = cases.make_case(lm=(0.008, 0.004), bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=8)
    c.smear = cases.smear_list(c, lm=(0.012, 0.006))
    _cmp_grid(c)
    _cmp_degrid(c)


def test_multi_facet_call_matches_single_calls():
    import torch
    from ddfacet_b200 import device as D
    cs = [cases.make_case(lm=lm, nw=3) for lm in [(0.0, 0.0), (0.01, 0.0), (0.0, -0.01)]]
    for c in cs[1:]:
        c.vis = cs[0].vis  # one visibility set, three facets
    singles = [cases.run_gpu_grid(c)["grid"] for c in cs]
    objs = [cases._gpu_objs(c) for c in cs]
    vs = objs[0][0]
    D.grid(vs, [o[1] for o in objs], D.make_pol([1], [1]))
    for o, s in zip(objs, singles):
        np.testing.assert_allclose(o[1].grid.cpu().numpy(), s, rtol=1e-5, atol=1e-6 * np.abs(s).max())
    # degrid: one call over three facets equals the sum of three single-facet predictions
    models = [cases.run_ref_grid(c)["grid"] for c in cs]
    vis0 = cs[0].vis
    want = vis0.copy()
    for c, m in zip(cs, models):
        want = want - (vis0 - cases.run_ref_degrid(c, m, vis0=vis0))
    objs = [cases._gpu_objs(c, model_grid=m, vis=vis0) for c, m in zip(cs, models)]
    D.degrid(objs[0][0], [o[1] for o in objs], D.make_pol([1], [1]))
    got = objs[0][0].vis.cpu().numpy()
    assert cases.rel_rms(vis0 - got, vis0 - want) < TOL


def test_uneven_facets_one_call():
    """Facets of different grid sizes (and more than one launch's worth) in one grid and one
    degrid call, each against the reference on that facet alone."""
    from ddfacet_b200 import device as D
    sizes = [255, 201, 311, 149] * 5  # 20 facets: two launches of facet descriptors
    lms = [(0.004 * (i % 5) - 0.008, 0.003 * (i // 5) - 0.004) for i in range(len(sizes))]
    cs = [cases.make_case(npix=n, lm=lm, nw=2, ncorr=4, stokes_ids=(1,), ntimes=10) for n, lm in zip(sizes, lms)]
    for c in cs[1:]:
        c.vis = cs[0].vis
    objs = [cases._gpu_objs(c) for c in cs]
    D.grid(objs[0][0], [o[1] for o in objs], D.make_pol(cs[0].corr_ids, [1]))
    refs = [cases.run_ref_grid(c) for c in cs]
    for o, r in zip(objs, refs):
        g = o[1].grid.cpu().numpy()
        assert cases.rel_rms(g, r["grid"]) < TOL
        np.testing.assert_array_equal(g != 0, r["grid"] != 0)
        np.testing.assert_allclose(o[1].sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)
    # degrid into zeros, so the comparison sees the predictions themselves rather than their
    # small difference from the visibilities (whose float32 rounding would dominate)
    vis0 = np.zeros_like(cs[0].vis)
    want = vis0.copy()
    for c, r in zip(cs, refs):
        want = want + cases.run_ref_degrid(c, r["grid"], vis0=vis0)
    objs = [cases._gpu_objs(c, model_grid=r["grid"], vis=vis0) for c, r in zip(cs, refs)]
    D.degrid(objs[0][0], [o[1] for o in objs], D.make_pol(cs[0].corr_ids, [1]))
    got = objs[0][0].vis.cpu().numpy()
    assert cases.rel_rms(vis0 - got, vis0 - want) < TOL


def test_unsupported_combination_raises():
    c = cases.make_case(ncorr=2, corr_ids=[9, 12], stokes_ids=(3,), nw=3)
    with pytest.raises(ValueError, match="Cannot convert input correlations"):
        cases.run_gpu_grid(c)
