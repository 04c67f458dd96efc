"""The batched calls (ddfg_grid_batched / ddfg_degrid_batched: one persistent launch whose CTAs
take work items from a queue in device memory), FP64-accumulated gridding and the large-block
list check.

* batched grid / degrid against the reference on single-visibility maps, averaged BDA blocks
  (modes 1 and 2), large blocks given a warp each, Jones, flags and PSF -- the same tolerances as
  tests/test_parity_gpu.py;
* an uneven multi-facet call under several schedules (facets per pack, stripes per item, CTAs
  per SM, static order, region spreading) against single-facet reference calls;
* FP64-accumulated gridding: within 1e-4 of the reference, at least as close to the FP64
  restatement as float32 accumulation (below 1e-6), and the accumulator left zero;
* ddfg_check_large_blocks rejects lists with an out-of-range, repeated, small or missing block.
"""
import functools

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

TOL = 1e-4


@functools.lru_cache(maxsize=None)
def _case(name):
    if name == "single":
        return cases.make_case(ncorr=4, stokes_ids=(1,), nw=3, lm=(0.006, -0.004))
    if name == "bda1_jones":
        c = cases.make_case(bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=16, flag_frac=0.1, ncorr=4)
        return cases.add_jones(c, mode=1, beam=True)
    if name == "bda2_blockjones":
        c = cases.make_case(bda_mode=2, dphi=np.sqrt(6 * 0.05), nchan=16, flag_frac=0.1, ncorr=4)
        return cases.add_jones(c, mode=2)
    return cases.make_case(ncorr=4, stokes_ids=(1, 2, 3, 4), nw=3, bda_mode=1, dphi=np.sqrt(6 * 0.05))


@pytest.mark.parametrize("name", ["single", "bda1_jones", "bda2_blockjones", "iquv"])
@pytest.mark.parametrize("batch_kw", [{}, {"stripes_per_item": 1, "ctas_per_sm": 1}, {"static": True},
                                      {"tiles": True}, {"tiles": True, "stripes_per_item": 2},
                                      {"spread": True, "stripes_per_item": 1},
                                      {"spread": True, "static": True, "stripes_per_item": 2}])
def test_batched_against_reference(name, batch_kw):
    c = _case(name)
    r = cases.run_ref_grid(c)
    g = cases.run_gpu_grid(c, batched=True, batch_kw=batch_kw)
    assert cases.rel_rms(g["grid"], r["grid"]) < TOL
    np.testing.assert_array_equal(g["grid"] != 0, r["grid"] != 0)
    np.testing.assert_allclose(g["sumwt"], r["sumwt"], rtol=1e-9)
    if c.jones:
        np.testing.assert_allclose(g["sumjones"], r["sumjones"], rtol=1e-5)
        np.testing.assert_allclose(g["sumjones_chan"], r["sumjones_chan"], rtol=1e-5)
    vr = cases.run_ref_degrid(c, r["grid"], vis0=c.vis)
    vg = cases.run_gpu_degrid(c, r["grid"], vis0=c.vis, batched=True, batch_kw=batch_kw)
    assert cases.rel_rms(c.vis - vg, c.vis - vr) < TOL


def test_batched_large_block_items():
    from ddfacet_b200 import device as D

    c = cases.make_case(bda_mode=1, dphi=np.sqrt(6 * 1.0), nchan=16, ntimes=60, flag_frac=0.1, ncorr=4)
    cases.add_jones(c, mode=1, nt=3, nd=3)
    r = cases.run_ref_grid(c)
    pol = D.make_pol(c.corr_ids, c.stokes_ids)
    for kw in ({}, {"stripes_per_item": 2, "ctas_per_sm": 1}):
        vs, fg, jd = cases._gpu_objs(c)
        vs = vs.with_large_blocks(128)
        assert vs.large_blocks is not None and vs.large_blocks.numel() >= 32
        D.grid(vs, [fg], pol, jd, batch=D.Batch.create(vs.vis.device, **kw))
        g = fg.grid.cpu().numpy()
        assert cases.rel_rms(g, r["grid"]) < TOL
        np.testing.assert_array_equal(g != 0, r["grid"] != 0)
        np.testing.assert_allclose(fg.sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)
        np.testing.assert_allclose(fg.sumjones_chan.cpu().numpy(), r["sumjones_chan"], rtol=1e-5)
        vr = cases.run_ref_degrid(c, r["grid"], vis0=c.vis)
        vs2, fm, jd2 = cases._gpu_objs(c, model_grid=r["grid"])
        vs2 = vs2.with_large_blocks(128)
        D.degrid(vs2, [fm], pol, jd2, batch=D.Batch.create(vs.vis.device, **kw))
        assert cases.rel_rms(c.vis - vs2.vis.cpu().numpy(), c.vis - vr) < TOL


@pytest.mark.parametrize("batch_kw", [{}, {"facets_per_pack": 3}, {"facets_per_pack": 1, "stripes_per_item": 3},
                                      {"facets_per_pack": 7, "static": True}, {"ctas_per_sm": 1},
                                      {"tiles": True, "facets_per_pack": 5},
                                      {"spread": True, "facets_per_pack": 4, "stripes_per_item": 1}])
def test_batched_uneven_facets(batch_kw):
    """20 facets of four grid sizes in one batched grid and one batched degrid call, each against
    the reference on that facet alone, under several schedules."""
    from ddfacet_b200 import device as D

    sizes = [255, 201, 311, 149] * 5
    lms = [(0.004 * (i % 5) - 0.008, 0.003 * (i // 5) - 0.004) for i in range(len(sizes))]
    cs = [cases.make_case(npix=n, lm=lm, nw=2, ncorr=4, stokes_ids=(1,), ntimes=10) for n, lm in zip(sizes, lms)]
    for c in cs[1:]:
        c.vis = cs[0].vis
    objs = [cases._gpu_objs(c) for c in cs]
    dev = objs[0][0].vis.device
    D.grid(objs[0][0], [o[1] for o in objs], D.make_pol(cs[0].corr_ids, [1]), batch=D.Batch.create(dev, **batch_kw))
    refs = [cases.run_ref_grid(c) for c in cs]
    for o, r in zip(objs, refs):
        g = o[1].grid.cpu().numpy()
        assert cases.rel_rms(g, r["grid"]) < TOL
        np.testing.assert_array_equal(g != 0, r["grid"] != 0)
        np.testing.assert_allclose(o[1].sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)
    vis0 = np.zeros_like(cs[0].vis)
    want = vis0.copy()
    for c, r in zip(cs, refs):
        want = want + cases.run_ref_degrid(c, r["grid"], vis0=vis0)
    objs = [cases._gpu_objs(c, model_grid=r["grid"], vis=vis0) for c, r in zip(cs, refs)]
    D.degrid(objs[0][0], [o[1] for o in objs], D.make_pol(cs[0].corr_ids, [1]), batch=D.Batch.create(dev, **batch_kw))
    got = objs[0][0].vis.cpu().numpy()
    assert cases.rel_rms(vis0 - got, vis0 - want) < TOL


@pytest.mark.parametrize("batched,stokes,tiles", [(False, (1, 2), False), (True, (1, 2), False), (True, (1,), True)])
def test_fp64_accumulated_grid(batched, stokes, tiles):
    c = cases.make_case(ncorr=4, stokes_ids=stokes, nw=3, ntimes=120, nant=16, lm=(0.004, 0.002))
    f64 = cases.run_fp64_grid(c)["grid"]
    r = cases.run_ref_grid(c)["grid"]
    kw = {"tiles": True} if tiles else None
    plain = cases.run_gpu_grid(c, batched=batched, batch_kw=kw)
    comp = cases.run_gpu_grid(c, batched=batched, fp64_acc=True, batch_kw=kw)
    e_plain, e_comp = cases.rel_rms(plain["grid"], f64), cases.rel_rms(comp["grid"], f64)
    print(f"rel RMS vs FP64: float32 sums {e_plain:.2e}, FP64 sums {e_comp:.2e}, reference {cases.rel_rms(r, f64):.2e}")
    assert cases.rel_rms(comp["grid"], r) < TOL
    np.testing.assert_array_equal(comp["grid"] != 0, r != 0)
    np.testing.assert_allclose(comp["sumwt"], plain["sumwt"], rtol=1e-12)
    assert e_comp <= e_plain * 1.01 and e_comp < 1e-6
    assert comp["acc_after"] == 0.0


def test_large_block_check_rejects_bad_lists():
    import torch

    from dataclasses import replace

    from ddfacet_b200 import _abi

    c = cases.make_case(bda_mode=1, dphi=np.sqrt(6 * 1.0), nchan=16, ntimes=60, ncorr=4)
    vs = cases._gpu_objs(c)[0].with_large_blocks(128)
    lb = vs.large_blocks
    assert lb is not None and lb.numel() >= 4
    listed = set(lb.cpu().tolist())
    small = next(b for b in range(vs.nblocks) if b not in listed)  # a block at or below the threshold
    bad = {
        "out of range": torch.cat([lb[:-1], torch.tensor([vs.nblocks], device=lb.device)]),
        "repeated": torch.cat([lb[:-1], lb[:1]]),
        "missing": lb[1:].contiguous(),
        "small": torch.cat([lb, torch.tensor([small], device=lb.device)]),
    }
    for why, lst in bad.items():
        with pytest.raises(_abi.DDFGError) as ei:
            replace(vs, large_blocks=lst.contiguous()).check_large_blocks()
        assert ei.value.code == _abi.DDFG_EMAP, why
    vs.check_large_blocks()

