"""The facet-sharded residual step (ddfacet_b200.parallel.sharded_residual_step) with the library's
own batched kernels on one GPU: with one rank it must equal a plain degrid-then-grid step over
every facet (the same kernels in the same order, and vis + (0 - P) == vis - P exactly), and two
emulated ranks whose degridded predictions are summed by hand must give the same residuals and
grids (every facet gridded once).  The multi-rank exchange itself is tested on CPU ranks
(tests/test_parallel_cpu.py)."""
import dataclasses

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _problem():
    from ddfacet_b200 import device as D

    sizes = [255, 201, 149, 311, 201]
    lms = [(0.004 * i - 0.008, 0.003 * (i % 2) - 0.002) for i in range(len(sizes))]
    cs = [cases.make_case(npix=n, lm=lm, nw=2, ncorr=4, stokes_ids=(1,), ntimes=10) for n, lm in zip(sizes, lms)]
    for c in cs[1:]:
        c.vis = cs[0].vis
    rng = np.random.default_rng(3)
    models = [(rng.standard_normal((1, 1, n, n)) + 1j * rng.standard_normal((1, 1, n, n))).astype(np.complex64) * 1e-2
              for n in sizes]
    vis = cs[0].vis.copy()
    objs_m = [cases._gpu_objs(c, model_grid=m, vis=vis) for c, m in zip(cs, models)]
    objs_g = [cases._gpu_objs(c) for c in cs]
    vs = objs_m[0][0]
    return vs, [o[1] for o in objs_m], [o[1] for o in objs_g], D.make_pol(cs[0].corr_ids, [1])


def test_one_rank_equals_plain_step():
    import torch

    from ddfacet_b200 import device as D, parallel

    vs, models, grids, pol = _problem()
    dev = vs.vis.device
    bd, bg = D.Batch.create(dev), D.Batch.create(dev)
    vis_in = vs.vis.clone()
    mine = parallel.sharded_residual_step(vs, models, grids, pol, None, 0, 1, batch_degrid=bd, batch_grid=bg)
    torch.cuda.synchronize()
    assert mine == list(range(len(models)))
    res_sharded = vs.vis.cpu().numpy()
    g_sharded = [g.grid.cpu().numpy() for g in grids]
    vs2, models2, grids2, _ = _problem()
    vs2.vis.copy_(vis_in)
    D.degrid(vs2, models2, pol, None, batch=bd)
    D.grid(vs2, grids2, pol, None, batch=bg)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(res_sharded, vs2.vis.cpu().numpy())
    for a, g in zip(g_sharded, grids2):
        assert cases.rel_rms(a, g.grid.cpu().numpy()) < 1e-6  # grid additions commute up to rounding


def test_two_emulated_ranks():
    """Two ranks on one GPU, run one after the other, with the all-reduce done by hand between the
    degrid and grid halves (the library calls sharded_residual_step makes, in its order)."""
    import torch

    from ddfacet_b200 import device as D, parallel

    vs, models, grids, pol = _problem()
    dev = vs.vis.device
    vis_in = vs.vis.clone()
    preds, shards = [], []
    for rank in range(2):
        mine = parallel.shard_facets(len(models), rank, 2)
        pred = torch.zeros_like(vis_in)
        D.degrid(dataclasses.replace(vs, vis=pred), [models[i] for i in mine], pol, None, batch=D.Batch.create(dev))
        preds.append(pred)
        shards.append(mine)
    total = preds[0] + preds[1]
    vs.vis.copy_(vis_in + total)
    for mine in shards:
        D.grid(vs, [grids[i] for i in mine], pol, None, batch=D.Batch.create(dev))
    torch.cuda.synchronize()
    assert sorted(shards[0] + shards[1]) == list(range(len(models)))
    vs1, models1, grids1, _ = _problem()
    vs1.vis.copy_(vis_in)
    parallel.sharded_residual_step(vs1, models1, grids1, pol, None, 0, 1)
    torch.cuda.synchronize()
    assert cases.rel_rms(vs.vis.cpu().numpy(), vs1.vis.cpu().numpy()) < 1e-6
    for a, b in zip(grids, grids1):
        assert cases.rel_rms(a.grid.cpu().numpy(), b.grid.cpu().numpy()) < 1e-6
