"""Parity on the benchmark's own workload geometry (ddfacet_b200.configs.multifacet_dde: 81 regular
facets of 735^2, 32 w-planes, oversampling 11, four linear correlations gridded to Stokes I,
per-facet per-antenna Jones in 5-minute slots), at a reduced number of dumps, through the batched
calls the benchmark makes.

* grids of corner, edge and centre facets against the reference's own gridder on those facets
  (<= 1e-4 relative RMS, identical touched cells, weight sums to 1e-9) and against the FP64
  restatement (FP64-accumulated gridding: <= 1e-5 relative RMS);
* the summed prediction of the same facets (one batched degrid call into zeros) against the sum of
  the reference's per-facet predictions (<= 1e-4);
* every block's integer footprint -- w-plane, CF table (conjugate or not), centre cell,
  oversampling offsets, sub-kernel -- word for word against the FP64 restatement of
  gridder.h:321-351 / degridder.h:168-200, for the gridder's and the degridder's block means;
* at a quarter of the track (58 M visibilities, ~2e4 grid additions per cell on average) the
  FP64-accumulated grid of two facets against the FP64 restatement over all rows, beside float32
  accumulation.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

PICK = [0, 4, 8, 40, 72, 80]  # corners, an edge and the centre of the 9 x 9 tessellation


def _case(w, fi, vis, host):
    """A tests.cases.Case for facet fi of workload w (host arrays shared between facets)."""
    obs = w.host["obs"]
    f = w.host["tess"].facets[fi]
    wt = w.host["wterms"][fi]
    c = cases.Case()
    c.obs = obs
    c.uvw, c.freqs, c.nrow, c.nchan, c.ncorr = obs.uvw, obs.freqs, obs.nrow, w.nchan, w.ncorr
    c.corr_ids, c.stokes_ids = [9, 10, 11, 12], [1]
    c.vis = vis
    c.flags = host["flags"]
    c.weights = host["weights"]
    c.npix = w.info["npix_padded"]
    c.incr = np.array(w.facets_grid[fi].incr)
    c.wt = wt
    c.winfos = np.array([wt.RefWave, wt.wmax, len(wt.Wplanes), 11], np.float64)
    c.lm = (f.l0, f.m0)
    c.facet_infos = np.array([wt.Cu, wt.Cv, f.l0, f.m0, fi], np.float64)
    c.nband, c.npol = 1, 1
    c.chan_map = w.host["chan_map"]
    c.bda = host["bda"]
    c.smear = None
    c.jones = {"A0": obs.A0.astype(np.int32), "A1": obs.A1.astype(np.int32), "mode": 1, "interp_mode": 0,
               "apply_amp": 1, "apply_phase": 1, "scale": 0, "calib_err": 0.0, "idir_kms": w.facets_grid[fi].idir_kms,
               "idir_beam": 0, "kms": host["J"], "kms_tmap": host["tmap"],
               "kms_cmap": np.zeros(w.nchan, np.int32)}
    return c


def _host(w):
    from ddfacet_b200 import bda

    obs = w.host["obs"]
    return {"vis": w.host["vis"].numpy().copy(), "flags": np.zeros((obs.nrow, w.nchan, w.ncorr), bool),
            "weights": np.ones((obs.nrow, w.nchan), np.float32), "bda": bda.plain_map(obs.A0, obs.A1, w.nchan),
            "J": w.jones.kms.cpu().numpy(), "tmap": w.jones.kms_tmap.cpu().numpy()}


@pytest.fixture(scope="module")
def small():
    import torch

    from ddfacet_b200 import configs

    w = configs.multifacet_dde(device=torch.device("cuda", 0), scale=0.01, nsrc=40)
    return w, _host(w)


def test_workload_grid_against_reference_and_fp64(small):
    import torch

    from ddfacet_b200 import device as D

    w, host = small
    for f in w.facets_grid:
        f.grid.zero_()
        f.sumwt.zero_()
        f.with_fp64_accumulation()
    D.grid(w.vs, w.facets_grid, w.pol, w.jones, batch=D.Batch.create(w.vs.vis.device, tiles=True))
    torch.cuda.synchronize()
    for fi in PICK:
        c = _case(w, fi, host["vis"], host)
        g = w.facets_grid[fi].grid.cpu().numpy()
        r = cases.run_ref_grid(c)
        f64 = cases.run_fp64_grid(c)
        e_ref, e64, e_ref64 = (cases.rel_rms(g, r["grid"]), cases.rel_rms(g, f64["grid"]),
                               cases.rel_rms(r["grid"], f64["grid"]))
        print(f"facet {fi}: gpu vs reference {e_ref:.2e}; vs FP64: gpu (FP64 sums) {e64:.2e}, "
              f"reference {e_ref64:.2e}")
        assert e_ref < 1e-4
        assert e64 < 1e-5
        np.testing.assert_array_equal(g != 0, r["grid"] != 0)
        np.testing.assert_allclose(w.facets_grid[fi].sumwt.cpu().numpy(), r["sumwt"], rtol=1e-9)
        assert float(w.facets_grid[fi].grid_acc.abs().max()) == 0.0
    for f in w.facets_grid:
        f.grid_acc = None


def test_workload_degrid_against_reference(small):
    import torch

    from ddfacet_b200 import device as D

    w, host = small
    obs = w.host["obs"]
    zeros = torch.zeros_like(w.vs.vis)
    vs0 = D.VisData.create(zeros, w.vs.uvw, w.vs.flags, w.vs.weights, obs.freqs, w.host["chan_map"], w.vs.bda_map,
                           device=zeros.device, block_start=w.vs.block_start)
    vs0.single_vis_blocks = w.vs.single_vis_blocks
    D.degrid(vs0, [w.facets_model[fi] for fi in PICK], w.pol, w.jones, batch=D.Batch.create(zeros.device))
    torch.cuda.synchronize()
    got = -vs0.vis.cpu().numpy()
    want = np.zeros_like(got)
    z = np.zeros_like(host["vis"])
    for fi in PICK:
        c = _case(w, fi, z, host)
        want -= cases.run_ref_degrid(c, w.facets_model[fi].grid.cpu().numpy(), vis0=z)
    e = cases.rel_rms(got, want)
    print(f"summed prediction of {len(PICK)} facets vs reference: {e:.2e}")
    assert e < 1e-4


@pytest.mark.parametrize("degrid", [False, True])
def test_workload_integer_indices(small, degrid):
    from ddfacet_b200 import device as D
    from oracle import fp64

    w, host = small
    obs = w.host["obs"]
    for fi in (0, 40, 80):
        fg = w.facets_model[fi] if degrid else w.facets_grid[fi]
        got = D.block_geometry(w.vs, fg, degrid=degrid).cpu().numpy()
        # the kernels read blocks through the plan's order, which for this map is the map order
        wt = w.host["wterms"][fi]
        want = fp64.block_indices(obs.uvw, host["flags"], obs.freqs, w.host["chan_map"], host["bda"], wt.Wplanes,
                                  wt.WplanesConj, 11, wt.RefWave, wt.wmax, fg.incr, wt.Cu, wt.Cv, 1,
                                  w.info["npix_padded"], degrid=degrid)
        assert got.shape == want.shape
        bad = np.flatnonzero(np.any(got != want, axis=1))
        assert bad.size == 0, f"facet {fi}: {bad.size} blocks differ, first {bad[:5]}: {got[bad[:3]]} vs {want[bad[:3]]}"
        ok = got[:, 0] == 1
        assert ok.mean() > 0.9
        # both CF tables (w > 0 and w <= 0) and many oversampling phases are exercised
        assert (got[ok, 2] < 32).any() and (got[ok, 2] >= 32).any()
        assert np.unique(got[ok, 7]).size > 100


def test_full_depth_fp64_accumulation_vs_fp64():
    """A quarter of the 4-hour track (58 M visibilities x 4 correlations) gridded onto a corner and
    the centre facet: float32 and FP64 accumulation against the FP64 restatement."""
    import torch

    from ddfacet_b200 import configs, device as D

    w = configs.multifacet_dde(device=torch.device("cuda", 0), scale=0.25, nsrc=200)
    host = _host(w)
    pick = [0, 40]
    errs = {}
    for comp in (False, True):
        fs = [w.facets_grid[fi] for fi in pick]
        for f in fs:
            f.grid.zero_()
            f.grid_acc = None
            if comp:
                f.with_fp64_accumulation()
        D.grid(w.vs, fs, w.pol, w.jones, batch=D.Batch.create(w.vs.vis.device, tiles=comp))
        torch.cuda.synchronize()
        errs[comp] = [fs[i].grid.cpu().numpy() for i in range(len(pick))]
    for i, fi in enumerate(pick):
        c = _case(w, fi, host["vis"], host)
        f64 = cases.run_fp64_grid(c)["grid"]
        e_plain, e_comp = cases.rel_rms(errs[False][i], f64), cases.rel_rms(errs[True][i], f64)
        print(f"facet {fi}, {w.nvis/1e6:.0f} Mvis: rel RMS vs FP64: float32 sums {e_plain:.2e}, FP64 sums {e_comp:.2e}")
        assert e_comp < 1e-5
        assert e_comp <= e_plain * 1.01
