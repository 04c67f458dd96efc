"""Small seeded gridding problems shared by the parity tests (CPU oracle vs GPU kernels)."""
from __future__ import annotations

import numpy as np

from ddfacet_b200 import bda, cf, synth

ARCSEC = np.pi / 180 / 3600


class Case:
    pass


def make_case(seed=1, nant=10, ntimes=30, nchan=8, ncorr=1, npix=255, cell_arcsec=3.0, nw=4, sup=7, overs=11,
              lm=(0.0, 0.0), dump_s=30.0, radius=2000.0, nsrc=5, nband=1, bda_mode=None, dphi=0.0, flag_frac=0.0,
              jones=None, corr_ids=None, stokes_ids=(1,), smear=None, weights="random", f_lo=1.30e9, f_hi=1.45e9):
    rng = np.random.default_rng(seed)
    c = Case()
    obs = synth.make_observation(seed, nant, radius, 34.0, 40.0, ntimes * dump_s / 3600.0, dump_s, nchan, f_lo, f_hi)
    c.obs = obs
    c.uvw = obs.uvw
    c.freqs = obs.freqs
    c.nrow = obs.nrow
    c.nchan = nchan
    c.ncorr = ncorr
    if corr_ids is None:
        corr_ids = {1: [1], 2: [9, 12], 4: [9, 10, 11, 12]}[ncorr]
    c.corr_ids = list(corr_ids)
    c.stokes_ids = list(stokes_ids)
    field = npix * cell_arcsec * ARCSEC / 2 * 0.6
    l, m, s = synth.point_sky(seed + 7, nsrc, field, center=lm)
    v = synth.dft_predict(obs.uvw, obs.freqs, l, m, s, ncorr=ncorr)
    if ncorr == 4:
        v[:, :, 1] = 0.1 * v[:, :, 0]
        v[:, :, 2] = -0.05j * v[:, :, 0]
    v = synth.add_noise(rng, v, 1e-3)
    c.vis = np.ascontiguousarray(v.astype(np.complex64))
    fl = np.zeros(c.vis.shape, bool)
    if flag_frac > 0:
        f1 = rng.uniform(size=(c.nrow, nchan)) < flag_frac
        fl[:] = f1[:, :, None]
    c.flags = fl
    c.weights = (rng.uniform(0.5, 1.5, (c.nrow, nchan)) if weights == "random" else np.ones((c.nrow, nchan))).astype(np.float32)
    c.npix = npix
    c.cell = cell_arcsec
    c.incr = np.array([-cell_arcsec, cell_arcsec]) * ARCSEC
    wmax = float(np.max(np.abs(obs.uvw[:, 2]))) * 1.01
    c.wt = cf.WTerms(Cell=cell_arcsec, Sup=sup, Nw=nw, wmax=wmax, Npix=npix, Freqs=obs.freqs, OverS=overs, lmShift=lm)
    c.winfos = np.array([c.wt.RefWave, c.wt.wmax, len(c.wt.Wplanes), overs], np.float64)
    c.lm = lm
    c.facet_infos = np.array([c.wt.Cu, c.wt.Cv, lm[0], lm[1], 0], np.float64)
    c.nband = nband
    c.chan_map = (np.arange(nchan) * nband // nchan).astype(np.int32)
    c.npol = len(stokes_ids)
    if bda_mode is None:
        c.bda = bda.plain_map(obs.A0, obs.A1, nchan)
    else:
        dfreq = float(obs.freqs[1] - obs.freqs[0]) if nchan > 1 else 1e6
        lrad = npix * cell_arcsec * ARCSEC * np.sqrt(2) / 2
        c.bda = bda.smear_mapping(obs.A0, obs.A1, obs.uvw, obs.freqs, dfreq, dphi, lrad, c.chan_map, mode=bda_mode)
    c.jones = jones
    c.smear = smear
    return c


def add_jones(c, nt=4, nd=3, sigma=0.1, mode=1, beam=False, kms=True, interp_mode=0, seed=5, nch=1,
              apply_amp=1, apply_phase=1, scale=0, calib_err=0.0, idir=1):
    na = c.obs.nant
    t = c.obs.times
    tmap = np.minimum(((t - t.min()) / (t.max() - t.min() + 1e-9) * nt).astype(np.int32), nt - 1)
    cmap = (np.arange(c.nchan) * nch // c.nchan).astype(np.int32)
    j = {"A0": c.obs.A0.astype(np.int32), "A1": c.obs.A1.astype(np.int32), "mode": mode,
         "interp_mode": interp_mode, "apply_amp": apply_amp, "apply_phase": apply_phase, "scale": scale,
         "calib_err": calib_err, "idir_kms": idir, "idir_beam": max(0, idir - 1)}
    if kms:
        j["kms"] = synth.random_jones(seed, nt, nd, na, nch, sigma)
        j["kms_tmap"] = tmap
        j["kms_cmap"] = cmap
    if beam:
        j["beam"] = synth.random_jones(seed + 1, nt, nd, na, nch, sigma * 0.5)
        j["beam_tmap"] = tmap
        j["beam_cmap"] = cmap
    if interp_mode == 1:
        w = np.abs(np.random.default_rng(seed + 2).standard_normal(nd)).astype(np.float32)
        w[0] = 0
        j["coefs"] = w / w.sum()
    c.jones = j
    return c


def smear_list(c, dt=30.0, dnu=None, do_t=1, do_f=1, lm=None):
    dnu = float(c.freqs[1] - c.freqs[0]) if dnu is None else dnu
    lmin = c.lm if lm is None else lm
    return [c.obs.uvw_dt.copy(), dt, dnu, do_t, do_f, lmin[0], lmin[1]]


def run_ref_grid(c, dopsf=False, sparsification=None):
    from oracle import ref

    g = np.zeros((c.nband, c.npol, c.npix, c.npix), np.complex64)
    sumwt = np.zeros((c.nband, c.npol), np.float64)
    lj = []
    if c.jones:
        c.jones["sumjones"] = np.zeros((2, c.nband), np.float64)
        c.jones["sumjones_chan"] = np.zeros((2, c.nchan), np.float64)
        lj = ref.ljones_list(c.jones, c.nrow, c.nchan, c.nband)
    ref.grid(g, c.vis, c.uvw, c.flags, c.weights, sumwt, c.wt.Wplanes, c.wt.WplanesConj, c.winfos, c.incr, c.freqs,
             c.facet_infos, c.bda, c.chan_map, c.corr_ids, c.stokes_ids, ljones=lj, lsmear=c.smear or [],
             sparsification=sparsification, dopsf=dopsf)
    out = {"grid": g, "sumwt": sumwt}
    if c.jones:
        out["sumjones"] = c.jones["sumjones"].copy()
        out["sumjones_chan"] = c.jones["sumjones_chan"].copy()
    return out


def run_ref_degrid(c, model_grid, vis0=None):
    from oracle import ref

    vis = np.zeros_like(c.vis) if vis0 is None else vis0.copy()
    lj = []
    if c.jones:
        c.jones["sumjones"] = np.zeros((2, c.nband), np.float64)
        c.jones["sumjones_chan"] = np.zeros((2, c.nchan), np.float64)
        lj = ref.ljones_list(c.jones, c.nrow, c.nchan, c.nband, gridder=False)
    ref.degrid(model_grid, vis, c.uvw, c.flags, c.wt.Wplanes, c.wt.WplanesConj, c.winfos, c.incr, c.freqs,
               c.facet_infos, c.bda, c.chan_map, c.corr_ids, c.stokes_ids, ljones=lj, lsmear=c.smear or [])
    return vis


def _gpu_objs(c, model_grid=None, vis=None):
    import torch

    from ddfacet_b200 import device as D

    dev = torch.device("cuda", 0)
    vs = D.VisData.create(c.vis if vis is None else vis, c.uvw, c.flags, c.weights, c.freqs, c.chan_map, c.bda,
                          device=dev, smear=c.smear[:5] if c.smear else None)
    tabs = D.CFTables.create(c.wt.Wplanes, c.wt.WplanesConj, c.winfos[3], c.wt.RefWave, c.wt.wmax, device=dev)
    g = (torch.zeros((c.nband, c.npol, c.npix, c.npix), dtype=torch.complex64, device=dev) if model_grid is None
         else torch.from_numpy(model_grid).to(dev))
    fg = D.FacetGrid(grid=g, cf=tabs, incr=tuple(c.incr), cu=c.wt.Cu, cv=c.wt.Cv, l0=c.lm[0], m0=c.lm[1],
                     decorr_lm=(c.smear[5], c.smear[6]) if c.smear else (0.0, 0.0),
                     sumwt=torch.zeros((c.nband, c.npol), dtype=torch.float64, device=dev),
                     sumjones=torch.zeros((2, c.nband), dtype=torch.float64, device=dev),
                     sumjones_chan=torch.zeros((2, c.nchan), dtype=torch.float64, device=dev))
    jd = None
    if c.jones:
        j = c.jones
        t = lambda a, dt=torch.int32: D.to_device(a, dt, dev)  # noqa: E731
        jd = D.JonesData(mode=j["mode"], a0=t(j["A0"]), a1=t(j["A1"]), interp_mode=j["interp_mode"],
                         apply_amp=j["apply_amp"], apply_phase=j["apply_phase"], scale_jones=j["scale"],
                         calib_error=j["calib_err"], wavelength_mean=float(np.mean(299792458.0 / c.freqs)))
        if "kms" in j:
            jd.kms = t(j["kms"], torch.complex64)
            jd.kms_tmap, jd.kms_cmap = t(j["kms_tmap"]), t(j["kms_cmap"])
        if "beam" in j:
            jd.beam = t(j["beam"], torch.complex64)
            jd.beam_tmap, jd.beam_cmap = t(j["beam_tmap"]), t(j["beam_cmap"])
        if "coefs" in j:
            jd.interp_coefs = t(j["coefs"], torch.float32)
        fg.idir_kms, fg.idir_beam = j["idir_kms"], j["idir_beam"]
    return vs, fg, jd


def run_gpu_grid(c, dopsf=False, batched=False, fp64_acc=False, batch_kw=None):
    """GPU grid of case c through ddfg_grid, or ddfg_grid_batched (``batched``, with ``batch_kw``
    for the scheduling); ``fp64_acc`` gives the facet an FP64 accumulator."""
    import torch

    from ddfacet_b200 import device as D

    vs, fg, jd = _gpu_objs(c)
    if fp64_acc:
        fg.with_fp64_accumulation()
    batch = D.Batch.create(vs.vis.device, **(batch_kw or {})) if batched else None
    D.grid(vs, [fg], D.make_pol(c.corr_ids, c.stokes_ids), jd, dopsf=dopsf, batch=batch)
    torch.cuda.synchronize()
    out = {"grid": fg.grid.cpu().numpy(), "sumwt": fg.sumwt.cpu().numpy()}
    if fp64_acc:
        out["acc_after"] = float(fg.grid_acc.abs().max().item())
    if c.jones:
        out["sumjones"] = fg.sumjones.cpu().numpy()
        out["sumjones_chan"] = fg.sumjones_chan.cpu().numpy()
    return out


def run_gpu_degrid(c, model_grid, vis0=None, batched=False, batch_kw=None):
    import torch

    from ddfacet_b200 import device as D

    vis = np.zeros_like(c.vis) if vis0 is None else vis0.copy()
    vs, fg, jd = _gpu_objs(c, model_grid=model_grid, vis=vis)
    batch = D.Batch.create(vs.vis.device, **(batch_kw or {})) if batched else None
    D.degrid(vs, [fg], D.make_pol(c.corr_ids, c.stokes_ids), jd, batch=batch)
    torch.cuda.synchronize()
    return vs.vis.cpu().numpy()


def rel_rms(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    den = np.sqrt(np.mean(np.abs(b) ** 2))
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2)) / (den if den > 0 else 1.0))


def run_fp64_grid(c, dopsf=False, sparsification=None):
    from oracle import fp64

    g, sw, sj, sjc = fp64.grid(c.vis, c.uvw, c.flags, c.weights, c.freqs, c.chan_map, c.bda, c.wt.Wplanes,
                               c.wt.WplanesConj, c.winfos[3], c.wt.RefWave, c.wt.wmax, c.incr, c.wt.Cu, c.wt.Cv, c.lm,
                               c.corr_ids, c.stokes_ids, c.nband, c.npix, jones=c.jones, smear=c.smear, dopsf=dopsf,
                               sparsification=sparsification)
    return {"grid": g, "sumwt": sw, "sumjones": sj, "sumjones_chan": sjc}


def run_fp64_degrid(c, model_grid, vis0=None):
    from oracle import fp64

    v0 = np.zeros_like(c.vis) if vis0 is None else vis0
    return fp64.degrid(model_grid, v0, c.uvw, c.freqs, c.chan_map, c.bda, c.wt.Wplanes, c.wt.WplanesConj, c.winfos[3],
                       c.wt.RefWave, c.wt.wmax, c.incr, c.wt.Cu, c.wt.Cv, c.lm, c.corr_ids, c.stokes_ids,
                       jones=c.jones, smear=c.smear)
