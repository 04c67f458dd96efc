"""The benchmark workloads, built from seeded synthetic data directly in device memory.

``multifacet_dde`` is the multi-facet direction-dependent imaging workload: a 4096^2 image at
1.5 arcsec in 9 x 9 regular facets (padding 1.7, 735^2 padded grids), 64 antennas uniform in a
disk of 4 km radius (8 km across) at latitude +34 deg observing dec +40 deg for 4 h at 8 s
(1800 dumps, 2016 baselines, 3.63 M rows), 64 channels over 0.90-1.67 GHz, 4 linear
correlations gridded to Stokes I, 200 power-law point sources plus 1 mJy noise, per-facet
per-antenna 2x2 Jones in 5-min slots (identity + 0.1 complex Gaussian), W-projection with
32 planes, supports from 7, oversampling 11.  Every (row, channel) is its own block (no BDA).

``combined_at_scale`` is one 1-hour chunk of the 8-hour, 121-facet, 256-channel workload (1485^2
padded grids, 64 w-planes, 1000 point sources and 20 Gaussians, per-facet Jones): 232.2 M
visibilities x 4 correlations per chunk, the full track being eight such chunks.

``plain_small`` is the single-facet, Stokes-I, 1024^2 image case (27 antennas in a 20 km
radius, 2 h at 10 s, 16 channels over 1.30-1.45 GHz, 8 w-planes, support 7).

``scale`` shrinks the number of dumps (and so rows) for quick runs; 1.0 is the full size.
"""
from __future__ import annotations

import concurrent.futures as cfut
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import bda, cf, device as D, geometry, pipeline, synth

C_LIGHT = 299792458.0


@dataclass
class Workload:
    name: str
    vs: D.VisData
    facets_grid: List[D.FacetGrid]      # residual grids (gridding target)
    facets_model: List[D.FacetGrid]     # model grids (degridding source), same CF tables
    jones: Optional[D.JonesData]
    pol: object
    nvis: int
    nrow: int
    nchan: int
    ncorr: int
    nfacets: int
    host: dict = field(default_factory=dict)   # host copies for the end-to-end path
    info: dict = field(default_factory=dict)


def _gen_vis_gpu(uvw_d, freqs_d, l, m, s, ncorr, noise_sigma, seed, dev, row_chunk=1 << 14):
    """Point-source visibilities + complex noise on the GPU (FP64 phase, complex64 result).
    All sources of a row chunk in one pass, so generation takes a few thousand launches."""
    nrow = uvw_d.shape[0]
    nchan = freqs_d.numel()
    out = torch.empty((nrow, nchan, ncorr), dtype=torch.complex64, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    lt = torch.tensor(l, dtype=torch.float64, device=dev)
    mt = torch.tensor(m, dtype=torch.float64, device=dev)
    nt = torch.sqrt(1 - lt ** 2 - mt ** 2) - 1
    lmn = torch.stack([lt, mt, nt])                                             # [3][nsrc]
    st = torch.tensor(s, dtype=torch.float32, device=dev)
    fr = (freqs_d / C_LIGHT).to(torch.float64)
    for r0 in range(0, nrow, row_chunk):
        uu = uvw_d[r0:r0 + row_chunk]
        turns = (uu @ lmn)[:, :, None] * fr[None, None, :]                        # [rows][nsrc][nchan]
        frac = (turns - torch.round(turns)).to(torch.float32)
        del turns
        acc = (torch.polar(st[None, :, None].expand_as(frac), 2 * np.pi * frac)).sum(dim=1)
        del frac
        noise = torch.randn((uu.shape[0], nchan, ncorr, 2), generator=g, device=dev) * noise_sigma
        blk = torch.view_as_complex(noise.contiguous())
        blk[:, :, 0] += acc
        if ncorr > 1:
            blk[:, :, ncorr - 1] += acc
        out[r0:r0 + row_chunk] = blk
    return out


def _plain_map_gpu(A0, A1, nchan, dev):
    """bda.plain_map built with device tensors (same words)."""
    groups = bda._baseline_rows(A0, A1)
    keys = sorted(groups.keys(), key=lambda k: "%d:%d" % k)
    rows = np.concatenate([groups[k] for k in keys]).astype(np.int32)
    nb = rows.size * nchan
    rows_d = torch.from_numpy(rows).to(dev)
    m = torch.empty(2 + nb + 3 * nb, dtype=torch.int32, device=dev)
    m[0:2] = torch.from_numpy(bda._header(nb)).to(dev)
    m[2:2 + nb] = 3
    body = m[2 + nb:].view(nb, 3)
    ch = torch.arange(nchan, dtype=torch.int32, device=dev).repeat(rows.size)
    body[:, 0] = ch
    body[:, 1] = ch + 1
    body[:, 2] = rows_d.repeat_interleave(nchan)
    return m


def _wterms(args):
    (cell, sup, nw, wmax, npix, freqs, overs, lm, i) = args
    return cf.WTerms(Cell=cell, Sup=sup, Nw=nw, wmax=wmax, Npix=npix, Freqs=freqs, OverS=overs, lmShift=lm,
                     IDFacet=i)


def build_wterms(tess_facets, cell, sup, nw, wmax, npix, freqs, overs, threads=8):
    """W-term tables of every facet; npix is one padded grid side for all or one per facet."""
    sides = list(npix) if np.ndim(npix) else [npix] * len(tess_facets)
    args = [(cell, sup, nw, wmax, n, freqs, overs, (f.l0, f.m0), f.index) for f, n in zip(tess_facets, sides)]
    with cfut.ThreadPoolExecutor(threads) as ex:
        return list(ex.map(_wterms, args))


def multifacet_dde(device=None, scale=1.0, seed=1002, nfacets_side=9, nchan=64, nw=32, with_jones=True,
                   keep_host=True, nsrc=200, jones_sigma=0.1):
    dev = D._dev(device)
    hours = 4.0 * scale
    obs = synth.make_observation(seed, 64, 4000.0, 34.0, 40.0, hours, 8.0, nchan, 0.90e9, 1.67e9)
    tess = geometry.regular_facets(4096, nfacets_side, 1.5, 1.7)
    npix_pad = tess.npix_padded
    cell = 1.5
    wmax = float(np.max(np.abs(obs.uvw[:, 2]))) * 1.001
    wts = build_wterms(tess.facets, cell, 7, nw, wmax, tess.npix_facet * 0 + npix_pad, obs.freqs, 11)
    field_rad = tess.npix * tess.cell_rad / 2
    l, m, s = synth.point_sky(seed + 1, nsrc, field_rad * 0.95, flux=("powerlaw", 1e-4, 1.0))
    uvw_d = torch.from_numpy(obs.uvw).to(dev)
    freqs_d = torch.from_numpy(obs.freqs).to(dev)
    ncorr = 4
    vis = _gen_vis_gpu(uvw_d, freqs_d, l, m, s, ncorr, 1e-3, seed + 2, dev)
    nrow = obs.nrow
    flags = torch.zeros((nrow, nchan, ncorr), dtype=torch.uint8, device=dev)
    weights = torch.ones((nrow, nchan), dtype=torch.float32, device=dev)
    chan_map = np.zeros(nchan, np.int32)
    bmap = _plain_map_gpu(obs.A0, obs.A1, nchan, dev)
    vs = D.VisData.create(vis, uvw_d, flags, weights, obs.freqs, chan_map, bmap, device=dev)
    jd = None
    if with_jones:
        nt = int(np.ceil(hours * 3600 / 300.0))
        J = synth.random_jones(seed + 3, nt, len(tess.facets), 64, 1, jones_sigma)
        tmap = np.minimum(((obs.times - obs.times.min()) // 300.0).astype(np.int32), nt - 1)
        jd = D.JonesData(mode=1, kms=torch.from_numpy(J).to(dev), kms_tmap=torch.from_numpy(tmap).to(dev),
                         kms_cmap=torch.zeros(nchan, dtype=torch.int32, device=dev),
                         a0=torch.from_numpy(obs.A0).to(dev), a1=torch.from_numpy(obs.A1).to(dev),
                         wavelength_mean=float(np.mean(C_LIGHT / obs.freqs)))
    fg, fm = [], []
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 4)
    for f, wt in zip(tess.facets, wts):
        tabs = D.CFTables.create(wt.Wplanes, wt.WplanesConj, 11, wt.RefWave, wt.wmax, device=dev)
        incr = (-cell / 3600 * np.pi / 180, cell / 3600 * np.pi / 180)
        g = torch.zeros((1, 1, npix_pad, npix_pad), dtype=torch.complex64, device=dev)
        mg = torch.randn((1, 1, npix_pad, npix_pad, 2), generator=gen, device=dev)
        mg = torch.view_as_complex(mg.contiguous()) * 1e-3
        common = dict(cf=tabs, incr=incr, cu=wt.Cu, cv=wt.Cv, l0=f.l0, m0=f.m0, idir_kms=f.index, idir_beam=0)
        fg.append(D.FacetGrid(grid=g, sumwt=torch.zeros((1, 1), dtype=torch.float64, device=dev),
                              sumjones=torch.zeros((2, 1), dtype=torch.float64, device=dev),
                              sumjones_chan=torch.zeros((2, nchan), dtype=torch.float64, device=dev), **common))
        fm.append(D.FacetGrid(grid=mg, **common))
    pol = D.make_pol([9, 10, 11, 12], [1])
    w = Workload("multifacet_dde", vs, fg, fm, jd, pol, nvis=nrow * nchan, nrow=nrow, nchan=nchan, ncorr=ncorr,
                 nfacets=len(fg))
    w.info = dict(npix=tess.npix, npix_facet=tess.npix_facet, npix_padded=npix_pad, nw=nw,
                  supports=sorted(set(int(x) for x in wts[0].Sups)), wmax=wmax, nant=64, ntimes=obs.ntimes,
                  nbl=obs.nbl, cell_arcsec=cell)
    w.host = {"obs": obs, "wterms": wts, "tess": tess, "chan_map": chan_map}
    if keep_host:
        w.host["vis"] = vis.cpu().pin_memory()
    return w


def _gen_sky_vis_gpu(uvw_d, freqs, l, m, s, fwhm_rad, ncorr, noise_sigma, seed, dev, rows=2048, chans=32):
    """Visibilities of point and circular Gaussian sources plus complex noise on the GPU:
    V = sum_k S_k g_k exp(+2 pi i (u l + v m + w (n - 1)) nu / c) with g_k = exp(-2 pi^2 sigma_k^2
    (u^2 + v^2) (nu / c)^2) (sigma = FWHM / sqrt(8 ln 2); points have FWHM 0).  The phase in turns is
    formed in FP64 and reduced before the FP32 cos/sin; rows and channels go in blocks so the
    [rows][sources][channels] intermediates stay near 1 GB."""
    nrow = uvw_d.shape[0]
    nchan = len(freqs)
    out = torch.empty((nrow, nchan, ncorr), dtype=torch.complex64, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    lt = torch.tensor(l, dtype=torch.float64, device=dev)
    mt = torch.tensor(m, dtype=torch.float64, device=dev)
    lmn = torch.stack([lt, mt, torch.sqrt(1 - lt ** 2 - mt ** 2) - 1])          # [3][nsrc]
    st = torch.tensor(s, dtype=torch.float32, device=dev)
    sig2 = torch.tensor((np.asarray(fwhm_rad) / np.sqrt(8 * np.log(2))) ** 2, dtype=torch.float32, device=dev)
    gauss = bool(np.any(np.asarray(fwhm_rad) > 0))
    fr = torch.tensor(np.asarray(freqs) / C_LIGHT, dtype=torch.float64, device=dev)
    for r0 in range(0, nrow, rows):
        uu = uvw_d[r0:r0 + rows]
        turns_rs = uu @ lmn                                                      # [r][s] (metres)
        uv2 = (uu[:, 0] ** 2 + uu[:, 1] ** 2).to(torch.float32)                   # [r]
        blk = torch.empty((uu.shape[0], nchan), dtype=torch.complex64, device=dev)
        for c0 in range(0, nchan, chans):
            f = fr[c0:c0 + chans]
            t = turns_rs[:, :, None] * f[None, None, :]                             # [r][s][c]
            frac = (t - torch.round(t)).to(torch.float32)
            del t
            amp = st[None, :, None].expand_as(frac)
            if gauss:
                amp = amp * torch.exp(-2 * np.pi ** 2 * sig2[None, :, None] * uv2[:, None, None] *
                                      (f.to(torch.float32) ** 2)[None, None, :])
            blk[:, c0:c0 + chans] = torch.polar(amp, 2 * np.pi * frac).sum(dim=1)
            del frac, amp
        noise = torch.randn((uu.shape[0], nchan, ncorr, 2), generator=g, device=dev) * noise_sigma
        v = torch.view_as_complex(noise.contiguous())
        v[:, :, 0] += blk
        if ncorr > 1:
            v[:, :, ncorr - 1] += blk
        out[r0:r0 + rows] = v
    return out


def combined_at_scale(device=None, scale=1.0, seed=1005, hour=0, nfacets_side=11, nchan=256, nw=64, nsrc=1000,
                      ngauss=20, keep_host=True):
    """The combined at-scale workload, one 1-hour chunk of it: a 10000^2 image at 1 arcsec in 11 x 11
    regular facets (padding 1.7: 891-pixel facets, 1485^2 padded grids, 9801^2 image), 64 antennas
    uniform in a disk of 4 km radius (8 km across) at latitude +34 deg observing dec +40 deg for 8 h
    at 8 s (3600 dumps, 2016 baselines), 256 channels over 0.90-1.67 GHz, 4 linear correlations
    gridded to Stokes I, 1000 power-law point sources (0.1 mJy - 1 Jy) plus 20 circular Gaussians
    (FWHM 5-60 arcsec) plus 1 mJy noise, per-facet per-antenna 2x2 Jones in 5-minute slots
    (identity + 0.1 complex Gaussian, 96 slots), W-projection with 64 planes (wmax of the whole
    8-hour track; ClassWTermModified's support rule gives support 7 at this facet size), oversampling
    11, every (row, channel) its own block.  The chunk is hour ``hour`` (450 dumps, 907,200 rows,
    232.2 M visibilities, 7.4 GB of visibilities); ``scale`` keeps that fraction of its dumps."""
    dev = D._dev(device)
    full = synth.make_observation(seed, 64, 4000.0, 34.0, 40.0, 8.0, 8.0, nchan, 0.90e9, 1.67e9)
    wmax = float(np.max(np.abs(full.uvw[:, 2]))) * 1.001
    nbl = full.nbl
    d0 = hour * 450
    d1 = d0 + max(1, int(round(450 * scale)))
    rows = slice(d0 * nbl, d1 * nbl)
    obs = synth.Observation(uvw=np.ascontiguousarray(full.uvw[rows]), uvw_dt=np.ascontiguousarray(full.uvw_dt[rows]),
                            A0=full.A0[rows], A1=full.A1[rows], times=full.times[rows], freqs=full.freqs,
                            nant=full.nant, ntimes=d1 - d0, dump_s=full.dump_s)
    tess = geometry.regular_facets(10000, nfacets_side, 1.0, 1.7)
    npix_pad = tess.npix_padded
    cell = 1.0
    wts = build_wterms(tess.facets, cell, 7, nw, wmax, npix_pad, obs.freqs, 11)
    field_rad = tess.npix * tess.cell_rad / 2
    l, m, s = synth.point_sky(seed + 1, nsrc, field_rad * 0.95, flux=("powerlaw", 1e-4, 1.0))
    lg, mg, sg = synth.point_sky(seed + 6, ngauss, field_rad * 0.9, flux=("powerlaw", 1e-3, 1.0))
    fw = np.random.default_rng(seed + 7).uniform(5.0, 60.0, ngauss) / 3600 * np.pi / 180
    uvw_d = torch.from_numpy(obs.uvw).to(dev)
    ncorr = 4
    vis = _gen_sky_vis_gpu(uvw_d, obs.freqs, np.concatenate([l, lg]), np.concatenate([m, mg]),
                           np.concatenate([s, sg]), np.concatenate([np.zeros(nsrc), fw]), ncorr, 1e-3, seed + 2, dev)
    nrow = obs.nrow
    flags = torch.zeros((nrow, nchan, ncorr), dtype=torch.uint8, device=dev)
    weights = torch.ones((nrow, nchan), dtype=torch.float32, device=dev)
    chan_map = np.zeros(nchan, np.int32)
    bmap = _plain_map_gpu(obs.A0, obs.A1, nchan, dev)
    vs = D.VisData.create(vis, uvw_d, flags, weights, obs.freqs, chan_map, bmap, device=dev)
    nt = 96
    J = synth.random_jones(seed + 3, nt, len(tess.facets), 64, 1, 0.1)
    tmap = np.minimum(((obs.times - full.times.min()) // 300.0).astype(np.int32), nt - 1)
    jd = D.JonesData(mode=1, kms=torch.from_numpy(J).to(dev), kms_tmap=torch.from_numpy(tmap).to(dev),
                     kms_cmap=torch.zeros(nchan, dtype=torch.int32, device=dev),
                     a0=torch.from_numpy(obs.A0).to(dev), a1=torch.from_numpy(obs.A1).to(dev),
                     wavelength_mean=float(np.mean(C_LIGHT / obs.freqs)))
    fg, fm = [], []
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 4)
    incr = (-cell / 3600 * np.pi / 180, cell / 3600 * np.pi / 180)
    for f, wt in zip(tess.facets, wts):
        tabs = D.CFTables.create(wt.Wplanes, wt.WplanesConj, 11, wt.RefWave, wt.wmax, device=dev)
        g = torch.zeros((1, 1, npix_pad, npix_pad), dtype=torch.complex64, device=dev)
        mg = torch.view_as_complex(torch.randn((1, 1, npix_pad, npix_pad, 2), generator=gen, device=dev)) * 1e-3
        common = dict(cf=tabs, incr=incr, cu=wt.Cu, cv=wt.Cv, l0=f.l0, m0=f.m0, idir_kms=f.index, idir_beam=0)
        fg.append(D.FacetGrid(grid=g, sumwt=torch.zeros((1, 1), dtype=torch.float64, device=dev),
                              sumjones=torch.zeros((2, 1), dtype=torch.float64, device=dev),
                              sumjones_chan=torch.zeros((2, nchan), dtype=torch.float64, device=dev), **common))
        fm.append(D.FacetGrid(grid=mg, **common))
    pol = D.make_pol([9, 10, 11, 12], [1])
    w = Workload("combined_at_scale", vs, fg, fm, jd, pol, nvis=nrow * nchan, nrow=nrow, nchan=nchan, ncorr=ncorr,
                 nfacets=len(fg))
    w.info = dict(npix=tess.npix, npix_facet=tess.npix_facet, npix_padded=npix_pad, nw=nw,
                  supports=sorted(set(int(x) for x in wts[0].Sups)), wmax=wmax, nant=64, ntimes=obs.ntimes,
                  nbl=nbl, chunk=f"hour {hour} of 8: dumps {d0}-{d1 - 1} of 3600", nsrc=nsrc, ngauss=ngauss,
                  full_track_nvis=full.nrow * nchan, cell_arcsec=cell)
    w.host = {"obs": obs, "wterms": wts, "tess": tess, "chan_map": chan_map, "J": J, "tmap": tmap}
    if keep_host:
        w.host["vis"] = vis.cpu().pin_memory()
    return w


def row_chunks(w: Workload, nchunks: int) -> List[pipeline.Chunk]:
    """The workload's rows in nchunks time ranges (whole dumps), each with its own block map
    (chunk-relative rows) and Jones row maps, as views of the device buffers."""
    obs = w.host["obs"]
    nbl = obs.nrow // obs.ntimes
    dev = w.vs.vis.device
    edges = np.round(np.linspace(0, obs.ntimes, nchunks + 1)).astype(np.int64) * nbl
    out = []
    for r0, r1 in zip(edges[:-1], edges[1:]):
        r0, r1 = int(r0), int(r1)
        if r1 <= r0:
            continue
        bmap = _plain_map_gpu(obs.A0[r0:r1], obs.A1[r0:r1], w.nchan, dev)
        vs = D.VisData.create(w.vs.vis[r0:r1], w.vs.uvw[r0:r1], w.vs.flags[r0:r1], w.vs.weights[r0:r1], obs.freqs,
                              w.host["chan_map"], bmap, device=dev)
        out.append(pipeline.Chunk((r0, r1), vs, pipeline.jones_rows(w.jones, r0, r1)))
    return out


def uneven_bda(device=None, scale=1.0, seed=1003, nfacets=25, npix_image=6000, cell=1.0, nchan=128, nw=32,
               grid_decorr=0.02, nsrc=200, block_order_tile=64, large_min_vis=2048):
    """Uneven facets with baseline-dependent averaging: a 6000^2 image at 1"/pixel in a Voronoi
    tessellation around 25 directions, 48 antennas in a 12 km log-radial layout, 6 h at 4 s,
    128 channels 0.9-1.7 GHz, 4 correlations, per-facet per-antenna 5-min Jones; block map of
    DDFacet's default mode 1 with GridDecorr 0.02 over the largest facet's field, built on the
    GPU (every block averages a few rows and channels, more on short baselines), its blocks
    visited in uv Z order (``block_order_tile`` cells per tile; 0 keeps the map order) and blocks of
    more than ``large_min_vis`` visibilities walked by a whole warp each (0: none)."""
    dev = D._dev(device)
    hours = 6.0 * scale
    obs = synth.make_observation(seed, 48, 12000.0, 34.0, 40.0, hours, 4.0, nchan, 0.90e9, 1.70e9, layout="lograd")
    rng = np.random.default_rng(seed + 5)
    r = npix_image * cell / 3600 * np.pi / 180 / 2
    tess = geometry.voronoi_facets(npix_image, cell, rng.uniform(-r, r, nfacets), rng.uniform(-r, r, nfacets), 1.7)
    wmax = float(np.max(np.abs(obs.uvw[:, 2]))) * 1.001
    wts = build_wterms(tess.facets, cell, 7, nw, wmax, [f.npix_padded for f in tess.facets], obs.freqs, 11)
    l, m, s = synth.point_sky(seed + 1, nsrc, r * 0.95, flux=("powerlaw", 1e-4, 1.0))
    uvw_d = torch.from_numpy(obs.uvw).to(dev)
    freqs_d = torch.from_numpy(obs.freqs).to(dev)
    ncorr = 4
    vis = _gen_vis_gpu(uvw_d, freqs_d, l, m, s, ncorr, 1e-3, seed + 2, dev)
    nrow = obs.nrow
    flags = torch.zeros((nrow, nchan, ncorr), dtype=torch.uint8, device=dev)
    weights = torch.ones((nrow, nchan), dtype=torch.float32, device=dev)
    chan_map = np.zeros(nchan, np.int32)
    lmax = max(f.npix_facet for f in tess.facets) * tess.cell_rad * np.sqrt(2) / 2
    dfreq = float(obs.freqs[1] - obs.freqs[0])
    bmap = bda.smear_mapping_gpu(obs.A0, obs.A1, uvw_d, obs.freqs, dfreq, np.sqrt(6 * grid_decorr), lmax, chan_map,
                                 device=dev)
    vs = D.VisData.create(vis, uvw_d, flags, weights, obs.freqs, chan_map, bmap, device=dev)
    if block_order_tile:
        # blocks in Z order of uv tiles of `block_order_tile` cells of the largest facet's grid:
        # the blocks in flight at once share a small piece of every facet's grid (L2-resident)
        # while a stripe of 32 blocks stays on one baseline
        tile = block_order_tile / (max(f.npix_padded for f in tess.facets) * tess.cell_rad)
        vs = vs.with_block_order(bda.uv_locality_order(vs.bda_map, vs.block_start, vs.uvw, vs.freqs, tile))
        del bmap
    if large_min_vis:
        vs = vs.with_large_blocks(large_min_vis)
    nt = int(np.ceil(hours * 3600 / 300.0))
    J = synth.random_jones(seed + 3, nt, nfacets, 48, 1, 0.1)
    tmap = np.minimum(((obs.times - obs.times.min()) // 300.0).astype(np.int32), nt - 1)
    jd = D.JonesData(mode=1, kms=torch.from_numpy(J).to(dev), kms_tmap=torch.from_numpy(tmap).to(dev),
                     kms_cmap=torch.zeros(nchan, dtype=torch.int32, device=dev),
                     a0=torch.from_numpy(obs.A0).to(dev), a1=torch.from_numpy(obs.A1).to(dev),
                     wavelength_mean=float(np.mean(C_LIGHT / obs.freqs)))
    fg, fm = [], []
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 4)
    incr = (-cell / 3600 * np.pi / 180, cell / 3600 * np.pi / 180)
    for f, wt in zip(tess.facets, wts):
        n = f.npix_padded
        tabs = D.CFTables.create(wt.Wplanes, wt.WplanesConj, 11, wt.RefWave, wt.wmax, device=dev)
        mg = torch.view_as_complex(torch.randn((1, 1, n, n, 2), generator=gen, device=dev).contiguous()) * 1e-3
        common = dict(cf=tabs, incr=incr, cu=wt.Cu, cv=wt.Cv, l0=f.l0, m0=f.m0, idir_kms=f.isol, idir_beam=0)
        fg.append(D.FacetGrid(grid=torch.zeros((1, 1, n, n), dtype=torch.complex64, device=dev),
                              sumwt=torch.zeros((1, 1), dtype=torch.float64, device=dev),
                              sumjones=torch.zeros((2, 1), dtype=torch.float64, device=dev),
                              sumjones_chan=torch.zeros((2, nchan), dtype=torch.float64, device=dev), **common))
        fm.append(D.FacetGrid(grid=mg, **common))
    pol = D.make_pol([9, 10, 11, 12], [1])
    w = Workload("uneven_bda", vs, fg, fm, jd, pol, nvis=nrow * nchan, nrow=nrow, nchan=nchan, ncorr=ncorr,
                 nfacets=len(fg))
    w.info = dict(npix=tess.npix, grids=[f.npix_padded for f in tess.facets], nw=nw, nblocks=vs.nblocks,
                  large_blocks=(0 if vs.large_blocks is None else int(vs.large_blocks.numel())),
                  large_min_vis=large_min_vis,
                  block_order=(f"uv Z order, tiles of {block_order_tile} cells" if block_order_tile else "map order"),
                  vis_per_block=nrow * nchan / max(vs.nblocks, 1), wmax=wmax, nant=48, ntimes=obs.ntimes)
    w.host = {"obs": obs, "wterms": wts, "tess": tess, "chan_map": chan_map}
    return w
