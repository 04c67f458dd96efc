"""Benchmark: Mvis/s through one grid+degrid pass over all facets, on synthetic data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload combined_at_scale|multifacet_dde|uneven_bda] [--scale S] [--fp32-accumulation]

Default workload: the combined at-scale configuration -- a 10000^2 image at 1 arcsec in 11 x 11
facets (121 padded grids of 1485^2), 64 antennas, 8 h at 8 s, 256 channels, 4 correlations,
1000 point sources + 20 Gaussians, per-facet per-antenna Jones in 5-minute slots, 64 w-planes,
oversampling 11 (ddfacet_b200/configs.py combined_at_scale) -- streamed in 1-hour chunks.  A step
is one chunk (232.2 M visibilities x 4 correlations, 7.4 GB) through one major-cycle pass of the
hot path: degrid every facet's model grid and subtract the prediction from the visibilities, then
grid the residuals onto every facet's residual grid.  Both calls are the batched ones (one
persistent, queue-driven launch per call, schedule chosen by ddfacet_b200.autotune) with
FP64-accumulated grid sums unless --fp32-accumulation.  ``plain`` in the JSON line times the same
kernels one facet per call on the same chunk.  The visibilities (7.4 GB) exceed L2, so no flush is
needed between steps.

``e2e`` runs the same step through the public API from pinned host buffers: the chunk's
visibilities, uvw, flags and weights are copied in and the residual visibilities copied out every
step (pipeline.PipelinedStep, copies overlapped with the kernels).

Multi-GPU: the path shards by chunk (independent visibility sets), so each rank runs its own
replica (weak scaling, no data-path collective); the timed region is bracketed by barriers and the
maximum over ranks is reported.

``--impl reference`` times the reference's own CPU gridder/degridder (oracle/_ref, built from
DDFacet's sources) on the host cores, one process per facet, on a bounded row sample of the same
configuration, and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mvis/s grid+degrid on 1 B200, batched vs plain, at <=1e-5 rel err vs FP64"
UNIT = "Mvis/s"
E2E_CHUNKS = 4  # sub-chunks of the end-to-end leg (copies of one overlap the kernels of the next)
C_LIGHT = 299792458.0


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------------------------------
# Workload descriptions shared by the GPU arm and the CPU reference arm
# ------------------------------------------------------------------------------------------
WORKLOADS = {
    "combined_at_scale": dict(seed=1005, nant=64, radius=4000.0, hours=8.0, dump=8.0, nchan=256, npix=10000,
                              side=11, cell=1.0, nw=64, chunk_dumps=450, nsrc_cpu=20),
    "multifacet_dde": dict(seed=1002, nant=64, radius=4000.0, hours=4.0, dump=8.0, nchan=64, npix=4096,
                           side=9, cell=1.5, nw=32, chunk_dumps=1800, nsrc_cpu=20),
}


# ------------------------------------------------------------------------------------------
# CPU reference on a bounded sample (test-infrastructure checker, run only here and in tests)
# ------------------------------------------------------------------------------------------
def _cpu_worker(args):
    path, ifacet = args
    sys.path.insert(0, ROOT)
    from oracle import ref

    d = np.load(path, allow_pickle=True).item()
    f = d["facets"][ifacet]
    grid = np.zeros((1, 1, d["npix"], d["npix"]), np.complex64)
    sumwt = np.zeros((1, 1), np.float64)
    jon = dict(d["jones"])
    jon["idir_kms"] = f["idir"]
    jon["sumjones"] = np.zeros((2, 1), np.float64)
    jon["sumjones_chan"] = np.zeros((2, d["nchan"]), np.float64)
    lj = ref.ljones_list(jon, d["nrow"], d["nchan"], 1)
    vis = d["vis"].copy()
    t0 = time.perf_counter()
    ref.degrid(f["model"], vis, d["uvw"], d["flags"], f["wp"], f["wc"], f["winfos"], d["incr"], d["freqs"],
               f["finfo"], d["bda"], d["chan_map"], d["corr"], d["stokes"], ljones=lj)
    ref.grid(grid, vis, d["uvw"], d["flags"], d["weights"], sumwt, f["wp"], f["wc"], f["winfos"], d["incr"],
             d["freqs"], f["finfo"], d["bda"], d["chan_map"], d["corr"], d["stokes"], ljones=lj)
    dt = time.perf_counter() - t0
    ref.delete_semaphores()
    return dt


def cpu_reference(workload="combined_at_scale", nrow_frac=0.005, nprocs=None):
    """The reference's grid+degrid of the workload's chunk on a row sample, one process per facet
    on the host cores, extrapolated to every row and facet of the chunk.  Returns (Mvis/s, cores,
    sample description)."""
    from ddfacet_b200 import bda, cf, geometry, synth

    p = WORKLOADS[workload]
    nchan = p["nchan"]
    ncpu = os.cpu_count() or 1
    tess = geometry.regular_facets(p["npix"], p["side"], p["cell"], 1.7)
    nfacets_total = len(tess.facets)
    nprocs = nprocs or min(ncpu, nfacets_total)
    full = synth.make_observation(p["seed"], p["nant"], p["radius"], 34.0, 40.0, p["hours"], p["dump"], nchan,
                                  0.90e9, 1.67e9)
    wmax = float(np.max(np.abs(full.uvw[:, 2]))) * 1.001
    chunk_rows = p["chunk_dumps"] * full.nbl
    nrow_s = max(full.nbl, int(chunk_rows * nrow_frac))
    rows = np.arange(nrow_s)
    uvw = full.uvw[rows].copy()
    l, m, s = synth.point_sky(p["seed"] + 1, p["nsrc_cpu"], tess.npix * tess.cell_rad / 2 * 0.95,
                              flux=("powerlaw", 1e-3, 1.0))
    rng = np.random.default_rng(p["seed"] + 2)
    vis = synth.add_noise(rng, synth.dft_predict(uvw, full.freqs, l, m, s, ncorr=4), 1e-3).astype(np.complex64)
    flags = np.zeros(vis.shape, bool)
    weights = np.ones((nrow_s, nchan), np.float32)
    bmap = bda.plain_map(full.A0[rows], full.A1[rows], nchan)
    nt = int(np.ceil(p["hours"] * 3600 / 300.0))
    J = synth.random_jones(p["seed"] + 3, nt, nfacets_total, p["nant"], 1, 0.1)
    tmap = np.minimum(((full.times[rows] - full.times.min()) // 300.0).astype(np.int32), nt - 1)
    cell = p["cell"]
    facets = []
    pick = [tess.facets[i] for i in np.linspace(0, nfacets_total - 1, nprocs).astype(int)]
    for fgeo in pick:
        wt = cf.WTerms(Cell=cell, Sup=7, Nw=p["nw"], wmax=wmax, Npix=tess.npix_padded, Freqs=full.freqs, OverS=11,
                       lmShift=(fgeo.l0, fgeo.m0))
        model = (rng.standard_normal((1, 1, tess.npix_padded, tess.npix_padded)) * 1e-3).astype(np.complex64)
        facets.append(dict(wp=wt.Wplanes, wc=wt.WplanesConj, winfos=np.array([wt.RefWave, wt.wmax, p["nw"], 11.]),
                           finfo=np.array([wt.Cu, wt.Cv, fgeo.l0, fgeo.m0, fgeo.index]), idir=fgeo.index,
                           model=model))
    d = dict(vis=vis, uvw=uvw, flags=flags, weights=weights, freqs=full.freqs, chan_map=np.zeros(nchan, np.int32),
             bda=bmap, corr=[9, 10, 11, 12], stokes=[1], npix=tess.npix_padded, nrow=nrow_s, nchan=nchan,
             incr=np.array([-cell, cell]) / 3600 * np.pi / 180, facets=facets,
             jones=dict(kms=J, kms_tmap=tmap, kms_cmap=np.zeros(nchan, np.int32), A0=full.A0[rows].astype(np.int32),
                        A1=full.A1[rows].astype(np.int32), mode=1, interp_mode=0, apply_amp=1, apply_phase=1,
                        scale=0, calib_err=0.0))
    fd, path = tempfile.mkstemp(suffix=".npy", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    os.close(fd)
    np.save(path, d, allow_pickle=True)
    try:
        ctx = mp.get_context("spawn")
        with ctx.Pool(nprocs) as pool:
            t0 = time.perf_counter()
            times = pool.map(_cpu_worker, [(path, i) for i in range(nprocs)])
            wall = time.perf_counter() - t0
    finally:
        os.unlink(path)
    nvis_s = nrow_s * nchan
    # nprocs facets processed concurrently, each timed around its grid+degrid calls (the slowest
    # bounds the round); the job is every facet over every row of the chunk.
    per_facet_vis_rate = nprocs * nvis_s / max(max(times), 1e-9)  # facet-visibilities per second
    chunk_nvis = chunk_rows * nchan
    job_time = chunk_nvis * nfacets_total / per_facet_vis_rate
    mvis = chunk_nvis / job_time / 1e6
    sample = (f"{nrow_s} rows x {nchan} ch x 4 corr ({nvis_s/1e6:.2f} Mvis, {p['nsrc_cpu']}-source sky + noise) "
              f"of the {chunk_rows}-row chunk, {nprocs} of {nfacets_total} facets in parallel (one process each), "
              f"grid+degrid with per-vis Jones, wall {wall:.2f}s (per-process {min(times):.2f}-{max(times):.2f}s), "
              "scaled to all rows and facets of the chunk")
    return mvis, nprocs, sample


def err_vs_fp64(w, fp64_acc, pick=(0, None), sample_rows=None):
    """Errors of the GPU path against the FP64 restatement (oracle/gridder_fp64.c) on the benchmark's
    own data: the grid of a corner and the centre facet over every row of the chunk (the full
    accumulation depth), and the prediction of the same facets on a row sample."""
    import torch

    from ddfacet_b200 import device as D
    from oracle import fp64

    nf = w.nfacets
    pick = [0, nf // 2] if pick == (0, None) else list(pick)
    obs = w.host["obs"]
    dev = w.vs.vis.device
    vis_h = w.vs.vis.cpu().numpy()
    bmap_h = w.vs.bda_map.cpu().numpy()
    flags = np.zeros(vis_h.shape, bool)
    weights = np.ones(vis_h.shape[:2], np.float32)
    jh = {"A0": obs.A0.astype(np.int32), "A1": obs.A1.astype(np.int32), "mode": 1, "interp_mode": 0, "apply_amp": 1,
          "apply_phase": 1, "scale": 0, "calib_err": 0.0, "idir_beam": 0, "kms": w.host["J"],
          "kms_tmap": w.host["tmap"], "kms_cmap": np.zeros(w.nchan, np.int32)}
    out = {"grid": {}, "degrid": {}}
    t0 = time.perf_counter()
    fs = [w.facets_grid[i] for i in pick]
    saved = [(f.grid.clone(), f.grid_acc) for f in fs]
    for f in fs:
        f.grid.zero_()
        f.grid_acc = None
        if fp64_acc:
            f.with_fp64_accumulation()
    D.grid(w.vs, fs, w.pol, w.jones, batch=D.Batch.create(dev))
    torch.cuda.synchronize()
    gpu_grids = [f.grid.cpu().numpy() for f in fs]
    for f, (g, lo) in zip(fs, saved):
        f.grid.copy_(g)
        f.grid_acc = lo
    for i, g in zip(pick, gpu_grids):
        wt = w.host["wterms"][i]
        fgeo = w.host["tess"].facets[i]
        ref64 = fp64.grid(vis_h, obs.uvw, flags, weights, obs.freqs, w.host["chan_map"], bmap_h, wt.Wplanes,
                          wt.WplanesConj, 11, wt.RefWave, wt.wmax, w.facets_grid[i].incr, wt.Cu, wt.Cv,
                          (fgeo.l0, fgeo.m0), [9, 10, 11, 12], [1], 1, w.info["npix_padded"],
                          jones=dict(jh, idir_kms=w.facets_grid[i].idir_kms))[0]
        d = g.astype(np.complex128) - ref64
        out["grid"][str(i)] = float(np.sqrt(np.mean(np.abs(d) ** 2) / np.mean(np.abs(ref64) ** 2)))
    # prediction on a row sample: degrid the picked facets into zeros
    from ddfacet_b200 import bda

    nr = sample_rows or max(obs.nbl, min(obs.nrow, 64 * obs.nbl))
    zeros = torch.zeros((nr, w.nchan, w.ncorr), dtype=torch.complex64, device=dev)
    bm = bda.plain_map(obs.A0[:nr], obs.A1[:nr], w.nchan)
    vs_s = D.VisData.create(zeros, w.vs.uvw[:nr], w.vs.flags[:nr], w.vs.weights[:nr], obs.freqs, w.host["chan_map"],
                            bm, device=dev)
    jd = dict(jh, A0=jh["A0"][:nr], A1=jh["A1"][:nr], kms_tmap=jh["kms_tmap"][:nr])
    from ddfacet_b200 import pipeline

    D.degrid(vs_s, [w.facets_model[i] for i in pick], w.pol, pipeline.jones_rows(w.jones, 0, nr),
             batch=D.Batch.create(dev))
    torch.cuda.synchronize()
    got = vs_s.vis.cpu().numpy().astype(np.complex128)
    want = np.zeros_like(got)
    for i in pick:
        wt = w.host["wterms"][i]
        fgeo = w.host["tess"].facets[i]
        want += fp64.degrid(w.facets_model[i].grid.cpu().numpy(), np.zeros_like(got), obs.uvw[:nr], obs.freqs,
                            w.host["chan_map"], bm, wt.Wplanes, wt.WplanesConj, 11, wt.RefWave, wt.wmax,
                            w.facets_model[i].incr, wt.Cu, wt.Cv, (fgeo.l0, fgeo.m0), [9, 10, 11, 12], [1],
                            jones=dict(jd, idir_kms=w.facets_model[i].idir_kms))
    out["degrid"]["facets " + ",".join(map(str, pick))] = float(
        np.sqrt(np.mean(np.abs(got - want) ** 2) / np.mean(np.abs(want) ** 2)))
    out["max"] = max(list(out["grid"].values()) + list(out["degrid"].values()))
    out["how"] = (f"grid: facets {pick} over all {obs.nrow} rows of the chunk ({w.nvis/1e6:.1f} Mvis) against the "
                  f"FP64 restatement; degrid: the same facets' summed prediction on the first {nr} rows; "
                  f"relative RMS; {time.perf_counter() - t0:.0f} s on {os.cpu_count()} host threads")
    return out


# ------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, path, gpu_id=None):
        self.path = path
        self.p = None
        self.gpu_id = gpu_id

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"] + (["-i", self.gpu_id] if self.gpu_id else []),
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
            rows = [[x.strip() for x in r] for r in rows if len(r) >= 9]
            sm = [float(r[1]) for r in rows]
            mx = max(float(r[2]) for r in rows)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(sm)}
        except Exception:
            return None


def tap_stats(w, sample_rows=20000):
    """Mean taps per (facet, visibility) from the w-plane each visibility falls in (row sample)."""
    obs = w.host["obs"]
    wt = w.host["wterms"][0]
    rows = np.linspace(0, obs.nrow - 1, min(sample_rows, obs.nrow)).astype(int)
    wabs = np.abs(obs.uvw[rows, 2])[:, None]
    nu = obs.freqs[None, :]
    iw = np.rint((wt.Nw - 1) * wabs * (wt.RefWave * nu / C_LIGHT) / wt.wmax).astype(int)
    sups = np.array([p.shape[0] // 11 for p in wt.Wplanes])
    ok = iw < len(sups)
    s2 = np.where(ok, sups[np.minimum(iw, len(sups) - 1)] ** 2, 0)
    return float(s2.mean())


def fp32_peak_tflops(dev):
    """FP32 (CUDA-core) dense throughput measured with a cuBLAS SGEMM (TF32 off), TFLOP/s."""
    import torch

    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn((n, n), device=dev)
        b = torch.randn((n, n), device=dev)
        torch.mm(a, b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for _ in range(5):
            e0.record()
            torch.mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2 * n ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def dropin_leg(w, ndumps=32):
    """One facet through the drop-in ClassDDEGridMachine, the way a DDFacet facet worker calls it:
    ``put`` then ``get`` with pageable numpy arrays (copied to the device and back inside each
    call) on the first ``ndumps`` dumps of the chunk, with its CF tables computed by the machine
    itself (not timed).  Host wall time of the two calls; facet-visibilities per second."""
    from ddfacet_b200 import bda
    from ddfacet_b200.gridmachine import ClassDDEGridMachine, default_gd

    obs = w.host["obs"]
    fi = 0
    tess = w.host["tess"]
    fg, wt = tess.facets[fi], w.host["wterms"][fi]
    nr = min(obs.nrow, obs.nbl * ndumps)
    nchan = w.nchan
    gd = default_gd()
    gd["Image"]["Cell"] = w.info["cell_arcsec"]
    gd["CF"]["Nw"] = len(wt.Wplanes)
    bmap = bda.plain_map(obs.A0[:nr], obs.A1[:nr], nchan)
    gm = ClassDDEGridMachine(gd, obs.freqs, fg.npix_facet, lmShift=(fg.l0, fg.m0), compute_cf=True, wmax=wt.wmax,
                             bda_grid=bmap, bda_degrid=bmap, DataCorrelationFormat=[9, 10, 11, 12],
                             ExpectedOutputStokes=[1], NFreqBands=1, Padding=1.7)
    dirs = {"l": np.array([f.l0 for f in tess.facets]), "m": np.array([f.m0 for f in tess.facets]),
            "I": np.ones(len(tess.facets))}
    J = w.host["J"] if "J" in w.host else w.jones.kms.cpu().numpy()
    tmap = w.host["tmap"] if "tmap" in w.host else w.jones.kms_tmap.cpu().numpy()
    dico = {"DicoJones_killMS": {"Dirs": dirs, "Jones": {"Jones": np.ascontiguousarray(J, np.complex64),
                                                          "VisToJonesChanMapping": np.zeros(nchan, np.int32)},
                                 "TimeMapping": np.ascontiguousarray(tmap[:nr])}}
    vis = np.ascontiguousarray(w.vs.vis[:nr].cpu().numpy())
    uvw = np.ascontiguousarray(obs.uvw[:nr])
    flags = np.zeros(vis.shape, bool)
    weights = np.ones((nr, nchan), np.float32)
    a0a1 = (np.ascontiguousarray(obs.A0[:nr]), np.ascontiguousarray(obs.A1[:nr]))
    times = np.ascontiguousarray(obs.times[:nr])
    chan_map = np.zeros(nchan, np.int64)
    n = gm.GridShape[-1]
    grid = np.zeros((1, 1, n, n), np.complex64)
    model = np.ascontiguousarray(w.facets_model[fi].grid.cpu().numpy())
    kw = dict(DicoJonesMatrices=dico, freqs=obs.freqs, ChanMapping=chan_map)
    gm.put(times, uvw, vis.copy(), flags, a0a1, W=weights, ResidueGrid=grid, **kw)  # warm-up
    gm.get(times, uvw, vis.copy(), flags, a0a1, model, ImToGrid=False, **kw)
    t0 = time.perf_counter()
    gm.put(times, uvw, vis, flags, a0a1, W=weights, ResidueGrid=grid, **kw)
    t1 = time.perf_counter()
    gm.get(times, uvw, vis, flags, a0a1, model, ImToGrid=False, **kw)
    t2 = time.perf_counter()
    return {"facet_Mvis_per_s": round(nr * nchan / (t2 - t0) / 1e6, 2), "put_ms": round((t1 - t0) * 1e3, 1),
            "get_ms": round((t2 - t1) * 1e3, 1),
            "what": (f"facet {fi}: ClassDDEGridMachine.put + get with pageable numpy arrays (a DDFacet facet "
                     f"worker's calls), first {ndumps} dumps ({nr} rows x {nchan} ch x 4 corr, "
                     f"{vis.nbytes / 1e6:.0f} MB of visibilities copied in and out by each call), host wall time")}


def algorithmic(w, s2):
    """Compulsory bytes and FLOPs of one grid call and one degrid call (one pass over the chunk):
    every stream touched once.  Grid: visibilities (K complex64), flags (K bytes), weights, uvw,
    the residual grids written, one CF table set, the Jones array.  Degrid: visibilities read and
    written, uvw, the model grids read, CF, Jones.  FLOPs: S^2 complex multiply-adds per facet and
    visibility (8 flops each) plus the 2x2 Jones products (112) and phasor/weight (20)."""
    K, F = w.ncorr, w.nfacets
    G2 = sum(int(f.grid.numel()) for f in w.facets_grid)
    cf_bytes = sum(int(f.cf.data.numel()) * 8 for f in w.facets_grid) // 2
    jones_bytes = int(w.jones.kms.numel()) * 8 if w.jones is not None else 0
    grid_b = w.nvis * (K * 8 + K + 4) + w.nrow * 24 + G2 * 8 + cf_bytes + jones_bytes
    degrid_b = w.nvis * (K * 16) + w.nrow * 24 + G2 * 8 + cf_bytes + jones_bytes
    flops_call = F * w.nvis * (8 * s2 + 112 + 20)
    return grid_b, degrid_b, flops_call


def run_gpu(args):
    import torch
    import torch.distributed as dist

    from ddfacet_b200 import autotune, configs, device as D, pipeline

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    comp = not args.fp32_accumulation

    t_build = time.perf_counter()
    if args.workload == "multifacet_dde":
        w = configs.multifacet_dde(device=dev, scale=args.scale)
    else:
        w = configs.combined_at_scale(device=dev, scale=args.scale)
    if comp:
        for f in w.facets_grid:
            f.with_fp64_accumulation()
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
    stream = torch.cuda.current_stream()

    t_tune = time.perf_counter()
    tuned = autotune.tune(w.vs, w.facets_grid, w.facets_model, w.pol, w.jones, use_cache=not args.retune)
    t_tune = time.perf_counter() - t_tune
    bg, bd = tuned.grid, tuned.degrid

    def step(ev=None):
        for f in w.facets_grid:
            f.grid.zero_()
        if ev:
            ev[0].record(stream)
        D.degrid(w.vs, w.facets_model, w.pol, w.jones, batch=bd)
        if ev:
            ev[1].record(stream)
        D.grid(w.vs, w.facets_grid, w.pol, w.jones, batch=bg)
        if ev:
            ev[2].record(stream)

    def plain_step():
        # the same kernels with one facet per call (one launch per facet and direction)
        for fm in w.facets_model:
            D.degrid(w.vs, [fm], w.pol, w.jones)
        for fg in w.facets_grid:
            fg.grid.zero_()
            D.grid(w.vs, [fg], w.pol, w.jones)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    gpu_id = None
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid).replace("GPU-", "")
    except Exception:
        cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        gpu_id = cvd.split(",")[dev.index or 0] if cvd else None
    clk = ClockSampler(os.path.join(tempfile.gettempdir(), f"ddfg_clocks_{os.getpid()}.csv"), gpu_id)
    with clk:
        torch.cuda.synchronize()
        start.record(stream)
        for k in range(args.steps):
            step(evs[k])
        stop.record(stream)
        torch.cuda.synchronize()
    ms_total = start.elapsed_time(stop)
    if world > 1:
        t = torch.tensor([ms_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    degrid_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    grid_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))

    # The same step captured once in a CUDA graph and replayed (device.capture_graph).
    graph = D.capture_graph(step)
    torch.cuda.synchronize()
    gr0 = torch.cuda.Event(enable_timing=True)
    gr1 = torch.cuda.Event(enable_timing=True)
    gr0.record(stream)
    graph.replay()
    gr1.record(stream)
    torch.cuda.synchronize()
    graph_ms = gr0.elapsed_time(gr1)
    del graph

    # End to end through the public API with host buffers: every step copies its inputs from
    # pinned memory and its residual visibilities back, in E2E_CHUNKS sub-chunks whose copies
    # overlap the kernels of the neighbouring sub-chunk (pipeline.PipelinedStep).
    host = {"vis": w.host["vis"], "uvw": w.vs.uvw.cpu().pin_memory(), "flags": w.vs.flags.cpu().pin_memory(),
            "weights": w.vs.weights.cpu().pin_memory()}
    host["out"] = torch.empty_like(host["vis"]).pin_memory()
    h2d = (host["vis"].numel() * 8 + host["uvw"].numel() * 8 + host["flags"].numel() + host["weights"].numel() * 4)
    d2h = host["out"].numel() * 8
    piped = pipeline.PipelinedStep(configs.row_chunks(w, E2E_CHUNKS), w.facets_grid, w.facets_model, w.pol, dev,
                                   batch_grid=bg, batch_degrid=bd)

    def e2e_step():
        for f in w.facets_grid:
            f.grid.zero_()
        piped.run(host, stream)

    e2e_steps = max(1, min(args.steps, 3))
    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    s1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = s0.elapsed_time(s1) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    del piped

    # The gridder with float32 grid sums (no FP64 accumulator), for comparison: one call.
    plain_grid_ms = None
    if comp:
        lo = [f.grid_acc for f in w.facets_grid]
        for f in w.facets_grid:
            f.grid_acc = None
        bnc = D.Batch.create(dev, facets_per_pack=bg.facets_per_pack, stripes_per_item=bg.stripes_per_item)
        D.grid(w.vs, w.facets_grid, w.pol, w.jones, batch=bnc)
        torch.cuda.synchronize()
        u0, u1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        u0.record(stream)
        D.grid(w.vs, w.facets_grid, w.pol, w.jones, batch=bnc)
        u1.record(stream)
        torch.cuda.synchronize()
        plain_grid_ms = u0.elapsed_time(u1)
        for f, g in zip(w.facets_grid, lo):
            f.grid_acc = g

    # The plain path on the same chunk: one facet per call.
    plain_step()
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    plain_step()
    p1.record(stream)
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)

    # Differentiation (the prediction as a torch.autograd.Function, ddfacet_b200.autograd): the
    # forward prediction, then the backward passes for every facet's model grid (adjoint gridding
    # kernel) and the per-facet per-antenna Jones, timed on the device.
    diff_info = None
    if w.jones is not None and not args.no_diff:
        from ddfacet_b200.autograd import PredictSetup, predict
        setup = PredictSetup(vs=w.vs, facets=w.facets_model, pol=w.pol, jones=w.jones)
        leaves = [f.grid.detach().clone().requires_grad_(True) for f in w.facets_model]
        kms_leaf = w.jones.kms.detach().clone().requires_grad_(True)
        de = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        de[0].record(stream)
        P = predict(setup, leaves, kms_leaf)
        de[1].record(stream)
        grads = torch.autograd.grad(P, [*leaves, kms_leaf], grad_outputs=w.vs.vis)
        de[2].record(stream)
        torch.cuda.synchronize()
        fwd_ms, bwd_ms = de[0].elapsed_time(de[1]), de[1].elapsed_time(de[2])
        del grads, leaves, kms_leaf, P
        diff_info = {"forward_ms": round(fwd_ms, 1), "backward_ms": round(bwd_ms, 1),
                     "Mvis_per_s": round(w.nvis / ((fwd_ms + bwd_ms) * 1e-3) / 1e6, 2),
                     "what": "predict (all facets) + backward for all model grids and the kMS Jones"}
        torch.cuda.empty_cache()

    nvis = w.nvis
    value = world * nvis / (ms_step * 1e-3) / 1e6
    e2e_value = world * nvis / (e2e_ms * 1e-3) / 1e6
    plain_value = world * nvis / (plain_ms * 1e-3) / 1e6

    s2 = tap_stats(w)
    grid_b, degrid_b, flops_call = algorithmic(w, s2)
    hbm_peak, peak_kind = _peaks()
    fp32_peak = fp32_peak_tflops(dev)
    dom = "grid" if grid_ms >= degrid_ms else "degrid"
    dom_ms = max(grid_ms, degrid_ms)
    dom_bytes = grid_b if dom == "grid" else degrid_b
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    # DRAM bytes (read + write) of one call of each kernel, per visibility, from the one-pass ncu
    # capture of the full chunk with the benchmark's schedules (profiles/traffic_combined_at_scale_full.md):
    # grid 194.2 GB in one launch (FP64 accumulators), degrid 229.7 GB in eight launches of 16 facets
    # (each re-reads and rewrites the visibilities), for 232,243,200 visibilities
    traffic_per_vis = {"grid": 194.172e9 / 232243200, "degrid": 229.674e9 / 232243200}
    K, F, G = w.ncorr, w.nfacets, w.info["npix_padded"]
    launches_grid = math.ceil(F / 128) * (2 if comp else 1)
    dpp = bd.facets_per_pack if bd.facets_per_pack > 0 else 128
    launches_degrid = math.ceil(F / min(dpp, 128))
    if args.workload == "combined_at_scale":
        desc = (f"combined at scale, one 1-h chunk: {F} facets x {G}^2 grids, {w.nrow} rows x "
                f"{w.nchan} ch x {K} corr ({nvis/1e6:.1f} Mvis, 7.4 GB) of the 8-h track "
                f"({w.info['full_track_nvis']/1e9:.2f} G vis in 8 chunks), per-vis Jones, "
                f"{w.info['nw']} w-planes, OverS 11, 1000 point + 20 Gaussian sources; step = degrid "
                "all facets (subtract) + grid all facets")
    else:
        desc = (f"multi-facet DDE: {F} facets x {G}^2 grid, {w.nrow} rows x {w.nchan} ch x {K} corr "
                f"({nvis/1e6:.1f} Mvis), per-vis Jones, {w.info['nw']} w-planes, OverS 11; step = degrid "
                "all facets (subtract) + grid all facets")
    out = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(3, args.warmup),
        "ms_per_step": round(ms_step, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" + (" (FP64 grid sums)" if comp else "") + "; FP64 phase/index arithmetic",
        "data": "synthetic (seeded; generated on device)",
        "config": {
            "workload": desc, "facets": F, "grid": G, "nvis": nvis, "ncorr": K, "nchan": w.nchan, "nrow": w.nrow,
            "w_planes": w.info["nw"], "supports": w.info["supports"], "mean_taps_per_vis": round(s2, 1),
            "array": "64 antennas uniform in a disk of 4 km radius (the '8 km disk' read as its diameter)",
            "bda": "none: every (row, channel) its own block",
            "chunk": w.info.get("chunk", "whole set"),
            "l2": f"inputs ({nvis * K * 8 / 1e9:.1f} GB visibilities) larger than L2; no flush",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "scale": args.scale,
            "fp64_accumulation": comp,
        },
        "kernels_ms": {"degrid_call": round(degrid_ms, 3), "grid_call": round(grid_ms, 3),
                       "graph_replay_step": round(graph_ms, 3)},
        "plain": {"ms_per_step": round(plain_ms, 1), "value": round(plain_value, 3),
                  "what": "the same kernels, one facet per call (one launch per facet and direction), same chunk",
                  "batched_speedup": round(plain_ms / ms_step, 3)},
        "schedule": dict(tuned.describe(), tune_s=round(t_tune, 1)),
        "fp32_accumulation_grid_ms": None if plain_grid_ms is None else round(plain_grid_ms, 1),
        "differentiation": diff_info,
        "roofline": {
            "bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 6), "peak_kind": peak_kind,
            "traffic": int(traffic_per_vis[dom] * nvis) if args.workload == "combined_at_scale" else None,
            "alg_bytes_per_launch": int(dom_bytes),
            "how": ("achieved = compulsory bytes of one call (visibilities, flags, weights, uvw, grids, one CF "
                    "table set, Jones; one launch per call) / the call's CUDA-event time; traffic = DRAM "
                    "read+write of one call in the one-pass ncu capture of the full chunk, per visibility x "
                    "visibilities"),
            "fp32": {"achieved_tflops": round(flops_call / (dom_ms * 1e-3) / 1e12, 3),
                     "peak_tflops": round(fp32_peak, 1), "peak_kind": "measured (cuBLAS SGEMM, TF32 off)",
                     "frac": round(flops_call / (dom_ms * 1e-3) / 1e12 / fp32_peak, 4),
                     "flops_per_call": int(flops_call)},
        },
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3),
                "how": f"pinned host buffers, {E2E_CHUNKS} sub-chunks, copies overlapped with the kernels"},
        "gpu_launches": args.steps * (launches_grid + launches_degrid),
        "clocks": clk.summary(),
        "setup_s": round(t_build, 1),
    }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and args.cpu_baseline and world == 1:
        torch.cuda.empty_cache()
        try:
            out["err_vs_fp64"] = err_vs_fp64(w, comp)
        except Exception as e:  # the check is reported, not allowed to drop the measurement
            out["err_vs_fp64"] = {"error": repr(e)[:300]}
        try:
            out["dropin"] = dropin_leg(w)
        except Exception as e:  # reported, not allowed to drop the measurement
            out["dropin"] = {"error": repr(e)[:300]}
        if args.workload in WORKLOADS:
            mv, cores, sample = cpu_reference(args.workload)
            out["cpu_baseline"] = {"value": round(mv, 4), "unit": UNIT, "cores": cores, "kind": "reference",
                                   "sample": sample}
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_uneven(args):
    """Uneven Voronoi facets with averaged BDA blocks (the batching-form workload): one degrid + grid
    step over all facets, device-resident, CUDA-event timed, batched and plain."""
    import torch

    from ddfacet_b200 import autotune, configs, device as D

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    w = configs.uneven_bda(device=dev, scale=args.scale)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    if not args.fp32_accumulation:
        for f in w.facets_grid:
            f.with_fp64_accumulation()
    tuned = autotune.tune(w.vs, w.facets_grid, w.facets_model, w.pol, w.jones, use_cache=not args.retune)

    def step(batched=True):
        for f in w.facets_grid:
            f.grid.zero_()
        if batched:
            D.degrid(w.vs, w.facets_model, w.pol, w.jones, batch=tuned.degrid)
            D.grid(w.vs, w.facets_grid, w.pol, w.jones, batch=tuned.grid)
        else:
            for fm in w.facets_model:
                D.degrid(w.vs, [fm], w.pol, w.jones)
            for fg in w.facets_grid:
                D.grid(w.vs, [fg], w.pol, w.jones)

    def timed(batched, n):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            step(batched)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    ms = timed(True, args.steps)
    step(False)
    torch.cuda.synchronize()
    plain_ms = timed(False, 1)

    def call_ms(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return round(e0.elapsed_time(e1), 1)

    kernels_ms = {"degrid_call": call_ms(lambda: D.degrid(w.vs, w.facets_model, w.pol, w.jones, batch=tuned.degrid)),
                  "grid_call": call_ms(lambda: D.grid(w.vs, w.facets_grid, w.pol, w.jones, batch=tuned.grid))}
    info = dict(w.info)
    g = info.pop("grids")
    print(json.dumps({"metric": METRIC, "value": round(w.nvis / (ms * 1e-3) / 1e6, 3), "unit": UNIT,
                      "ms_per_step": round(ms, 1), "steps": args.steps, "warmup": max(1, args.warmup),
                      "kernels_ms": kernels_ms, "fp64_accumulation": not args.fp32_accumulation,
                      "plain": {"ms_per_step": round(plain_ms, 1),
                                "value": round(w.nvis / (plain_ms * 1e-3) / 1e6, 3),
                                "batched_speedup": round(plain_ms / ms, 3)},
                      "schedule": tuned.describe(),
                      "config": {"workload": f"uneven BDA: {w.nfacets} Voronoi facets (grids {min(g)}..{max(g)}), "
                                             f"{w.nrow} rows x {w.nchan} ch x 4 corr ({w.nvis/1e6:.1f} Mvis), "
                                             f"{info['nblocks']} BDA blocks, per-vis Jones", **info,
                                 "scale": args.scale},
                      "setup_s": round(setup_s, 1)}), flush=True)


def run_profile_call(args):
    """One grid or one degrid call of the workload with a fixed schedule and nothing else on the GPU
    before it but the data generation: the launch an ncu capture selects with -k and -c."""
    import torch

    from ddfacet_b200 import configs, device as D

    dev = torch.device("cuda", 0)
    w = (configs.multifacet_dde if args.workload == "multifacet_dde" else configs.combined_at_scale)(
        device=dev, scale=args.scale, keep_host=False)
    if not args.fp32_accumulation:
        for f in w.facets_grid:
            f.with_fp64_accumulation()
    b = D.Batch.create(dev, facets_per_pack=args.fpp, stripes_per_item=args.spi, tiles=args.tiles)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    if args.profile_call == "grid":
        D.grid(w.vs, w.facets_grid, w.pol, w.jones, batch=b)
    else:
        D.degrid(w.vs, w.facets_model, w.pol, w.jones, batch=b)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"call": args.profile_call, "ms": round(e0.elapsed_time(e1), 3), "nvis": w.nvis,
                      "schedule": b.describe(), "fp64_accumulation": not args.fp32_accumulation}), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (oracle/build_ref.sh)"}))
        return
    wl = args.workload if args.workload in WORKLOADS else "combined_at_scale"
    vals = []
    cores = sample = None
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps)):
        mv, cores, sample = cpu_reference(wl)
        vals.append(mv)
    wall = time.perf_counter() - t0
    v = float(np.median(vals))
    p = WORKLOADS[wl]
    out = {"metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
           "steps": args.steps, "warmup": 0, "ms_per_step": round(wall / max(1, args.steps) * 1e3, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64 grid / f64 internal",
           "data": "synthetic (seeded)",
           "config": {"workload": f"{wl}: {p['side']}x{p['side']} facets, {p['nchan']} ch x 4 corr, per-vis Jones, "
                                  f"{p['nw']} w-planes; reference CPU gridder+degridder on a row sample of one "
                                  "chunk, extrapolated to the chunk"},
           "impl": "reference",
           "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": cores, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--fp32-accumulation", action="store_true", help="float32 grid sums (no FP64 accumulator)")
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiation timing")
    ap.add_argument("--retune", action="store_true", help="ignore the autotuner's cache")
    ap.add_argument("--workload", default="combined_at_scale",
                    choices=["combined_at_scale", "multifacet_dde", "uneven_bda"])
    ap.add_argument("--profile-call", choices=["grid", "degrid"],
                    help="run one batched call with the schedule below and exit (for ncu captures)")
    ap.add_argument("--fpp", type=int, default=16, help="--profile-call: facets per pack")
    ap.add_argument("--spi", type=int, default=64, help="--profile-call: stripes per queue item")
    ap.add_argument("--tiles", action="store_true", help="--profile-call: warp grid tiles")

    args = ap.parse_args()
    if args.profile_call:
        run_profile_call(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "uneven_bda":
        run_uneven(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
