"""Benchmark: Mvis/s through one grid+degrid pass over all facets, on synthetic data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--scale S]

A step is one major-cycle pass of the hot path over the whole visibility set: degrid every
facet's model grid and subtract the prediction from the visibilities, then grid the residual
visibilities onto every facet's (zeroed) residual grid.  The workload is the multi-facet DDE
configuration (81 facets of 735^2, 232 M visibilities x 4 correlations, per-visibility Jones,
32 w-planes); see ddfacet_b200/configs.py.  Inputs (7.4 GB of visibilities) are larger than L2,
so no flush is needed between steps.

Multi-GPU: the path shards by facet-independent visibility sets, so each rank runs its own
replica of the workload (weak scaling, no data-path collective); the timed region is bracketed
by barriers and the maximum over ranks is reported.

``--impl reference`` times the reference's own CPU gridder/degridder (oracle/_ref, built from
DDFacet's sources) on the host cores, one process per facet, on a bounded sample of the same
workload, and prints the same metric.
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
E2E_CHUNKS = 8  # time chunks of the end-to-end leg


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


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


def cpu_reference(nfacets_total=81, nrow_frac=0.02, nprocs=None, seed=1002):
    """Reference grid+degrid of the multi-facet DDE workload on a row sample; one process per
    facet on the host cores.  Returns (Mvis/s for the full job, cores, sample description)."""
    from ddfacet_b200 import bda, cf, geometry, synth

    ncpu = os.cpu_count() or 1
    nprocs = nprocs or min(ncpu, nfacets_total)
    nchan = 64
    obs = synth.make_observation(seed, 64, 4000.0, 34.0, 40.0, 4.0, 8.0, nchan, 0.90e9, 1.67e9)
    tess = geometry.regular_facets(4096, 9, 1.5, 1.7)
    nrow_s = max(1, int(obs.nrow * nrow_frac))
    rows = np.arange(nrow_s)
    uvw = obs.uvw[rows].copy()
    l, m, s = synth.point_sky(seed + 1, 20, tess.npix * tess.cell_rad / 2 * 0.95, flux=("powerlaw", 1e-3, 1.0))
    rng = np.random.default_rng(seed + 2)
    vis = synth.add_noise(rng, synth.dft_predict(uvw, obs.freqs, l, m, s, ncorr=4), 1e-3).astype(np.complex64)
    flags = np.zeros(vis.shape, bool)
    weights = np.ones((nrow_s, nchan), np.float32)
    bmap = bda.plain_map(obs.A0[rows], obs.A1[rows], nchan)
    nt = int(np.ceil(4.0 * 3600 / 300.0))
    J = synth.random_jones(seed + 3, nt, len(tess.facets), 64, 1, 0.1)
    tmap = np.minimum(((obs.times[rows] - obs.times.min()) // 300.0).astype(np.int32), nt - 1)
    wmax = float(np.max(np.abs(obs.uvw[:, 2]))) * 1.001
    cell = 1.5
    facets = []
    pick = [tess.facets[i] for i in np.linspace(0, len(tess.facets) - 1, nprocs).astype(int)]
    for fgeo in pick:
        wt = cf.WTerms(Cell=cell, Sup=7, Nw=32, wmax=wmax, Npix=tess.npix_padded, Freqs=obs.freqs, OverS=11,
                       lmShift=(fgeo.l0, fgeo.m0))
        model = (rng.standard_normal((1, 1, tess.npix_padded, tess.npix_padded)) * 1e-3).astype(np.complex64)
        facets.append(dict(wp=wt.Wplanes, wc=wt.WplanesConj, winfos=np.array([wt.RefWave, wt.wmax, 32, 11.]),
                           finfo=np.array([wt.Cu, wt.Cv, fgeo.l0, fgeo.m0, fgeo.index]), idir=fgeo.index,
                           model=model))
    d = dict(vis=vis, uvw=uvw, flags=flags, weights=weights, freqs=obs.freqs, chan_map=np.zeros(nchan, np.int32),
             bda=bmap, corr=[9, 10, 11, 12], stokes=[1], npix=tess.npix_padded, nrow=nrow_s, nchan=nchan,
             incr=np.array([-cell, cell]) / 3600 * np.pi / 180, facets=facets,
             jones=dict(kms=J, kms_tmap=tmap, kms_cmap=np.zeros(nchan, np.int32), A0=obs.A0[rows].astype(np.int32),
                        A1=obs.A1[rows].astype(np.int32), mode=1, interp_mode=0, apply_amp=1, apply_phase=1,
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
    # bounds the round); the full job is nfacets_total facets over all rows.
    per_facet_vis_rate = nprocs * nvis_s / max(max(times), 1e-9)  # facet-visibilities per second
    full_nvis = obs.nrow * nchan
    job_time = full_nvis * nfacets_total / per_facet_vis_rate
    mvis = full_nvis / job_time / 1e6
    sample = (f"{nrow_s} rows x {nchan} ch x 4 corr ({nvis_s/1e6:.2f} Mvis) of the {obs.nrow}-row set, "
              f"{nprocs} of {nfacets_total} facets in parallel (one process each), grid+degrid with per-vis Jones, "
              f"wall {wall:.2f}s (per-process {min(times):.2f}-{max(times):.2f}s), scaled to all rows and facets")
    return mvis, nprocs, sample


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
    iw = np.rint((wt.Nw - 1) * wabs * (wt.RefWave * nu / 299792458.0) / wt.wmax).astype(int)
    sups = np.array([p.shape[0] // 11 for p in wt.Wplanes])
    ok = iw < len(sups)
    s2 = np.where(ok, sups[np.minimum(iw, len(sups) - 1)] ** 2, 0)
    return float(s2.mean())


def run_gpu(args):
    import torch
    import torch.distributed as dist

    from ddfacet_b200 import configs, device as D, pipeline

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    t_build = time.perf_counter()
    w = configs.multifacet_dde(device=dev, scale=args.scale)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
    stream = torch.cuda.current_stream()
    fpl = 16

    def step(ev=None):
        for f in w.facets_grid:
            f.grid.zero_()
        if ev:
            ev[0].record(stream)
        D.degrid(w.vs, w.facets_model, w.pol, w.jones)
        if ev:
            ev[1].record(stream)
        D.grid(w.vs, w.facets_grid, w.pol, w.jones)
        if ev:
            ev[2].record(stream)

    def plain_step():
        # the same physics with one facet per launch, blocks in map order (direct kernels)
        for fm, fg in zip(w.facets_model, w.facets_grid):
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

    # The same step captured once in a CUDA graph and replayed (device.capture_graph).
    graph = D.capture_graph(step)
    torch.cuda.synchronize()
    gr0 = torch.cuda.Event(enable_timing=True)
    gr1 = torch.cuda.Event(enable_timing=True)
    gr0.record(stream)
    for _ in range(max(1, min(args.steps, 3))):
        graph.replay()
    gr1.record(stream)
    torch.cuda.synchronize()
    graph_ms = gr0.elapsed_time(gr1) / max(1, min(args.steps, 3))
    del graph
    degrid_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    grid_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))

    # End to end through the public API with host buffers: every step copies its inputs from
    # pinned memory and its residual visibilities back, in E2E_CHUNKS time chunks whose copies
    # overlap the kernels of the neighbouring chunk (pipeline.PipelinedStep).
    host = {"vis": w.host["vis"], "uvw": w.vs.uvw.cpu().pin_memory(), "flags": w.vs.flags.cpu().pin_memory(),
            "weights": w.vs.weights.cpu().pin_memory()}
    host["out"] = torch.empty_like(host["vis"]).pin_memory()
    h2d = (host["vis"].numel() * 8 + host["uvw"].numel() * 8 + host["flags"].numel() + host["weights"].numel() * 4)
    d2h = host["out"].numel() * 8
    piped = pipeline.PipelinedStep(configs.row_chunks(w, E2E_CHUNKS), w.facets_grid, w.facets_model, w.pol, dev)

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

    # Imaging weights (Briggs, robust 0) of the same visibilities: index, density accumulation,
    # Briggs transform and normalisation, device-resident, timed on the device.
    from ddfacet_b200.weights import ImagingWeights, uvmax_wavelengths
    obs = w.host["obs"]
    uvmax = uvmax_wavelengths(w.vs.uvw, None, obs.freqs)
    tess = w.host["tess"]

    def weights_pass():
        iw = ImagingWeights(uvmax, tess.cell_rad, tess.npix, mode="briggs", robust=0.0, device=dev)
        iw.accumulate(w.vs.uvw, obs.freqs, w.vs.weights)
        iw.finish()
        return iw, iw.apply(w.vs.uvw, obs.freqs, w.vs.weights)

    weights_pass()
    torch.cuda.synchronize()
    q0 = torch.cuda.Event(enable_timing=True)
    q1 = torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    iw, _ = weights_pass()
    q1.record(stream)
    torch.cuda.synchronize()
    weights_ms = q0.elapsed_time(q1)
    # bytes: uvw and weights read twice (index for accumulation, index for normalisation), index
    # written and read twice, weights written once; the density grid is small and L2-resident
    wbytes = 2 * (w.nrow * 24 + nvis_w(w) * 4) + 4 * nvis_w(w) * 4 + nvis_w(w) * 4
    weights_info = {"ms": round(weights_ms, 3), "Mvis_per_s": round(w.nvis / (weights_ms * 1e-3) / 1e6, 1),
                    "achieved_GBs": round(wbytes / (weights_ms * 1e-3) / 1e9, 1),
                    "grid": [int(iw.npixx), int(iw.npixy)], "mode": "briggs robust 0"}
    del iw

    # Mode-1 BDA block map (DDFacet's default averaging, GridDecorr 0.02) of the same rows, built
    # on the GPU; reported beside the metric (the timed step itself uses single-visibility blocks).
    from ddfacet_b200 import bda as bda_mod
    dfreq = float(obs.freqs[1] - obs.freqs[0])
    lmax = tess.npix * tess.cell_rad * np.sqrt(2) / 2
    bargs = (obs.A0, obs.A1, w.vs.uvw, obs.freqs, dfreq, np.sqrt(6 * 0.02), lmax, w.host["chan_map"])
    bda_mod.smear_mapping_gpu(*bargs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bmap = bda_mod.smear_mapping_gpu(*bargs)
    torch.cuda.synchronize()
    bda_ms = (time.perf_counter() - t0) * 1e3
    nb_bda = int(bmap[0].item()) & 0xFFFFFFFF
    bda_info = {"ms": round(bda_ms, 2), "blocks": nb_bda, "vis_per_block": round(w.nvis / max(nb_bda, 1), 2),
                "what": "mode-1 map, GridDecorr 0.02, l = image radius x sqrt 2, wall time incl. host grouping"}
    del bmap

    # Differentiation (the prediction as a torch.autograd.Function, ddfacet_b200.autograd): the
    # forward prediction, then the backward passes for every facet's model grid (adjoint gridding
    # kernel) and the per-facet per-antenna Jones, timed on the device.
    diff_info = None
    if w.jones is not None:
        from ddfacet_b200.autograd import PredictSetup, predict
        setup = PredictSetup(vs=w.vs, facets=w.facets_model, pol=w.pol, jones=w.jones)
        leaves = [f.grid.detach().clone().requires_grad_(True) for f in w.facets_model]
        kms_leaf = w.jones.kms.detach().clone().requires_grad_(True)

        def diff_pass(ev=None):
            if ev:
                ev[0].record(stream)
            P = predict(setup, leaves, kms_leaf)
            if ev:
                ev[1].record(stream)
            grads = torch.autograd.grad(P, [*leaves, kms_leaf], grad_outputs=w.vs.vis)
            if ev:
                ev[2].record(stream)
            return grads

        diff_pass()
        torch.cuda.synchronize()
        de = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        grads = diff_pass(de)
        torch.cuda.synchronize()
        fwd_ms, bwd_ms = de[0].elapsed_time(de[1]), de[1].elapsed_time(de[2])
        del grads, leaves, kms_leaf
        diff_info = {"forward_ms": round(fwd_ms, 1), "backward_ms": round(bwd_ms, 1),
                     "Mvis_per_s": round(w.nvis / ((fwd_ms + bwd_ms) * 1e-3) / 1e6, 2),
                     "what": "predict (all facets) + backward for all model grids and the kMS Jones"}

    plain_ms = None
    if args.plain:
        plain_step()
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        plain_step()
        p1.record(stream)
        torch.cuda.synchronize()
        plain_ms = p0.elapsed_time(p1)

    nvis = w.nvis
    value = world * nvis / (ms_step * 1e-3) / 1e6
    e2e_value = world * nvis / (e2e_ms * 1e-3) / 1e6

    # Roofline of the dominant kernel: algorithmic bytes per call (inputs read once per 16-facet
    # launch, grids and CF tables once per call).
    K = w.ncorr
    F = w.nfacets
    G = w.info["npix_padded"]
    cf_bytes = sum(int(f.cf.data.numel()) * 8 for f in w.facets_grid)
    jones_bytes = int(w.jones.kms.numel()) * 8 if w.jones is not None else 0
    launches_per_call = math.ceil(F / (fpl if fpl > 0 else 16))
    grid_bytes = (launches_per_call * (nvis * (K * 8 + K + 4) + w.nrow * 24 + jones_bytes)
                  + F * G * G * 8 * 2 + cf_bytes // 2)
    degrid_bytes = (launches_per_call * (nvis * (K * 16) + w.nrow * 24 + jones_bytes)
                    + F * G * G * 8 + cf_bytes // 2)
    s2 = tap_stats(w)
    flops_pass = F * nvis * (2 * s2 * 8 + 2 * (112 + 40))
    hbm_peak, peak_kind = _peaks()
    dom = "grid" if grid_ms >= degrid_ms else "degrid"
    dom_ms = max(grid_ms, degrid_ms)
    dom_bytes = grid_bytes if dom == "grid" else degrid_bytes
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
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
        "dtype": "f32 (FP64 phase/index arithmetic)",
        "data": "synthetic (seeded; generated on device)",
        "config": {
            "workload": f"multi-facet DDE: {F} facets x {G}^2 grid, {w.nrow} rows x {w.nchan} ch x {K} corr "
                        f"({nvis/1e6:.1f} Mvis), per-vis Jones, {w.info['nw']} w-planes, OverS 11; "
                        "step = degrid all facets (subtract) + grid all facets",
            "facets": F, "grid": G, "nvis": nvis, "ncorr": K, "nchan": w.nchan, "nrow": w.nrow,
            "w_planes": w.info["nw"], "mean_taps_per_vis": round(s2, 1),
            "l2": "inputs (7.4 GB visibilities) larger than L2; no flush",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "scale": args.scale,
        },
        "kernels_ms": {"degrid_call": round(degrid_ms, 3), "grid_call": round(grid_ms, 3),
                       "graph_replay_step": round(graph_ms, 3)},
        "plain": (None if plain_ms is None else
                  {"ms_per_step": round(plain_ms, 1), "value": round(world * nvis / (plain_ms * 1e-3) / 1e6, 3),
                   "what": "the same kernels, one facet per call (one launch per facet and direction)",
                   "batched_speedup": round(plain_ms / ms_step, 2)}),
        "facets_per_launch": fpl,
        "bda_map": bda_info,
        "differentiation": diff_info,
        "imaging_weights": dict(weights_info, frac_of_hbm=round(weights_info["achieved_GBs"] / _peaks()[0], 4)),
        "roofline": {
            "bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 5), "peak_kind": peak_kind,
            # DRAM bytes (read + write) of one 16-facet launch of the dominant kernel: 95.0 B per
            # visibility (grid) / 113 B (degrid), measured by ncu on the 0.05-scale workload and
            # scaled by visibilities
            "traffic": int((95.0 if dom == "grid" else 113.0) * nvis),
            "alg_bytes_per_launch": int(dom_bytes / launches_per_call),
            "fp32": {"achieved_tflops": round(flops_pass / (ms_step * 1e-3) / 1e12, 2),
                     "peak_tflops_nominal": round(fp32_peak, 1),
                     "frac": round(flops_pass / (ms_step * 1e-3) / 1e12 / fp32_peak, 4)},
        },
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3),
                "how": f"pinned host buffers, {E2E_CHUNKS} time chunks, copies overlapped with the kernels"},
        "gpu_launches": args.steps * 2 * launches_per_call,
        "clocks": clk.summary(),
        "setup_s": round(t_build, 1),
    }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and args.cpu_baseline and world == 1:
        mv, cores, sample = cpu_reference(F)
        out["cpu_baseline"] = {"value": round(mv, 4), "unit": UNIT, "cores": cores, "kind": "reference",
                               "sample": sample}
    if rank == 0:
        print(json.dumps(out), flush=True)


def nvis_w(w):
    return w.nrow * w.nchan


def run_uneven(args):
    """Uneven Voronoi facets with averaged BDA blocks (an additional workload, not the metric's
    configuration): one degrid + grid step over all facets, device-resident, CUDA-event timed."""
    import torch

    from ddfacet_b200 import configs, device as D

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    w = configs.uneven_bda(device=dev, scale=args.scale)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()

    def step():
        for f in w.facets_grid:
            f.grid.zero_()
        D.degrid(w.vs, w.facets_model, w.pol, w.jones)
        D.grid(w.vs, w.facets_grid, w.pol, w.jones)

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    info = dict(w.info)
    g = info.pop("grids")
    print(json.dumps({"metric": METRIC, "value": round(w.nvis / (ms * 1e-3) / 1e6, 3), "unit": UNIT,
                      "ms_per_step": round(ms, 1), "steps": args.steps, "warmup": max(1, args.warmup),
                      "config": {"workload": f"uneven BDA: {w.nfacets} Voronoi facets (grids {min(g)}..{max(g)}), "
                                             f"{w.nrow} rows x {w.nchan} ch x 4 corr ({w.nvis/1e6:.1f} Mvis), "
                                             f"{info['nblocks']} BDA blocks, per-vis Jones", **info,
                                 "scale": args.scale},
                      "setup_s": round(setup_s, 1)}), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (oracle/build_ref.sh)"}))
        return
    vals = []
    cores = sample = None
    for _ in range(max(1, args.steps)):
        mv, cores, sample = cpu_reference(81)
        vals.append(mv)
    v = float(np.median(vals))
    out = {"metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
           "steps": args.steps, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c64 grid / f64 internal", "data": "synthetic (seeded)",
           "config": {"workload": "multi-facet DDE (81 facets x 735^2, 232 Mvis x 4 corr, per-vis Jones), "
                                  "reference CPU gridder+degridder on a row sample"},
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
    ap.add_argument("--plain", action="store_true", help="also time the one-facet-per-launch direct path")
    ap.add_argument("--workload", default="multifacet_dde", choices=["multifacet_dde", "uneven_bda"],
                    help="uneven_bda: an additional workload (Voronoi facets, averaged blocks)")

    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "uneven_bda":
        run_uneven(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
