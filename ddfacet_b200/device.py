"""Device-resident inputs of the gridder/degridder and the calls through the C ABI.

PyTorch tensors own all device memory (plumbing only); the work is done by libddfg.so.

* ``VisData``   -- visibilities, uvw, flags, weights, frequencies, channel map, the BDA block
                   map and its plan (block starts), optional smearing inputs.
* ``CFTables``  -- one facet's W-projection planes packed in one complex64 buffer, with the
                   plane offsets in the order the gridder wants them (Wplanes first) and in the
                   order the degridder wants them (WplanesConj first), mirroring
                   ClassDDEGridMachine.put/get (ClassDDEGridMachine.py:830-831, 1091-1092).
* ``FacetGrid`` -- a facet's grid tensor, geometry and float64 output sums.
* ``JonesData`` -- LJones as device tensors (ClassDDEGridMachine.py:571-679).
* ``grid`` / ``degrid`` -- one ABI call over any number of facets.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, replace
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _abi

C_LIGHT = 299792458.0


def _dev(device=None):
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return torch.device(device)


def to_device(x, dtype, device, copy_ok=True, non_blocking=False):
    """numpy / torch -> contiguous device tensor of ``dtype`` (no copy if already right)."""
    if isinstance(x, torch.Tensor):
        t = x
        if t.dtype != dtype:
            t = t.to(dtype)
        if t.device != device:
            t = t.to(device, non_blocking=non_blocking)
        return t.contiguous()
    a = np.ascontiguousarray(x)
    t = torch.from_numpy(a)
    if t.dtype != dtype:
        t = t.to(dtype)
    return t.to(device, non_blocking=non_blocking).contiguous()


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


@dataclass
class VisData:
    vis: torch.Tensor            # complex64 [nrow, nchan, ncorr]
    uvw: torch.Tensor            # float64 [nrow, 3]
    flags: torch.Tensor          # uint8 [nrow, nchan, ncorr]
    weights: torch.Tensor        # float32 [nrow, nchan]
    freqs: torch.Tensor          # float64 [nchan]
    freqs_host: np.ndarray
    recip_wvl: torch.Tensor      # float64 [nchan] freqs / c (the IEEE quotient the reference forms)
    chan_map: torch.Tensor       # int32 [nchan]
    bda_map: torch.Tensor        # int32
    block_start: torch.Tensor    # int64 [nblocks]
    nblocks: int
    chan_equidistant: int
    single_vis_blocks: int = 0
    sparsification: Optional[torch.Tensor] = None
    uvw_dt: Optional[torch.Tensor] = None
    dt: float = 0.0
    dnu: float = 0.0
    do_tsmear: int = 0
    do_fsmear: int = 0
    large_blocks: Optional[torch.Tensor] = None   # int64 [nlarge] (with_large_blocks)
    large_min_vis: int = 0

    @staticmethod
    def plan_map(bda_map: torch.Tensor, nrow: int, nchan: int, stream=None):
        """(block starts, every-block-single-visibility flag) of a packed BDA map (checked);
        see ddfg_bda_plan."""
        lib = _abi.lib()
        m = bda_map
        lo, hi = (int(x) for x in m[:2].cpu().numpy().view(np.uint32)) if m.is_cuda else (int(np.uint32(m[0])), int(m[1]))
        nb = lo + (hi << 32)
        starts = torch.empty(max(nb, 1), dtype=torch.int64, device=m.device)
        ws = torch.empty(int(lib.ddfg_bda_plan_workspace_size(nb)), dtype=torch.uint8, device=m.device)
        single = C.c_int32(0)
        _abi.check(lib.ddfg_bda_plan(m.data_ptr(), m.numel(), nb, nrow, nchan, starts.data_ptr(), ws.data_ptr(),
                                     ws.numel(), _stream_ptr(stream), C.byref(single)))
        return (starts[:nb] if nb > 0 else starts[:0]), int(single.value)

    @classmethod
    def create(cls, vis, uvw, flags, weights, freqs, chan_map, bda_map, device=None, sparsification=None,
               smear=None, block_start=None, non_blocking=False):
        device = _dev(device)
        freqs_host = np.asarray(freqs.cpu().numpy() if isinstance(freqs, torch.Tensor) else freqs, np.float64)
        if freqs_host.size > 1:
            df = freqs_host[1:] - freqs_host[:-1]
            cheq = int(np.max(np.abs(df - np.mean(df))) < 1.)
        else:
            cheq = 0
        v = to_device(vis, torch.complex64, device, non_blocking=non_blocking)
        if v.dim() != 3:
            raise NameError("vis has to be [nrow, nchan, ncorr]")
        nrow, nchan, ncorr = v.shape
        f = flags
        if isinstance(f, np.ndarray):
            f = f.view(np.uint8) if f.dtype == np.bool_ else f.astype(np.uint8)
        elif isinstance(f, torch.Tensor) and f.dtype == torch.bool:
            f = f.view(torch.uint8)
        fl = to_device(f, torch.uint8, device, non_blocking=non_blocking)
        bm = to_device(bda_map, torch.int32, device, non_blocking=non_blocking)
        single = 0
        if block_start is None:
            block_start, single = cls.plan_map(bm, nrow, nchan)
        nb = int(block_start.numel())
        sp = None
        if sparsification is not None and np.size(sparsification) > 0:
            sp_np = np.asarray(sparsification)
            if sp_np.size != nb:
                raise ValueError("sparsification argument must be an array of length NTotBlocks")
            sp = to_device(sp_np.astype(np.uint8), torch.uint8, device)
        out = cls(
            vis=v,
            uvw=to_device(uvw, torch.float64, device, non_blocking=non_blocking),
            flags=fl,
            weights=to_device(weights, torch.float32, device, non_blocking=non_blocking),
            freqs=to_device(freqs_host, torch.float64, device),
            freqs_host=freqs_host,
            recip_wvl=to_device(freqs_host / C_LIGHT, torch.float64, device),
            chan_map=to_device(np.asarray(chan_map, np.int32) if not isinstance(chan_map, torch.Tensor) else chan_map,
                               torch.int32, device),
            bda_map=bm,
            block_start=block_start,
            nblocks=nb,
            chan_equidistant=cheq,
            single_vis_blocks=single,
            sparsification=sp,
        )
        if smear is not None and len(smear) > 0:
            uvw_dt, dt, dnu, do_t, do_f = smear[:5]
            out.uvw_dt = to_device(uvw_dt, torch.float64, device)
            out.dt, out.dnu, out.do_tsmear, out.do_fsmear = float(dt), float(dnu), int(do_t), int(do_f)
        return out

    def with_block_order(self, order: torch.Tensor) -> "VisData":
        """The same visibilities with the map's blocks visited in ``order`` (a permutation of block
        indices, e.g. ``bda.uv_locality_order``): the map is rewritten by ``bda.reorder_blocks``
        and planned again, and a sparsification mask is permuted with the blocks.  The degridder's
        output changes only by the order of its tap sums, the gridder's by the order of its grid
        sums."""
        from . import bda

        m = bda.reorder_blocks(self.bda_map, self.block_start, order)
        starts, single = self.plan_map(m, int(self.vis.shape[0]), int(self.vis.shape[1]))
        sp = None if self.sparsification is None else self.sparsification[order].contiguous()
        out = replace(self, bda_map=m, block_start=starts, single_vis_blocks=single, sparsification=sp,
                      large_blocks=None, large_min_vis=0)
        return out.with_large_blocks(self.large_min_vis) if self.large_blocks is not None else out

    def with_large_blocks(self, min_vis: int = 128) -> "VisData":
        """The same visibilities with the list of blocks of more than ``min_vis`` visibilities
        (rows x channels) that the averaged-block kernels give a whole warp each (ddfg_vis
        large_blocks).  Mode-1 maps give the shortest baselines blocks spanning the whole track;
        one lane per block would hold its warp for the whole walk.  Needs Jones terms that do
        not depend on uv (no scale_jones)."""
        if min_vis < 1:
            raise ValueError("min_vis must be positive")
        nb = self.nblocks
        if nb == 0 or self.single_vis_blocks:
            return replace(self, large_blocks=None, large_min_vis=0)
        sizes = self.bda_map[2:2 + nb].to(torch.int64) - 2
        st = self.block_start
        nv = sizes * (self.bda_map[st + 1].to(torch.int64) - self.bda_map[st].to(torch.int64))
        idx = torch.nonzero(nv > int(min_vis)).flatten().contiguous()
        out = replace(self, large_blocks=idx if idx.numel() else None, large_min_vis=int(min_vis))
        if out.vis.is_cuda:
            out.check_large_blocks()
        return out

    def check_large_blocks(self, stream=None):
        """Validates the large-block list on the device (ddfg_check_large_blocks): raises if an entry
        is not a block index, is listed twice or is not above the threshold, or if a block above
        the threshold is missing."""
        if self.large_blocks is None or self.large_blocks.numel() == 0:
            return
        lib = _abi.lib()
        ws = torch.empty(int(lib.ddfg_check_large_blocks_workspace_size(self.nblocks)), dtype=torch.uint8,
                         device=self.vis.device)
        vss = self.struct()
        _abi.check(lib.ddfg_check_large_blocks(C.byref(vss), ws.data_ptr(), ws.numel(), _stream_ptr(stream)))

    def struct(self) -> _abi.VisSet:
        s = _abi.VisSet()
        nrow, nchan, ncorr = self.vis.shape
        s.vis = self.vis.data_ptr()
        s.uvw = self.uvw.data_ptr()
        s.flags = self.flags.data_ptr()
        s.weights = self.weights.data_ptr()
        s.freqs = self.freqs.data_ptr()
        s.freq_mean = float(np.mean(self.freqs_host)) if self.freqs_host.size else 0.0
        s.recip_wvl = self.recip_wvl.data_ptr()
        s.chan_map = self.chan_map.data_ptr()
        s.nrow, s.nchan, s.ncorr = nrow, nchan, ncorr
        s.chan_equidistant = self.chan_equidistant
        s.single_vis_blocks = int(self.single_vis_blocks)
        s.bda_map = self.bda_map.data_ptr()
        s.bda_len = self.bda_map.numel()
        s.block_start = self.block_start.data_ptr() if self.nblocks > 0 else None
        s.nblocks = self.nblocks
        s.sparsification = _ptr(self.sparsification)
        s.uvw_dt = _ptr(self.uvw_dt)
        s.dt, s.dnu = self.dt, self.dnu
        s.do_tsmear, s.do_fsmear = self.do_tsmear, self.do_fsmear
        if self.large_blocks is not None and self.large_blocks.numel() > 0:
            s.large_blocks = self.large_blocks.data_ptr()
            s.nlarge = int(self.large_blocks.numel())
            s.large_min_vis = int(self.large_min_vis)
        return s


@dataclass
class CFTables:
    data: torch.Tensor           # complex64 packed planes (Wplanes then WplanesConj)
    off_grid: torch.Tensor       # int64 [2*nw]: Wplanes offsets then WplanesConj offsets
    off_degrid: torch.Tensor     # int64 [2*nw]: WplanesConj offsets then Wplanes offsets
    sup: torch.Tensor            # int32 [2*nw]
    nw: int
    overs: int
    ref_wave: float
    wmax: float
    max_support: int = 0

    @classmethod
    def create(cls, wplanes: Sequence[np.ndarray], wplanes_conj: Sequence[np.ndarray], overs: int, ref_wave: float,
               wmax: float, device=None):
        device = _dev(device)
        nw = len(wplanes)
        planes = list(wplanes) + list(wplanes_conj)
        sizes = [int(p.size) for p in planes]
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        packed = np.concatenate([np.ascontiguousarray(p, np.complex64).ravel() for p in planes])
        sup = np.array([p.shape[0] // overs for p in planes], np.int32)
        off_d = np.concatenate([offs[nw:], offs[:nw]])
        sup_d = np.concatenate([sup[nw:], sup[:nw]])
        if not np.array_equal(sup_d, sup):
            raise ValueError("W planes and their conjugates must have the same supports")
        return cls(data=to_device(packed, torch.complex64, device), off_grid=to_device(offs, torch.int64, device),
                   off_degrid=to_device(off_d, torch.int64, device), sup=to_device(sup, torch.int32, device), nw=nw,
                   overs=int(overs), ref_wave=float(ref_wave), wmax=float(wmax), max_support=int(sup.max()))


@dataclass
class FacetGrid:
    grid: torch.Tensor           # complex64 [nband, npol, ny, nx]
    cf: CFTables
    incr: tuple                  # (incr_x, incr_y) radians
    cu: float
    cv: float
    l0: float
    m0: float
    idir_kms: int = 0
    idir_beam: int = 0
    decorr_lm: tuple = (0.0, 0.0)
    sumwt: Optional[torch.Tensor] = None        # float64 [nband, npol]
    sumjones: Optional[torch.Tensor] = None     # float64 [2, nband]
    sumjones_chan: Optional[torch.Tensor] = None  # float64 [2, nchan]
    grid_acc: Optional[torch.Tensor] = None     # complex128 like grid: FP64 accumulation (all zero)

    def with_fp64_accumulation(self) -> "FacetGrid":
        """This facet with an FP64 accumulator (ddfg_facet.grid_acc): gridding adds every tap
        product into it with FP64 atomics and, at the end of each call, adds it into the float32
        grid (one rounding per cell) and zeroes it, so each call adds the correctly rounded sum of
        its contributions.  The atomics do not return a value, so the call costs little more than
        with float32 sums (10-16 % on the combined at-scale chunk, more when the accumulators of a
        pack overflow L2 badly), and the accumulator takes twice the grid's memory."""
        if self.grid_acc is None:
            self.grid_acc = torch.zeros(self.grid.shape, dtype=torch.complex128, device=self.grid.device)
        return self

    def struct(self, degrid=False) -> _abi.Facet:
        s = _abi.Facet()
        nband, npol, ny, nx = self.grid.shape
        s.grid = self.grid.data_ptr()
        s.nband, s.npol, s.ny, s.nx = nband, npol, ny, nx
        s.incr_x, s.incr_y = float(self.incr[0]), float(self.incr[1])
        s.cu, s.cv, s.l0, s.m0 = float(self.cu), float(self.cv), float(self.l0), float(self.m0)
        s.cf_data = self.cf.data.data_ptr()
        s.cf_offset = (self.cf.off_degrid if degrid else self.cf.off_grid).data_ptr()
        s.cf_support = self.cf.sup.data_ptr()
        s.nw, s.overs = self.cf.nw, self.cf.overs
        s.max_support = int(self.cf.max_support)
        s.ref_wave, s.wmax = self.cf.ref_wave, self.cf.wmax
        s.idir_kms, s.idir_beam = int(self.idir_kms), int(self.idir_beam)
        s.decorr_l, s.decorr_m = float(self.decorr_lm[0]), float(self.decorr_lm[1])
        s.sumwt = _ptr(self.sumwt)
        s.sumjones = _ptr(self.sumjones)
        s.sumjones_chan = _ptr(self.sumjones_chan)
        s.grid_acc = None if degrid else _ptr(self.grid_acc)
        return s


@dataclass
class JonesData:
    mode: int = 0
    kms: Optional[torch.Tensor] = None
    kms_tmap: Optional[torch.Tensor] = None
    kms_cmap: Optional[torch.Tensor] = None
    beam: Optional[torch.Tensor] = None
    beam_tmap: Optional[torch.Tensor] = None
    beam_cmap: Optional[torch.Tensor] = None
    a0: Optional[torch.Tensor] = None
    a1: Optional[torch.Tensor] = None
    interp_coefs: Optional[torch.Tensor] = None
    interp_mode: int = 0
    apply_amp: int = 1
    apply_phase: int = 1
    scale_jones: int = 0
    calib_error: float = 0.0
    wavelength_mean: float = 1.0

    def struct(self) -> _abi.Jones:
        s = _abi.Jones()
        s.mode = int(self.mode)
        if self.kms is not None:
            s.kms = self.kms.data_ptr()
            for i in range(4):
                s.kms_dims[i] = int(self.kms.shape[i])
            s.kms_tmap, s.kms_cmap = _ptr(self.kms_tmap), _ptr(self.kms_cmap)
        if self.beam is not None:
            s.beam = self.beam.data_ptr()
            for i in range(4):
                s.beam_dims[i] = int(self.beam.shape[i])
            s.beam_tmap, s.beam_cmap = _ptr(self.beam_tmap), _ptr(self.beam_cmap)
        s.a0, s.a1 = _ptr(self.a0), _ptr(self.a1)
        s.interp_coefs = _ptr(self.interp_coefs)
        s.interp_mode = int(self.interp_mode)
        s.apply_amp, s.apply_phase, s.scale_jones = int(self.apply_amp), int(self.apply_phase), int(self.scale_jones)
        s.calib_error = float(self.calib_error)
        s.wavelength_mean = float(self.wavelength_mean)
        return s


def make_pol(corr_ids, stokes_ids) -> _abi.Pol:
    p = _abi.Pol()
    corr_ids = [int(c) for c in corr_ids]
    stokes_ids = [int(s) for s in stokes_ids]
    if len(corr_ids) > 4 or len(stokes_ids) > 4:
        raise ValueError("at most 4 correlations and 4 Stokes parameters")
    p.ncorr, p.npol = len(corr_ids), len(stokes_ids)
    for i, c in enumerate(corr_ids):
        p.corr_ids[i] = c
    for i, s in enumerate(stokes_ids):
        p.stokes_ids[i] = s
    return p


@dataclass
class Batch:
    """Scheduling of the batched (persistent, queue-driven) calls and their workspace
    (ddfg_batch): facets per pack, stripes per queue item, resident CTAs per SM (0 = library
    default); ``static`` replaces the queue by a fixed item order (for measurements), ``tiles``
    has the gridder's warps sum each stripe in a shared-memory tile before adding it to the grid,
    and ``spread`` interleaves the items over one contiguous region of the block order per CTA
    (concurrent CTAs work on distant parts of a uv-ordered map)."""
    workspace: torch.Tensor
    facets_per_pack: int = 0
    stripes_per_item: int = 0
    ctas_per_sm: int = 0
    static: bool = False
    tiles: bool = False
    spread: bool = False

    @classmethod
    def create(cls, device=None, **kw) -> "Batch":
        lib = _abi.lib()
        ws = torch.zeros(int(lib.ddfg_batch_workspace_size()), dtype=torch.uint8, device=_dev(device))
        return cls(workspace=ws, **kw)

    def struct(self) -> _abi.Batch:
        b = _abi.Batch()
        b.workspace = self.workspace.data_ptr()
        b.workspace_bytes = self.workspace.numel()
        b.facets_per_pack = int(self.facets_per_pack)
        b.stripes_per_item = int(self.stripes_per_item)
        b.ctas_per_sm = int(self.ctas_per_sm)
        b.flags = (1 if self.static else 0) | (2 if self.tiles else 0) | (4 if self.spread else 0)
        return b

    def describe(self) -> dict:
        return {"facets_per_pack": int(self.facets_per_pack), "stripes_per_item": int(self.stripes_per_item),
                "ctas_per_sm": int(self.ctas_per_sm), "queue": not self.static, "tiles": bool(self.tiles),
                "spread": bool(self.spread)}


def grid(vs: VisData, facets: List[FacetGrid], pol: _abi.Pol, jones: Optional[JonesData] = None, dopsf=False,
         stream=None, batch: Optional[Batch] = None):
    """Grid ``vs`` onto every facet: ddfg_grid, or ddfg_grid_batched with a ``batch``."""
    lib = _abi.lib()
    arr = (_abi.Facet * max(1, len(facets)))(*[f.struct(degrid=False) for f in facets])
    js = (jones or JonesData()).struct()
    vss = vs.struct()
    if batch is None:
        _abi.check(lib.ddfg_grid(C.byref(vss), C.byref(js), C.byref(pol), arr, len(facets), int(bool(dopsf)),
                                 _stream_ptr(stream)))
    else:
        bs = batch.struct()
        _abi.check(lib.ddfg_grid_batched(C.byref(vss), C.byref(js), C.byref(pol), arr, len(facets),
                                         int(bool(dopsf)), C.byref(bs), _stream_ptr(stream)))


def degrid(vs: VisData, facets: List[FacetGrid], pol: _abi.Pol, jones: Optional[JonesData] = None, stream=None,
           batch: Optional[Batch] = None):
    """Subtract every facet's prediction from ``vs.vis``: ddfg_degrid, or ddfg_degrid_batched with
    a ``batch``."""
    lib = _abi.lib()
    arr = (_abi.Facet * max(1, len(facets)))(*[f.struct(degrid=True) for f in facets])
    js = (jones or JonesData()).struct()
    vss = vs.struct()
    if batch is None:
        _abi.check(lib.ddfg_degrid(C.byref(vss), C.byref(js), C.byref(pol), arr, len(facets), _stream_ptr(stream)))
    else:
        bs = batch.struct()
        _abi.check(lib.ddfg_degrid_batched(C.byref(vss), C.byref(js), C.byref(pol), arr, len(facets), C.byref(bs),
                                           _stream_ptr(stream)))


def block_geometry(vs: VisData, facet: FacetGrid, degrid=False, stream=None) -> torch.Tensor:
    """int32 [nblocks, 8] = (status, iw, plane, locx, locy, offx, offy, k) of every block on
    ``facet`` as the gridder (or, with ``degrid``, the degridder) computes them
    (ddfg_block_geometry)."""
    lib = _abi.lib()
    out = torch.full((max(vs.nblocks, 1), 8), -1, dtype=torch.int32, device=vs.vis.device)
    vss = vs.struct()
    fs = facet.struct(degrid=degrid)
    _abi.check(lib.ddfg_block_geometry(C.byref(vss), C.byref(fs), int(bool(degrid)), out.data_ptr(),
                                       _stream_ptr(stream)))
    return out[:vs.nblocks]


def capture_graph(fn, warmup: int = 1):
    """Record ``fn()`` -- a sequence of library calls on the current stream, such as a
    degrid-then-grid step -- into a CUDA graph and return it (``g.replay()`` reruns it).  The
    library's grid / degrid / FFT calls allocate nothing and never synchronise, so they capture
    as they are; ``fn`` is run ``warmup`` times first on a side stream (this sets the kernels'
    shared-memory attributes and loads the kernels before capture)."""
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(warmup):
            fn()
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g
