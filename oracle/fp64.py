"""ctypes driver of the FP64 gridder/degridder restatement (test infrastructure only).

``grid(case, ...)`` and ``degrid(case, model, ...)`` run oracle/gridder_fp64.c on the same
inputs as the GPU path and the reference module, accumulating in complex128.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libddfg_fp64.so")
_lib = None

_vp = C.c_void_p


class JonesIn(C.Structure):
    _fields_ = [("mode", C.c_int), ("kms", _vp), ("kdims", C.c_int * 4), ("ktmap", _vp), ("kcmap", _vp),
                ("beam", _vp), ("bdims", C.c_int * 4), ("btmap", _vp), ("bcmap", _vp), ("a0", _vp), ("a1", _vp),
                ("idir_kms", C.c_int), ("idir_beam", C.c_int), ("coefs", _vp), ("interp_mode", C.c_int),
                ("apply_amp", C.c_int), ("apply_phase", C.c_int), ("scale", C.c_int), ("calib_err", C.c_double),
                ("wl_mean", C.c_double)]


class SmearIn(C.Structure):
    _fields_ = [("uvw_dt", _vp), ("dt", C.c_double), ("dnu", C.c_double), ("l", C.c_double), ("m", C.c_double),
                ("do_t", C.c_int), ("do_f", C.c_int)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["bash", os.path.join(HERE, "build_fp64.sh")], check=True)
        _lib = C.CDLL(LIB)
    return _lib


def _p(a):
    return C.c_void_p(None if a is None else a.ctypes.data)


def _pack_cf(wplanes, wconj, overs, degrid):
    first, second = (wconj, wplanes) if degrid else (wplanes, wconj)
    planes = list(first) + list(second)
    sizes = [p.size for p in planes]
    off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    data = np.concatenate([np.ascontiguousarray(p, np.complex64).ravel() for p in planes])
    sup = np.array([p.shape[0] // overs for p in planes], np.int32)
    return data, off, sup


def _jones(j, keep):
    ji = JonesIn()
    if not j:
        ji.mode = 0
        return ji
    ji.mode = int(j["mode"])
    for key, dims, tm, cm in (("kms", "kdims", "ktmap", "kcmap"), ("beam", "bdims", "btmap", "bcmap")):
        if key in j:
            arr = np.ascontiguousarray(j[key], np.complex64)
            keep.append(arr)
            setattr(ji, key, arr.ctypes.data)
            for i in range(4):
                getattr(ji, dims)[i] = arr.shape[i]
            t = np.ascontiguousarray(j[key + "_tmap"], np.int32)
            c = np.ascontiguousarray(j[key + "_cmap"], np.int32)
            keep += [t, c]
            setattr(ji, tm, t.ctypes.data)
            setattr(ji, cm, c.ctypes.data)
    a0 = np.ascontiguousarray(j["A0"], np.int32)
    a1 = np.ascontiguousarray(j["A1"], np.int32)
    keep += [a0, a1]
    ji.a0, ji.a1 = a0.ctypes.data, a1.ctypes.data
    ji.idir_kms, ji.idir_beam = int(j.get("idir_kms", 0)), int(j.get("idir_beam", 0))
    if "coefs" in j:
        co = np.ascontiguousarray(j["coefs"], np.float32)
        keep.append(co)
        ji.coefs = co.ctypes.data
    ji.interp_mode = int(j.get("interp_mode", 0))
    ji.apply_amp, ji.apply_phase, ji.scale = int(j.get("apply_amp", 1)), int(j.get("apply_phase", 1)), int(j.get("scale", 0))
    ji.calib_err = float(j.get("calib_err", 0.0))
    ji.wl_mean = float(j.get("wl_mean", 1.0))
    return ji


def _smear(s, keep):
    si = SmearIn()
    if s:
        dt = np.ascontiguousarray(s[0], np.float64)
        keep.append(dt)
        si.uvw_dt = dt.ctypes.data
        si.dt, si.dnu, si.do_t, si.do_f, si.l, si.m = float(s[1]), float(s[2]), int(s[3]), int(s[4]), float(s[5]), float(s[6])
    return si


def grid(vis, uvw, flags, weights, freqs, chan_map, bda_map, wplanes, wconj, overs, ref_wave, wmax, incr, cu, cv, lm,
         corr_ids, stokes_ids, nband, npix, jones=None, smear=None, dopsf=False, sparsification=None):
    """FP64 grid [nband, npol, npix, npix] complex128, sumwt, sumjones, sumjones_chan."""
    keep = []
    npol = len(stokes_ids)
    nrow, nchan, ncorr = vis.shape
    g = np.zeros((nband, npol, npix, npix), np.complex128)
    sumwt = np.zeros((nband, npol))
    sj = np.zeros((2, nband))
    sjc = np.zeros((2, nchan))
    cf, off, sup = _pack_cf(wplanes, wconj, overs, degrid=False)
    arrs = [np.ascontiguousarray(vis, np.complex64), np.ascontiguousarray(uvw, np.float64),
            np.ascontiguousarray(flags).view(np.uint8) if flags.dtype == bool else np.ascontiguousarray(flags, np.uint8),
            np.ascontiguousarray(weights, np.float32), np.ascontiguousarray(freqs, np.float64),
            np.ascontiguousarray(chan_map, np.int32), np.ascontiguousarray(bda_map, np.int32),
            np.array(corr_ids, np.int32), np.array(stokes_ids, np.int32)]
    sp = None if sparsification is None else np.ascontiguousarray(sparsification, np.uint8)
    if jones:
        jones = dict(jones, wl_mean=float(np.mean(299792458.0 / np.asarray(freqs))))
    ji, si = _jones(jones, keep), _smear(smear, keep)
    f = lib().fp64_grid
    f.restype = C.c_int
    rc = f(_p(g), nband, npol, npix, npix, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]), _p(arrs[3]), C.c_int64(nrow), nchan,
           ncorr, _p(arrs[4]), _p(arrs[5]), _p(arrs[6]), _p(cf), _p(off), _p(sup), len(wplanes), int(overs),
           C.c_double(ref_wave), C.c_double(wmax), C.c_double(incr[0]), C.c_double(incr[1]), C.c_double(cu),
           C.c_double(cv), C.c_double(lm[0]), C.c_double(lm[1]), _p(arrs[7]), len(corr_ids), _p(arrs[8]),
           len(stokes_ids), int(bool(dopsf)), C.byref(ji), C.byref(si), _p(sp), _p(sumwt), _p(sj), _p(sjc))
    if rc:
        raise ValueError("unsupported correlation/Stokes combination")
    return g, sumwt, sj, sjc


def degrid(model, vis0, uvw, freqs, chan_map, bda_map, wplanes, wconj, overs, ref_wave, wmax, incr, cu, cv, lm, corr_ids,
           stokes_ids, jones=None, smear=None):
    """vis0 - prediction, complex128 [nrow, nchan, ncorr]."""
    keep = []
    nband, npol, ny, nx = model.shape
    nrow, nchan, ncorr = vis0.shape
    v = np.ascontiguousarray(vis0, np.complex128).copy()
    cf, off, sup = _pack_cf(wplanes, wconj, overs, degrid=True)
    m = np.ascontiguousarray(model, np.complex64)
    arrs = [np.ascontiguousarray(uvw, np.float64), np.ascontiguousarray(freqs, np.float64),
            np.ascontiguousarray(chan_map, np.int32), np.ascontiguousarray(bda_map, np.int32),
            np.array(corr_ids, np.int32), np.array(stokes_ids, np.int32)]
    if jones:
        jones = dict(jones, wl_mean=float(np.mean(299792458.0 / np.asarray(freqs))))
    ji, si = _jones(jones, keep), _smear(smear, keep)
    f = lib().fp64_degrid
    f.restype = C.c_int
    rc = f(_p(m), nband, npol, ny, nx, _p(v), _p(arrs[0]), C.c_int64(nrow), nchan, ncorr, _p(arrs[1]), _p(arrs[2]),
           _p(arrs[3]), _p(cf), _p(off), _p(sup), len(wplanes), int(overs), C.c_double(ref_wave), C.c_double(wmax),
           C.c_double(incr[0]), C.c_double(incr[1]), C.c_double(cu), C.c_double(cv), C.c_double(lm[0]),
           C.c_double(lm[1]), _p(arrs[4]), len(corr_ids), _p(arrs[5]), len(stokes_ids), C.byref(ji), C.byref(si))
    if rc:
        raise ValueError("unsupported correlation/Stokes combination")
    return v


def block_indices(uvw, flags, freqs, chan_map, bda_map, wplanes, wconj, overs, ref_wave, wmax, incr, cu, cv, nband,
                  npix, degrid=False):
    """int32 [nblocks, 8] = (status, iw, plane, locx, locy, offx, offy, k) of every block, from the
    gridder's (flag-aware) or the degridder's block means: the integer indices of gridder.h:321-351
    restated in FP64 C, for a word-by-word comparison with ddfg_block_geometry."""
    nrow, nchan, ncorr = flags.shape
    cf, off, sup = _pack_cf(wplanes, wconj, overs, degrid=degrid)
    bm = np.ascontiguousarray(bda_map, np.int32)
    nb = int(np.uint32(bm[0])) + (int(bm[1]) << 32)
    out = np.full((max(nb, 1), 8), -1, np.int32)
    fl = np.ascontiguousarray(flags).view(np.uint8) if flags.dtype == bool else np.ascontiguousarray(flags, np.uint8)
    arrs = [np.ascontiguousarray(uvw, np.float64), fl, np.ascontiguousarray(freqs, np.float64),
            np.ascontiguousarray(chan_map, np.int32)]
    f = lib().fp64_block_indices
    f.restype = C.c_int
    f(_p(arrs[0]), _p(arrs[1]), nchan, ncorr, _p(arrs[2]), _p(arrs[3]), _p(bm), _p(off), _p(sup), len(wplanes),
      int(overs), C.c_double(ref_wave), C.c_double(wmax), int(npix), int(npix), int(nband), C.c_double(incr[0]),
      C.c_double(incr[1]), C.c_double(cu), C.c_double(cv), int(bool(degrid)), _p(out))
    return out[:nb]


def predict_np(bda_map, uvw, freqs, chan_map, a0, a1, facets, kms=None, kms_tmap=None, kms_cmap=None,
               only=None, beam=None, beam_tmap=None, beam_cmap=None, coefs=None, apply_amp=True, apply_phase=True,
               scale=False, calib_err=0.0, wavelength_mean=1.0):
    """Per-facet FP64 predictions P_f (complex128 [nrow][nchan][4]) of the differentiable prediction
    P = sum_f J0 (s_f I) J1^H exp(+2 pi i nu (u l0 + v m0 + w (n0 - 1)) / c), s_f the degridder's tap
    sum sum CF G_f at each block's footprint (Stokes I from four linear correlations, XX = YY = I;
    kMS Jones at the facet's direction per visibility, no normalisation; no smearing), in numpy
    float64 with complex128 grids and Jones -- so finite differences can take steps float32 cannot
    hold.  The integer footprints come from block_indices (the FP64 restatement of
    degridder.h:138-200).  facets: dicts with grid (complex [1][1][N][N]), wplanes, wconj, overs,
    ref_wave, wmax, incr, cu, cv, l0, m0, idir (and idir_beam with a beam).  ``only``: indices of
    the facets to evaluate.  With ``beam`` each antenna's Jones is J = K B (JonesServer.cc:276-289);
    with interpolation ``coefs`` (mode 1) every matrix is scaled by (sum of coefs)^2, which is what
    the reference's GiveJones loop (JonesServer.cc:71-93) returns for the facet's direction; without
    ``apply_amp`` / ``apply_phase`` the kMS elements are normalised as NormJones does
    (JonesServer.cc:25-52): z / |z| (phase only), |z| (amplitude only); with ``scale`` each is
    then scaled by (1 - alpha)/|z| + alpha, alpha = exp(-2 pi calib_err^2 (u^2 + v^2) /
    wavelength_mean^2) at the uv of the visibility where the reference's Jones cache last
    recomputed the kMS terms (per block, rows then channels: the first visibility of each run of
    equal time slot, antennas and Jones channel)."""
    bm = np.ascontiguousarray(bda_map, np.int32)
    nb = int(np.uint32(bm[0])) + (int(bm[1]) << 32)
    sizes = bm[2:2 + nb].astype(np.int64)
    starts = 2 + nb + np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    nrow = uvw.shape[0]
    nchan = len(freqs)
    # visibilities of every block: (block, row, channel)
    vb, vr, vc = [], [], []
    for b in range(nb):
        s = starts[b]
        c0, c1 = int(bm[s]), int(bm[s + 1])
        rows = bm[s + 2:s + sizes[b]]
        rr, cc = np.meshgrid(rows, np.arange(c0, c1), indexing="ij")
        vb.append(np.full(rr.size, b))
        vr.append(rr.ravel())
        vc.append(cc.ravel())
    vb, vr, vc = np.concatenate(vb), np.concatenate(vr).astype(np.int64), np.concatenate(vc).astype(np.int64)
    flags = np.zeros((nrow, nchan, 4), np.uint8)
    k_nu = np.asarray(freqs, np.float64) / 299792458.0
    out = []
    for fi, f in enumerate(facets):
        if only is not None and fi not in only:
            out.append(None)
            continue
        G = np.asarray(f["grid"], np.complex128)[0, 0]
        N = G.shape[-1]
        idx = block_indices(uvw, flags, freqs, chan_map, bm, f["wplanes"], f["wconj"], f["overs"], f["ref_wave"],
                            f["wmax"], f["incr"], f["cu"], f["cv"], 1, N, degrid=True)
        planes = list(f["wconj"]) + list(f["wplanes"])   # the degridder's table order
        O = int(f["overs"])
        sblk = np.zeros(nb, np.complex128)
        ok = idx[:, 0] == 1
        for p in np.unique(idx[ok, 2]):
            sel = np.flatnonzero(ok & (idx[:, 2] == p))
            S = planes[p].shape[0] // O
            sup = (S - 1) // 2
            sub = np.asarray(planes[p], np.complex128).reshape(O * O, S, S)[idx[sel, 7]]
            ry = idx[sel, 4][:, None] - sup + np.arange(S)[None, :]
            rx = idx[sel, 3][:, None] - sup + np.arange(S)[None, :]
            win = G[ry[:, :, None], rx[:, None, :]]
            sblk[sel] = np.sum(sub * win, axis=(1, 2))
        s = sblk[vb]
        n0m1 = np.sqrt(1.0 - f["l0"] ** 2 - f["m0"] ** 2) - 1.0
        u = uvw[vr]
        ph = np.exp(2j * np.pi * k_nu[vc] * (u[:, 0] * f["l0"] + u[:, 1] * f["m0"] + u[:, 2] * n0m1))
        P = np.zeros((nrow, nchan, 4), np.complex128)
        if kms is not None:
            kf = 1.0 if coefs is None else float(np.sum(np.asarray(coefs, np.float64))) ** 2
            J = np.asarray(kms, np.complex128)
            t, ch = np.asarray(kms_tmap)[vr], np.asarray(kms_cmap)[vc]
            J0 = kf * J[t, f["idir"], np.asarray(a0)[vr], ch].reshape(-1, 2, 2)
            J1 = kf * J[t, f["idir"], np.asarray(a1)[vr], ch].reshape(-1, 2, 2)
            if scale:
                key = np.stack([t, np.asarray(a0)[vr], np.asarray(a1)[vr], ch, vb], axis=1)
                start = np.ones(vr.size, bool)
                start[1:] = np.any(key[1:] != key[:-1], axis=1)
                first = np.maximum.accumulate(np.where(start, np.arange(vr.size), 0))
                uk = uvw[vr[first]]
                r2 = (uk[:, 0] ** 2 + uk[:, 1] ** 2) / wavelength_mean ** 2
                alpha = np.exp(-2 * np.pi * calib_err ** 2 * r2)[:, None, None]
            for K in (J0, J1):
                if not apply_amp:
                    a = np.abs(K)
                    K[a != 0] /= a[a != 0]
                if not apply_phase:
                    K[...] = np.abs(K)
                if scale:
                    a = np.abs(K)
                    fac = np.where(a != 0, (1 - alpha) / np.where(a != 0, a, 1) + alpha, 1.0)
                    K[...] = K * fac
            if beam is not None:
                B = np.asarray(beam, np.complex128)
                tb, cb, db = np.asarray(beam_tmap)[vr], np.asarray(beam_cmap)[vc], f.get("idir_beam", 0)
                J0 = J0 @ (kf * B[tb, db, np.asarray(a0)[vr], cb].reshape(-1, 2, 2))
                J1 = J1 @ (kf * B[tb, db, np.asarray(a1)[vr], cb].reshape(-1, 2, 2))
            M = np.einsum("nij,nkj->nik", J0, np.conj(J1))             # J0 J1^H
        else:
            M = np.broadcast_to(np.eye(2, dtype=np.complex128), (vr.size, 2, 2))
        P[vr, vc, :] = (M.reshape(-1, 4) * (s * ph)[:, None])
        out.append(P)
    return out
