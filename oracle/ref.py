"""Driver of the reference's own compiled gridder/degridder (test infrastructure only).

Loads ``oracle/_ref/_pyGridderSmearPols3x*.so`` -- DDFacet/Gridder/GridderSmearPols.cc built
from source by ``oracle/build_ref.sh`` -- and calls ``pyGridderWPol32`` / ``pyDeGridderWPol``
with the positional argument lists ClassDDEGridMachine.put/get build
(DDFacet/Imager/ClassDDEGridMachine.py:809-831, 1084-1108).  Used as the parity checker by the
tests and as the timed CPU baseline by bench.py.
"""
from __future__ import annotations

import glob
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_mod = None
_sems = False


def available() -> bool:
    return bool(glob.glob(os.path.join(REF_DIR, "_pyGridderSmearPols3x*.so")))


def module():
    global _mod
    if _mod is None:
        paths = glob.glob(os.path.join(REF_DIR, "_pyGridderSmearPols3x*.so"))
        if not paths:
            raise RuntimeError("reference gridder not built: run oracle/build_ref.sh")
        spec = importlib.util.spec_from_file_location("_pyGridderSmearPols3x", paths[0])
        _mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_mod)
    return _mod


def set_semaphores(n=16):
    """The degridder locks row % N semaphores; N must be set before any degrid
    (ClassFacetMachine.py:160-169)."""
    global _sems
    if not _sems:
        names = ["/ddfg_oracle_%d_%d" % (os.getpid(), i) for i in range(n)]
        module().pySetSemaphores(names)
        _sems = True


def delete_semaphores():
    global _sems
    if _sems:
        module().pyDeleteSemaphore()
        _sems = False


def ljones_list(jones: dict, nrow, nchan, nband, gridder=True):
    """LJones (ClassDDEGridMachine.py:665-677, 772-776) from a plain dict, or [] without Jones.

    keys: kms, kms_tmap, kms_cmap, beam, beam_tmap, beam_cmap, A0, A1, idir_kms, idir_beam,
    coefs, interp_mode, mode (1 per vis / 2 per block), apply_amp, apply_phase, scale, calib_err,
    sumjones [2, nband] (out), sumjones_chan [2, nchan] (out)."""
    if not jones:
        return []
    e4 = np.array([], np.complex64).reshape((0, 0, 0, 0))
    ei = np.array([], np.int32)
    return [
        jones.get("kms", e4), jones.get("kms_tmap", ei), jones.get("beam", e4), jones.get("beam_tmap", ei),
        jones["A0"], jones["A1"],
        np.array([jones.get("idir_kms", 0)], np.int32), np.float32(jones.get("coefs", np.array([], np.float32))),
        np.array([jones.get("idir_beam", 0)], np.int32),
        np.array([jones.get("interp_mode", 0), jones.get("mode", 1)], np.int32),
        jones.get("kms_cmap", ei), jones.get("beam_cmap", ei), np.array([], np.float32).reshape((0, 0)),
        int(jones.get("apply_amp", 1)), int(jones.get("apply_phase", 1)), int(jones.get("scale", 0)),
        float(jones.get("calib_err", 0.0)),
        jones["sumjones"], jones["sumjones_chan"], np.float32(0.0),
    ]


def grid(grid, vis, uvw, flags, weights, sumwt, wplanes, wplanes_conj, winfos, incr, freqs, facet_infos, bda_map,
         chan_map, corr_ids, stokes_ids, ljones=(), lsmear=(), sparsification=None, dopsf=False, chan_equidistant=None):
    """pyGridderWPol32 (GridderSmearPols.cc:76-209): accumulates into ``grid`` and ``sumwt``."""
    if chan_equidistant is None:
        chan_equidistant = _chan_equidistant(freqs)
    module().pyGridderWPol32(
        grid, vis, uvw, flags, weights, sumwt, bool(dopsf), list(wplanes), list(wplanes_conj),
        np.asarray(winfos, np.float64), np.asarray(incr, np.float64), np.asarray(freqs, np.float64),
        [np.array([0, 5, 5, 0], np.int32), np.asarray(facet_infos, np.float64)], list(ljones), bda_map,
        sparsification if sparsification is not None else np.array([], dtype=bool),
        [2, int(chan_equidistant), 1, 0], list(lsmear), np.int32(chan_map),
        np.array(corr_ids).astype(np.uint16), np.array(stokes_ids).astype(np.uint16))


def degrid(grid, vis, uvw, flags, wplanes, wplanes_conj, winfos, incr, freqs, facet_infos, bda_map, chan_map,
           corr_ids, stokes_ids, ljones=(), lsmear=(), chan_equidistant=None):
    """pyDeGridderWPol (GridderSmearPols.cc:212-348): subtracts the prediction from ``vis``.
    Lcfs=WplanesConj, LcfsConj=Wplanes as ClassDDEGridMachine.get passes them (:1091-1092)."""
    set_semaphores()
    if chan_equidistant is None:
        chan_equidistant = _chan_equidistant(freqs)
    sumwt = np.zeros((grid.shape[0], grid.shape[1]), np.float64)
    row_infos = np.array([0, uvw.shape[0]], np.int32)
    return module().pyDeGridderWPol(
        grid, vis, uvw, flags, sumwt, 0, list(wplanes_conj), list(wplanes), np.asarray(winfos, np.float64),
        np.asarray(incr, np.float64), np.asarray(freqs, np.float64),
        [np.array([0, 5, 5, 0], np.int32), np.asarray(facet_infos, np.float64), row_infos], list(ljones), bda_map,
        np.array([], dtype=bool), [2, int(chan_equidistant), 1, 0], list(lsmear), np.int32(chan_map),
        np.array(corr_ids).astype(np.uint16), np.array(stokes_ids).astype(np.uint16))


def _chan_equidistant(freqs):
    freqs = np.asarray(freqs)
    if freqs.size > 1:
        df = freqs[1:] - freqs[:-1]
        return int(np.max(np.abs(df - np.mean(df))) < 1.)
    return 0
