"""Imaging weights (natural / uniform / Briggs) on the GPU.

Mirrors the weight pipeline of DDFacet's visibility server (DDFacet/Data/ClassVisServer.py:
``_loadWeights_handler`` :930-975, ``_CalcWeights_serial`` :857-913, ``_uv_to_index`` :981-1003,
``_accumulateWeights_handler`` :1005-1023, ``_finalizeWeights_handler`` :1025-1062): the uv extent
of the unflagged data sizes a float64 uv-density grid, every chunk's weights are accumulated onto
it, Briggs weighting transforms it, and every chunk's weights are divided by their cell's density.
The per-visibility passes run in libddfg.so (``ddfg_weights_*``).

    iw = ImagingWeights(chunks_uvmax, cell_rad, npix_image, mode="briggs", robust=0.0,
                        nbands=1, super_uniform=1.0)
    for chunk in chunks: iw.accumulate(uvw, freqs, weights, band_of_chan)
    iw.finish()
    for chunk in chunks: w_img = iw.apply(uvw, freqs, weights, band_of_chan)
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np
import torch

from . import _abi, device as D

C_LIGHT = 299792458.0


def uvmax_wavelengths(uvw: torch.Tensor, rowflags: Optional[torch.Tensor], freqs) -> float:
    """max |u|, |v| of the unflagged rows, in wavelengths at the highest frequency
    (ClassVisServer.py:947-951)."""
    uv = uvw[:, :2]
    if rowflags is not None:
        uv = uv[~rowflags]
    return float(uv.abs().max().item()) * float(np.max(np.asarray(freqs))) / C_LIGHT


class ImagingWeights:
    def __init__(self, uvmax: float, cell_rad: float, npix_image: int, mode: str = "briggs", robust: float = 0.0,
                 nbands: int = 1, super_uniform: float = 1.0, device=None):
        if mode not in ("natural", "uniform", "briggs", "robust"):
            raise ValueError("unknown weighting mode %s" % mode)
        self.mode = mode
        self.robust = robust
        self.nbands = nbands
        self.device = D._dev(device)
        self.grid = None
        if mode != "natural":
            fov = cell_rad * npix_image
            self.cell = 1. / (super_uniform * fov)
            self.xymax = int(math.floor(uvmax / self.cell)) + 1
            self.npixx = self.xymax * 2 + 1
            self.npixy = self.xymax + 1
            self.npix = self.npixx * self.npixy
            self.grid = torch.zeros((nbands, self.npix), dtype=torch.float64, device=self.device)
            self._bad = torch.zeros(1, dtype=torch.int32, device=self.device)

    def _index(self, uvw, freqs, weights, band_of_chan):
        lib = _abi.lib()
        uvw = D.to_device(uvw, torch.float64, self.device)
        fr = D.to_device(np.asarray(freqs, np.float64), torch.float64, self.device)
        w = D.to_device(weights, torch.float32, self.device)
        nrow, nchan = w.shape
        bmap = None
        if self.nbands > 1:
            bmap = D.to_device(np.asarray(band_of_chan, np.int32), torch.int32, self.device)
        index = torch.empty((nrow, nchan), dtype=torch.int32, device=self.device)
        _abi.check(lib.ddfg_weights_uv_index(uvw.data_ptr(), nrow, fr.data_ptr(), nchan, w.data_ptr(),
                                             None if bmap is None else bmap.data_ptr(), self.nbands, self.cell,
                                             self.xymax, self.npixx, self.npix, index.data_ptr(), D._stream_ptr()))
        return w, index

    def accumulate(self, uvw, freqs, weights, band_of_chan=None):
        """Add one chunk's weights (float32 [nrow][nchan], flagged visibilities already 0) to the
        density grid."""
        if self.grid is None:
            return
        w, index = self._index(uvw, freqs, weights, band_of_chan)
        _abi.check(_abi.lib().ddfg_weights_accumulate(self.grid.data_ptr(), self.grid.numel(), w.data_ptr(),
                                                      index.data_ptr(), index.numel(), self._bad.data_ptr(),
                                                      D._stream_ptr()))

    def finish(self):
        """Briggs transform of the density grid (after every chunk was accumulated)."""
        if int(self._bad.item() if self.grid is not None else 0):
            raise RuntimeError("a visibility fell outside the weight grid (uvmax too small)")
        if self.mode in ("briggs", "robust"):
            numerator_sqrt = 5.0 * 10 ** (-self.robust)
            ws = torch.empty(2 * self.nbands, dtype=torch.float64, device=self.device)
            _abi.check(_abi.lib().ddfg_weights_robust(self.grid.data_ptr(), self.npix, self.nbands, numerator_sqrt,
                                                      ws.data_ptr(), D._stream_ptr()))

    def apply(self, uvw, freqs, weights, band_of_chan=None) -> torch.Tensor:
        """The chunk's imaging weights (float32 [nrow][nchan], a new tensor)."""
        w = D.to_device(weights, torch.float32, self.device).clone()
        if self.grid is None:
            return w
        w, index = self._index(uvw, freqs, w, band_of_chan)
        _abi.check(_abi.lib().ddfg_weights_finalize(w.data_ptr(), index.data_ptr(), index.numel(),
                                                    self.grid.data_ptr(), self.grid.numel(), D._stream_ptr()))
        return w
