"""Integer maps that feed the gridder and degridder.

* ``jones_time_map``      -- row -> Jones time slot: ClassJones.GiveTimeMapping
                             (DDFacet/Data/ClassJones.py:415-439): for every slot it in order, the
                             rows with t0[it] <= time < t1[it] get it (a later slot overrides an
                             earlier one where they overlap; rows in no slot keep 0; the times need
                             not be sorted).  ``jones_time_map_gpu`` is the same on the device
                             (ddfg_jones_time_map), one thread per row.
* ``jones_chan_map``      -- visibility channel -> Jones channel: the nearest solution-interval
                             centre (ClassJones.GiveVisToJonesChanMapping, ClassJones.py:1004-1012;
                             the first on a tie, as numpy's argmin).
* ``ChannelMaps``         -- the grid-band and degrid-band channel maps of every measurement set
                             (ClassVisServer.Init, DDFacet/Data/ClassVisServer.py:135-355): the band
                             width and count from the data's frequency span (BandMHz, else NBand),
                             grid_band = floor((nu - nu_min) / band width) over the sorted global
                             frequencies, each channel's index within its band, and per measurement
                             set the degridding bands (DegridBandMHz, else NDegridBand) with
                             floor((nu - nu_min_ms) / degrid width) and their centre frequencies.

All integer results are what the reference computes, word for word (tests/test_maps_cpu.py and
tests/test_maps_gpu.py against fixtures made by running the reference's own functions).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


def jones_time_map(times, t0, t1) -> np.ndarray:
    """int32 [nrow] Jones time slot of every row (GiveTimeMapping)."""
    times = np.asarray(times, np.float64)
    t0 = np.asarray(t0, np.float64)
    t1 = np.asarray(t1, np.float64)
    ind = np.zeros(times.size, np.int32)
    for it in range(t0.size):
        ind[(times >= t0[it]) & (times < t1[it])] = it
    return ind


def jones_time_map_gpu(times, t0, t1, stream=None):
    """jones_time_map on the device (ddfg_jones_time_map): times a float64 CUDA tensor [nrow];
    returns an int32 CUDA tensor."""
    import torch

    from . import _abi, device as D

    dev = times.device
    tt = D.to_device(times, torch.float64, dev)
    a = D.to_device(np.asarray(t0, np.float64), torch.float64, dev)
    b = D.to_device(np.asarray(t1, np.float64), torch.float64, dev)
    out = torch.empty(tt.numel(), dtype=torch.int32, device=dev)
    lib = _abi.lib()
    _abi.check(lib.ddfg_jones_time_map(tt.data_ptr(), tt.numel(), a.data_ptr(), b.data_ptr(), a.numel(),
                                       out.data_ptr(), D._stream_ptr(stream)))
    return out


def jones_chan_map(chan_freqs, freq_domains) -> np.ndarray:
    """Jones channel of every visibility channel: argmin |nu - (domain lo + hi) / 2|
    (GiveVisToJonesChanMapping)."""
    fd = np.asarray(freq_domains, np.float64).reshape(-1, 2)
    mean = (fd[:, 0] + fd[:, 1]) / 2.
    nu = np.asarray(chan_freqs, np.float64).reshape(-1, 1)
    return np.argmin(np.abs(nu - mean.reshape(1, -1)), axis=1)


@dataclass
class MSChannels:
    """One measurement set's channels (MS.ChanFreq, MS.ChanWidth)."""
    chan_freq: np.ndarray
    chan_width: np.ndarray


@dataclass
class ChannelMaps:
    nbands: int
    grid_bw: float
    band_centers: np.ndarray
    band_channels: List[List[float]]
    chan_mapping: Dict[int, np.ndarray] = field(default_factory=dict)          # MS channel -> grid band
    chan_mapping_chan: Dict[int, np.ndarray] = field(default_factory=dict)     # -> channel within its band
    chan_mapping_degrid: Dict[int, np.ndarray] = field(default_factory=dict)   # -> degridding band
    degrid_freqs: Dict[int, np.ndarray] = field(default_factory=dict)          # degridding band centres

    @classmethod
    def build(cls, ms_list: Sequence[MSChannels], band_mhz: float = 0.0, nband: int = 1,
              degrid_band_mhz: float = 0.0, ndegrid_band: int = 0) -> "ChannelMaps":
        global_freqs = set()
        lo, hi = 1e+999, 0.
        for ms in ms_list:
            global_freqs.update(np.asarray(ms.chan_freq).tolist())
            lo = min(lo, (ms.chan_freq - ms.chan_width / 2).min())
            hi = max(hi, (ms.chan_freq + ms.chan_width / 2).max())
        gfreqs = np.array(sorted(global_freqs))
        span = hi - lo
        grid_bw = band_mhz * 1e+6
        if grid_bw:
            grid_bw = min(grid_bw, span)
            nbands = int(math.ceil(span / grid_bw))
        else:
            nbands = int(np.min([nband, len(gfreqs)]))
            grid_bw = span / nbands
        grid_band = np.floor((gfreqs - lo) / grid_bw).astype(int)
        band_of = dict(zip(gfreqs.tolist(), grid_band.tolist()))
        centers = np.linspace(lo + grid_bw / 2, hi - grid_bw / 2, nbands)
        band_channels, chan_in_band = [], {}
        for ib in range(nbands):
            fl = sorted([f for f, b in band_of.items() if b == ib])
            band_channels.append(fl)
            chan_in_band.update({f: c for c, f in enumerate(fl)})
        out = cls(nbands=nbands, grid_bw=grid_bw, band_centers=centers, band_channels=band_channels)
        for ims, ms in enumerate(ms_list):
            nu = np.asarray(ms.chan_freq, np.float64)
            mlo = (nu - ms.chan_width / 2).min()
            mhi = (nu + ms.chan_width / 2).max()
            bw = mhi - mlo
            out.chan_mapping[ims] = np.array([band_of[f] for f in nu.tolist()])
            out.chan_mapping_chan[ims] = np.array([chan_in_band[f] for f in nu.tolist()])
            dbw = degrid_band_mhz * 1e+6
            if dbw:
                dbw = min(dbw, bw)
                dbw = max(dbw, ms.chan_width[0])
            else:
                nd = min(ndegrid_band or nu.size, nu.size)
                dbw = bw / nd
            out.chan_mapping_degrid[ims] = np.floor((nu - mlo) / dbw).astype(int)
            edges = np.arange(mlo, mhi + dbw, dbw)
            out.degrid_freqs[ims] = (edges[:-1] + edges[1:]) / 2
        return out
