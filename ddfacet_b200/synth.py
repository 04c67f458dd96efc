"""Seeded synthetic observations with the shapes of the benchmark configurations.

No measurement set is read: antenna layouts, uvw tracks, frequencies, skies, visibilities and
Jones terms are generated from a seed (numpy ``default_rng``), so every run sees the same data.

* array: antennas uniform in a disk (r = R sqrt(U)) or log-radial, rotated to equatorial XYZ at
  the site latitude; uvw from hour angle H and declination d:
      u = sin H X + cos H Y
      v = -sin d cos H X + sin d sin H Y + cos d Z
      w = cos d cos H X - cos d sin H Y + sin d Z
  rows ordered time-major, baselines (a0 < a1) minor; ``uvw_dt`` is the analytic derivative.
* frequencies: linspace(f_lo, f_hi, nchan).
* sky: point sources uniform in the field, flux log-uniform or power-law.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

C_LIGHT = 299792458.0
OMEGA_EARTH = 7.2921150e-5  # rad/s


@dataclass
class Observation:
    uvw: np.ndarray      # float64 [nrow, 3]
    uvw_dt: np.ndarray   # float64 [nrow, 3] (m/s)
    A0: np.ndarray       # int32 [nrow]
    A1: np.ndarray       # int32 [nrow]
    times: np.ndarray    # float64 [nrow]
    freqs: np.ndarray    # float64 [nchan]
    nant: int
    ntimes: int
    dump_s: float

    @property
    def nrow(self):
        return self.uvw.shape[0]

    @property
    def nbl(self):
        return self.nant * (self.nant - 1) // 2


def antenna_layout(rng, nant, radius_m, layout="disk", rmin=50.0):
    th = rng.uniform(0, 2 * np.pi, nant)
    if layout == "disk":
        r = radius_m * np.sqrt(rng.uniform(0, 1, nant))
    elif layout == "lograd":
        r = np.exp(rng.uniform(np.log(rmin), np.log(radius_m), nant))
    else:
        raise ValueError(layout)
    east = r * np.cos(th)
    north = r * np.sin(th)
    return east, north, np.zeros(nant)


def make_observation(seed, nant, radius_m, lat_deg, dec_deg, hours, dump_s, nchan, f_lo, f_hi, layout="disk"):
    rng = np.random.default_rng(seed)
    e, n, up = antenna_layout(rng, nant, radius_m, layout)
    lat = np.deg2rad(lat_deg)
    # ENU -> equatorial XYZ (X towards H=0 meridian, Z to the pole)
    X = -np.sin(lat) * n + np.cos(lat) * up
    Y = e
    Z = np.cos(lat) * n + np.sin(lat) * up
    ntimes = int(round(hours * 3600.0 / dump_s))
    t = (np.arange(ntimes) - (ntimes - 1) / 2.0) * dump_s
    H = OMEGA_EARTH * t
    d = np.deg2rad(dec_deg)
    a0, a1 = np.triu_indices(nant, 1)
    bx, by, bz = X[a1] - X[a0], Y[a1] - Y[a0], Z[a1] - Z[a0]
    sH, cH = np.sin(H)[:, None], np.cos(H)[:, None]
    u = sH * bx + cH * by
    v = -np.sin(d) * cH * bx + np.sin(d) * sH * by + np.cos(d) * bz
    w = np.cos(d) * cH * bx - np.cos(d) * sH * by + np.sin(d) * bz
    du = OMEGA_EARTH * (cH * bx - sH * by)
    dv = OMEGA_EARTH * (np.sin(d) * sH * bx + np.sin(d) * cH * by)
    dw = OMEGA_EARTH * (-np.cos(d) * sH * bx - np.cos(d) * cH * by)
    uvw = np.stack([u.ravel(), v.ravel(), w.ravel()], axis=1)
    uvw_dt = np.stack([du.ravel(), dv.ravel(), dw.ravel()], axis=1)
    nbl = a0.size
    A0 = np.tile(a0, ntimes).astype(np.int32)
    A1 = np.tile(a1, ntimes).astype(np.int32)
    times = np.repeat(t, nbl)
    freqs = np.linspace(f_lo, f_hi, nchan)
    return Observation(uvw=np.ascontiguousarray(uvw), uvw_dt=np.ascontiguousarray(uvw_dt), A0=A0, A1=A1,
                       times=times, freqs=freqs, nant=nant, ntimes=ntimes, dump_s=dump_s)


def point_sky(seed, nsrc, field_rad, flux=("loguniform", 1e-3, 1.0), center=(0.0, 0.0)):
    """(l, m, S) of nsrc point sources uniform in a square field of half-width field_rad."""
    rng = np.random.default_rng(seed)
    l = center[0] + rng.uniform(-field_rad, field_rad, nsrc)
    m = center[1] + rng.uniform(-field_rad, field_rad, nsrc)
    kind, lo, hi = flux
    if kind == "loguniform":
        s = np.exp(rng.uniform(np.log(lo), np.log(hi), nsrc))
    elif kind == "powerlaw":  # N(>S) ~ S^-1.5 between lo and hi
        a = 1.5
        u = rng.uniform(0, 1, nsrc)
        s = (lo ** -a - u * (lo ** -a - hi ** -a)) ** (-1.0 / a)
    else:
        raise ValueError(kind)
    return l, m, s


def dft_predict(uvw, freqs, l, m, s, ncorr=1, chunk=4096):
    """V = sum_k S_k exp(+2 pi i (u l + v m + w (n-1)) nu / c), FP64 (sign of
    ClassDDEGridMachine.py:264-271).  Used only to make synthetic visibilities."""
    n1 = np.sqrt(1 - l ** 2 - m ** 2) - 1
    nrow = uvw.shape[0]
    out = np.zeros((nrow, freqs.size), np.complex128)
    for r0 in range(0, nrow, chunk):
        uu = uvw[r0:r0 + chunk]
        ph = uu[:, 0:1] * l[None] + uu[:, 1:2] * m[None] + uu[:, 2:3] * n1[None]  # [r, k]
        arg = 2j * np.pi * ph[:, :, None] * (freqs[None, None, :] / C_LIGHT)
        out[r0:r0 + chunk] = np.einsum("k,rkc->rc", s, np.exp(arg))
    if ncorr == 1:
        return out[:, :, None]
    res = np.zeros((nrow, freqs.size, ncorr), np.complex128)
    res[:, :, 0] = out
    res[:, :, -1] = out
    return res


def add_noise(rng, vis, sigma):
    return vis + sigma * (rng.standard_normal(vis.shape) + 1j * rng.standard_normal(vis.shape))


def random_jones(seed, nt, nd, na, nch, sigma):
    """I + sigma (N + iN), complex64 [nt, nd, na, nch, 2, 2]."""
    rng = np.random.default_rng(seed)
    j = sigma * (rng.standard_normal((nt, nd, na, nch, 2, 2)) + 1j * rng.standard_normal((nt, nd, na, nch, 2, 2)))
    j[..., 0, 0] += 1
    j[..., 1, 1] += 1
    return j.astype(np.complex64)
