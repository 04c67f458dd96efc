"""W-projection convolution functions and the prolate-spheroidal taper (FP64, host, one-off).

A from-scratch restatement of DDFacet's CF generation, computed once per facet before any
gridding:

* ``eval_sphe``        -- rational approximation of the 0-order prolate spheroidal
                          (DDFacet/ToolsDir/ModTaper.py:76-111, ``EvalSphe``), vectorised.
* ``sphe2d``           -- the 2-D radial spheroidal on an ``N x N`` grid over [-1, 1]^2
                          (ModTaper.py:38-47, ``Sphe2D``).
* ``SpheroidalTaper``  -- cut of the spheroidal's spectrum to the CF support, and its
                          zero-padded inverse transform on an image grid (ModCF.py:87-172,
                          ``SpheMachine``); ``taper(n)`` is the reference's ``ifzfCF``.
* ``fit_n_minus_n0``   -- degree-5 2-D polynomial fit of n(l, m) - n0 around a facet centre;
                          its linear terms become the uvw shift (Cu, Cv) (ModCF.py:267-295,
                          ``Give_dn``; ModFitPoly2D.py:30-58).
* ``WTerms``           -- oversampled W-kernels ``Wplanes`` and their conjugate-phase twins
                          ``WplanesConj`` re-ordered as ``[OverS][OverS][S][S]`` so that one
                          oversampling phase is a contiguous S*S tap table
                          (ModCF.py:297-597, ``ClassWTermModified``; ``GiveReorgCF`` :364-372).

The arithmetic follows the reference step for step (same FFT library, same normalisations,
same order of operations), so the complex64 tables agree with the reference's bit-for-bit or to
the last ulp; the CF tables are then uploaded once and stay resident on the GPU.
"""
from __future__ import annotations

import functools
import itertools
import math

import numpy as np
import scipy.fftpack
from scipy.interpolate import interp1d

C_LIGHT = 299792458.0

# Rational approximation coefficients of the spheroidal function (ModTaper.py:77-80): these are
# the published Schwab (1984) prolate-spheroidal coefficients for alpha=1, m=6 support.
_P = np.array([[8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1],
               [4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2]])
_Q = np.array([[1.0000000e0, 8.212018e-1, 2.078043e-1],
               [1.0000000e0, 9.599102e-1, 2.918724e-1]])


def eval_sphe(nu):
    """Vectorised ``EvalSphe`` (ModTaper.py:76-111): 0 outside [0, 1]."""
    nu = np.asarray(nu, dtype=np.float64)
    out = np.zeros_like(nu)
    for part, (lo, hi, end, closed) in enumerate(((0.0, 0.75, 0.75, False), (0.75, 1.0, 1.0, True))):
        sel = (nu >= lo) & ((nu <= hi) if closed else (nu < hi))
        if not np.any(sel):
            continue
        x = nu[sel]
        nusq = x * x
        d = nusq - end * end
        dp = d
        top = np.full_like(x, _P[part][0])
        for k in range(1, 5):
            top = top + _P[part][k] * dp
            dp = dp * d
        bot = np.full_like(x, _Q[part][0])
        dp = d
        for k in range(1, 3):
            bot = bot + _Q[part][k] * dp
            dp = dp * d
        out[sel] = (1.0 - nusq) * (top / bot)
    return out


def sphe2d(npix, factor=1.0):
    """``Sphe2D`` (ModTaper.py:38-47): spheroidal of the radius on linspace(-1, 1, npix)^2."""
    x, y = np.mgrid[-1:1:1j * npix, -1:1:1j * npix]
    r = np.sqrt(x ** 2 + y ** 2)
    return eval_sphe(np.abs(r) * factor)


def fft2c(a):
    """Centred forward FFT normalised by 1/N (ModCF.py:46-49)."""
    return scipy.fftpack.fftshift(scipy.fftpack.fft2(scipy.fftpack.ifftshift(a))) / np.float64(a.size)


def ifft2c(a):
    """Centred inverse FFT scaled by N (ModCF.py:52-60)."""
    return scipy.fftpack.fftshift(scipy.fftpack.ifft2(scipy.fftpack.ifftshift(a))) * np.float64(a.size)


def zero_pad(a, outshape):
    """``ZeroPad`` (ModCF.py:63-79): centre ``a`` in a zero square of side ``outshape``."""
    nx = a.shape[0]
    b = np.zeros((outshape, outshape), dtype=a.dtype)
    off = (outshape - nx) // 2 + (1 if outshape % 2 == 0 else 0)
    b[off:off + nx, off:off + nx] = a
    return b


@functools.lru_cache(maxsize=64)
def _taper_cached(support, npix):
    z = SpheroidalTaper(support)._taper(npix)
    z.setflags(write=False)
    return z


class SpheroidalTaper:
    """``SpheMachine`` (ModCF.py:87-172) for the "Sphe" type."""

    SUPPORT_CALC = 111

    def __init__(self, support):
        self.support = int(support)
        ns = self.SUPPORT_CALC
        xc = ns // 2
        cf = np.complex128(sphe2d(ns))
        fcf = fft2c(cf)
        h = self.support // 2
        self.small_fcf = fcf[xc - h:xc + h + 1, xc - h:xc + h + 1].copy()
        self.small_cf = cf

    def taper(self, npix):
        """The image-plane taper ``ifzfCF`` of side ``npix`` (ModCF.py:120-170); memoised per
        (support, npix) since it does not depend on the facet."""
        return _taper_cached(self.support, int(npix)).copy()

    def _taper(self, npix):
        z = ifft2c(zero_pad(self.small_fcf, npix))
        # ModCF.py:170 compares complex values lexicographically (real part first).
        neg = (z.real < 0) | ((z.real == 0) & (z.imag < 0))
        z[neg] = 1e-10
        return z


def polyfit2d(x, y, z, order=3):
    """Least-squares 2-D polynomial, coefficient k <-> x**i * y**j (ModFitPoly2D.py:30-48)."""
    ncols = (order + 1) ** 2
    g = np.zeros((x.size, ncols))
    for k, (i, j) in enumerate(itertools.product(range(order + 1), range(order + 1))):
        g[:, k] = x ** i * y ** j
    m, _, _, _ = np.linalg.lstsq(g, z, rcond=-1)
    return m


def polyval2d(x, y, m):
    """Evaluate ``polyfit2d`` coefficients (ModFitPoly2D.py:50-58)."""
    order = int(np.sqrt(len(m))) - 1
    z = np.zeros_like(x)
    for a, (i, j) in zip(m, itertools.product(range(order + 1), range(order + 1))):
        z += a * x ** i * y ** j
    return z


def fit_n_minus_n0(l0, m0, rad=1.0, order=4):
    """``Give_dn`` (ModCF.py:267-295).  Returns (Cl, Cm, coefs) with the linear terms zeroed."""
    npts = 100
    l, m = np.mgrid[l0 - rad:l0 + rad:npts * 1j, m0 - rad:m0 + rad:npts * 1j]
    dl = (l - l0).flatten()
    dm = (m - m0).flatten()
    mll = np.max(np.abs((dl + l0) ** 2 + (dm + m0) ** 2))
    if mll > 1.0:
        return 0.0, 0.0, np.zeros((order + 1, order + 1), np.float32).flatten()
    y = np.sqrt(1 - (dl + l0) ** 2 - (dm + m0) ** 2) - np.sqrt(1 - l0 ** 2 - m0 ** 2)
    coef = polyfit2d(dl, dm, y, order=order)
    c = coef.reshape((order + 1, order + 1))
    cl = c[0, 1]
    cm = c[1, 0]
    c[0, 1] = 0
    c[1, 0] = 0
    return cl, cm, c.flatten()


def reorg_cf(a, overs):
    """``GiveReorgCF`` (ModCF.py:364-372): [S*O][S*O] -> [O][O][S][S] flattened back to 2-D."""
    sup = a.shape[0] // overs
    b = np.zeros((overs, overs, sup, sup), dtype=a.dtype)
    for i in range(overs):
        for j in range(overs):
            b[i, j] = a[i::overs, j::overs]
    return b.reshape((a.shape[0], a.shape[0]))


class WTerms:
    """Per-facet W-projection tables (``ClassWTermModified``, ModCF.py:297-597).

    Attributes mirror the reference's: ``Wplanes``, ``WplanesConj`` (lists of complex64
    ``[S*O, S*O]`` arrays in ``[O][O][S][S]`` order), ``Sups``, ``Cu``, ``Cv``, ``RefWave``,
    ``wmax``, ``Nw``, ``OverS``, ``ifzfCF`` (complex128 ``[Npix, Npix]`` taper).
    """

    def __init__(self, Cell=10, Sup=15, Nw=11, wmax=30000, Npix=101, Freqs=np.array([100.e6]),
                 OverS=11, lmShift=None, IDFacet=None):
        self.Nw = Nw
        self.Cell = Cell
        self.Sup = Sup
        self.Npix = Npix
        self.Freqs = np.asarray(Freqs)
        self.OverS = OverS
        self.lmShift = lmShift
        self.IDFacet = IDFacet
        self.RefWave = C_LIGHT / self.Freqs[-1]
        self.wmax = wmax
        self.sphe = SpheroidalTaper(Sup)
        self.ifzfCF = self.sphe.taper(Npix)
        self._init_w()

    def _init_w(self):
        nw, cell, sup, wmax, npix, overs = self.Nw, self.Cell, self.Sup, self.wmax, self.Npix, self.OverS
        supmax = 501
        sphe_w = self.sphe.taper(supmax)
        radius_deg = (npix / 2.0) * cell / 3600.0
        lrad = radius_deg * np.pi / 180.0
        l, m = np.mgrid[-lrad * np.sqrt(2.):np.sqrt(2.) * lrad:supmax * 1j,
                        -lrad * np.sqrt(2.):np.sqrt(2.) * lrad:supmax * 1j]
        n_1 = np.sqrt(1. - l ** 2 - m ** 2) - 1
        wave_min = C_LIGHT / self.Freqs[-1]
        w_screen = np.exp(-2. * 1j * np.pi * (wmax / wave_min) * n_1) * sphe_w
        fw = fft2c(w_screen)
        fw1d = np.abs(fw[(supmax - 1) // 2, :])
        fw1d /= np.max(fw1d)
        fw1d = fw1d[(supmax - 1) // 2::]
        ind = np.argsort(fw1d)
        try:
            interp = interp1d(fw1d[ind], np.arange(fw1d.shape[0])[ind])
            supmax = np.int64(interp(np.array([1. / 1000]))[0])
        except Exception:  # the reference falls back to the base support (ModCF.py:414-420)
            supmax = sup
        sups = np.int64(np.linspace(sup, np.max([supmax, sup]), nw))
        wgrid = np.linspace(0, wmax, nw)
        self.Sups = sups

        l0, m0 = (0., 0.) if self.lmShift is None else self.lmShift
        radmax = (1. - np.sqrt(l0 ** 2 + m0 ** 2)) / np.sqrt(2)
        rad = 3 * lrad
        rad = np.min([rad, 0.99 * radmax])
        rad = np.max([rad, lrad])
        self.Cv, self.Cu, coef_poly = fit_n_minus_n0(l0, m0, rad=rad, order=5)

        wplanes, wplanes_conj = [], []
        if nw <= 1:
            if not (sups[0] % 2):
                sups[0] += 1
            w = np.abs(self.sphe.taper(int(sups[0])))
            planes = [(w, int(sups[0]))]
        else:
            planes = []
            for i in range(nw):
                if not (sups[i] % 2):
                    sups[i] += 1
                s = int(sups[i])
                this_sphe = self.sphe.taper(s)
                wl = wgrid[i] / wave_min
                dx = 2 * lrad / s
                l, m = np.mgrid[-lrad + dx / 2:lrad - dx / 2:s * 1j, -lrad + dx / 2:lrad - dx / 2:s * 1j]
                n_1 = polyval2d(l, m, coef_poly)
                w = np.exp(-2. * 1j * np.pi * wl * n_1)
                w *= np.abs(this_sphe)
                planes.append((w, s))
        for w, s in planes:
            zw = zero_pad(w, outshape=w.shape[0] * overs)
            fzw = np.complex64(fft2c(zw))
            fzw_conj = np.complex64(fft2c(np.conj(zw)))
            wplanes.append(np.ascontiguousarray(reorg_cf(fzw, overs)))
            wplanes_conj.append(np.ascontiguousarray(reorg_cf(fzw_conj, overs)))
        self.Wplanes = wplanes
        self.WplanesConj = wplanes_conj
        self.wmap = wgrid

    @property
    def supports(self):
        return [int(p.shape[0] // self.OverS) for p in self.Wplanes]


def n0_minus_one(l0, m0):
    """n0 - 1 = sqrt(1 - l0^2 - m0^2) - 1 (gridder.h:108)."""
    return math.sqrt(1 - l0 * l0 - m0 * m0) - 1
