"""The batched facet machine: every facet of a tessellation gridded and degridded together.

Mirrors the parts of DDFacet's ``ClassFacetMachine`` that sit on the hot path
(DDFacet/Imager/ClassFacetMachine.py):

* set-up (``appendMainField`` / ``setFacetsLocs`` / ``_initcf_worker``, :232-548, :766-838):
  regular tessellation, per-facet W-projection tables and taper, spatial-weight masks (facet
  polygon convolved with a Gaussian of ``MixingWidth`` pixels, normalised, zeroed below 1e-3),
  the facet-normalisation image (``BuildFacetNormImage``, :1289-1330);
* ``grid_all_facets`` / ``degrid_all_facets`` -- ``putChunkInBackground`` /
  ``getChunkInBackground`` (:912-927) for all facets in one call of the GPU gridder/degridder;
* ``facets_to_image`` -- ``FacetsToIm`` (:1012-1249) with ``FacetsToIm_Channel`` (:1331-1416):
  per-facet GridToIm on the GPU (cuFFT), weight and taper normalisation, stitching, facet norm;
* ``image_to_facets`` -- ``set_model_grid`` / ``GiveModelTessel`` (ClassImToGrid.py:138-264):
  model image to every facet's model grid on the GPU.

Host code here builds one-off geometry and tables (FP64 numpy); every per-visibility and
per-pixel pass runs in libddfg.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _abi, cf, device as D, geometry

C_LIGHT = 299792458.0


# ------------------------------------------------------------------------------------------
# spatial weights (host, one-off)
# ------------------------------------------------------------------------------------------
def give_gauss(npix, cell_rad, gauss_pars):
    """``GiveGauss`` (DDFacet/ToolsDir/ModFFTW.py:654-690)."""
    uvscale = npix * cell_rad / 2
    sig_maj, sig_min, ang = gauss_pars
    ang = 2 * np.pi - ang
    U, V = np.mgrid[-uvscale:uvscale:npix * 1j, -uvscale:uvscale:npix * 1j]
    ct, st, c2t, s2t = np.cos(ang), np.sin(ang), np.cos(2 * ang), np.sin(2 * ang)
    sx2, sy2 = sig_maj ** 2, sig_min ** 2
    a = (ct ** 2 / (2. * sx2)) + (st ** 2 / (2. * sy2))
    b = -(s2t / (4. * sx2)) + (s2t / (4. * sy2))
    c = (st ** 2 / (2. * sx2)) + (ct ** 2 / (2. * sy2))
    return np.exp(-(a * U ** 2 + 2 * b * U * V + c * V ** 2)).astype(np.float32)


def convolve_gaussian(img, gauss_pars, cell_rad=1.0):
    """``_convolveSingleGaussianFFTW`` for one plane (ModFFTW.py:779-849): zero-pad to the next
    FFT size, multiply spectra with |FFT(gaussian)|, crop."""
    npix = img.shape[-1]
    pad = max(int(np.ceil((geometry.estimate_npix(npix)[1] - npix) / 2.0) * 2), 0)
    psf = np.pad(give_gauss(npix, cell_rad, gauss_pars), ((pad // 2, pad // 2), (pad // 2, pad // 2)))
    fpsf = np.abs(np.fft.rfft2(np.fft.ifftshift(psf)))
    a = np.fft.ifftshift(np.pad(img, ((pad // 2, pad // 2), (pad // 2, pad // 2))))
    out = np.fft.fftshift(np.fft.irfft2(np.fft.rfft2(a) * fpsf, s=a.shape))
    return out[pad // 2:pad // 2 + npix, pad // 2:pad // 2 + npix]


def _inside_convex(px, py, poly):
    """Points strictly inside a convex polygon (either winding)."""
    n = len(poly)
    sgn = None
    inside = np.ones(px.shape, bool)
    signs = []
    for i in range(n):
        x0, y0 = poly[i]
        x1, y1 = poly[(i + 1) % n]
        cross = (x1 - x0) * (py - y0) - (y1 - y0) * (px - x0)
        signs.append(cross)
    s = np.stack(signs)
    return np.all(s > 0, axis=0) | np.all(s < 0, axis=0)


def spatial_weight(polygon, extent_padded, npix, corners_tot, mixing_width):
    """Spatial-weight mask of a facet (``_initcf_worker``, ClassFacetMachine.py:785-820), in
    image orientation: polygon mask (inside the main-image square too), Gaussian-smoothed with
    sigma ``mixing_width`` pixels, divided by its maximum, zero below 1e-3."""
    l0, l1, m0, m1 = extent_padded
    X, Y = np.mgrid[l0:l1:npix * 1j, m0:m1:npix * 1j]
    mask = _inside_convex(X, Y, np.asarray(polygon)) & _inside_convex(X, Y, np.asarray(corners_tot))
    sw = convolve_gaussian(mask.astype(np.float32), (mixing_width, mixing_width, 0), cell_rad=1.0)
    sw = sw.astype(np.float32)
    mx = np.max(sw)
    if mx > 0:
        sw /= mx
    sw[sw < 1e-3] = 0.
    return sw


# ------------------------------------------------------------------------------------------
# the facet machine
# ------------------------------------------------------------------------------------------
@dataclass
class FacetState:
    geom: geometry.FacetGeom
    wterms: cf.WTerms
    grid: D.FacetGrid        # residual grid (gridding target)
    model: D.FacetGrid       # model grid (degridding source)
    sphe: torch.Tensor       # float32 [N][N] taper (grid orientation; symmetric)
    invsphe: torch.Tensor    # float32 [N][N]
    sw_img: torch.Tensor     # float32 [N][N] spatial weight, image orientation
    sw_grid: torch.Tensor    # float32 [N][N] spatial weight, grid orientation (SW.T[::-1, :])
    sw_host: np.ndarray


class FacetMachine:
    """All facets of a tessellation on one GPU: a regular ``nfacets_side`` x ``nfacets_side`` one
    (ClassFacetMachine), or any ``tessellation`` such as ``geometry.voronoi_facets``
    (ClassFacetMachineTessel), whose facets may differ in size."""

    def __init__(self, npix, cell_arcsec, nfacets_side, freqs, padding=1.7, nband=1, stokes_ids=(1,),
                 corr_ids=(9, 10, 11, 12), overs=11, support=7, nw=32, wmax=None, mixing_width=10.0, device=None,
                 threads=8, tessellation=None):
        self.device = D._dev(device)
        self.tess = tessellation or geometry.regular_facets(npix, nfacets_side, cell_arcsec, padding)
        self.cell = cell_arcsec
        self.freqs = np.asarray(freqs, np.float64)
        self.nband = nband
        self.stokes_ids = list(stokes_ids)
        self.corr_ids = list(corr_ids)
        self.npol = len(stokes_ids)
        self.overs = overs
        if wmax is None:
            raise ValueError("wmax must be given (the largest |w| to grid)")
        self.wmax = float(wmax)
        self.pol = D.make_pol(corr_ids, stokes_ids)
        t = self.tess
        self.npix_out = t.npix
        from .configs import build_wterms

        wts = build_wterms(t.facets, cell_arcsec, support, nw, self.wmax, [g.npix_padded for g in t.facets],
                           self.freqs, overs, threads=threads)
        incr = (-cell_arcsec / 3600 * np.pi / 180, cell_arcsec / 3600 * np.pi / 180)
        radius_tot = t.cell_rad * t.npix * 0.5
        corners = [[-radius_tot, -radius_tot], [radius_tot, -radius_tot], [radius_tot, radius_tot],
                   [-radius_tot, radius_tot]]
        self.facets: List[FacetState] = []
        norm = np.zeros((t.npix, t.npix), np.float32)
        dev = self.device
        for g, wt in zip(t.facets, wts):
            N = g.npix_padded
            rf = g.npix_facet * t.cell_rad * 0.5
            rfp = N * t.cell_rad * 0.5
            if g.polygon is not None:
                poly = g.polygon
            elif len(t.facets) > 1:
                poly = [[g.l0 + rf, g.m0 - rf], [g.l0 - rf, g.m0 - rf], [g.l0 - rf, g.m0 + rf], [g.l0 + rf, g.m0 + rf]]
            else:
                poly = corners
            sw = spatial_weight(poly, (g.l0 - rfp, g.l0 + rfp, g.m0 - rfp, g.m0 + rfp), N, corners, mixing_width)
            self._add_norm(norm, sw, g, N)
            tabs = D.CFTables.create(wt.Wplanes, wt.WplanesConj, overs, wt.RefWave, wt.wmax, device=dev)
            common = dict(cf=tabs, incr=incr, cu=wt.Cu, cv=wt.Cv, l0=g.l0, m0=g.m0, idir_kms=g.isol, idir_beam=0)
            z = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)  # noqa: E731
            fg = D.FacetGrid(grid=torch.zeros((nband, self.npol, N, N), dtype=torch.complex64, device=dev),
                             sumwt=z(nband, self.npol), sumjones=z(2, nband), sumjones_chan=z(2, self.freqs.size),
                             **common)
            fm = D.FacetGrid(grid=torch.zeros((nband, self.npol, N, N), dtype=torch.complex64, device=dev), **common)
            sphe = np.float32(wt.ifzfCF.real)
            inv = np.float32(1. / np.float64(wt.ifzfCF.real))
            self.facets.append(FacetState(g, wt, fg, fm, torch.from_numpy(sphe).to(dev), torch.from_numpy(inv).to(dev),
                                          torch.from_numpy(sw).to(dev),
                                          torch.from_numpy(np.ascontiguousarray(sw.T[::-1, :])).to(dev), sw))
        self.facet_norm_host = norm
        self.facet_norm = torch.from_numpy(norm).to(dev)
        self._plans = {}
        self._work = None

    @staticmethod
    def _add_norm(norm, sw, g, n):
        """``BuildFacetNormImage`` (ClassFacetMachine.py:1289-1330) for one facet."""
        m = norm.shape[0]
        xc, yc = g.pix_central
        e = _edges(xc, yc, m, n)
        norm[e[0]:e[1], e[2]:e[3]] += sw[e[4]:e[5], e[6]:e[7]]

    # --------------------------------------------------------------------------------------
    def _plan(self, n):
        if n not in self._plans:
            p = C.c_void_p()
            lib = _abi.lib()
            _abi.check(lib.ddfg_fft_plan_create(n, self.nband * self.npol, C.byref(p)))
            self._plans[n] = p
        return self._plans[n]

    def close(self):
        lib = _abi.lib()
        for p in self._plans.values():
            lib.ddfg_fft_plan_destroy(p)
        self._plans = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _work_for(self, n):
        need = self.nband * self.npol * n * n
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.complex64, device=self.device)
        return self._work

    # --------------------------------------------------------------------------------------
    def reset_grids(self):
        for f in self.facets:
            f.grid.grid.zero_()
            f.grid.sumwt.zero_()
            f.grid.sumjones.zero_()
            f.grid.sumjones_chan.zero_()

    def grid_all_facets(self, vs: D.VisData, jones: Optional[D.JonesData] = None, dopsf=False):
        """Grid ``vs`` onto every facet's residual grid (accumulating) in one library call."""
        D.grid(vs, [f.grid for f in self.facets], self.pol, jones, dopsf=dopsf)

    def degrid_all_facets(self, vs: D.VisData, jones: Optional[D.JonesData] = None):
        """Subtract every facet's model prediction from ``vs.vis`` in one library call."""
        D.degrid(vs, [f.model for f in self.facets], self.pol, jones)

    def facets_to_image(self, stream=None) -> torch.Tensor:
        """Dirty image float32 [nband, npol, M, M] from the residual grids (``FacetsToIm``).
        The facet grids are transformed in place, as ``GridToIm`` does."""
        lib = _abi.lib()
        st = D._stream_ptr(stream)
        m = self.npix_out
        image = torch.zeros((self.nband, self.npol, m, m), dtype=torch.float32, device=self.device)
        for f in self.facets:
            n = f.grid.grid.shape[-1]
            _abi.check(lib.ddfg_grid_to_image(self._plan(n), C.c_void_p(f.grid.grid.data_ptr()),
                                              C.c_double(float(self.overs) ** 2),
                                              C.c_void_p(self._work_for(n).data_ptr()), st))
            w = self._norm_weights(f)
            xc, yc = f.geom.pix_central
            _abi.check(lib.ddfg_stitch_facet(C.c_void_p(f.grid.grid.data_ptr()), self.nband, self.npol, n,
                                             C.c_void_p(f.sphe.data_ptr()), C.c_void_p(f.invsphe.data_ptr()),
                                             C.c_void_p(f.sw_grid.data_ptr()), C.c_void_p(w.data_ptr()),
                                             C.c_void_p(image.data_ptr()), m, xc, yc, st))
        if bool((self.facet_norm_host != 0).any()):
            _abi.check(lib.ddfg_image_normalise(C.c_void_p(image.data_ptr()), self.nband * self.npol, m,
                                                C.c_void_p(self.facet_norm.data_ptr()), st))
        return image

    def _norm_weights(self, f):
        """SumWeights[band][pol] * sqrt(SumJonesNorm[band]) (ClassFacetMachine.py:1066-1076, 1385-1391)."""
        sw = f.grid.sumwt
        sj = f.grid.sumjones
        if float(sj.abs().sum().item()) == 0.0:
            norm = torch.ones(self.nband, dtype=torch.float64, device=self.device)
        else:
            den = torch.where(sj[1] == 0, torch.ones_like(sj[1]), sj[1])
            norm = sj[0] / den
            norm = torch.where(norm == 0, torch.ones_like(norm), norm)
        return (sw * torch.sqrt(norm)[:, None]).contiguous()

    def image_to_facets(self, model_image: torch.Tensor, stream=None, out: Optional[List[torch.Tensor]] = None):
        """Every facet's model grid from the model image float32 [nband, npol, M, M]
        (``set_model_grid`` with ``GiveModelTessel(ToGrid=True)``), written into the facets' model
        grids or into ``out`` (one complex64 [nband, npol, N, N] tensor per facet)."""
        lib = _abi.lib()
        st = D._stream_ptr(stream)
        img = model_image.to(self.device, torch.float32).contiguous()
        m = img.shape[-1]
        targets = [f.model.grid for f in self.facets] if out is None else out
        if len(targets) != len(self.facets):
            raise ValueError("one output grid per facet")
        for f, g in zip(self.facets, targets):
            n = f.model.grid.shape[-1]
            if g.shape != f.model.grid.shape or g.dtype != torch.complex64 or not g.is_contiguous():
                raise ValueError(f"output grid must be contiguous complex64 {tuple(f.model.grid.shape)}")
            xc, yc = f.geom.pix_central
            _abi.check(lib.ddfg_image_to_grid(self._plan(n), C.c_void_p(img.data_ptr()), m,
                                              C.c_void_p(self.facet_norm.data_ptr()), C.c_void_p(f.sw_img.data_ptr()),
                                              C.c_void_p(f.sphe.data_ptr()), xc, yc, C.c_double(float(self.overs)),
                                              C.c_void_p(g.data_ptr()), C.c_void_p(self._work_for(n).data_ptr()), st))

    def image_to_facets_adjoint(self, grid_grads: Sequence[torch.Tensor], stream=None) -> torch.Tensor:
        """The adjoint of ``image_to_facets`` with respect to the real model image: the gradient
        float32 [nband, npol, M, M] of a real loss given its gradients with respect to every facet's
        model grid (PyTorch's complex convention), summed over facets."""
        lib = _abi.lib()
        st = D._stream_ptr(stream)
        m = self.npix_out
        if len(grid_grads) != len(self.facets):
            raise ValueError("one grid gradient per facet")
        grad = torch.zeros((self.nband, self.npol, m, m), dtype=torch.float32, device=self.device)
        for f, g in zip(self.facets, grid_grads):
            if g is None:
                continue
            n = f.model.grid.shape[-1]
            g = g.to(self.device, torch.complex64).contiguous()
            if g.shape != f.model.grid.shape:
                raise ValueError(f"grid gradient must have shape {tuple(f.model.grid.shape)}")
            xc, yc = f.geom.pix_central
            _abi.check(lib.ddfg_image_to_grid_adjoint(self._plan(n), C.c_void_p(g.data_ptr()), m,
                                                      C.c_void_p(self.facet_norm.data_ptr()),
                                                      C.c_void_p(f.sw_img.data_ptr()), C.c_void_p(f.sphe.data_ptr()),
                                                      xc, yc, C.c_double(float(self.overs)),
                                                      C.c_void_p(grad.data_ptr()),
                                                      C.c_void_p(self._work_for(n).data_ptr()), st))
        return grad


def _edges(xc, yc, m, n):
    """``GiveEdges(xc, yc, m, n//2, n//2, n)`` (DDFacet/ToolsDir/GiveEdges.py:29-80):
    (x0main, x1main, y0main, y1main, x0facet, x1facet, y0facet, y1facet)."""
    mx0 = xc - n // 2
    x0m = max(0, mx0)
    x0f = x0m - mx0
    mx1 = xc + n // 2
    x1m = min(m - 1, mx1)
    x1f = n - (mx1 - x1m)
    x1m += 1
    my0 = yc - n // 2
    y0m = max(0, my0)
    y0f = y0m - my0
    my1 = yc + n // 2
    y1m = min(m - 1, my1)
    y1f = n - (my1 - y1m)
    y1m += 1
    return x0m, x1m, y0m, y1m, x0f, x1f, y0f, y1f
