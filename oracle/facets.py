"""NumPy restatements of the per-facet transforms and the stitching (test infrastructure only).

Each function follows the reference line by line in float64/complex128 where the reference uses
NumPy, so the GPU kernels (cuFFT + fused passes) can be compared with it:
  * grid_to_im          -- ClassDDEGridMachine.GridToIm (ClassDDEGridMachine.py:1186-1190) with
                           FFTW_2Donly_np.ifft (ModFFTW.py:631-648);
  * facets_to_im_channel-- ClassFacetMachine.FacetsToIm_Channel (ClassFacetMachine.py:1331-1416);
  * facet_norm          -- ClassFacetMachine.BuildFacetNormImage (ClassFacetMachine.py:1289-1330);
  * give_model_tessel   -- ClassImToGrid.GiveModelTessel(ToGrid=True) (ClassImToGrid.py:138-264)
                           with FFTW_2Donly_np.fft (ModFFTW.py:611-629);
  * give_model_tessel_adjoint -- the adjoint of give_model_tessel with respect to the real model
                           image (no reference counterpart), each step of the forward undone in
                           reverse order in float64.
"""
import numpy as np


def give_edges(xc, yc, n0, n1):
    """GiveEdges(xc, yc, N0, N1//2, N1//2, N1) (GiveEdges.py:29-80)."""
    mx0 = xc - n1 // 2
    x0m = max(0, mx0)
    x0f = x0m - mx0
    mx1 = xc + n1 // 2
    x1m = min(n0 - 1, mx1)
    x1f = n1 - (mx1 - x1m)
    x1m += 1
    my0 = yc - n1 // 2
    y0m = max(0, my0)
    y0f = y0m - my0
    my1 = yc + n1 // 2
    y1m = min(n0 - 1, my1)
    y1f = n1 - (my1 - y1m)
    y1m += 1
    return (x0m, x1m, y0m, y1m), (x0f, x1f, y0f, y1f)


def grid_to_im(grid, overs):
    g = np.asarray(grid, np.complex128) * overs ** 2
    out = np.empty_like(g)
    for ich in range(g.shape[0]):
        for ipol in range(g.shape[1]):
            b = np.fft.ifftshift(g[ich, ipol])
            b = np.fft.ifft2(b)
            out[ich, ipol] = np.fft.fftshift(b) * (g.shape[-1] * g.shape[-2])
    return out


def facets_to_im_channel(dirties, sphes, invsphes, sws_img, weights, pix_centrals, npix_out, facet_norm):
    """dirties[f]: complex [nband, npol, N, N]; sws_img[f]: SW as stored (image orientation);
    weights[f]: [nband, npol] = SumWeights * sqrt(SumJonesNorm)."""
    nband, npol = dirties[0].shape[:2]
    image = np.zeros((nband, npol, npix_out, npix_out), np.float32)
    for d, sphe, inv, sw, w, (xc, yc) in zip(dirties, sphes, invsphes, sws_img, weights, pix_centrals):
        n = d.shape[-1]
        spw = sw.T[::-1, :]
        (x0m, x1m, y0m, y1m), (x0f, x1f, y0f, y1f) = give_edges(xc, yc, npix_out, n)
        for ch in range(nband):
            for pol in range(npol):
                im = d[ch, pol].real.astype(np.float32).copy()
                ww = w[ch, pol]
                ww = ww if ww != 0 else 1.0
                im = (im.astype(np.float64) * inv.astype(np.float64) * spw.astype(np.float64) / ww).astype(np.float32)
                im[sphe < 1e-3] = 0
                im = im[::-1, :].T[x0f:x1f, y0f:y1f]
                image[ch, pol, x0m:x1m, y0m:y1m] += im
    if (facet_norm != 0).any():
        image /= facet_norm
    return image


def facet_norm(sws_img, pix_centrals, sizes, npix_out):
    """BuildFacetNormImage (ClassFacetMachine.py:1289-1330): the sum of the facets' spatial
    weights (image orientation) placed with GiveEdges, float32."""
    norm = np.zeros((npix_out, npix_out), np.float32)
    for sw, (xc, yc), n in zip(sws_img, pix_centrals, sizes):
        (x0m, x1m, y0m, y1m), (x0f, x1f, y0f, y1f) = give_edges(xc, yc, npix_out, n)
        norm[x0m:x1m, y0m:y1m] += np.real(np.asarray(sw)[x0f:x1f, y0f:y1f])
    return norm


def give_model_tessel(image, norm_im, sphe, sw_img, xc, yc, n, overs, transform=True):
    """With ``transform=False`` returns the scaled facet model before the FFT, which is what the
    reference returns for a facet whose normalised model has no positive pixel (SumFlux == 0,
    ClassImToGrid.py:249-256)."""
    nch, npol, npix_out, _ = image.shape
    (x0d, x1d, y0d, y1d), (x0p, x1p, y0p, y1p) = give_edges(xc, yc, npix_out, n)
    model = np.zeros((nch, npol, n, n), np.float32)
    for ch in range(nch):
        for pol in range(npol):
            model[ch, pol][x0p:x1p, y0p:y1p] = image[ch, pol][x0d:x1d, y0d:y1d].real
            model[ch, pol][x0p:x1p, y0p:y1p] /= norm_im[x0d:x1d, y0d:y1d].real
            model[ch, pol][x0p:x1p, y0p:y1p] *= sw_img[x0p:x1p, y0p:y1p]
            model[ch, pol][x0p:x1p, y0p:y1p] /= sphe[x0p:x1p, y0p:y1p].real
            model[ch, pol][sphe < 1e-3] = 0
            model[ch, pol] = model[ch, pol].T[::-1, :]
    model *= np.float32((overs * n) ** 2)
    if not transform:
        return model.astype(np.complex128)
    out = np.zeros(model.shape, np.complex128)
    for ch in range(nch):
        for pol in range(npol):
            b = np.fft.ifftshift(model[ch, pol].astype(np.complex128))
            b = np.fft.fft2(b)
            out[ch, pol] = np.fft.fftshift(b) / (n * n)
    return out


def give_model_tessel_adjoint(grid_grad, norm_im, sphe, sw_img, xc, yc, npix_out, overs):
    """Re(A^H y) for A = give_model_tessel(., norm_im, sphe, sw_img, xc, yc, n, overs) acting on a
    real image [nch, npol, M, M]; y is complex [nch, npol, n, n]. Returns float64 [nch, npol, M, M]."""
    y = np.asarray(grid_grad, np.complex128)
    nch, npol, n, _ = y.shape
    (x0d, x1d, y0d, y1d), (x0p, x1p, y0p, y1p) = give_edges(xc, yc, npix_out, n)
    out = np.zeros((nch, npol, npix_out, npix_out), np.float64)
    mask = np.asarray(sphe) < 1e-3
    for ch in range(nch):
        for pol in range(npol):
            b = np.fft.ifftshift(y[ch, pol]) / (n * n)       # adjoint of fftshift(.) / n^2
            b = np.fft.ifft2(b) * (n * n)                    # adjoint of the unnormalised fft2
            b = np.fft.fftshift(b) * float(overs * n) ** 2   # adjoint of ifftshift, then the scale
            b = b[::-1, :].T                                 # adjoint of .T[::-1, :]
            b = np.where(mask, 0, b.real)
            box = b[x0p:x1p, y0p:y1p] / np.asarray(norm_im, np.float64)[x0d:x1d, y0d:y1d]
            box = box * np.asarray(sw_img, np.float64)[x0p:x1p, y0p:y1p] / np.asarray(sphe, np.float64)[x0p:x1p, y0p:y1p]
            out[ch, pol, x0d:x1d, y0d:y1d] += box
    return out
