"""FP64 direct Fourier transforms -- test infrastructure only (the "direct-DFT oracle").

* ``predict(uvw, freqs, l, m, s)``: V(row, chan) = sum_k S_k exp(+2 pi i (u l_k + v m_k + w (n_k - 1)) nu / c),
  the sign convention of the reference's own check (ClassDDEGridMachine.py:264-272, testGrid; the
  degridder subtracts, so its output for zero input visibilities is -V).
* ``dirty(uvw, freqs, vis, weights, l, m)``: the weighted direct dirty image at arbitrary (l, m),
  I(l, m) = Re sum_rc w V exp(-2 pi i (u l + v m + w (n - 1)) nu / c) / sum_rc w.

Both evaluate every term in float64 numpy, row-chunked; they state the error of the W-projection
grid/degrid path against the exact transform (tests/test_dft_gpu.py).  Not used by the product.
"""
from __future__ import annotations

import numpy as np

C_LIGHT = 299792458.0


def predict(uvw, freqs, l, m, s, chunk=2048):
    uvw = np.asarray(uvw, np.float64)
    l = np.atleast_1d(np.asarray(l, np.float64))
    m = np.atleast_1d(np.asarray(m, np.float64))
    s = np.atleast_1d(np.asarray(s, np.float64))
    n1 = np.sqrt(1.0 - l ** 2 - m ** 2) - 1.0
    k = np.asarray(freqs, np.float64) / C_LIGHT
    out = np.zeros((uvw.shape[0], k.size), np.complex128)
    for r0 in range(0, uvw.shape[0], chunk):
        u = uvw[r0:r0 + chunk]
        ph = u[:, 0:1] * l[None] + u[:, 1:2] * m[None] + u[:, 2:3] * n1[None]          # [r][src] metres
        out[r0:r0 + chunk] = np.einsum("s,rsc->rc", s, np.exp(2j * np.pi * ph[:, :, None] * k[None, None, :]))
    return out


def dirty(uvw, freqs, vis, weights, l, m, chunk=2048):
    uvw = np.asarray(uvw, np.float64)
    l = np.atleast_1d(np.asarray(l, np.float64))
    m = np.atleast_1d(np.asarray(m, np.float64))
    n1 = np.sqrt(1.0 - l ** 2 - m ** 2) - 1.0
    k = np.asarray(freqs, np.float64) / C_LIGHT
    vis = np.asarray(vis, np.complex128)
    w = np.asarray(weights, np.float64)
    acc = np.zeros(l.size, np.float64)
    for r0 in range(0, uvw.shape[0], chunk):
        u = uvw[r0:r0 + chunk]
        ph = u[:, 0:1] * l[None] + u[:, 1:2] * m[None] + u[:, 2:3] * n1[None]          # [r][pix]
        e = np.exp(-2j * np.pi * ph[:, :, None] * k[None, None, :])                       # [r][pix][c]
        acc += np.real(np.einsum("rc,rpc->p", w[r0:r0 + chunk] * vis[r0:r0 + chunk], e))
    return acc / w.sum()
