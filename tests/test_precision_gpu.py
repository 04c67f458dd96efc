"""Errors of the GPU kernels against the FP64 oracle (oracle/gridder_fp64.c).

The oracle accumulates in complex128 with double products; the GPU path is FP32 with FP64
phase/index arithmetic.  Bounds:
  * gridding: <= 1e-5 relative RMS of the grid and weight sums to 1e-9;
  * degridding: within 2x of the reference's own complex64 error against the same oracle (the
    prediction sums S*S products whose terms cancel, which the reference's float products
    already bound) and <= 1e-4.
Each test prints both errors, so the figures appear in the test log.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [
    dict(),
    dict(ncorr=4, stokes_ids=(1, 2, 3, 4), nw=3, lm=(0.01, -0.005)),
    dict(ncorr=4, stokes_ids=(1,), bda_mode=1, dphi=np.sqrt(6 * 0.05), flag_frac=0.1, nband=2),
])
def test_grid_vs_fp64(kw):
    c = cases.make_case(**kw)
    if kw.get("bda_mode"):
        cases.add_jones(c, mode=1, beam=True)
        c.smear = cases.smear_list(c)
    f = cases.run_fp64_grid(c)
    g = cases.run_gpu_grid(c)
    r = cases.run_ref_grid(c)
    eg, er = cases.rel_rms(g["grid"], f["grid"]), cases.rel_rms(r["grid"], f["grid"])
    print(f"grid rel RMS vs FP64: gpu {eg:.2e}  reference {er:.2e}")
    assert eg < 1e-5
    np.testing.assert_allclose(g["sumwt"], f["sumwt"], rtol=1e-9)


@pytest.mark.parametrize("model", ["point", "dirty"])
def test_degrid_vs_fp64(model):
    c = cases.make_case(ncorr=4, stokes_ids=(1,), nw=3, lm=(0.004, 0.002))
    cases.add_jones(c, mode=1)
    if model == "dirty":
        m = cases.run_ref_grid(c)["grid"]
    else:  # a few point sources on the facet image, taper-corrected and transformed
        rng = np.random.default_rng(11)
        img = np.zeros((c.npix, c.npix), np.complex128)
        for _ in range(8):
            img[rng.integers(40, c.npix - 40), rng.integers(40, c.npix - 40)] = rng.uniform(0.1, 1.0)
        img /= c.wt.ifzfCF.real
        m = np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(img))).astype(np.complex64)[None, None]
    vf = cases.run_fp64_degrid(c, m)
    vg = cases.run_gpu_degrid(c, m)
    vr = cases.run_ref_degrid(c, m)
    eg, er = cases.rel_rms(vg, vf), cases.rel_rms(vr, vf)
    print(f"degrid ({model} model) rel RMS vs FP64: gpu {eg:.2e}  reference {er:.2e}")
    assert eg < max(2 * er, 1e-6) and eg < 1e-4
