"""The drop-in ClassDDEGridMachine (numpy in, numpy out) against the reference's gridder and
degridder called with the same tables, the way ClassDDEGridMachine.put/get call them.

Tolerances as the kernel parity tests: 1e-4 relative RMS on grids and predictions, identical
touched-cell sets, 1e-9 relative on weight sums, 1e-5 on Jones sums; the cuFFT transforms within
1e-5 relative RMS of numpy's FFT in float64.
"""
import numpy as np
import pytest
import torch

import cases
from ddfacet_b200.gridmachine import ClassDDEGridMachine, default_gd

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _machine(c, stokes=(1,), bda_jones=0, interp="Nearest", nw=3):
    GD = default_gd()
    GD["Image"]["Cell"] = c.cell
    GD["CF"]["Nw"] = nw
    GD["Comp"]["BDAJones"] = bda_jones
    GD["DDESolutions"]["Type"] = interp
    wmax = float(np.max(np.abs(c.uvw[:, 2]))) * 1.01
    gm = ClassDDEGridMachine(GD, c.freqs, c.npix, lmShift=c.lm, compute_cf=True, wmax=wmax, bda_grid=c.bda,
                             bda_degrid=c.bda, DataCorrelationFormat=c.corr_ids, ExpectedOutputStokes=list(stokes),
                             NFreqBands=c.nband, Padding=1.0)
    # the oracle is called with the machine's own tables and geometry
    c.wt = gm.WTerm
    c.npix = gm.Npix
    c.incr = gm.incr
    c.winfos = np.array([gm.WTerm.RefWave, gm.WTerm.wmax, len(gm.WTerm.Wplanes), gm.OverS], np.float64)
    c.facet_infos = np.array([gm.WTerm.Cu, gm.WTerm.Cv, c.lm[0], c.lm[1], 0], np.float64)
    return gm


def _dico(c, lm):
    j = c.jones
    nd = j["kms"].shape[1]
    l = np.linspace(-0.05, 0.05, nd)
    m = np.zeros(nd)
    l[j["idir_kms"]], m[j["idir_kms"]] = lm
    return {"DicoJones_killMS": {"Dirs": {"l": l, "m": m, "I": np.ones(nd)},
                                 "Jones": {"Jones": np.ascontiguousarray(j["kms"], np.complex64),
                                           "VisToJonesChanMapping": j["kms_cmap"]},
                                 "TimeMapping": j["kms_tmap"]}}


def _case(jones=False, **kw):
    args = dict(seed=31, nant=8, ntimes=16, nchan=8, ncorr=4, npix=255, cell_arcsec=6.0, nw=3, bda_mode=1,
                dphi=np.sqrt(6 * 0.05), flag_frac=0.05, lm=(0.01, -0.004))
    args.update(kw)
    c = cases.make_case(**args)
    if jones:
        cases.add_jones(c, mode=1, nt=3, nd=3, idir=1)
    return c


@pytest.mark.parametrize("jones", [False, True])
def test_put_matches_reference(jones):
    c = _case(jones=jones)
    gm = _machine(c)
    grid = np.zeros(gm.GridShape, np.complex64)
    dico = _dico(c, c.lm) if jones else None
    gm.put(c.obs.times, c.uvw, c.vis, c.flags, (c.obs.A0.astype(np.int32), c.obs.A1.astype(np.int32)), W=c.weights,
           DicoJonesMatrices=dico, freqs=c.freqs, ChanMapping=c.chan_map, ResidueGrid=grid)
    r = cases.run_ref_grid(c)
    assert cases.rel_rms(grid, r["grid"]) < TOL
    np.testing.assert_array_equal(grid != 0, r["grid"] != 0)
    np.testing.assert_allclose(gm.SumWeigths, r["sumwt"], rtol=1e-9)
    if jones:
        np.testing.assert_allclose(gm.SumJones, r["sumjones"], rtol=1e-5)
        np.testing.assert_allclose(gm.SumJonesChan, r["sumjones_chan"], rtol=1e-5)
    # a second put accumulates into the grid and the weight sums
    g1, s1 = grid.copy(), gm.SumWeigths.copy()
    gm.put(c.obs.times, c.uvw, c.vis, c.flags, (c.obs.A0.astype(np.int32), c.obs.A1.astype(np.int32)), W=c.weights,
           DicoJonesMatrices=dico, freqs=c.freqs, ChanMapping=c.chan_map, ResidueGrid=grid)
    assert cases.rel_rms(grid, 2 * g1) < 1e-6
    np.testing.assert_allclose(gm.SumWeigths, 2 * s1, rtol=1e-12)


@pytest.mark.parametrize("jones", [False, True])
def test_get_matches_reference(jones):
    c = _case(jones=jones)
    gm = _machine(c)
    model = cases.run_ref_grid(c)["grid"]
    dico = _dico(c, c.lm) if jones else None
    vis = c.vis.copy()
    out = gm.get(c.obs.times, c.uvw, vis, c.flags, (c.obs.A0.astype(np.int32), c.obs.A1.astype(np.int32)), model,
                 DicoJonesMatrices=dico, freqs=c.freqs, ImToGrid=False, ChanMapping=c.chan_map)
    assert out is vis  # subtracted in place, as the reference does
    vr = cases.run_ref_degrid(c, model, vis0=c.vis)
    assert cases.rel_rms(c.vis - vis, c.vis - vr) < TOL


def test_get_accepts_device_tensors():
    c = _case()
    gm = _machine(c)
    model = cases.run_ref_grid(c)["grid"]
    dev = torch.device("cuda", 0)
    vis = torch.from_numpy(c.vis.copy()).to(dev)
    out = gm.get(c.obs.times, torch.from_numpy(c.uvw).to(dev), vis, torch.from_numpy(c.flags).to(dev),
                 (c.obs.A0.astype(np.int32), c.obs.A1.astype(np.int32)), torch.from_numpy(model).to(dev),
                 freqs=c.freqs, ImToGrid=False, ChanMapping=c.chan_map)
    assert out.data_ptr() == vis.data_ptr()
    vr = cases.run_ref_degrid(c, model, vis0=c.vis)
    assert cases.rel_rms(c.vis - vis.cpu().numpy(), c.vis - vr) < TOL


def _np_fft(a):
    return np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(a, axes=(-1, -2))), axes=(-1, -2)) / (a.shape[-1] * a.shape[-2])


def _np_ifft(a):
    return np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(a, axes=(-1, -2))), axes=(-1, -2)) * (a.shape[-1] * a.shape[-2])


def test_fft_machine_and_grid_to_im():
    c = _case(nchan=8)
    c.nband = 2
    c.chan_map = (np.arange(8) * 2 // 8).astype(np.int32)
    gm = _machine(c, stokes=(1, 2))
    rng = np.random.default_rng(4)
    a = (rng.standard_normal(gm.GridShape) + 1j * rng.standard_normal(gm.GridShape)).astype(np.complex64)
    f = gm.getFFTWMachine().fft(a.copy())
    assert cases.rel_rms(f, _np_fft(a.astype(np.complex128))) < 1e-5
    g = a.copy()
    d = gm.GridToIm(g)
    assert d is g
    assert cases.rel_rms(d, _np_ifft(a.astype(np.complex128) * gm.OverS ** 2)) < 1e-5


def test_get_model_image_paths():
    """ImToGrid=True (image -> padded, tapered, transformed grid) and TranformModelInput='FT' give the
    grids that the degridder is then fed, so each equals a get() on that grid."""
    c = _case(ncorr=1, corr_ids=[1], stokes_ids=(1,))
    gm = _machine(c)
    rng = np.random.default_rng(8)
    n = gm.NonPaddedNpix
    img = np.zeros((1, 1, n, n), np.float32)
    img[0, 0, rng.integers(0, n, 6), rng.integers(0, n, 6)] = 1.0
    A = (c.obs.A0.astype(np.int32), c.obs.A1.astype(np.int32))
    v_img = gm.get(c.obs.times, c.uvw, c.vis.copy(), c.flags, A, img, freqs=c.freqs, ImToGrid=True,
                   ChanMapping=c.chan_map)
    x0, x1 = gm.PaddingInnerCoord
    pad = np.zeros(gm.GridShape, np.complex128)
    pad[:, :, x0:x1, x0:x1] = img
    corr = (pad * (gm.OverS * gm.Padding) ** 2).real / gm.ifzfCF.real
    grid = (_np_fft(corr) * n ** 2).astype(np.complex64)
    vr = cases.run_ref_degrid(c, grid, vis0=c.vis)
    assert cases.rel_rms(c.vis - v_img, c.vis - vr) < 1e-4
    big = np.zeros(gm.GridShape, np.complex64)
    big[0, 0, gm.Npix // 2 + 3, gm.Npix // 2 - 2] = 1.0
    v_ft = gm.get(c.obs.times, c.uvw, c.vis.copy(), c.flags, A, big, freqs=c.freqs, ImToGrid=False,
                  TranformModelInput="FT", ChanMapping=c.chan_map)
    vr = cases.run_ref_degrid(c, _np_fft(big.astype(np.complex128)).astype(np.complex64), vis0=c.vis)
    assert cases.rel_rms(c.vis - v_ft, c.vis - vr) < 1e-4
    # an all-zero model returns the visibilities untouched
    v0 = c.vis.copy()
    assert gm.get(c.obs.times, c.uvw, v0, c.flags, A, np.zeros_like(img), freqs=c.freqs) is v0
    np.testing.assert_array_equal(v0, c.vis)
