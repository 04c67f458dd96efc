"""Differentiable prediction (ddfacet_b200.autograd): the backward kernels against three checks.

* dot-product test: <A x, y> = <x, A^H y> for random model grids x and visibility-space y
  (256 pairs on single-visibility maps, 64 on averaged blocks): norm-wise <= 1e-6 for every pair,
  relative <= 1e-6 in the mean;
* central differences with h = 1e-6 in float64 (numpy FP64 prediction on complex128 inputs) at 64
  coordinates, and the same checks at the benchmark's 81-facet geometry;
* central finite differences of a float64 loss, L = 1/2 sum w |V - P|^2 with P from the FP64
  oracle degridder, at 64 random coordinates of the model grids and of the kMS Jones array
  (perturbations of 2^-10, exactly representable in the float32 inputs; L is a polynomial, so
  the central difference has no step error beyond its own rounding): norm-wise relative
  difference <= 1e-4 against the GPU gradient;
* the reference's own gridder applied to the weighted residuals: for Stokes I from XX/YY the
  gradient of L with respect to a model grid is -2 x the reference gridder's grid of w (V - P)
  (its Stokes I is (XX + YY) / 2), up to the reference's conj(flip(W)) vs W tap difference:
  relative RMS <= 1e-4.
"""
import numpy as np
import pytest
import torch

import cases
from ddfacet_b200 import device as D
from ddfacet_b200.autograd import PredictSetup, predict

pytestmark = pytest.mark.gpu

LMS = [(0.004, -0.002), (-0.006, 0.005)]


# maps: "single" (every block one visibility) or "bda" (DDFacet's mode-1 map with averaged blocks)
MAPS = {"single": {}, "bda": dict(bda_mode=1, dphi=np.sqrt(6 * 0.05))}


def _setup(jones=True, kind="single", jones_mode=1, beam=False, interp_mode=0, apply_amp=1, apply_phase=1, scale=0,
           calib_err=0.0):
    cs = [cases.make_case(seed=17, nant=8, ntimes=12, nchan=8, ncorr=4, stokes_ids=(1,), nw=3, lm=lm, **MAPS[kind])
          for lm in LMS]
    for c in cs[1:]:
        c.vis = cs[0].vis
    if kind == "bda":
        nb = int(np.uint32(cs[0].bda[0]))
        assert cs[0].nrow * cs[0].nchan / nb > 1.5  # the blocks do average
    if jones:
        for i, c in enumerate(cs):
            cases.add_jones(c, mode=jones_mode, nt=3, nd=3, idir=i + 1, beam=beam, interp_mode=interp_mode,
                            apply_amp=apply_amp, apply_phase=apply_phase, scale=scale, calib_err=calib_err)
    objs = [cases._gpu_objs(c) for c in cs]
    setup = PredictSetup(vs=objs[0][0], facets=[o[1] for o in objs], pol=D.make_pol(cs[0].corr_ids, [1]),
                         jones=objs[0][2])
    return cs, setup


def _rand_grids(setup, rng):
    out = []
    for f in setup.facets:
        a = rng.standard_normal(f.grid.shape) + 1j * rng.standard_normal(f.grid.shape)
        out.append(torch.from_numpy(a.astype(np.complex64)).cuda())
    return out


def _vdot(a, b):
    return complex(torch.sum(torch.conj(a.to(torch.complex128)) * b.to(torch.complex128)).item())


def _dot_product_errors(setup, shape_v, rng, npairs):
    """|<y, A x> - <A^H y, x>| over npairs random pairs, in float64, relative to |<y, A x>| and
    norm-wise (relative to ||y|| ||A x||, the Cauchy-Schwarz bound of either product)."""
    kms = setup.jones.kms
    rel, nw = [], []
    for _ in range(npairs):
        x = [g.requires_grad_(True) for g in _rand_grids(setup, rng)]
        y = torch.from_numpy((rng.standard_normal(shape_v) + 1j * rng.standard_normal(shape_v))
                             .astype(np.complex64)).cuda()
        P = predict(setup, x, kms)
        gx = torch.autograd.grad(P, x, grad_outputs=y)
        lhs = _vdot(y, P.detach())
        rhs = sum(_vdot(g, xi.detach()) for g, xi in zip(gx, x))
        rel.append(abs(lhs - rhs) / abs(lhs))
        nw.append(abs(lhs - rhs) / (float(torch.linalg.vector_norm(y.double())) *
                                    float(torch.linalg.vector_norm(P.detach().to(torch.complex128)))))
    return np.array(rel), np.array(nw)


@pytest.mark.parametrize("kind,jones_mode,npairs", [("single", 1, 256), ("bda", 1, 64), ("bda", 2, 64)])
def test_dot_product_adjoint(kind, jones_mode, npairs):
    """Norm-wise <= 1e-6 for every pair.  Relative to the product itself: <= 1e-6 in the mean; the
    largest is stated -- float32 operators give each product a rounding error of ~eps sqrt(n) times
    its terms' size, and a pair whose terms cancel (|<y, A x>| well below ||y|| ||A x||) shows it
    magnified."""
    cs, setup = _setup(jones=True, kind=kind, jones_mode=jones_mode)
    rel, nw = _dot_product_errors(setup, cs[0].vis.shape, np.random.default_rng(0), npairs)
    print(f"dot-product test ({kind}, Jones mode {jones_mode}, {npairs} pairs): norm-wise max {nw.max():.2e}; "
          f"relative mean {rel.mean():.2e} max {rel.max():.2e}")
    assert nw.max() < 1e-6
    assert rel.mean() < 1e-6 and rel.max() < 1e-5


def _np_facets(cs, grids):
    return [dict(grid=g.astype(np.complex128), wplanes=c.wt.Wplanes, wconj=c.wt.WplanesConj, overs=int(c.winfos[3]),
                 ref_wave=c.wt.RefWave, wmax=c.wt.wmax, incr=c.incr, cu=c.wt.Cu, cv=c.wt.Cv, l0=c.lm[0], m0=c.lm[1],
                 idir=c.jones["idir_kms"], idir_beam=c.jones["idir_beam"]) for c, g in zip(cs, grids)]


def _fd_check(bda, uvw, freqs, chan_map, a0, a1, facets, kms, tmap, cmap, V, w, g_grids, g_kms, rng, ncoord, h=1e-6,
              **extra):
    """Central differences of L = 1/2 sum w |V - sum_f P_f|^2 at h (float64 steps on complex128
    grids and Jones) at ncoord random coordinates, half Jones and half model grid, against the GPU
    gradient: norm-wise relative differences (Jones, grids).  ``extra``: beam / interpolation
    arguments of oracle/fp64.py predict_np."""
    from oracle import fp64

    kms = np.asarray(kms, np.complex128)
    Ps = fp64.predict_np(bda, uvw, freqs, chan_map, a0, a1, facets, kms, tmap, cmap, **extra)
    total = sum(Ps)
    wv = np.asarray(w, np.float64)[:, :, None]
    Vd = np.asarray(V, np.complex128)

    def dloss(aff, Pp, Pm):
        """L(+h) - L(-h) without forming L: with r = V - P, |r+|^2 - |r-|^2 = Re[(r+ - r-) conj(r+ + r-)],
        r+ - r- = -(P+ - P-) and r+ + r- = 2 (V - P_others) - (P+ + P-), so the large |V|^2 terms
        never meet the small difference."""
        dp = sum(Pp[i] for i in aff) - sum(Pm[i] for i in aff)
        sp = 2 * (Vd - (total - sum(Ps[i] for i in aff))) - (sum(Pp[i] for i in aff) + sum(Pm[i] for i in aff))
        return 0.5 * float(np.sum(wv * np.real(-dp * np.conj(sp))))

    used_t = np.unique(tmap)
    fd, an = [], []
    for n in range(ncoord):
        imag = bool(rng.integers(2))
        step = 1j * h if imag else h
        if n < ncoord // 2:  # a Jones coordinate of a direction some facet uses
            fi = int(rng.integers(len(facets)))
            d = facets[fi]["idir"]
            idx = (int(rng.choice(used_t)), d, int(rng.integers(0, kms.shape[2])), 0, int(rng.integers(2)),
                   int(rng.integers(2)))
            aff = [i for i, f in enumerate(facets) if f["idir"] == d]
            Pn = []
            for sgn in (1, -1):
                k2 = kms.copy()
                k2[idx] += sgn * step
                Pn.append(fp64.predict_np(bda, uvw, freqs, chan_map, a0, a1, facets, k2, tmap, cmap, only=aff, **extra))
            dl = dloss(aff, Pn[0], Pn[1])
            g = g_kms[idx]
        else:
            fi = int(rng.integers(len(facets)))
            nz = np.argwhere(np.abs(g_grids[fi]) > 0)
            idx = tuple(nz[rng.integers(len(nz))])
            Pn = []
            for sgn in (1, -1):
                f2 = [dict(f) for f in facets]
                gg = f2[fi]["grid"].copy()
                gg[idx] += sgn * step
                f2[fi]["grid"] = gg
                Pn.append(fp64.predict_np(bda, uvw, freqs, chan_map, a0, a1, f2, kms, tmap, cmap, only=[fi], **extra))
            dl = dloss([fi], Pn[0], Pn[1])
            g = g_grids[fi][idx]
        fd.append(dl / (2 * h))
        an.append(g.imag if imag else g.real)
    fd, an = np.array(fd), np.array(an)
    k = ncoord // 2
    return (np.linalg.norm(fd[:k] - an[:k]) / np.linalg.norm(fd[:k]),
            np.linalg.norm(fd[k:] - an[k:]) / np.linalg.norm(fd[k:]))


@pytest.mark.parametrize("kind", ["single", "bda"])
def test_finite_differences_h1e6(kind):
    """Central differences with h = 1e-6 in float64 (complex128 grids and Jones through the numpy
    FP64 prediction, oracle/fp64.py predict_np) at 64 random coordinates -- 32 of the kMS Jones, 32
    of the model grids -- against the GPU gradient: norm-wise <= 1e-5."""
    cs, setup = _setup(jones=True, kind=kind, jones_mode=1)
    rng = np.random.default_rng(11)
    grids = [g.cpu().numpy() * np.float32(0.01) for g in _rand_grids(setup, rng)]
    kms = np.ascontiguousarray(cs[0].jones["kms"], np.complex64)
    V, w = cs[0].vis, cs[0].weights
    gg, gk, _ = _gpu_loss_grads(setup, grids, kms, V, w)
    j = cs[0].jones
    ej, eg = _fd_check(cs[0].bda, cs[0].uvw, cs[0].freqs, cs[0].chan_map, j["A0"], j["A1"], _np_facets(cs, grids), kms,
                       j["kms_tmap"], j["kms_cmap"], V, w, gg, gk, rng, 64)
    print(f"central differences h=1e-6 (FP64, {kind}) vs GPU gradient: Jones {ej:.2e}  grid {eg:.2e}")
    assert ej < 1e-5 and eg < 1e-5


@pytest.mark.parametrize("kind,beam,interp,amp,phase,scale", [
    ("single", True, 0, 1, 1, 0), ("bda", True, 0, 1, 1, 0), ("single", False, 1, 1, 1, 0), ("bda", True, 1, 1, 1, 0),
    ("single", False, 0, 0, 1, 0), ("bda", True, 0, 0, 1, 0), ("single", False, 0, 1, 0, 0),
    ("single", False, 0, 1, 1, 1), ("bda", False, 0, 1, 1, 1), ("bda", True, 0, 0, 1, 1)])
def test_jones_gradient_beam_weighted_normalised(kind, beam, interp, amp, phase, scale):
    """The kMS Jones gradient with a beam (J = K B, the beam held constant), with weighted directions
    (interpolation mode 1) and through the phase-only / amplitude-only normalisation: central
    differences h = 1e-6 in FP64 (oracle/fp64.py predict_np with the same Jones model) at 32
    coordinates, norm-wise <= 1e-5."""
    # a calibration error that gives alpha well inside (0, 1) at these baselines
    ce = 0.3 * 2.998e8 / 1.375e9 / 1500.0 if scale else 0.0
    cs, setup = _setup(jones=True, kind=kind, jones_mode=1, beam=beam, interp_mode=interp, apply_amp=amp,
                       apply_phase=phase, scale=scale, calib_err=ce)
    rng = np.random.default_rng(19)
    grids = [g.cpu().numpy() * np.float32(0.01) for g in _rand_grids(setup, rng)]
    kms = np.ascontiguousarray(cs[0].jones["kms"], np.complex64)
    V, w = cs[0].vis, cs[0].weights
    gg, gk, _ = _gpu_loss_grads(setup, grids, kms, V, w)
    j = cs[0].jones
    extra = {}
    if beam:
        extra.update(beam=j["beam"], beam_tmap=j["beam_tmap"], beam_cmap=j["beam_cmap"])
    if interp:
        extra.update(coefs=j["coefs"])
    extra.update(apply_amp=bool(amp), apply_phase=bool(phase))
    if scale:
        extra.update(scale=True, calib_err=ce, wavelength_mean=float(np.mean(299792458.0 / cs[0].freqs)))
    ej, eg = _fd_check(cs[0].bda, cs[0].uvw, cs[0].freqs, cs[0].chan_map, j["A0"], j["A1"], _np_facets(cs, grids), kms,
                       j["kms_tmap"], j["kms_cmap"], V, w, gg, gk, rng, 32, **extra)
    print(f"central differences h=1e-6 ({kind}, beam={beam}, interp mode {interp}, amp={amp}, phase={phase}, "
          f"scale={scale}) "
          f"vs GPU gradient: "
          f"Jones {ej:.2e}  grid {eg:.2e}")
    assert ej < 1e-5 and eg < 1e-5


def test_config4_geometry():
    """The differentiation checks at the benchmark's multi-facet geometry (81 facets of 735^2, 32
    w-planes, 64 channels, 4 correlations) on two dumps, with a 300-source sky and Jones of sigma
    0.15: dot-product test on 32 pairs (norm-wise <= 1e-6) and central differences (h = 1e-6, FP64)
    at 16 coordinates (<= 1e-5 norm-wise)."""
    from ddfacet_b200 import bda, configs

    w = configs.multifacet_dde(device=torch.device("cuda", 0), scale=0.001, nsrc=300, jones_sigma=0.15)
    setup = PredictSetup(vs=w.vs, facets=w.facets_model, pol=w.pol, jones=w.jones)
    rng = np.random.default_rng(13)
    rel, nw = _dot_product_errors(setup, tuple(w.vs.vis.shape), rng, 32)
    print(f"config-4 geometry ({w.nrow} rows x {w.nchan} ch, 81 facets): dot-product norm-wise max {nw.max():.2e}, "
          f"relative mean {rel.mean():.2e} max {rel.max():.2e}")
    assert nw.max() < 1e-6
    obs = w.host["obs"]
    grids = [(f.grid * 10).cpu().numpy() for f in w.facets_model]
    kms = w.jones.kms.cpu().numpy()
    V = w.vs.vis.cpu().numpy()
    wt = w.vs.weights.cpu().numpy()
    x = [torch.from_numpy(g).cuda().requires_grad_(True) for g in grids]
    k = torch.from_numpy(kms).cuda().requires_grad_(True)
    r = torch.from_numpy(V).cuda() - predict(setup, x, k)
    (0.5 * torch.sum(torch.from_numpy(wt).cuda()[:, :, None] * (r.real ** 2 + r.imag ** 2))).backward()
    facets = [dict(grid=g.astype(np.complex128), wplanes=wtm.Wplanes, wconj=wtm.WplanesConj, overs=11,
                   ref_wave=wtm.RefWave, wmax=wtm.wmax, incr=fm.incr, cu=wtm.Cu, cv=wtm.Cv, l0=fm.l0, m0=fm.m0,
                   idir=fm.idir_kms) for g, wtm, fm in zip(grids, w.host["wterms"], w.facets_model)]
    ej, eg = _fd_check(bda.plain_map(obs.A0, obs.A1, w.nchan), obs.uvw, obs.freqs, w.host["chan_map"], obs.A0, obs.A1,
                       facets, kms, w.jones.kms_tmap.cpu().numpy(), np.zeros(w.nchan, np.int32), V, wt,
                       [xi.grad.cpu().numpy() for xi in x], k.grad.cpu().numpy(), rng, 16)
    print(f"config-4 geometry central differences h=1e-6 vs GPU gradient: Jones {ej:.2e}  grid {eg:.2e}")
    assert ej < 1e-5 and eg < 1e-5


def _oracle_loss(cs, grids, kms, V, w):
    from oracle import fp64
    P = np.zeros(V.shape, np.complex128)
    for c, g in zip(cs, grids):
        j = dict(c.jones)
        j["kms"] = kms
        P -= fp64.degrid(g, np.zeros(V.shape, np.complex64), c.uvw, c.freqs, c.chan_map, c.bda, c.wt.Wplanes,
                         c.wt.WplanesConj, c.winfos[3], c.wt.RefWave, c.wt.wmax, c.incr, c.wt.Cu, c.wt.Cv, c.lm,
                         c.corr_ids, c.stokes_ids, jones=j, smear=c.smear)
    r = V.astype(np.complex128) - P
    return 0.5 * float(np.sum(w[:, :, None] * np.abs(r) ** 2))


def _gpu_loss_grads(setup, grids, kms, V, w):
    x = [torch.from_numpy(g).cuda().requires_grad_(True) for g in grids]
    k = torch.from_numpy(kms).cuda().requires_grad_(True)
    P = predict(setup, x, k)
    r = torch.from_numpy(V).cuda() - P
    loss = 0.5 * torch.sum(torch.from_numpy(w).cuda()[:, :, None] * (r.real ** 2 + r.imag ** 2))
    loss.backward()
    return [xi.grad.cpu().numpy() for xi in x], k.grad.cpu().numpy(), P.detach().cpu().numpy()


@pytest.mark.parametrize("kind,jones_mode", [("single", 1), ("bda", 1), ("bda", 2)])
def test_finite_differences_fp64(kind, jones_mode):
    cs, setup = _setup(jones=True, kind=kind, jones_mode=jones_mode)
    rng = np.random.default_rng(1)
    grids = [g.cpu().numpy() * np.float32(0.01) for g in _rand_grids(setup, rng)]
    kms = np.ascontiguousarray(cs[0].jones["kms"], np.complex64)
    V = cs[0].vis
    w = cs[0].weights
    gg, gk, _ = _gpu_loss_grads(setup, grids, kms, V, w)
    h = np.float32(2.0 ** -10)
    fd, an = [], []
    # 32 Jones coordinates (used slots, directions and antennas) and 32 model-grid coordinates
    used_t = np.unique(cs[0].jones["kms_tmap"])
    for n in range(64):
        coord = "jones" if n < 32 else "grid"
        imag = bool(rng.integers(2))
        if coord == "jones":
            idx = (int(rng.choice(used_t)), int(rng.integers(1, 3)), int(rng.integers(0, cs[0].obs.nant)), 0,
                   int(rng.integers(2)), int(rng.integers(2)))
            base = kms
            g_an = gk[idx]
        else:
            fi = int(rng.integers(len(grids)))
            nz = np.argwhere(np.abs(gg[fi]) > 0)
            idx = tuple(nz[rng.integers(len(nz))])
            base = grids[fi]
            g_an = gg[fi][idx]
        step = (1j * h) if imag else h
        plus, minus = base.copy(), base.copy()
        plus[idx] += np.complex64(step)
        minus[idx] -= np.complex64(step)
        if coord == "jones":
            lp = _oracle_loss(cs, grids, plus, V, w)
            lm = _oracle_loss(cs, grids, minus, V, w)
        else:
            gp = list(grids); gp[fi] = plus
            gm = list(grids); gm[fi] = minus
            lp = _oracle_loss(cs, gp, kms, V, w)
            lm = _oracle_loss(cs, gm, kms, V, w)
        # the step actually taken (x +- h is exact in float32 unless it crosses a power of two)
        d = complex(plus[idx]) - complex(minus[idx])
        fd.append((lp - lm) / (d.imag if imag else d.real))
        an.append(g_an.imag if imag else g_an.real)
    fd, an = np.array(fd), np.array(an)
    ej = np.linalg.norm(fd[:32] - an[:32]) / np.linalg.norm(fd[:32])
    eg = np.linalg.norm(fd[32:] - an[32:]) / np.linalg.norm(fd[32:])
    print(f"finite differences (FP64 oracle, {kind}, Jones mode {jones_mode}) vs GPU gradient: "
          f"Jones {ej:.2e}  grid {eg:.2e}")
    assert ej < 1e-4 and eg < 1e-4


def test_adjoint_matches_reference_gridder_on_residuals():
    cs, setup = _setup(jones=True)
    rng = np.random.default_rng(2)
    grids = [g.cpu().numpy() * np.float32(0.01) for g in _rand_grids(setup, rng)]
    kms = np.ascontiguousarray(cs[0].jones["kms"], np.complex64)
    V = cs[0].vis
    w = cs[0].weights
    gg, _, P = _gpu_loss_grads(setup, grids, kms, V, w)
    for c, g in zip(cs, gg):
        c.vis = np.ascontiguousarray((V - P).astype(np.complex64))
        c.weights = w
        ref = cases.run_ref_grid(c)["grid"]
        e = cases.rel_rms(g, -2.0 * ref)
        print(f"adjoint vs -2 x reference gridder on weighted residuals: {e:.2e}")
        assert e < 1e-4


def test_jones_gradient_needs_kms_jones():
    """The Jones gradient covers kMS Jones with or without a beam, any direction weighting and every
    normalisation (amplitude, phase, amplitude scaling); with beam-only Jones the model-grid
    gradient still works and the library refuses a Jones gradient with its message."""
    import ctypes as C

    from ddfacet_b200 import _abi

    c = cases.make_case(seed=3, bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=8, ncorr=4)
    cases.add_jones(c, mode=1, nt=3, nd=3, kms=False, beam=True)
    vs, fg, jd = cases._gpu_objs(c)
    pol = D.make_pol(c.corr_ids, c.stokes_ids)
    setup = PredictSetup(vs=vs, facets=[fg], pol=pol, jones=jd)
    x = torch.zeros_like(fg.grid).requires_grad_(True)
    (gx,) = torch.autograd.grad(predict(setup, [x], None).abs().sum(), [x])
    assert gx.shape == x.shape
    lib = _abi.lib()
    arr = (_abi.Facet * 1)(fg.struct(degrid=True))
    vss, js = vs.struct(), jd.struct()
    grad = torch.zeros(64, dtype=torch.complex64, device=fg.grid.device)
    rc = lib.ddfg_degrid_jones_grad(C.byref(vss), C.byref(js), C.byref(pol), arr, 1, C.c_void_p(grad.data_ptr()),
                                    None)
    assert rc == _abi.DDFG_EUNSUPPORTED and "kMS" in _abi.last_error()


# ---- the model image as the leaf: image -> facet grids (crop, norm, taper, FFT) -> prediction ----

def _image_problem(kind, seed=21):
    from ddfacet_b200 import bda, geometry, synth
    from ddfacet_b200.facetmachine import FacetMachine

    npix = 600
    obs = synth.make_observation(seed, 8, 2000.0, 34.0, 40.0, 12 * 30.0 / 3600.0, 30.0, 8, 1.30e9, 1.45e9)
    wmax = float(np.max(np.abs(obs.uvw[:, 2]))) * 1.01
    tess = None
    if kind == "voronoi":
        r = npix * 6.0 / 3600 * np.pi / 180 / 2
        rng = np.random.default_rng(seed)
        tess = geometry.voronoi_facets(npix, 6.0, rng.uniform(-0.8 * r, 0.8 * r, 4), rng.uniform(-0.8 * r, 0.8 * r, 4),
                                       1.7)
    fm = FacetMachine(npix, 6.0, 2, obs.freqs, padding=1.7, nband=1, stokes_ids=(1,), corr_ids=(9, 10, 11, 12),
                      support=7, nw=3, wmax=wmax, mixing_width=10.0, tessellation=tess)
    dev = fm.device
    vis = np.zeros((obs.nrow, obs.freqs.size, 4), np.complex64)
    vs = D.VisData.create(vis, obs.uvw, np.zeros(vis.shape, bool), np.ones((obs.nrow, obs.freqs.size), np.float32),
                          obs.freqs, np.zeros(obs.freqs.size, np.int32), bda.plain_map(obs.A0, obs.A1, obs.freqs.size),
                          device=dev)
    nd = len(fm.facets)
    t = obs.times
    tmap = np.minimum(((t - t.min()) / (t.max() - t.min() + 1e-9) * 3).astype(np.int32), 2)
    kms = torch.from_numpy(synth.random_jones(seed + 1, 3, nd, obs.nant, 1, 0.1)).to(dev)
    jd = D.JonesData(mode=1, kms=kms, kms_tmap=torch.from_numpy(tmap).to(dev),
                     kms_cmap=torch.zeros(obs.freqs.size, dtype=torch.int32, device=dev),
                     a0=torch.from_numpy(obs.A0.astype(np.int32)).to(dev),
                     a1=torch.from_numpy(obs.A1.astype(np.int32)).to(dev),
                     wavelength_mean=float(np.mean(299792458.0 / obs.freqs)))
    return fm, vs, jd


@pytest.mark.parametrize("kind", ["regular", "voronoi"])
def test_image_to_grid_adjoint_matches_oracle(kind):
    """ddfg_image_to_grid_adjoint summed over facets against the FP64 restatement of the adjoint
    (oracle/facets.py give_model_tessel_adjoint): 1e-5 relative RMS."""
    from oracle import facets as OF

    fm, _, _ = _image_problem(kind)
    rng = np.random.default_rng(3)
    ys = [torch.from_numpy((rng.standard_normal(f.model.grid.shape) + 1j * rng.standard_normal(f.model.grid.shape))
                           .astype(np.complex64)).cuda() for f in fm.facets]
    got = fm.image_to_facets_adjoint(ys).cpu().numpy()
    want = np.zeros(got.shape, np.float64)
    for f, y in zip(fm.facets, ys):
        want += OF.give_model_tessel_adjoint(y.cpu().numpy(), fm.facet_norm_host, f.sphe.cpu().numpy(), f.sw_host,
                                             *f.geom.pix_central, fm.npix_out, fm.overs)
    e = cases.rel_rms(got, want)
    print(f"image adjoint vs FP64 oracle ({kind}): {e:.2e}")
    assert e < 1e-5


def test_image_leaf_dot_product_256_pairs():
    """<y, P(x)> = <x, A^H y> for the whole chain real image x -> facet grids -> prediction with
    per-facet Jones, over 256 random pairs: relative difference <= 1e-6 in the mean, 1e-5 for any
    pair (float64 inner products of the float32 results).  For a real leaf the backward pass gives
    Re(A^H y) = d Re<y, P>/dx; the imaginary part comes from a second backward pass with i y
    (Re<i y, P> = Im<y, P>), so the complex products are compared as in the model-grid test."""
    from ddfacet_b200.autograd import model_grids, predict, setup_from_facet_machine

    fm, vs, jd = _image_problem("voronoi")
    setup = setup_from_facet_machine(fm, vs, jd)
    rng = np.random.default_rng(5)
    shape = (fm.nband, fm.npol, fm.npix_out, fm.npix_out)
    errs = []
    for _ in range(256):
        x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda().requires_grad_(True)
        y = torch.from_numpy((rng.standard_normal(vs.vis.shape) + 1j * rng.standard_normal(vs.vis.shape))
                             .astype(np.complex64)).cuda()
        P = predict(setup, model_grids(fm, x), jd.kms)
        (gr,) = torch.autograd.grad(P, [x], grad_outputs=y, retain_graph=True)
        (gi,) = torch.autograd.grad(P, [x], grad_outputs=1j * y)
        lhs = _vdot(y, P.detach())
        xd = x.detach().double()
        rhs = complex(float(torch.sum(gr.double() * xd).item()), float(torch.sum(gi.double() * xd).item()))
        errs.append(abs(lhs - rhs) / abs(lhs))
    print(f"image-leaf dot-product test: mean rel {np.mean(errs):.2e}  max {np.max(errs):.2e}")
    assert np.mean(errs) < 1e-6 and np.max(errs) < 1e-5


def test_image_leaf_gradient_is_adjoint_of_grid_gradient():
    """dL/dimage = Re(A^H dL/dgrids): the image gradient of L = 1/2 sum w |V - P|^2 through the
    facet machine equals the oracle adjoint applied to the grid gradients (1e-5 relative RMS), and
    the Jones gradient is the same whether the grids or the image are the leaf."""
    from oracle import facets as OF
    from ddfacet_b200.autograd import model_grids, predict, setup_from_facet_machine

    fm, vs, jd = _image_problem("regular")
    setup = setup_from_facet_machine(fm, vs, jd)
    rng = np.random.default_rng(9)
    img = np.zeros((fm.nband, fm.npol, fm.npix_out, fm.npix_out), np.float32)
    img[0, 0, rng.integers(0, fm.npix_out, 20), rng.integers(0, fm.npix_out, 20)] = rng.uniform(0.1, 1.0, 20)
    V = torch.from_numpy((rng.standard_normal(vs.vis.shape) + 1j * rng.standard_normal(vs.vis.shape))
                         .astype(np.complex64)).cuda() * 0.01
    w = vs.weights

    def loss_of(P):
        r = V - P
        return 0.5 * torch.sum(w[:, :, None] * (r.real ** 2 + r.imag ** 2))

    x = torch.from_numpy(img).cuda().requires_grad_(True)
    k1 = jd.kms.clone().requires_grad_(True)
    loss_of(predict(setup, model_grids(fm, x), k1)).backward()
    grids = [g.detach().requires_grad_(True) for g in model_grids(fm, torch.from_numpy(img).cuda())]
    k2 = jd.kms.clone().requires_grad_(True)
    loss_of(predict(setup, grids, k2)).backward()
    want = np.zeros(img.shape, np.float64)
    for f, g in zip(fm.facets, grids):
        want += OF.give_model_tessel_adjoint(g.grad.cpu().numpy(), fm.facet_norm_host, f.sphe.cpu().numpy(), f.sw_host,
                                             *f.geom.pix_central, fm.npix_out, fm.overs)
    e = cases.rel_rms(x.grad.cpu().numpy(), want)
    print(f"image gradient vs oracle adjoint of the grid gradients: {e:.2e}")
    assert e < 1e-5
    assert cases.rel_rms(k1.grad.cpu().numpy(), k2.grad.cpu().numpy()) < 1e-6


def test_model_grids_checks_shape():
    from ddfacet_b200.autograd import model_grids

    fm, _, _ = _image_problem("regular")
    with pytest.raises(ValueError, match="model image must be"):
        model_grids(fm, torch.zeros((1, 1, 10, 10), device="cuda"))
    with pytest.raises(ValueError, match="real"):
        model_grids(fm, torch.zeros((1, 1, fm.npix_out, fm.npix_out), dtype=torch.complex64, device="cuda"))
