"""Differentiable prediction (ddfacet_b200.autograd): the backward kernels against three checks.

* dot-product test: <A x, y> = <x, A^H y> for random model grids x and visibility-space y
  (32 pairs), relative difference <= 1e-6 in the mean and 1e-5 for any pair;
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


def _setup(jones=True):
    cs = [cases.make_case(seed=17, nant=8, ntimes=12, nchan=8, ncorr=4, stokes_ids=(1,), nw=3, lm=lm) for lm in LMS]
    for c in cs[1:]:
        c.vis = cs[0].vis
    if jones:
        for i, c in enumerate(cs):
            cases.add_jones(c, mode=1, nt=3, nd=3, idir=i + 1)
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


def test_dot_product_adjoint():
    cs, setup = _setup(jones=True)
    rng = np.random.default_rng(0)
    kms = setup.jones.kms
    errs = []
    for _ in range(32):
        x = [g.requires_grad_(True) for g in _rand_grids(setup, rng)]
        y = torch.from_numpy((rng.standard_normal(cs[0].vis.shape) +
                              1j * rng.standard_normal(cs[0].vis.shape)).astype(np.complex64)).cuda()
        P = predict(setup, x, kms)
        gx = torch.autograd.grad(P, x, grad_outputs=y)
        lhs = _vdot(y, P.detach())
        rhs = sum(_vdot(g, xi.detach()) for g, xi in zip(gx, x))
        errs.append(abs(lhs - rhs) / abs(lhs))
    print(f"dot-product test: mean rel {np.mean(errs):.2e}  max {np.max(errs):.2e}")
    assert np.mean(errs) < 1e-6 and np.max(errs) < 1e-5


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


def test_finite_differences_fp64():
    cs, setup = _setup(jones=True)
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
        kind = "jones" if n < 32 else "grid"
        imag = bool(rng.integers(2))
        if kind == "jones":
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
        if kind == "jones":
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
    print(f"finite differences (FP64 oracle) vs GPU gradient: Jones {ej:.2e}  grid {eg:.2e}")
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


def test_unsupported_maps_raise():
    c = cases.make_case(seed=3, bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=8)
    vs, fg, jd = cases._gpu_objs(c)
    setup = PredictSetup(vs=vs, facets=[fg], pol=D.make_pol(c.corr_ids, c.stokes_ids), jones=None)
    x = torch.zeros_like(fg.grid).requires_grad_(True)
    P = predict(setup, [x])
    with pytest.raises(ValueError, match="one visibility"):
        P.abs().sum().backward()
