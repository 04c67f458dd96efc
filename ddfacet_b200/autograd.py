"""Differentiable visibility prediction: degridding as a ``torch.autograd.Function``.

``predict(setup, model_grids, jones_kms)`` returns the model visibilities
``P = sum_f Degrid_f(G_f)`` (complex64 ``[nrow][nchan][ncorr]``) that ``ddfg_degrid`` would
subtract.  Its backward pass runs the library's hand-written adjoint kernels:

* ``ddfg_degrid_adjoint`` -- dLoss/dG_f for every facet's model grid (the exact adjoint of the
  prediction: conjugated CF taps at the degridder's footprint, adjoint Stokes map, conjugated
  phasor, J0^H g J1);
* ``ddfg_degrid_jones_grad`` -- dLoss/dJ for the per-facet, per-antenna kMS Jones terms.

``model_grids(fm, image)`` makes every facet's model grid from a model image (the facet machine's
``image_to_facets``: crop, facet norm, spatial weight, taper correction, FFT) differentiably, its
backward being ``ddfg_image_to_grid_adjoint``; composed with ``predict`` it gives the model image
as a leaf tensor.

Gradients follow PyTorch's complex convention (for a real loss, ``z.grad`` is
dLoss/dRe z + i dLoss/dIm z).  Phases, smearing factors and Jones products are recomputed in the
backward kernels from the same inputs rather than stored.  Supported: every BDA map (blocks of
one visibility or averaged, per-visibility or per-block Jones); for the Jones gradient, kMS Jones
alone or times a beam (the beam is held constant), nearest or weighted directions, through every
normalisation of the reference's Jones server (amplitude, phase, amplitude scaling).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence

import torch

from . import _abi, device as D


@dataclasses.dataclass
class PredictSetup:
    """The fixed inputs of a prediction: visibility geometry (its ``vis`` is not read), facets
    (CF tables and geometry; their ``grid`` is replaced by the model grids), polarisation and the
    Jones metadata (its ``kms`` is replaced by the Jones tensor)."""
    vs: D.VisData
    facets: List[D.FacetGrid]
    pol: object
    jones: Optional[D.JonesData] = None


def setup_from_facet_machine(fm, vs: D.VisData, jones: Optional[D.JonesData] = None) -> PredictSetup:
    """A prediction over every facet of a ``FacetMachine`` (its model facets' CF tables and
    geometry, its polarisation)."""
    return PredictSetup(vs=vs, facets=[f.model for f in fm.facets], pol=fm.pol, jones=jones)


def _facets_with(setup: PredictSetup, grids: Sequence[torch.Tensor]):
    return [dataclasses.replace(f, grid=g, sumwt=None, sumjones=None, sumjones_chan=None)
            for f, g in zip(setup.facets, grids)]


def _jones_with(setup: PredictSetup, kms: Optional[torch.Tensor]):
    if setup.jones is None:
        return None
    return dataclasses.replace(setup.jones, kms=kms) if kms is not None else setup.jones


class _Predict(torch.autograd.Function):
    @staticmethod
    def forward(ctx, setup: PredictSetup, kms, *grids):
        grids = [g.contiguous() for g in grids]
        out = torch.zeros_like(setup.vs.vis)
        vs = dataclasses.replace(setup.vs, vis=out)
        D.degrid(vs, _facets_with(setup, grids), setup.pol, _jones_with(setup, kms))
        ctx.setup = setup
        ctx.save_for_backward(kms if kms is not None else torch.empty(0), *grids)
        ctx.has_kms = kms is not None
        return out.neg_()  # ddfg_degrid subtracted the prediction from zeros

    @staticmethod
    def backward(ctx, grad_out):
        setup = ctx.setup
        saved = ctx.saved_tensors
        kms = saved[0] if ctx.has_kms else None
        grids = saved[1:]
        lib = _abi.lib()
        g = grad_out.to(torch.complex64).contiguous()
        vs = dataclasses.replace(setup.vs, vis=g)
        vss = vs.struct()
        jd = _jones_with(setup, kms)
        js = (jd or D.JonesData()).struct()
        grad_grids = [None] * len(grids)
        if any(ctx.needs_input_grad[2:]):
            gg = [torch.zeros_like(x) for x in grids]
            arr = (_abi.Facet * max(1, len(gg)))(*[f.struct(degrid=True) for f in _facets_with(setup, gg)])
            _abi.check(lib.ddfg_degrid_adjoint(C.byref(vss), C.byref(js), C.byref(setup.pol), arr, len(gg),
                                               D._stream_ptr()))
            grad_grids = gg
        grad_kms = None
        if ctx.has_kms and ctx.needs_input_grad[1]:
            grad_kms = torch.zeros_like(kms)
            arr = (_abi.Facet * max(1, len(grids)))(*[f.struct(degrid=True) for f in _facets_with(setup, grids)])
            _abi.check(lib.ddfg_degrid_jones_grad(C.byref(vss), C.byref(js), C.byref(setup.pol), arr, len(grids),
                                                  grad_kms.data_ptr(), D._stream_ptr()))
        return (None, grad_kms, *grad_grids)


def predict(setup: PredictSetup, model_grids: Sequence[torch.Tensor], jones_kms: Optional[torch.Tensor] = None):
    """Model visibilities of every facet's model grid (complex64 [nrow][nchan][ncorr]),
    differentiable with respect to the grids and the kMS Jones tensor."""
    if len(model_grids) != len(setup.facets):
        raise ValueError("one model grid per facet")
    return _Predict.apply(setup, jones_kms, *model_grids)


class _ModelGrids(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fm, image):
        out = [torch.empty(f.model.grid.shape, dtype=torch.complex64, device=fm.device) for f in fm.facets]
        fm.image_to_facets(image, out=out)
        ctx.fm = fm
        ctx.image_dtype = image.dtype
        return tuple(out)

    @staticmethod
    def backward(ctx, *grads):
        if not ctx.needs_input_grad[1]:
            return None, None
        g = ctx.fm.image_to_facets_adjoint(grads)
        return None, g.to(ctx.image_dtype)


def model_grids(fm, image: torch.Tensor) -> List[torch.Tensor]:
    """Every facet's model grid (complex64 [nband, npol, N, N]) from the real model image
    [nband, npol, M, M] of the facet machine ``fm``, differentiable with respect to the image."""
    if image.dim() != 4 or tuple(image.shape) != (fm.nband, fm.npol, fm.npix_out, fm.npix_out):
        raise ValueError(f"model image must be [{fm.nband}, {fm.npol}, {fm.npix_out}, {fm.npix_out}]")
    if image.is_complex():
        raise ValueError("the model image is real")
    return list(_ModelGrids.apply(fm, image))
