"""Per-facet GPU transforms and stitching against the NumPy restatement of the reference
(oracle/facets.py): GridToIm, FacetsToIm_Channel (+ facet norm), GiveModelTessel(ToGrid).
Tolerance: 1e-5 relative RMS (complex64 cuFFT against complex128 numpy)."""
import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def _fm(kind, nfs=3, npix=1200):
    from ddfacet_b200 import geometry
    from ddfacet_b200.facetmachine import FacetMachine

    freqs = np.linspace(1.3e9, 1.45e9, 8)
    tess = None
    if kind == "voronoi":  # five directions: uneven facets (ClassFacetMachineTessel)
        r = npix * 6.0 / 3600 * np.pi / 180 / 2
        rng = np.random.default_rng(4)
        tess = geometry.voronoi_facets(npix, 6.0, rng.uniform(-0.8 * r, 0.8 * r, 5), rng.uniform(-0.8 * r, 0.8 * r, 5),
                                       1.7)
        assert len({f.npix_padded for f in tess.facets}) > 1
    return FacetMachine(npix, 6.0, nfs, freqs, padding=1.7, nband=1, stokes_ids=(1,), corr_ids=(9, 10, 11, 12),
                        support=7, nw=3, wmax=2000.0, mixing_width=10.0, tessellation=tess)


@pytest.mark.parametrize("kind", ["regular", "voronoi"])
def test_grid_to_image_and_stitch(kind):
    from oracle import facets as OF

    fm = _fm(kind)
    rng = np.random.default_rng(0)
    grids = []
    for f in fm.facets:
        g = (rng.standard_normal(f.grid.grid.shape) + 1j * rng.standard_normal(f.grid.grid.shape)).astype(np.complex64)
        grids.append(g)
        f.grid.grid.copy_(torch.from_numpy(g))
        f.grid.sumwt.fill_(123.0)
    image = fm.facets_to_image().cpu().numpy()
    dirties = [OF.grid_to_im(g, fm.overs) for g in grids]
    for f, d in zip(fm.facets, dirties):
        got = f.grid.grid.cpu().numpy()  # transformed in place
        assert cases.rel_rms(got, d) < 1e-5
    want = OF.facets_to_im_channel(dirties, [f.sphe.cpu().numpy() for f in fm.facets],
                                   [f.invsphe.cpu().numpy() for f in fm.facets], [f.sw_host for f in fm.facets],
                                   [np.full((1, 1), 123.0) for _ in fm.facets], [f.geom.pix_central for f in fm.facets],
                                   fm.npix_out, fm.facet_norm_host)
    assert cases.rel_rms(image, want) < 1e-5


@pytest.mark.parametrize("kind", ["regular", "voronoi"])
def test_image_to_grid(kind):
    from oracle import facets as OF

    fm = _fm(kind)
    rng = np.random.default_rng(1)
    img = np.zeros((1, 1, fm.npix_out, fm.npix_out), np.float32)
    for _ in range(30):
        img[0, 0, rng.integers(0, fm.npix_out), rng.integers(0, fm.npix_out)] = rng.uniform(0.01, 1.0)
    fm.image_to_facets(torch.from_numpy(img))
    for f in fm.facets:
        want = OF.give_model_tessel(img, fm.facet_norm_host, f.sphe.cpu().numpy(), f.sw_host, *f.geom.pix_central,
                                    f.model.grid.shape[-1], fm.overs)
        got = f.model.grid.cpu().numpy()
        if np.abs(want).max() == 0:
            assert np.abs(got).max() == 0
        else:
            assert cases.rel_rms(got, want) < 1e-5


def _ptr(t):
    import ctypes as C

    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("name", ["reg", "vor"])
def test_against_reference_fixture(name):
    """The C-ABI transforms on the reference's own outputs (tests/golden/facets_golden.npz, from
    ClassDDEGridMachine.GridToIm, ClassFacetMachine.BuildFacetNormImage / FacetsToIm_Channel and
    ClassImToGrid.GiveModelTessel(ToGrid=True) on a regular 3 x 3 and an uneven 4-facet case):
    GridToIm to 1e-5 relative RMS; stitching the reference's dirty facets bit for bit (the same
    float64 products and float32 additions in the same facet order); the whole chain from the
    grids to 1e-5; the model grids to 1e-5.  For the facet whose padded box sees no positive model
    component the reference returns its scaled model without the FFT (SumFlux == 0,
    ClassImToGrid.py:249-256); the kernels transform it, which is checked against the transform of
    the reference's returned array."""
    import ctypes as C
    import os

    from ddfacet_b200 import _abi

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "facets_golden.npz"))
    lib = _abi.lib()
    dev = torch.device("cuda", 0)
    m, nband, npol, overs = int(g[f"{name}_m"]), int(g[f"{name}_nband"]), int(g[f"{name}_npol"]), int(g["overs"])
    norm = torch.from_numpy(g[f"{name}_facet_norm"]).to(dev)
    model = torch.from_numpy(g[f"{name}_model"]).to(dev)
    img_ref_dirty = torch.zeros((nband, npol, m, m), dtype=torch.float32, device=dev)
    img_chain = torch.zeros_like(img_ref_dirty)
    quirk = 0
    for k, (c, n) in enumerate(zip(g[f"{name}_centres"], g[f"{name}_sizes"])):
        p = f"{name}_f{k}_"
        n, xc, yc = int(n), int(c[0]), int(c[1])
        plan = C.c_void_p()
        _abi.check(lib.ddfg_fft_plan_create(n, nband * npol, C.byref(plan)))
        try:
            work = torch.empty((nband * npol * n * n,), dtype=torch.complex64, device=dev)
            grid = torch.from_numpy(g[p + "grid"]).to(dev)
            _abi.check(lib.ddfg_grid_to_image(plan, _ptr(grid), C.c_double(float(overs) ** 2), _ptr(work), None))
            torch.cuda.synchronize()
            assert cases.rel_rms(grid.cpu().numpy(), g[p + "dirty"]) < 1e-5
            sphe = torch.from_numpy(g[p + "sphe"]).to(dev)
            inv = torch.from_numpy(g[p + "invsphe"]).to(dev)
            sw_img = torch.from_numpy(g[p + "sw"]).to(dev)
            sw_grid = torch.from_numpy(np.ascontiguousarray(g[p + "sw"].T[::-1, :])).to(dev)
            w = torch.from_numpy(g[p + "sumweights"] * np.sqrt(g[p + "sumjonesnorm"])[:, None]).to(dev).contiguous()
            ref_dirty = torch.from_numpy(g[p + "dirty"]).to(dev)
            for src, dst in ((ref_dirty, img_ref_dirty), (grid, img_chain)):
                _abi.check(lib.ddfg_stitch_facet(_ptr(src), nband, npol, n, _ptr(sphe), _ptr(inv), _ptr(sw_grid),
                                                 _ptr(w), _ptr(dst), m, xc, yc, None))
            out = torch.empty((nband, npol, n, n), dtype=torch.complex64, device=dev)
            _abi.check(lib.ddfg_image_to_grid(plan, _ptr(model), m, _ptr(norm), _ptr(sw_img), _ptr(sphe), xc, yc,
                                              C.c_double(float(overs)), _ptr(out), _ptr(work), None))
            torch.cuda.synchronize()
            got, want = out.cpu().numpy(), g[p + "model_grid"]
            if float(g[p + "sumflux"]) == 0.0 and np.abs(want).max() > 0:
                b = np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(want.astype(np.complex128), axes=(-2, -1))),
                                    axes=(-2, -1)) / (n * n)
                assert cases.rel_rms(got, b) < 1e-5
                quirk += 1
            elif np.abs(want).max() == 0:
                assert np.abs(got).max() == 0
            else:
                assert cases.rel_rms(got, want) < 1e-5
        finally:
            lib.ddfg_fft_plan_destroy(plan)
    for img in (img_ref_dirty, img_chain):
        _abi.check(lib.ddfg_image_normalise(_ptr(img), nband * npol, m, _ptr(norm), None))
    torch.cuda.synchronize()
    want = g[f"{name}_image"]
    np.testing.assert_array_equal(img_ref_dirty.cpu().numpy(), want)
    assert cases.rel_rms(img_chain.cpu().numpy(), want) < 1e-5
    assert quirk == (1 if name == "reg" else 0)
