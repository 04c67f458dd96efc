"""Generates the golden fixtures under tests/golden/ by running the reference itself.

Run in a container that has the reference checkout (read-only) and the reference gridder built
by oracle/build_ref.sh:

    python tests/golden/make_golden.py [/path/to/reference]

The reference's Python modules are imported with stand-ins for the absent optional packages
(pyfftw -> numpy.fft, SharedArray, numexpr); nothing here is used by the product.  Fixtures:

  cf_golden.npz    ModCF.ClassWTermModified tables for two facet centres
  bda_golden.npz   ClassSmearMapping block maps (mode 1 and mode 2) of a small observation,
                   packed in collectSmearMapping's key order
  grid_golden.npz  inputs and outputs of pyGridderWPol32 / pyDeGridderWPol on a small case
                   (4 correlations, Stokes I, per-visibility Jones, BDA blocks, flags)
  sw_golden.npz    ModFFTW.ConvolveGaussian of a facet mask (the spatial-weight smoothing)
  weights_golden.npz  imaging weights: ClassVisServer._uv_to_index, the compiled
                   pyAccumulateWeightsOntoGridNoSem, the Briggs step and
                   ClassVisServer._finalizeWeights_handler on a small observation

  maps_golden.npz  ClassJones.GiveTimeMapping / GiveVisToJonesChanMapping and the channel maps
                   ClassVisServer.Init builds (grid bands, channels within bands, degridding bands)
                   for two measurement sets under three frequency settings
  facets_golden.npz  ClassDDEGridMachine.GridToIm, ClassFacetMachine.BuildFacetNormImage /
                   FacetsToIm_Channel and ClassImToGrid.GiveModelTessel(ToGrid=True) on a regular
                   3 x 3 and an uneven 4-facet tessellation of a small image

    python tests/golden/make_golden.py [/path/to/reference] [--only weights|maps|facets]
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
_args = [a for a in sys.argv[1:] if not a.startswith("--") and a not in ("weights", "maps", "facets")]
REF = _args[0] if _args else os.environ.get("DDFACET_REF", "")
if not REF or not os.path.isdir(REF):
    sys.exit("usage: make_golden.py <reference checkout> (or set DDFACET_REF)")
ONLY = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None


def _stub(name, **attrs):
    m = types.ModuleType(name)
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


def _numexpr_evaluate(expr, out=None, casting=None, local_dict=None):
    """numexpr.evaluate on numpy: evaluates expr with the caller's local variables, every array
    operand first cast to their common type (numexpr computes in the widest operand type)."""
    ns = dict(sys._getframe(1).f_locals if local_dict is None else local_dict)
    names = [k for k in compile(expr, "<numexpr>", "eval").co_names if isinstance(ns.get(k), (np.ndarray, np.generic))]
    if names:
        common = np.result_type(*[ns[k].dtype for k in names])
        for k in names:
            ns[k] = np.asarray(ns[k]).astype(common, copy=False)
    ns.update(exp=np.exp, sqrt=np.sqrt, sin=np.sin, cos=np.cos, abs=np.abs)
    res = eval(expr, {"__builtins__": {}}, ns)
    if out is not None:
        out[...] = res
        return out
    return res


def import_reference():
    sys.path.insert(0, REF)
    pf = _stub("pyfftw")
    pfi = _stub("pyfftw.interfaces")
    def _np_fft(fn):
        # pyfftw's numpy interface takes extra planner keywords that numpy.fft does not
        def call(*a, **kw):
            for k in ("overwrite_input", "threads", "planner_effort", "auto_align_input", "auto_contiguous"):
                kw.pop(k, None)
            return fn(*a, **kw)
        return call

    pfn = _stub("pyfftw.interfaces.numpy_fft",
                **{k: _np_fft(getattr(np.fft, k)) for k in dir(np.fft) if not k.startswith("_")})
    pf.interfaces = pfi
    pfi.numpy_fft = pfn
    pfi.cache = _stub("pyfftw.interfaces.cache", enable=lambda: None, set_keepalive_time=lambda t: None)
    pfi.scipy_fftpack = _stub("pyfftw.interfaces.scipy_fftpack")
    _stub("SharedArray")
    _stub("numexpr", evaluate=_numexpr_evaluate, set_num_threads=lambda n: 1)
    # the process pool imports a compiled helper module at import time; it is never called here
    cb = _stub("DDFacet.cbuild")
    cg = _stub("DDFacet.cbuild.Gridder")
    cb.Gridder = cg
    cg._pyArrays3x = _stub("DDFacet.cbuild.Gridder._pyArrays3x")
    from DDFacet.Imager import ModCF  # noqa: F401
    from DDFacet.Data import ClassSmearMapping  # noqa: F401
    from DDFacet.ToolsDir import ModFFTW  # noqa: F401
    return ModCF, ClassSmearMapping, ModFFTW


class CFDict(dict):
    def addSharedArray(self, name, shape, dtype):
        self[name] = np.zeros(shape, dtype)
        return self[name]


class _InertMeta(type):
    def __getattr__(cls, k):
        if k.startswith("__"):
            raise AttributeError(k)
        return cls

    def __call__(cls, *a, **k):
        return cls


_INERT = _InertMeta("Inert", (), {})


class _InertModule(types.ModuleType):
    """A module every attribute of which is an inert class (imports of names succeed)."""
    __path__ = []

    def __getattr__(self, k):
        if k.startswith("__"):
            raise AttributeError(k)
        return _INERT


def stub(name):
    """Registers inert modules for ``name`` and its parents that are not importable."""
    parts = name.split(".")
    for i in range(1, len(parts) + 1):
        n = ".".join(parts[:i])
        if n not in sys.modules:
            sys.modules[n] = _InertModule(n)
            if i > 1:
                setattr(sys.modules[".".join(parts[:i - 1])], parts[i - 1], sys.modules[n])


def import_visserver():
    """DDFacet.Data.ClassVisServer with inert stand-ins for the MS, beam and astronomy packages it
    imports at module level (none of them is used by the weight functions), and the compiled
    reference gridder module from oracle/_ref."""
    for n in ("pyrap.tables", "pyrap.measures", "pyrap.quanta", "casacore.tables", "casacore.measures",
              "casacore.quanta", "astropy.time", "astropy.io.fits", "astropy.wcs", "ephem"):
        if n not in sys.modules:
            stub(n)
    sys.path.insert(0, ROOT)
    from oracle import ref
    mod = ref.module()
    sys.modules["DDFacet.cbuild.Gridder._pyGridderSmearPols3x"] = mod
    sys.modules["DDFacet.cbuild.Gridder"].__dict__["_pyGridderSmearPols3x"] = mod
    for _ in range(60):
        try:
            from DDFacet.Data import ClassVisServer
            return ClassVisServer, mod
        except ModuleNotFoundError as e:
            for k in list(sys.modules):
                if k.startswith("DDFacet.Data.Class") or k.startswith("DDFacet.Imager.Class"):
                    del sys.modules[k]
            stub(e.name)
    raise RuntimeError("could not import ClassVisServer")


class _MSW(dict):
    def delete_item(self, k):
        self.pop(k, None)


def make_weights_golden():
    import tempfile

    V, mod = import_visserver()
    sys.path.insert(0, ROOT)
    from ddfacet_b200 import synth
    obs = synth.make_observation(31, 8, 1500.0, 34.0, 40.0, 20 * 30.0 / 3600.0, 30.0, 8, 1.30e9, 1.45e9)
    rng = np.random.default_rng(32)
    nrow, nchan = obs.nrow, 8
    freqs = obs.freqs
    weights = rng.uniform(0.5, 2.0, (nrow, nchan)).astype(np.float32)
    weights[rng.uniform(size=(nrow, nchan)) < 0.1] = 0          # flagged
    rowflags = np.zeros(nrow, bool)
    band_of_chan = np.array([0, 0, 0, 0, 1, 1, 1, 1], np.int32)
    cell_rad, npix_image, super_uniform = 3.0 / 3600 * np.pi / 180, 512, 1.0
    out = {"uvw": obs.uvw, "freqs": freqs, "weights_in": weights, "band_of_chan": band_of_chan,
           "cell_rad": cell_rad, "npix_image": npix_image, "super_uniform": super_uniform}
    uvmax = abs(obs.uvw[~rowflags, :2]).max() * freqs.max() / V._cc      # ClassVisServer.py:949
    fov = cell_rad * npix_image                                          # ClassVisServer.py:868-883
    cell = 1. / (super_uniform * fov)
    xymax = int(np.floor(uvmax / cell)) + 1
    npixx = xymax * 2 + 1
    npix = npixx * (xymax + 1)
    out.update(uvmax=uvmax, cell=cell, xymax=xymax, npixx=npixx, npix=npix)

    class Self:
        DicoMSChanMapping = {0: band_of_chan}
        ListMS = [types.SimpleNamespace(MSName="synthetic")]

    for nbands in (1, 2):
        self = Self()
        self.Weighting = "briggs"
        self._uv_to_index = lambda *a, _s=self: V.ClassVisServer._uv_to_index(_s, *a)
        uv = obs.uvw[:, :2].copy()
        index = V.ClassVisServer._uv_to_index(self, 0, uv, weights, freqs, cell, npix, npixx, nbands, xymax)
        grid = np.zeros((nbands, npix), np.float64)
        mod.pyAccumulateWeightsOntoGridNoSem(grid, weights.ravel(), index.ravel())
        out[f"index_{nbands}"] = index
        out[f"grid_{nbands}"] = grid.copy()
        robust = 0.5                                                    # ClassVisServer.py:897-904
        numeratorSqrt = 5.0 * 10 ** (-robust)
        for band in range(nbands):
            grid1 = grid[band, :]
            avgW = (grid1 ** 2).sum() / grid1.sum()
            sSq = numeratorSqrt ** 2 / avgW
            grid1[...] = 1 + grid1 * sSq
        out[f"grid_briggs_{nbands}"] = grid.copy()
        with tempfile.TemporaryDirectory() as td:
            msw = _MSW(weight=weights.copy(), uv=uv, cachepath=os.path.join(td, "w.npy"))
            V.ClassVisServer._finalizeWeights_handler(self, {"grid": grid}, msw, 0, 0, freqs, cell, npix, npixx,
                                                      nbands, xymax)
            assert msw.get("success"), msw.get("error")
            out[f"weights_briggs_{nbands}"] = np.load(os.path.join(td, "w.npy"))
    out["robust"] = 0.5
    np.savez_compressed(os.path.join(HERE, "weights_golden.npz"), **out)
    print("weights golden written")


class _FakeMS:
    """The measurement-set object ClassVisServer.Init reads: channel frequencies and widths, and the
    few methods its loop calls (no table is opened)."""
    SPECS = {}

    def __init__(self, msname, **kw):
        self.MSName = msname
        self.ChanFreq, self.ChanWidth = self.SPECS[msname]
        self.empty = False
        self.Ncorr = 4
        self.CorrelationIds = [9, 10, 11, 12]
        self.maincache = types.SimpleNamespace(dirname="/tmp")

    def getPerChunkRowCounts(self):
        return [100]

    def get_obs_details(self):
        return {}

    def numChunks(self):
        return 1

    def __str__(self):
        return self.MSName


def make_maps_golden():
    V, _ = import_visserver()
    from DDFacet.Data import ClassJones as CJ

    rng = np.random.default_rng(41)
    out = {}
    # ---- Jones time map: unsorted times, a gap between slots, an overlap, rows outside every slot
    times = rng.uniform(-100.0, 3700.0, 6000)
    t0 = np.array([0.0, 300.0, 600.0, 900.0, 1300.0, 1600.0, 1800.0, 2400.0, 3000.0])
    t1 = np.array([300.0, 600.0, 900.0, 1200.0, 1600.0, 1900.0, 2100.0, 3000.0, 3600.0])
    sols = {"Jones": np.zeros((t0.size, 1, 1, 1, 2, 2), np.complex64), "t0": t0, "t1": t1}
    out.update(times=times, t0=t0, t1=t1, time_map=CJ.ClassJones.GiveTimeMapping(None, sols, times))
    # ---- visibility channel -> Jones channel
    freqs = np.linspace(1.30e9, 1.45e9, 16)
    doms = np.array([[1.28e9, 1.33e9], [1.33e9, 1.38e9], [1.38e9, 1.43e9], [1.43e9, 1.48e9]])
    fake = types.SimpleNamespace(MS=types.SimpleNamespace(ChanFreq=freqs, NSPWChan=freqs.size))
    out.update(jchan_freqs=freqs, jchan_domains=doms, jchan_map=CJ.ClassJones.GiveVisToJonesChanMapping(fake, doms))
    # ---- grid / degrid channel maps of two measurement sets (ClassVisServer.Init)
    f1 = np.linspace(1.30e9, 1.45e9, 16)
    f2 = np.linspace(1.40e9, 1.62e9, 8)
    _FakeMS.SPECS = {"a.ms": (f1, np.full(16, f1[1] - f1[0])), "b.ms": (f2, np.full(8, f2[1] - f2[0]))}
    out.update(ms_a_freq=f1, ms_a_width=_FakeMS.SPECS["a.ms"][1], ms_b_freq=f2, ms_b_width=_FakeMS.SPECS["b.ms"][1])
    V.ClassMS = types.SimpleNamespace(ClassMS=_FakeMS)
    settings = [(0.0, 3, 0.0, 0), (40.0, 1, 25.0, 0), (0.0, 1, 0.0, 4), (100.0, 2, 0.0, 3)]
    for k, (band_mhz, nband, dband_mhz, ndband) in enumerate(settings):
        vs = V.ClassVisServer.__new__(V.ClassVisServer)
        vs.GD = {"Data": {"Dask": False, "MS": "a.ms"}, "Cache": {"Reset": 0, "Dir": ""},
                 "Freq": {"BandMHz": band_mhz, "NBand": nband, "DegridBandMHz": dband_mhz, "NDegridBand": ndband},
                 "RIME": {"PolMode": "I"}, "HMP": {"Alpha": [0., 0., 1.]}, "SSDClean": {"SSDSolvePars": ["S", "Alpha"]}}
        vs.MSList = ["a.ms", "b.ms"]
        vs.DicoSelectOptions = {"DDID": 0, "Field": 0}
        vs.ColName, vs.SubColName, vs.TaQL, vs.TMemChunkSize, vs.DATA = "DATA", None, None, 1.0, None
        V.ClassVisServer.Init(vs)
        out[f"s{k}_settings"] = np.array([band_mhz, nband, dband_mhz, ndband], np.float64)
        out[f"s{k}_nbands"] = np.array(vs.NFreqBands)
        out[f"s{k}_centers"] = np.asarray(vs.FreqBandCenters)
        for ims in (0, 1):
            out[f"s{k}_ms{ims}_map"] = np.asarray(vs.DicoMSChanMapping[ims])
            out[f"s{k}_ms{ims}_mapchan"] = np.asarray(vs.DicoMSChanMappingChan[ims])
            out[f"s{k}_ms{ims}_degrid"] = np.asarray(vs.DicoMSChanMappingDegridding[ims])
            out[f"s{k}_ms{ims}_degrid_freqs"] = np.asarray(vs.FreqBandChannelsDegrid[ims])
    out["nsettings"] = np.array(len(settings))
    np.savez_compressed(os.path.join(HERE, "maps_golden.npz"), **out)
    print("maps golden written")


def import_facetmachine():
    """ClassFacetMachine (FacetsToIm_Channel, BuildFacetNormImage), ClassImToGrid (GiveModelTessel)
    and ClassDDEGridMachine (GridToIm), with inert stand-ins for the plotting, polygon and image
    packages and for the compiled modules ClassDDEGridMachine imports at module level (none of
    them is called by those functions)."""
    import_visserver()
    for n in ("pyrap.images", "casacore.images", "matplotlib", "matplotlib.path", "Polygon",
              "DDFacet.cbuild.Gridder._pyGridderSmearPolsClassic3x", "DDFacet.cbuild.Gridder._pyGridder3x"):
        stub(n)
    for _ in range(60):
        try:
            from DDFacet.Imager import ClassDDEGridMachine, ClassFacetMachine, ClassImToGrid
            return ClassFacetMachine, ClassImToGrid, ClassDDEGridMachine
        except ModuleNotFoundError as e:
            for k in list(sys.modules):
                if k.startswith("DDFacet.Imager.Class"):
                    del sys.modules[k]
            stub(e.name)
    raise RuntimeError("could not import ClassFacetMachine")


def _cell_sw(ModFFTW, centres, k, xc, yc, n, m, mixing):
    """Spatial weight of facet k the way _initcf_worker (ClassFacetMachine.py:785-820) makes it,
    on the facet's padded pixel box [x, y] (image orientation): the facet's tessellation cell
    (pixels nearer to its centre than to any other centre) inside the main image,
    Gaussian-smoothed, divided by its maximum, zero below 1e-3."""
    i, j = np.mgrid[0:n, 0:n]
    x, y = xc - n // 2 + i, yc - n // 2 + j
    c = np.asarray(centres, np.float64)
    d = (x[None] - c[:, 0, None, None]) ** 2 + (y[None] - c[:, 1, None, None]) ** 2
    mask = (np.argmin(d, axis=0) == k) & (x >= 0) & (x < m) & (y >= 0) & (y < m)
    sw = np.float32(mask.reshape((1, 1, n, n)))
    sw = ModFFTW.ConvolveGaussian(shareddict={"in": sw, "out": sw}, field_in="in", field_out="out", ch=0,
                                  CellSizeRad=1, GaussPars_ch=(mixing, mixing, 0))
    sw = np.asarray(sw).reshape((n, n))
    sw /= np.max(sw)
    sw[sw < 1e-3] = 0.
    return sw


def make_facets_golden():
    """Stitching and model-image cutting on a regular 3 x 3 and an uneven 4-facet (Voronoi-like)
    tessellation of a small main image, through the reference's own functions:
    ClassDDEGridMachine.GridToIm, ClassFacetMachine.BuildFacetNormImage / FacetsToIm_Channel and
    ClassImToGrid.GiveModelTessel(ToGrid=True)."""
    ModCF, _, ModFFTW = import_reference()
    CFM, CIG, CDG = import_facetmachine()
    rng = np.random.default_rng(77)
    freqs = np.linspace(1.30e9, 1.45e9, 4)
    out = {}
    cases = {
        # name: main image side, facet centres (pixels), padded facet sizes, bands, Stokes planes
        "reg": (75, [(12 + 25 * a, 12 + 25 * b) for a in range(3) for b in range(3)], [43] * 9, 2, 1),
        "vor": (75, [(16, 22), (55, 14), (27, 57), (62, 60)], [61, 57, 67, 49], 1, 2),
    }
    for name, (m, centres, sizes, nband, npol) in cases.items():
        nf = len(centres)
        fm = types.SimpleNamespace()
        fm.OutImShape = (nband, npol, m, m)
        fm.nch, fm.npol, fm.stitchedType = nband, npol, np.float32
        fm.VS = types.SimpleNamespace(NFreqBands=nband)
        fm.GD = {"Parallel": {"NCPU": 1}}
        fm._norm_dict = {}
        fm.GiveEmptyMainField = lambda _s=fm: np.zeros(_s.OutImShape, dtype=_s.stitchedType)
        fm.DicoImager, fm._CF, fm.DicoGridMachine = {}, {}, {}
        for k, ((xc, yc), n) in enumerate(zip(centres, sizes)):
            cf = CFDict()
            ModCF.ClassWTermModified(Cell=6.0, Sup=7, Npix=n, Freqs=freqs, wmax=1000.0, Nw=2, OverS=11,
                                     lmShift=(0.0, 0.0), cf_dict=cf, compute_cf=True)
            sw = _cell_sw(ModFFTW, centres, k, xc, yc, n, m, 5.0)
            fm._CF[k] = {"Sphe": np.asarray(cf["Sphe"]), "InvSphe": np.asarray(cf["InvSphe"]), "SW": sw}
            sumw = rng.uniform(50.0, 200.0, (nband, npol))
            sjn = rng.uniform(0.5, 2.0, nband)
            if name == "reg" and k == 0:
                sumw[1, :] = 0.0  # a band with no weight: stitched without normalisation
            fm.DicoImager[k] = {"pixCentral": (xc, yc), "NpixFacetPadded": n, "SumWeights": sumw,
                                "SumJonesNorm": sjn}
            grid = (rng.standard_normal((nband, npol, n, n)) + 1j * rng.standard_normal((nband, npol, n, n)))
            grid = grid.astype(np.complex64)
            gm = types.SimpleNamespace(WTerm=types.SimpleNamespace(OverS=11),
                                       getFFTWMachine=lambda: ModFFTW.FFTW_2Donly_np())
            dirty = CDG.ClassDDEGridMachine.GridToIm(gm, grid.copy())
            fm.DicoGridMachine[k] = {"Dirty": dirty}
            p = f"{name}_f{k}_"
            out.update({p + "grid": grid, p + "dirty": np.asarray(dirty, np.complex64), p + "sphe": fm._CF[k]["Sphe"],
                        p + "invsphe": fm._CF[k]["InvSphe"], p + "sw": sw, p + "sumweights": sumw,
                        p + "sumjonesnorm": sjn})
        CFM.ClassFacetMachine.BuildFacetNormImage(fm)
        norm = np.asarray(fm._norm_dict["FacetNorm"])
        assert (norm > 0).all(), f"{name}: facet norm has empty pixels"
        image = CFM.ClassFacetMachine.FacetsToIm_Channel(fm, kind="Dirty")
        # model image: point components; in the regular case the first facet's padded box holds
        # negative components only, so the reference's SumFlux is zero there (ClassImToGrid.py:249-256)
        model = np.zeros((nband, npol, m, m), np.float32)
        for _ in range(40):
            x, y = rng.integers(0, m, 2)
            if name == "reg" and x < 34 and y < 34:
                continue
            model[rng.integers(0, nband), rng.integers(0, npol), x, y] = rng.uniform(0.05, 1.0)
        if name == "reg":
            model[0, 0, 5, 9], model[1, 0, 14, 3], model[0, 0, 20, 18] = -0.3, -0.2, -0.5
        i2g = CIG.ClassImToGrid(OverS=11, GD=None)
        for k in range(nf):
            g, sumflux = i2g.GiveModelTessel(model, fm.DicoImager, k, norm, fm._CF[k]["Sphe"], fm._CF[k]["SW"],
                                             ToGrid=True)
            out[f"{name}_f{k}_model_grid"] = np.asarray(g, np.complex64)
            out[f"{name}_f{k}_sumflux"] = np.float64(sumflux)
        out.update({f"{name}_m": m, f"{name}_centres": np.asarray(centres, np.int32),
                    f"{name}_sizes": np.asarray(sizes, np.int32), f"{name}_nband": nband, f"{name}_npol": npol,
                    f"{name}_facet_norm": norm, f"{name}_image": np.asarray(image, np.float32),
                    f"{name}_model": model})
    out["overs"] = 11
    np.savez_compressed(os.path.join(HERE, "facets_golden.npz"), **out)
    print("facets golden written")


def main():
    if ONLY == "facets":
        make_facets_golden()
        return
    if ONLY == "weights":
        import_reference()
        make_weights_golden()
        return
    if ONLY == "maps":
        import_reference()
        make_maps_golden()
        return
    ModCF, SM, ModFFTW = import_reference()
    sys.path.insert(0, ROOT)
    from ddfacet_b200 import synth

    freqs = np.linspace(1.30e9, 1.45e9, 8)
    # ---- CF tables
    out = {}
    for i, lm in enumerate([(0.0, 0.0), (0.02, -0.01)]):
        w = ModCF.ClassWTermModified(Cell=3.0, Sup=7, Npix=129, Freqs=freqs, wmax=3000.0, Nw=4, OverS=11,
                                     lmShift=lm, cf_dict=CFDict(), compute_cf=True)
        out[f"f{i}_lm"] = np.array(lm)
        out[f"f{i}_sups"] = np.array(w.Sups)
        out[f"f{i}_cucv"] = np.array([w.Cu, w.Cv])
        out[f"f{i}_ifzf"] = np.asarray(w.ifzfCF)
        for k, (a, b) in enumerate(zip(w.Wplanes, w.WplanesConj)):
            out[f"f{i}_w{k}"] = a
            out[f"f{i}_wc{k}"] = b
    out["freqs"] = freqs
    np.savez_compressed(os.path.join(HERE, "cf_golden.npz"), **out)

    # ---- BDA maps
    obs = synth.make_observation(7, 7, 1500.0, 34.0, 40.0, 0.25, 30.0, 8, 1.30e9, 1.45e9)
    chan_map = np.array([0, 0, 0, 0, 1, 1, 1, 1], np.int32)
    dfreq = float(freqs[1] - freqs[0])
    DATA = {"A0": obs.A0, "A1": obs.A1, "uvw": obs.uvw, "dfreqs": dfreq, "freqs": obs.freqs}
    bda = {"A0": obs.A0, "A1": obs.A1, "uvw": obs.uvw, "freqs": obs.freqs, "chan_map": chan_map, "dfreq": dfreq}
    for mode, fn in ((1, SM.GiveBlocksRowsListBL_old), (2, SM.GiveBlocksRowsListBL)):
        for dphi_name, decorr in (("a", 0.02), ("b", 0.002)):
            dPhi = np.sqrt(6. * (1. - (1. - decorr)))
            l = 0.01
            per = {}
            for a0 in range(obs.nant):
                for a1 in range(obs.nant):
                    if a0 == a1:
                        continue
                    r = fn(a0, a1, DATA, dPhi, l, chan_map)
                    if r[0] is not None:
                        per["%d:%d" % (a0, a1)] = (np.array(r[0]), np.array(r[1]))
            keys = sorted(per.keys())
            nb = sum(len(per[k][1]) for k in keys)
            body = np.concatenate([per[k][0] for k in keys]).astype(np.int32)
            sizes = np.concatenate([per[k][1] for k in keys]).astype(np.int32)
            m = np.concatenate([[nb, nb >> 32], sizes, body]).astype(np.int32)
            bda[f"map_mode{mode}_{dphi_name}"] = m
            bda[f"dphi_{dphi_name}"] = dPhi
    bda["l"] = 0.01
    np.savez_compressed(os.path.join(HERE, "bda_golden.npz"), **bda)

    # ---- reference gridder / degridder on a small case
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import cases

    c = cases.make_case(seed=21, nant=8, ntimes=12, nchan=8, ncorr=4, stokes_ids=(1,), npix=129, cell_arcsec=6.0,
                        nw=3, bda_mode=1, dphi=np.sqrt(6 * 0.05), flag_frac=0.05, lm=(0.01, -0.004))
    cases.add_jones(c, mode=1, nt=3, nd=2, idir=1)
    r = cases.run_ref_grid(c)
    vr = cases.run_ref_degrid(c, r["grid"], vis0=c.vis)
    g = dict(vis=c.vis, uvw=c.uvw, flags=c.flags, weights=c.weights, freqs=c.freqs, chan_map=c.chan_map, bda=c.bda,
             incr=c.incr, winfos=c.winfos, facet_infos=c.facet_infos, lm=np.array(c.lm),
             jones_kms=c.jones["kms"], jones_tmap=c.jones["kms_tmap"], jones_cmap=c.jones["kms_cmap"],
             A0=c.jones["A0"], A1=c.jones["A1"], idir=c.jones["idir_kms"],
             grid=r["grid"], sumwt=r["sumwt"], sumjones=r["sumjones"], sumjones_chan=r["sumjones_chan"], vis_degrid=vr)
    for k, (a, b) in enumerate(zip(c.wt.Wplanes, c.wt.WplanesConj)):
        g[f"w{k}"] = a
        g[f"wc{k}"] = b
    g["nw"] = len(c.wt.Wplanes)
    np.savez_compressed(os.path.join(HERE, "grid_golden.npz"), **g)

    # ---- spatial-weight smoothing
    mask = np.zeros((1, 1, 97, 97), np.float32)
    mask[0, 0, 20:70, 25:80] = 1
    sw = ModFFTW.ConvolveGaussian(shareddict={"in": mask, "out": mask.copy()}, field_in="in", field_out="out", ch=0,
                                  CellSizeRad=1, GaussPars_ch=(10, 10, 0))
    np.savez_compressed(os.path.join(HERE, "sw_golden.npz"), mask=mask[0, 0], sw=np.asarray(sw).reshape(97, 97))
    make_weights_golden()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
