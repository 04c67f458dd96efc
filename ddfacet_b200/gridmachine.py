"""Drop-in ``ClassDDEGridMachine`` whose put/get run on the B200 kernels.

Same constructor, methods, attributes and error behaviour as DDFacet's grid machine
(DDFacet/Imager/ClassDDEGridMachine.py:308-1190); only the work moves to libddfg.so:

* ``__init__``            -- :310-460: padded size from ``EstimateNpix``, ``incr=[-cell, cell]``,
                              Jones type, W-term tables (``cf.WTerms``, from ``cf_dict`` or computed);
* ``setDecorr``           -- :545-569;
* ``GiveParamJonesList``  -- :571-679: nearest-direction pick, interpolation weights, BDA Jones mode;
* ``put``                 -- :681-861: grids into ``ResidueGrid`` (accumulating), updates
                              ``SumWeigths``, ``SumJones`` and ``SumJonesChan``;
* ``get``                 -- :922-1152: subtracts the prediction from ``visIn`` in place and returns it;
* ``CheckTypes``          -- :863-920: the same ``NameError`` / ``TypeError`` messages;
* ``GridToIm``, ``getFFTWMachine`` -- :1186-1190, :471-491, on cuFFT.

Inputs may be numpy arrays (copied to the GPU and results copied back into the caller's arrays,
as the reference updates them in place) or CUDA tensors (used in place).  There is no CPU
implementation behind this class: without the CUDA library it raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _abi, cf, device as D
from .geometry import estimate_npix

C_LIGHT = 299792458.0


def default_gd():
    """The GD keys the grid machine reads, at DDFacet's defaults (DDFacet/Parset/DefaultParset.cfg:77-150, 259-276)."""
    return {
        "RIME": {"Precision": "S", "PolMode": "I", "FFTMachine": "FFTW", "ForwardMode": "BDA-degrid",
                 "BackwardMode": "BDA-grid", "DecorrMode": "", "DecorrLocation": "Edge"},
        "CF": {"OverS": 11, "Support": 7, "Nw": 100, "wmax": 0},
        "Image": {"Cell": 5.0, "NPix": 5000},
        "Facets": {"Padding": 1.7, "NFacets": 3, "MixingWidth": 10},
        "Comp": {"GridDecorr": 0.02, "DegridDecorr": 0.02, "GridFoV": "Facet", "DegridFoV": "Facet", "BDAMode": 1,
                 "BDAJones": 0, "Sparsification": 0},
        "DDESolutions": {"JonesMode": "Full", "DDModeGrid": "AP", "DDModeDeGrid": "AP", "ScaleAmpGrid": 0,
                         "ScaleAmpDeGrid": 0, "CalibErr": 10.0, "Type": "Nearest", "Scale": 1.0, "gamma": 4.0,
                         "ReWeightSNR": 0.0},
    }


class FFTMachine:
    """``FFTW_2Donly`` on cuFFT: fft = fftshift(fft2(ifftshift(A))) / N^2, ifft = the inverse * N^2,
    per [band, pol] plane, in place (ModFFTW.py:535-599)."""

    def __init__(self, shape, device=None):
        self.shape = tuple(shape)
        self.device = D._dev(device)
        nb, npol, n, n2 = self.shape
        if n != n2:
            raise ValueError("square grids only")
        self.n = n
        p = C.c_void_p()
        _abi.check(_abi.lib().ddfg_fft_plan_create(n, nb * npol, C.byref(p)))
        self._plan = p
        self._work = torch.empty(self.shape, dtype=torch.complex64, device=self.device)

    def __del__(self):
        try:
            _abi.lib().ddfg_fft_plan_destroy(self._plan)
        except Exception:
            pass

    def _run(self, A, inverse):
        host = not isinstance(A, torch.Tensor)
        t = D.to_device(A, torch.complex64, self.device) if host else A
        if t.dim() == 2 and self.shape[:2] == (1, 1):
            t = t.view(1, 1, *t.shape)  # a single plane, as FFTW_2Donly accepts
        if tuple(t.shape) != self.shape or t.dtype != torch.complex64 or not t.is_contiguous():
            raise ValueError("FFT machine built for %s complex64" % (self.shape,))
        scale = 1.0 if inverse else 1.0 / (self.n * self.n)
        _abi.check(_abi.lib().ddfg_fft_centred(self._plan, t.data_ptr(), int(inverse), scale, self._work.data_ptr(),
                                                D._stream_ptr()))
        if host:
            out = t.cpu().numpy().reshape(np.shape(A))
            if isinstance(A, np.ndarray) and A.dtype == np.complex64 and A.flags.c_contiguous:
                A[...] = out
                return A
            return out
        return t.view(A.shape)

    def fft(self, A, ChanList=None):
        return self._run(A, inverse=False)

    def ifft(self, A, norm=True):
        return self._run(A, inverse=True)


class ClassDDEGridMachine:
    _fft_machines = {}

    def __init__(self, GD, ChanFreq, Npix, lmShift=(0., 0.), IDFacet=0, SpheNorm=True, NFreqBands=1,
                 DataCorrelationFormat=[5, 6, 7, 8], ExpectedOutputStokes=[1], ListSemaphores=None, cf_dict=None,
                 compute_cf=False, wmax=None, bda_grid=None, bda_degrid=None, Padding=None, device=None):
        self.GD = GD
        self.IDFacet = IDFacet
        self.SpheNorm = SpheNorm
        self.ListSemaphores = ListSemaphores  # kept for the call surface; no host locks are used
        self._bda_grid = bda_grid
        self._bda_degrid = bda_degrid
        self.DoPSF = False
        self.device = D._dev(device)
        Precision = GD["RIME"]["Precision"]
        if Precision == "S":
            self.dtype = np.complex64
        elif Precision == "D":
            raise NotImplementedError("Precision=D (complex128 grids) is not supported on the GPU path; use S")
        if Padding is None:
            Padding = GD["Facets"]["Padding"]
        self.NonPaddedNpix, Npix = estimate_npix(Npix, Padding)
        self.Padding = Npix / float(self.NonPaddedNpix)
        self.LSmear = []
        self.PolMode = ExpectedOutputStokes
        self.npol = len(ExpectedOutputStokes)
        self.SkyType = 1
        self.PolMap = np.array([0, 5, 5, 0], np.int32)
        self.PolModeID = 0
        self.Npix = Npix
        self.NFreqBands = NFreqBands
        self.NonPaddedShape = (NFreqBands, self.npol, self.NonPaddedNpix, self.NonPaddedNpix)
        self.GridShape = (NFreqBands, self.npol, self.Npix, self.Npix)
        x0 = (self.Npix - self.NonPaddedNpix) // 2
        self.PaddingInnerCoord = (x0, x0 + self.NonPaddedNpix)
        self.OverS = GD["CF"]["OverS"]
        self.Sup = GD["CF"]["Support"]
        self.Nw = GD["CF"]["Nw"]
        self.Cell = GD["Image"]["Cell"]
        self.incr = (np.array([-self.Cell, self.Cell], dtype=np.float64) / 3600.) * (np.pi / 180)
        self.JonesType = {"Scalar": 0, "Diag": 1, "Full": 2}[GD["DDESolutions"]["JonesMode"]]
        self.ChanFreq = np.asarray(ChanFreq)
        self.WProj = True
        self.lmShift = lmShift
        if cf_dict is not None or compute_cf:
            self.InitCF(cf_dict, compute_cf, wmax)
        self.reinitGrid()
        self.DataCorrelationFormat = DataCorrelationFormat
        self.ExpectedOutputStokes = ExpectedOutputStokes
        self._fftw_machine = None
        self._cf_dev = None

    # ---------------------------------------------------------------------------------- set-up
    def InitCF(self, cf_dict, compute_cf, wmax):
        if compute_cf:
            self.WTerm = cf.WTerms(Cell=self.Cell, Sup=self.Sup, Npix=self.Npix, Freqs=self.ChanFreq, wmax=wmax,
                                   Nw=self.Nw, OverS=self.OverS, lmShift=self.lmShift, IDFacet=self.IDFacet)
            if cf_dict is not None:
                cf_dict["wmax"] = wmax
                cf_dict["Sphe"] = np.float32(self.WTerm.ifzfCF.real)
                cf_dict["InvSphe"] = np.float32(1. / np.float64(self.WTerm.ifzfCF.real))
                cf_dict["CuCv"] = np.array([self.WTerm.Cu, self.WTerm.Cv])
                cf_dict["W"] = pack_square_planes(list(self.WTerm.Wplanes) + list(self.WTerm.WplanesConj))
        else:
            w = cf.WTerms.__new__(cf.WTerms)
            w.wmax = cf_dict["wmax"]
            w.ifzfCF = cf_dict["Sphe"]
            w.Cu, w.Cv = cf_dict["CuCv"]
            ww = cf_dict["W"]
            if isinstance(ww, np.ndarray):
                ww = unpack_square_planes(ww)
            if len(ww) != self.Nw * 2:
                raise RuntimeError("mismatch in number of cached w-planes")
            w.Wplanes, w.WplanesConj = list(ww[:self.Nw]), list(ww[self.Nw:])
            w.OverS = self.OverS
            w.RefWave = C_LIGHT / self.ChanFreq[-1]
            w.Nw = self.Nw
            self.WTerm = w
        self.ifzfCF = self.WTerm.ifzfCF

    def reinitGrid(self):
        self.NChan, self.npol, _, _ = self.GridShape
        self.SumWeigths = np.zeros((self.NChan, self.npol), np.float64)
        self.SumJones = np.zeros((2, self.NChan), np.float64)

    def setDecorr(self, uvw_dt, DT, Dnu, SmearMode="FT", lm_min=None, lm_PhaseCenter=None):
        DoSmearFreq = 1 if "F" in SmearMode else 0
        DoSmearTime = 1 if "T" in SmearMode else 0
        lmin, mmin = self.lmShift
        if lm_min is not None:
            lmin, mmin = lm_min
        if lm_PhaseCenter is not None:
            lmin -= lm_PhaseCenter[0]
            mmin -= lm_PhaseCenter[1]
        if not (uvw_dt.dtype == np.float64):
            raise NameError('uvw_dt.dtype %s %s' % (str(uvw_dt.dtype), str(np.float64)))
        self.LSmear = [uvw_dt, DT, Dnu, DoSmearTime, DoSmearFreq, lmin, mmin]

    @staticmethod
    def _getGlobalFFTWMachine(GridShape, device):
        key = (tuple(GridShape), str(device))
        m = ClassDDEGridMachine._fft_machines.get(key)
        if m is None:
            m = ClassDDEGridMachine._fft_machines[key] = FFTMachine(GridShape, device)
        return m

    def getFFTWMachine(self):
        if self._fftw_machine is None:
            self._fftw_machine = self._getGlobalFFTWMachine(self.GridShape, self.device)
        return self._fftw_machine

    # ---------------------------------------------------------------------------------- Jones
    def GiveParamJonesList(self, DicoJonesMatrices, times, A0, A1, uvw, gridder=False, degridder=False):
        """Device Jones terms and the facet's Jones directions (ClassDDEGridMachine.py:571-679)."""
        idir_kMS, w_kMS, idir_Beam, InterpMode, BDAJonesMode = self.jones_directions(DicoJonesMatrices, gridder)
        if A0.size != uvw.shape[0]:
            raise RuntimeError("Antenna array is expected to have the same number of rows as the uvw array")
        dev = self.device
        jd = D.JonesData(mode=BDAJonesMode, interp_mode=int(InterpMode),
                         a0=D.to_device(A0, torch.int32, dev), a1=D.to_device(A1, torch.int32, dev),
                         wavelength_mean=float(np.mean(C_LIGHT / self.ChanFreq)))
        for key, attr in (("DicoJones_killMS", "kms"), ("DicoJones_Beam", "beam")):
            if key in DicoJonesMatrices:
                dj = DicoJonesMatrices[key]
                J = dj["Jones"]["Jones"]
                self.CheckTypes(A0=A0, A1=A1, Jones=J)
                setattr(jd, attr, D.to_device(J, torch.complex64, dev))
                setattr(jd, attr + "_tmap", D.to_device(np.int32(dj["TimeMapping"]), torch.int32, dev))
                setattr(jd, attr + "_cmap", D.to_device(np.int32(dj["Jones"]["VisToJonesChanMapping"]), torch.int32, dev))
                self._check_jones_maps(J, dj, A0, A1, idir_kMS if attr == "kms" else idir_Beam)
        if InterpMode == 1:
            jd.interp_coefs = D.to_device(np.float32(w_kMS), torch.float32, dev)
        return jd, idir_kMS, idir_Beam

    def jones_directions(self, DicoJonesMatrices, gridder=False):
        """(killMS direction, killMS interpolation weights, beam direction, interpolation mode,
        BDA Jones mode) for this facet: the host half of ClassDDEGridMachine.py:571-625."""
        l0, m0 = self.lmShift
        idir_kMS = 0
        w_kMS = np.array([], np.float32)
        d0 = self.GD["DDESolutions"]["Scale"] * np.pi / 180
        gamma = self.GD["DDESolutions"]["gamma"]
        if "DicoJones_killMS" in DicoJonesMatrices:
            dirs = DicoJonesMatrices["DicoJones_killMS"]["Dirs"]
            lc, mc, sI = dirs["l"], dirs["m"], dirs["I"]
            d = np.sqrt((l0 - lc) ** 2 + (m0 - mc) ** 2)
            idir_kMS = int(np.argmin(d))
            w = sI / (1. + d / d0) ** gamma
            w /= np.sum(w)
            w[w < (0.2 * w.max())] = 0       # drop directions below a fifth of the strongest
            w[np.argsort(w)[::-1][3:]] = 0    # keep the three strongest
            w /= np.sum(w)
            w_kMS = w
        idir_Beam = 0
        if "DicoJones_Beam" in DicoJonesMatrices:
            dirs = DicoJonesMatrices["DicoJones_Beam"]["Dirs"]
            d = np.sqrt((l0 - dirs["l"]) ** 2 + (m0 - dirs["m"]) ** 2)
            idir_Beam = int(np.argmin(d))
        InterpMode = self.GD["DDESolutions"]["Type"]
        InterpMode = {"Nearest": 0, "Krigging": 1}.get(InterpMode, InterpMode)
        mode = self.GD["Comp"]["BDAJones"]
        if gridder:
            BDAJonesMode = 2 if mode in ("grid", "both") else 1
        else:
            BDAJonesMode = 2 if mode == "both" else 1
        return idir_kMS, w_kMS, idir_Beam, InterpMode, BDAJonesMode

    @staticmethod
    def _check_jones_maps(J, dj, A0, A1, idir):
        """The kernels index the Jones array with these maps; out-of-range entries are refused here."""
        nt, nd, na, nch = J.shape[:4]
        tm = np.asarray(dj["TimeMapping"])
        cm = np.asarray(dj["Jones"]["VisToJonesChanMapping"])
        if tm.size and (tm.min() < 0 or tm.max() >= nt):
            raise ValueError("Jones time mapping outside [0, %d)" % nt)
        if cm.size and (cm.min() < 0 or cm.max() >= nch):
            raise ValueError("Jones channel mapping outside [0, %d)" % nch)
        if min(A0.min(), A1.min()) < 0 or max(A0.max(), A1.max()) >= na:
            raise ValueError("antenna index outside [0, %d)" % na)
        if not (0 <= idir < nd):
            raise ValueError("Jones direction outside [0, %d)" % nd)

    # ---------------------------------------------------------------------------------- plumbing
    def _cf_tables(self):
        if self._cf_dev is None:
            w = self.WTerm
            self._cf_dev = D.CFTables.create(w.Wplanes, w.WplanesConj, self.OverS, w.RefWave, w.wmax,
                                             device=self.device)
        return self._cf_dev

    def _facet(self, grid_t, sumwt=None, sumjones=None, sumjones_chan=None, idirs=(0, 0)):
        l0, m0 = self.lmShift
        dec = (self.LSmear[5], self.LSmear[6]) if self.LSmear else (0.0, 0.0)
        return D.FacetGrid(grid=grid_t, cf=self._cf_tables(), incr=tuple(self.incr), cu=self.WTerm.Cu,
                           cv=self.WTerm.Cv, l0=l0, m0=m0, idir_kms=idirs[0], idir_beam=idirs[1], decorr_lm=dec,
                           sumwt=sumwt, sumjones=sumjones, sumjones_chan=sumjones_chan)

    def _visdata(self, vis, uvw, flag, W, freqs, ChanMapping, bda, sparsification):
        smear = self.LSmear[:5] if self.LSmear else None
        return D.VisData.create(vis, uvw, flag, W, freqs, ChanMapping, bda, device=self.device,
                                sparsification=sparsification, smear=smear)

    # ---------------------------------------------------------------------------------- put / get
    def put(self, times, uvw, visIn, flag, A0A1, W=None, PointingID=0, DoNormWeights=True, DicoJonesMatrices=None,
            freqs=None, DoPSF=0, ChanMapping=None, ResidueGrid=None, sparsification=None):
        """Grid ``visIn`` into ``ResidueGrid`` (accumulating), as pyGridderWPol32 does."""
        vis = visIn
        self.DoNormWeights = DoNormWeights
        if not self.DoNormWeights:
            self.reinitGrid()
        if ChanMapping is None:
            ChanMapping = np.zeros((visIn.shape[1],), np.int64)
        self.ChanMappingGrid = ChanMapping
        Grid = ResidueGrid
        if _dtype(Grid) != self.dtype:
            raise TypeError("Grid must be of type " + str(self.dtype))
        A0, A1 = A0A1
        NVisChan = vis.shape[1]
        self.SumJonesChan = np.zeros((2, NVisChan), np.float64)
        if W is None:
            W = np.ones((uvw.shape[0], NVisChan), dtype=np.float64)
        if tuple(vis.shape) != tuple(flag.shape):
            raise Exception('vis[%s] and flag[%s] should have the same shape' % (str(vis.shape), str(flag.shape)))
        self.CheckTypes(Grid=Grid, vis=vis, uvw=uvw, flag=flag, ListWTerm=self.WTerm.Wplanes, W=W)
        if self.GD["RIME"]["BackwardMode"] != "BDA-grid":
            raise ValueError("unknown --RIME-BackwardMode %s" % self.GD["RIME"]["BackwardMode"])
        dev = self.device
        jd, idirs = None, (0, 0)
        if DicoJonesMatrices is not None:
            jd, ik, ib = self.GiveParamJonesList(DicoJonesMatrices, times, _np(A0), _np(A1), uvw, gridder=True)
            jd.apply_amp = 1 if "A" in self.GD["DDESolutions"]["DDModeGrid"] else 0
            jd.apply_phase = 1 if "P" in self.GD["DDESolutions"]["DDModeGrid"] else 0
            if self.GD["DDESolutions"]["ScaleAmpGrid"]:
                jd.scale_jones = 1
                jd.calib_error = (self.GD["DDESolutions"]["CalibErr"] / 3600.) * np.pi / 180
            idirs = (ik, ib)
        vs = self._visdata(vis, uvw, flag, W, freqs, np.int32(ChanMapping), self._bda_grid, sparsification)
        grid_t = Grid if isinstance(Grid, torch.Tensor) else torch.from_numpy(Grid).to(dev)
        z = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)  # noqa: E731
        fg = self._facet(grid_t, z(*self.SumWeigths.shape), z(*self.SumJones.shape), z(2, NVisChan), idirs)
        D.grid(vs, [fg], D.make_pol(self.DataCorrelationFormat, self.ExpectedOutputStokes), jd, dopsf=bool(DoPSF))
        if not isinstance(Grid, torch.Tensor):
            Grid[...] = grid_t.cpu().numpy()
        self.SumWeigths += fg.sumwt.cpu().numpy()
        if DicoJonesMatrices is not None:
            self.SumJones += fg.sumjones.cpu().numpy()
            self.SumJonesChan += fg.sumjones_chan.cpu().numpy()

    def get(self, times, uvw, visIn, flag, A0A1, ModelImage, PointingID=0, Row0Row1=(0, -1),
            DicoJonesMatrices=None, freqs=None, ImToGrid=True, TranformModelInput="", ChanMapping=None,
            sparsification=None):
        """Subtract the prediction of ``ModelImage`` (a model grid with ImToGrid=False) from
        ``visIn`` in place and return it, as pyDeGridderWPol does."""
        vis = visIn
        A0, A1 = A0A1
        if ImToGrid:
            if float(_absmax(ModelImage)) == 0:
                return vis
            Grid = self.setModelIm(_np(ModelImage))
        else:
            Grid = ModelImage
        if ChanMapping is None:
            ChanMapping = np.zeros((visIn.shape[1],), np.int32)
        if TranformModelInput == "FT":
            if float(_absmax(ModelImage)) == 0:
                return vis
            Grid = self.getFFTWMachine().fft(np.complex64(_np(ModelImage)).copy())
        self.ChanMappingDegrid = np.int32(ChanMapping)
        self.SumJonesChan = np.zeros((2, visIn.shape[1]), np.float64)
        if tuple(vis.shape) != tuple(flag.shape):
            raise Exception('vis[%s] and flag[%s] should have the same shape' % (str(vis.shape), str(flag.shape)))
        self.CheckTypes(Grid=Grid, vis=vis, uvw=uvw, flag=flag, ListWTerm=self.WTerm.Wplanes)
        if self.GD["RIME"]["ForwardMode"] != "BDA-degrid":
            raise ValueError("unknown --RIME-ForwardMode %s" % self.GD["RIME"]["ForwardMode"])
        jd, idirs = None, (0, 0)
        if DicoJonesMatrices is not None:
            jd, ik, ib = self.GiveParamJonesList(DicoJonesMatrices, times, _np(A0), _np(A1), uvw, degridder=True)
            jd.apply_amp = 1 if "A" in self.GD["DDESolutions"]["DDModeDeGrid"] else 0
            jd.apply_phase = 1 if "P" in self.GD["DDESolutions"]["DDModeDeGrid"] else 0
            if self.GD["DDESolutions"]["ScaleAmpDeGrid"]:
                jd.scale_jones = 1
                jd.calib_error = (self.GD["DDESolutions"]["CalibErr"] / 3600.) * np.pi / 180
            idirs = (ik, ib)
        dummy_w = np.ones(vis.shape[:2], np.float32)
        vs = self._visdata(vis, uvw, flag, dummy_w, freqs, np.int32(ChanMapping), self._bda_degrid, None)
        grid_t = Grid if isinstance(Grid, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(Grid)).to(self.device)
        fg = self._facet(grid_t, idirs=idirs)
        D.degrid(vs, [fg], D.make_pol(self.DataCorrelationFormat, self.ExpectedOutputStokes), jd)
        if isinstance(vis, torch.Tensor):
            if vs.vis.data_ptr() != vis.data_ptr():
                vis.copy_(vs.vis)
            return vis
        vis[...] = vs.vis.cpu().numpy()
        return vis

    # ---------------------------------------------------------------------------------- checks
    def CheckTypes(self, Grid=None, vis=None, uvw=None, flag=None, ListWTerm=None, W=None, A0=None, A1=None,
                   Jones=None):
        """ClassDDEGridMachine.CheckTypes (:863-920): NameError on dtype or contiguity mismatch."""
        def chk(x, dt, name, contig=True):
            if x is None:
                return
            if _dtype(x) != np.dtype(dt):
                raise NameError('%s.dtype %s' % (name, str(_dtype(x))))
            if contig and not _contig(x):
                raise NameError("%s has to be contiguous" % name)
        if Grid is not None:
            if _dtype(Grid) != self.dtype:
                raise NameError('Grid.dtype %s %s' % (str(_dtype(Grid)), str(self.dtype)))
            if not _contig(Grid):
                raise NameError("Grid has to be contiguous")
        chk(vis, np.complex64, "vis")
        chk(uvw, np.float64, "uvw")
        chk(flag, np.bool_, "flag")
        if ListWTerm is not None and ListWTerm[0].dtype != np.complex64:
            raise NameError('ListWTerm.dtype %s' % (str(ListWTerm[0].dtype)))
        chk(W, np.float32, "W")
        chk(A0, np.int32, "A0")
        chk(A1, np.int32, "A1")
        chk(Jones, np.complex64, "Jones")

    # ---------------------------------------------------------------------------------- images
    def setModelIm(self, ModelIm):
        _, _, n, n = ModelIm.shape
        x0, x1 = self.PaddingInnerCoord
        padded = np.zeros(self.GridShape, dtype=self.dtype)
        padded[:, :, x0:x1, x0:x1] = ModelIm
        return self.ImToGrid(padded) * n ** 2

    def ImToGrid(self, ModelIm):
        corr = ModelIm * (self.OverS * self.Padding) ** 2
        corr = (corr.real / self.ifzfCF.real).astype(np.complex64)
        return self.getFFTWMachine().fft(np.ascontiguousarray(corr))

    def GridToIm(self, Grid):
        """Grid *= OverS^2 and its inverse transform, in place (ClassDDEGridMachine.py:1186-1190)."""
        if isinstance(Grid, torch.Tensor):
            Grid.mul_(float(self.OverS) ** 2)
        else:
            Grid *= (self.OverS) ** 2
        return self.getFFTWMachine().ifft(Grid)


def pack_square_planes(planes):
    """One flat array ``[N, side_0 .. side_N-1, plane_0.ravel(), ...]`` holding N square planes,
    the layout a shared ``cf_dict["W"]`` carries (NpShared.PackListSquareMatrix, NpShared.py:288-308)."""
    dt = planes[0].dtype
    head = np.array([len(planes)] + [p.shape[0] for p in planes], dtype=dt)
    return np.concatenate([head] + [np.ascontiguousarray(p, dt).ravel() for p in planes])


def unpack_square_planes(flat):
    """Inverse of ``pack_square_planes`` (NpShared.UnPackListSquareMatrix, NpShared.py:311-331)."""
    n = int(np.real(flat[0]))
    sides = [int(np.real(x)) for x in flat[1:1 + n]]
    out, i = [], 1 + n
    for s in sides:
        out.append(flat[i:i + s * s].reshape(s, s))
        i += s * s
    return out


def _np(x):
    return x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def _dtype(x):
    if isinstance(x, torch.Tensor):
        return {torch.complex64: np.dtype(np.complex64), torch.complex128: np.dtype(np.complex128),
                torch.float32: np.dtype(np.float32), torch.float64: np.dtype(np.float64),
                torch.bool: np.dtype(np.bool_), torch.int32: np.dtype(np.int32)}.get(x.dtype, np.dtype(object))
    return np.asarray(x).dtype


def _contig(x):
    return x.is_contiguous() if isinstance(x, torch.Tensor) else bool(np.asarray(x).flags.c_contiguous)


def _absmax(x):
    return x.abs().max().item() if isinstance(x, torch.Tensor) else np.max(np.abs(x))
