"""Host logic of the drop-in ClassDDEGridMachine that runs without a GPU: the type checks and
their messages, the padded geometry, the shared cf_dict layout and the Jones direction choice
(ClassDDEGridMachine.py:308-679, 863-920; NpShared.py:288-331)."""
import numpy as np
import pytest

from ddfacet_b200.gridmachine import ClassDDEGridMachine, default_gd, pack_square_planes, unpack_square_planes


def _gm(**kw):
    GD = default_gd()
    GD["CF"]["Nw"] = 2
    GD["Image"]["Cell"] = 6.0
    args = dict(GD=GD, ChanFreq=np.linspace(1.3e9, 1.4e9, 4), Npix=301, lmShift=(0.01, -0.02), device="cpu")
    args.update(kw)
    return ClassDDEGridMachine(**args)


def test_geometry_matches_reference_rules():
    gm = _gm()
    # EstimateNpix: odd fast size, then padded and at least 513
    assert gm.NonPaddedNpix % 2 == 1 and gm.Npix % 2 == 1 and gm.Npix >= 513
    assert gm.GridShape == (1, 1, gm.Npix, gm.Npix)
    x0, x1 = gm.PaddingInnerCoord
    assert x1 - x0 == gm.NonPaddedNpix and x0 == (gm.Npix - gm.NonPaddedNpix) // 2
    np.testing.assert_allclose(gm.incr, np.array([-6.0, 6.0]) / 3600 * np.pi / 180)
    assert gm.SumWeigths.shape == (1, 1) and gm.SumJones.shape == (2, 1)


def test_check_types_messages():
    gm = _gm()
    with pytest.raises(NameError, match="vis.dtype"):
        gm.CheckTypes(vis=np.zeros((2, 2, 1), np.complex128))
    with pytest.raises(NameError, match="vis has to be contiguous"):
        gm.CheckTypes(vis=np.zeros((2, 4, 1), np.complex64)[:, ::2])
    with pytest.raises(NameError, match="uvw.dtype"):
        gm.CheckTypes(uvw=np.zeros((2, 3), np.float32))
    with pytest.raises(NameError, match="flag.dtype"):
        gm.CheckTypes(flag=np.zeros((2, 2, 1), np.uint8))
    with pytest.raises(NameError, match="W.dtype"):
        gm.CheckTypes(W=np.zeros((2, 2), np.float64))
    with pytest.raises(NameError, match="Grid.dtype"):
        gm.CheckTypes(Grid=np.zeros((1, 1, 3, 3), np.complex128))
    with pytest.raises(NameError, match="A0.dtype"):
        gm.CheckTypes(A0=np.zeros(3, np.int64))
    with pytest.raises(NameError, match="Jones.dtype"):
        gm.CheckTypes(Jones=np.zeros((1, 1, 1, 1, 2, 2), np.complex128))
    gm.CheckTypes(vis=np.zeros((2, 2, 1), np.complex64), uvw=np.zeros((2, 3)), flag=np.zeros((2, 2, 1), bool),
                  W=np.zeros((2, 2), np.float32))


def test_put_rejects_wrong_grid_dtype():
    gm = _gm()
    with pytest.raises(TypeError, match="Grid must be of type"):
        gm.put(None, np.zeros((2, 3)), np.zeros((2, 4, 1), np.complex64), np.zeros((2, 4, 1), bool),
               (np.zeros(2, np.int32), np.zeros(2, np.int32)), ResidueGrid=np.zeros(gm.GridShape, np.complex128))


def test_set_decorr():
    gm = _gm()
    with pytest.raises(NameError, match="uvw_dt.dtype"):
        gm.setDecorr(np.zeros((3, 3), np.float32), 10., 1e5)
    gm.setDecorr(np.zeros((3, 3)), 10., 1e5, SmearMode="F", lm_PhaseCenter=(0.001, 0.002))
    assert gm.LSmear[1:] == [10., 1e5, 0, 1, 0.01 - 0.001, -0.02 - 0.002]


def test_square_plane_packing_round_trip():
    rng = np.random.default_rng(0)
    planes = [(rng.standard_normal((s, s)) + 1j * rng.standard_normal((s, s))).astype(np.complex64) for s in (77, 33, 55)]
    flat = pack_square_planes(planes)
    assert flat.shape == (1 + 3 + sum(p.size for p in planes),) and flat[0] == 3
    for a, b in zip(unpack_square_planes(flat), planes):
        np.testing.assert_array_equal(a, b)


def test_cf_dict_round_trip():
    cfd = {}
    gm = _gm(cf_dict=cfd, compute_cf=True, wmax=2000.0)
    for k in ("Sphe", "InvSphe", "CuCv", "W", "wmax"):
        assert k in cfd
    gm2 = _gm(cf_dict=cfd, compute_cf=False)
    assert len(gm2.WTerm.Wplanes) == 2
    for a, b in zip(gm.WTerm.Wplanes + gm.WTerm.WplanesConj, gm2.WTerm.Wplanes + gm2.WTerm.WplanesConj):
        np.testing.assert_array_equal(a, b)
    assert (gm2.WTerm.Cu, gm2.WTerm.Cv) == (gm.WTerm.Cu, gm.WTerm.Cv)


def test_jones_directions():
    gm = _gm()
    dirs = {"l": np.array([0.5, 0.011, -0.3, 0.02]), "m": np.array([0.0, -0.019, 0.1, -0.02]), "I": np.ones(4)}
    dico = {"DicoJones_killMS": {"Dirs": dirs}, "DicoJones_Beam": {"Dirs": {"l": dirs["l"][::-1].copy(),
                                                                             "m": dirs["m"][::-1].copy()}}}
    ik, w, ib, interp, mode = gm.jones_directions(dico, gridder=True)
    assert ik == 1 and ib == 2 and interp == 0 and mode == 1
    assert abs(w.sum() - 1) < 1e-12 and np.count_nonzero(w) <= 3
    # the two nearby directions dominate the interpolation weights
    assert set(np.flatnonzero(w)) <= {1, 3, 2}
    gm.GD["Comp"]["BDAJones"] = "grid"
    assert gm.jones_directions(dico, gridder=True)[4] == 2
    assert gm.jones_directions(dico, gridder=False)[4] == 1
    gm.GD["Comp"]["BDAJones"] = "both"
    assert gm.jones_directions(dico, gridder=False)[4] == 2
