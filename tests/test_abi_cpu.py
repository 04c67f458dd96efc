"""The C ABI without a GPU: libddfg.so loads, exports every function include/ddfg.h declares,
and rejects bad arguments and unsupported correlation/Stokes combinations before touching a
device (messages as GridderSmearPols.cc:107-208, 243-346)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "ddfg.h")).read()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(ddfg_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_function():
    from ddfacet_b200 import _abi

    lib = _abi.lib()
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
        assert n in _abi.SIGNATURES, f"{n} has no ctypes signature"
    assert lib.ddfg_version() >= 1


def _call_grid(corr, stokes, nblocks=0):
    from ddfacet_b200 import _abi, device as D

    lib = _abi.lib()
    vs = _abi.VisSet()
    vs.ncorr = len(corr)
    vs.nblocks = nblocks
    js = _abi.Jones()
    pol = D.make_pol(corr, stokes)
    f = _abi.Facet()
    f.grid = f.cf_data = f.cf_offset = f.cf_support = 0x100
    f.nx = f.ny = 33
    f.nband = f.npol = f.nw = 1
    f.overs = 11
    f.max_support = 7
    f.wmax = 1.0
    arr = (_abi.Facet * 1)(f)
    return lib.ddfg_grid(C.byref(vs), C.byref(js), C.byref(pol), arr, 1, 0, None), _abi.last_error()


@pytest.mark.parametrize("corr,stokes,msg", [
    ([9, 12], [3], "Cannot convert input correlations"),
    ([2, 3], [1], "Only accepts I,RR,RL,LR,LL,XX,XY,YX,YY"),
    ([9, 10, 11, 12], [7], "Only accepts I,Q,U,V"),
])
def test_grid_dispatch_errors(corr, stokes, msg):
    from ddfacet_b200 import _abi

    rc, err = _call_grid(corr, stokes)
    assert rc == _abi.DDFG_EUNSUPPORTED
    assert msg in err


def test_null_and_size_checks():
    from ddfacet_b200 import _abi, device as D

    lib = _abi.lib()
    assert lib.ddfg_grid(None, None, None, None, 0, 0, None) == _abi.DDFG_EINVAL
    vs = _abi.VisSet()
    vs.ncorr = 1
    js = _abi.Jones()
    pol = D.make_pol([1], [1])
    arr = (_abi.Facet * 1)()
    assert lib.ddfg_grid(C.byref(vs), C.byref(js), C.byref(pol), arr, 5000, 0, None) == _abi.DDFG_ESIZE
    js.mode = 1  # Jones requested without any Jones arrays
    rc = lib.ddfg_degrid(C.byref(vs), C.byref(js), C.byref(pol), arr, 0, None)
    assert rc == _abi.DDFG_EINVAL and "neither E or DD Jones" in _abi.last_error()
    assert lib.ddfg_bda_plan_noalloc(None, 0, (1 << 24) + 1, 0, 0, None, None, None) == _abi.DDFG_ESIZE
