"""The allocation-free block-map planner, ddfg_bda_plan_noalloc, against ddfg_bda_plan.

ddfg_bda_plan_noalloc serves callers that cannot allocate device memory at planning time (an
application whose pool allocator owns the GPU, a pipeline that forbids allocation after
start-up): it keeps its scratch in a fixed array inside the library instead of taking a
workspace.  This test calls it through the C ABI, twice in a row, and checks that each call's
block starts equal the workspace-taking entry point's exactly (the plan is integer work), that a
malformed map is still rejected and a good map after it still plans (the shared error word is
cleared on every call), that a map above the fixed limit is refused with a clear error, and that
a call leaves the device's free memory unchanged (it allocates nothing).
Run alone in a fresh process or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from ddfacet_b200 import _abi

    return _abi.lib(), _abi


def _maps():
    import cases
    from ddfacet_b200 import bda

    c = cases.make_case(nant=12, ntimes=40, nchan=16)
    plain = bda.plain_map(c.obs.A0, c.obs.A1, c.nchan)
    c2 = cases.make_case(nant=12, ntimes=40, nchan=16, bda_mode=1, dphi=np.sqrt(6 * 0.05))
    return [(plain, c.nrow, c.nchan), (c2.bda, c2.nrow, c2.nchan)]


def _plan_with_workspace(lib, abi, m, nrow, nchan):
    import torch

    nb = int(m[0]) + (int(m[1]) << 32)
    md = torch.from_numpy(m).cuda()
    out = torch.full((nb,), -1, dtype=torch.int64, device="cuda")
    ws = torch.empty(int(lib.ddfg_bda_plan_workspace_size(nb)), dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    single = C.c_int32(-1)
    abi.check(lib.ddfg_bda_plan(md.data_ptr(), md.numel(), nb, nrow, nchan, out.data_ptr(), ws.data_ptr(), ws.numel(), s,
                                C.byref(single)))
    return out.cpu().numpy(), single.value


def _plan_noalloc(lib, m, nrow, nchan, nb=None):
    import torch

    nb = int(m[0]) + (int(m[1]) << 32) if nb is None else nb
    md = torch.from_numpy(m).cuda()
    out = torch.full((max(min(nb, md.numel()), 1),), -1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    single = C.c_int32(-1)
    rc = lib.ddfg_bda_plan_noalloc(md.data_ptr(), md.numel(), nb, nrow, nchan, out.data_ptr(), s, C.byref(single))
    return rc, out.cpu().numpy()[:nb], single.value


def test_noalloc_plan_matches_workspace_plan_twice():
    lib, abi = _lib()
    for m, nrow, nchan in _maps():
        want, want_single = _plan_with_workspace(lib, abi, m, nrow, nchan)
        for _ in range(2):
            rc, got, single = _plan_noalloc(lib, m, nrow, nchan)
            assert rc == 0, abi.last_error()
            np.testing.assert_array_equal(got, want)
            assert single == want_single


def test_noalloc_rejects_bad_map_then_plans_again():
    lib, abi = _lib()
    m, nrow, nchan = _maps()[0]
    bad = m.copy()
    nb = int(m[0])
    bad[2 + nb + 2] = nrow  # first block's row == nrow: out of range
    rc, _, _ = _plan_noalloc(lib, bad, nrow, nchan)
    assert rc == abi.DDFG_EMAP
    assert "row outside" in abi.last_error()
    rc, got, _ = _plan_noalloc(lib, m, nrow, nchan)
    assert rc == 0, abi.last_error()
    np.testing.assert_array_equal(got, _plan_with_workspace(lib, abi, m, nrow, nchan)[0])


def test_noalloc_refuses_maps_above_its_limit():
    lib, abi = _lib()
    m, nrow, nchan = _maps()[0]
    limit = 1 << 24
    rc, _, _ = _plan_noalloc(lib, m, nrow, nchan, nb=limit + 1)
    assert rc == abi.DDFG_ESIZE
    assert "fixed scratch limit" in abi.last_error()


def test_noalloc_call_allocates_no_device_memory():
    import torch

    lib, abi = _lib()
    m, nrow, nchan = _maps()[1]
    nb = int(m[0]) + (int(m[1]) << 32)
    md = torch.from_numpy(m).cuda()
    out = torch.full((nb,), -1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    single = C.c_int32(-1)
    assert lib.ddfg_bda_plan_noalloc(md.data_ptr(), md.numel(), nb, nrow, nchan, out.data_ptr(), s,
                                     C.byref(single)) == 0, abi.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert lib.ddfg_bda_plan_noalloc(md.data_ptr(), md.numel(), nb, nrow, nchan, out.data_ptr(), s,
                                         C.byref(single)) == 0, abi.last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
