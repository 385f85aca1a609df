"""agd_eikonal_solve_fixed_scratch: the eikonal solve for callers that cannot
allocate device memory (host applications that own the device allocator,
code that must not call cudaMalloc at that point).  Its scratch is a fixed
device array inside the library instead of a caller workspace.

Checked through the C ABI against agd_eikonal_solve (caller workspace) on the
same instances, on two calls in a row, within the float32 tolerance of the
other parity tests.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import load_case, make_dictin

pytestmark = pytest.mark.gpu
REL = 1e-5


def _prepared(names):
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface
    itfs = []
    for name in names:
        case, _ = load_case(name)
        case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
        it = Interface(make_dictin(case))
        it.SetKernelTraits()
        it.SetGeometry()
        it.SetArgs()
        itfs.append(it)
    return itfs


def _solve(itfs, fixed):
    from adaptivegriddiscretizations_b200 import _lib
    L = _lib.lib()
    for it in itfs:
        it.values_t.fill_(float("inf"))
    arr = (_lib.AgdInstance * len(itfs))(*[it.instance() for it in itfs])
    stats = torch.zeros((len(itfs), 2), dtype=torch.int64, device="cuda")
    if fixed:
        _lib.check(L.agd_eikonal_solve_fixed_scratch(arr, len(itfs), _lib.ptr(stats), None, _lib.stream_ptr()))
    else:
        nbytes = L.agd_eikonal_workspace_bytes(arr, len(itfs))
        ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        _lib.check(L.agd_eikonal_solve(arr, len(itfs), _lib.ptr(ws), nbytes, _lib.ptr(stats), None,
                                       _lib.stream_ptr()))
    torch.cuda.synchronize()
    s = stats.cpu().numpy()
    assert not ((s[:, 0] >> 32) & 0xffffffff).any(), "solver status"
    return [it.squeeze(it.values_t).cpu().numpy() for it in itfs]


def _rel(a, b):
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a))
    return (np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1e-30)).max()


@pytest.mark.parametrize("names", [["riem2", "riem2_aniso", "iso2"], ["riem3", "iso3"]], ids=["2d", "3d"])
def test_fixed_scratch_matches_workspace_solve(names):
    itfs = _prepared(names)
    want = _solve(itfs, fixed=False)
    for _ in range(2):  # the array keeps the previous call's contents
        got = _solve(itfs, fixed=True)
        for g, w in zip(got, want):
            assert _rel(g, w) < REL


def test_fixed_scratch_rejects_oversized_requests():
    from adaptivegriddiscretizations_b200 import _lib
    L = _lib.lib()
    big = _lib.AgdInstance(model=_lib.AGD_MODEL_ISOTROPIC, ndim=3, niter_i=8, fim_front_width=4, nitermax_o=10)
    for k in range(3):
        big.shape[k] = 640
        big.shape_i[k] = 4
    dummy = torch.empty(4, device="cuda")
    big.values = big.rhs = big.seedbits = dummy.data_ptr()
    rc = L.agd_eikonal_solve_fixed_scratch(ctypes.byref(big), 1, None, None, _lib.stream_ptr())
    assert rc == _lib.AGD_STATUS_WORKSPACE
    assert b"AGD_FIXED_SCRATCH_BYTES" in L.agd_last_error()
