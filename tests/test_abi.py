"""The C ABI library loads and exports every entry point include/*.h declares
(no device work: runs without a GPU)."""
import os
import re

from conftest import REPO


def _declared():
    names = set()
    inc = os.path.join(REPO, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            src = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, f)).read(), flags=re.S)
            names |= set(re.findall(r"\b(agd_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_declared_symbols():
    from adaptivegriddiscretizations_b200 import _lib
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 19
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_no_gpu_entry_points_report_errors_cleanly():
    import ctypes
    from adaptivegriddiscretizations_b200 import _lib
    L = _lib.lib()
    plan = ctypes.c_void_p()
    assert L.agd_plan_create(None, 0, ctypes.byref(plan)) == _lib.AGD_STATUS_INVALID
    assert b"no instance" in L.agd_last_error()
    inst = _lib.AgdInstance(model=1, ndim=2, niter_i=8, fim_front_width=4, nitermax_o=10)
    inst.shape[0], inst.shape[1], inst.shape[2] = 10, 10, 1
    inst.shape_i[0], inst.shape_i[1], inst.shape_i[2] = 5, 5, 1
    assert L.agd_plan_create(ctypes.byref(inst), 1, ctypes.byref(plan)) == _lib.AGD_STATUS_UNSUPPORTED
