"""CPU-side checks of the C ABI: the library loads, exports every function that
include/*.h declares, and validates arguments on the host (no GPU compute here)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(af_[A-Za-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_all_declared_symbols():
    from atmospheric_flows_b200 import operator as O
    L = O.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert _declared(), "no declarations found"
    assert not missing, missing


def test_error_strings():
    from atmospheric_flows_b200 import operator as O
    L = O.lib()
    assert L.af_error_string(O.AF_OK) == b"ok"
    assert L.af_error_string(O.AF_NO_CONVERGENCE) == b"no convergence"
    assert L.af_error_string(O.AF_TIMEOUT) == b"a kernel gave up a bounded wait"


def test_stage_wait_test_hook_validates_on_host():
    """The failure-detection test hook rejects a null handle and negative poll counts
    without touching a device."""
    from atmospheric_flows_b200 import operator as O
    L = O.lib()
    assert L.af_set_stage_wait_test(None, 4) == O.AF_BAD_ARG


def test_create_rejects_bad_arguments_on_host():
    """Argument validation happens before any device call."""
    from atmospheric_flows_b200 import operator as O
    from atmospheric_flows_b200 import mesh as M
    L = O.lib()
    m = M.box_mesh(4, 2)
    v = np.ascontiguousarray(m.vertices)
    desc = O._MeshDesc(4, 2, 0, v.ctypes.data, 0, 0.0)
    h = ctypes.c_void_p()
    assert L.af_create(ctypes.byref(desc), 4, 7, 1.0, 1.0, 1.0, ctypes.byref(h)) == O.AF_BAD_ARG  # n_q != 2p+1
    assert b"2*degree+1" in L.af_last_error_message()
    assert L.af_create(ctypes.byref(desc), 9, 19, 1.0, 1.0, 1.0, ctypes.byref(h)) == O.AF_UNSUPPORTED
    bad = O._MeshDesc(0, 2, 0, v.ctypes.data, 0, 0.0)
    assert L.af_create(ctypes.byref(bad), 4, 9, 1.0, 1.0, 1.0, ctypes.byref(h)) == O.AF_BAD_ARG
    assert L.af_set_NS_stage(None, 7) == O.AF_BAD_ARG


def test_cpp_header_compiles():
    """include/af_euler_operator.hpp is self-contained C++17 over af_gpu.h."""
    import subprocess
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = "#include \"af_euler_operator.hpp\"\nint main() { return 0; }\n"
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
                        "-x", "c++", "-"], input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_imex_options_are_checked_on_the_host_and_no_device_fails_loudly():
    """af_imex_create rejects bad options before any device call; with valid arguments and no
    CUDA device (this CPU run) the library returns AF_NO_DEVICE and no handle, with no CPU
    fallback."""
    from atmospheric_flows_b200 import operator as O
    from atmospheric_flows_b200 import imex as I
    from atmospheric_flows_b200 import mesh as M
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present: the no-device path is not reachable")
    except ImportError:
        pass
    L = O.lib()
    m = M.hill_mesh(4, 2)
    v = np.ascontiguousarray(m.vertices)
    desc = O._MeshDesc(4, 2, 0, v.ctypes.data, 0, 0.0)
    d = I.Options()
    L.af_imex_default_options(ctypes.byref(d))
    assert d.schur_poly_degree == 0 and d.schur_preconditioner == -1 and d.eps == 1e-8
    h = ctypes.c_void_p()
    args = (ctypes.c_double(1.0), ctypes.c_double(1.0), ctypes.c_double(0.5))
    for field, bad in (("eps", -1.0), ("gmres_restart", 61), ("schur_poly_degree", -1),
                       ("schur_preconditioner", 9), ("mass_solver", 2), ("fixed_point_max_iterations", 0)):
        o = I.Options()
        L.af_imex_default_options(ctypes.byref(o))
        setattr(o, field, bad)
        assert L.af_imex_create(ctypes.byref(desc), 4, *args, ctypes.byref(o), ctypes.byref(h)) == O.AF_BAD_ARG, field
        assert b"bad options" in L.af_last_error_message()
        assert h.value is None
    assert L.af_imex_create(ctypes.byref(desc), 4, *args, ctypes.byref(d), ctypes.byref(h)) == O.AF_NO_DEVICE
    assert h.value is None
    op = ctypes.c_void_p()
    assert L.af_create(ctypes.byref(desc), 4, 9, *args, ctypes.byref(op)) == O.AF_NO_DEVICE
    assert op.value is None


def test_noalloc_schur_apply_checks_arguments_on_the_host():
    """af_schur_apply_noalloc validates its arguments before it touches a device: null or
    unaligned pointers, the stage, the degree and the static scratch limit (65536 pressure
    DoFs) are rejected on the host; with valid arguments and no CUDA device it returns
    AF_NO_DEVICE.  No pointer is dereferenced on these paths."""
    from atmospheric_flows_b200 import operator as O
    from atmospheric_flows_b200 import mesh as M
    L = O.lib()
    vp = ctypes.c_void_p
    L.af_schur_apply_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, vp, vp, vp, vp, vp,
                                         ctypes.POINTER(ctypes.c_int)]
    L.af_schur_apply_noalloc.restype = ctypes.c_int
    m = M.hill_mesh(4, 2)
    buf = np.zeros(4096, dtype=np.float64)  # stands in for device memory: never read here
    base = buf.ctypes.data + (-buf.ctypes.data) % 16
    p = vp(base)
    it = ctypes.c_int(-1)

    def call(nx=4, nz=2, degree=4, stage=1, ptrs=None, mach=1.0, dt=1.0):
        a = ptrs or [p] * 5
        return L.af_schur_apply_noalloc(nx, nz, 0, a[0], degree, mach, dt, stage, a[1], a[2], a[3], a[4], None,
                                        ctypes.byref(it))

    assert call(ptrs=[p, p, None, p, p]) == O.AF_BAD_ARG
    assert b"null pointer" in L.af_last_error_message()
    assert call(stage=3) == O.AF_BAD_ARG
    assert call(mach=0.0) == O.AF_BAD_ARG
    assert call(degree=9) == O.AF_UNSUPPORTED
    assert call(nx=64, nz=64) == O.AF_BAD_ARG  # 4096 cells x 25 = 102400 pressure DoFs
    assert b"static scratch limit" in L.af_last_error_message()
    assert call(ptrs=[p, p, p, vp(base + 8), p]) == O.AF_BAD_ARG
    assert b"16-byte aligned" in L.af_last_error_message()
    assert m.n_cells * 25 <= 65536
    try:
        import torch
        if torch.cuda.is_available():
            return  # a CUDA device is present: the no-device path is not reachable
    except ImportError:
        pass
    assert call() == O.AF_NO_DEVICE
    assert it.value == -1
