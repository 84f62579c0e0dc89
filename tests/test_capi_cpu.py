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
