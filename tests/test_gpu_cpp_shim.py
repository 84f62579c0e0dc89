"""The C++ header (include/af_euler_operator.hpp) driving libaf_gpu.so from a C++ program in
the shape of the reference's stage drivers (tests/cpp/shim_test.cpp)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_shim(tmp_path):
    pytest.importorskip("torch")
    libdir = os.path.join(ROOT, "atmospheric_flows_b200")
    exe = tmp_path / "shim_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "shim_test.cpp"), "-o", str(exe), "-L", libdir, "-laf_gpu",
                    "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}",
                    "-Wl,-rpath,/usr/local/cuda/lib64"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
