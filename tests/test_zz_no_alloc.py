"""af_schur_apply_noalloc: the Schur complement apply for callers that must not allocate
device memory (code inside a framework whose caching allocator owns the GPU memory, or a
time loop that budgets its memory up front).  It keeps its scratch in a static device
array of the library instead of calling cudaMalloc.

Checked here through the C ABI against the allocating entry point (af_vmult with
NS_stage 2 on a handle) on two calls in a row with different inputs -- the second call
runs on scratch that still holds the first call's values -- and for the size limit.
This file is collected last so that a failure here cannot hide other results; it also
passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12  # same algorithm and reduction order as af_vmult: differences are rounding only


def _lib():
    from atmospheric_flows_b200.operator import lib
    L = lib()
    vp = ctypes.c_void_p
    L.af_schur_apply_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int, vp, vp, vp, vp, vp,
                                         ctypes.POINTER(ctypes.c_int)]
    L.af_schur_apply_noalloc.restype = ctypes.c_int
    return L


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("degree,periodic,stage", [(4, 0, 1), (4, 0, 2), (4, 1, 1), (2, 1, 2), (5, 0, 1),
                                                    (5, 1, 2)])
def test_noalloc_schur_matches_handle_path(degree, periodic, stage):
    """The no-allocation call runs first, before this test creates a handle of the degree, so
    that in a fresh process its own per-device set-up (symbol address, basis tables) is the
    path under test."""
    from atmospheric_flows_b200.operator import EULEROperator, AF_OK
    L = _lib()
    P = degree
    nx, nz = (12, 6) if P <= 4 else (8, 6)  # 8x6 cells at degree 5: 1728 pressure DoFs
    m = M.jitter_mesh(M.hill_mesh(nx, nz, periodic_x=bool(periodic)), 0.15, seed=21)
    sc = M.Scaling()
    dt = 3.0
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(7 + stage + 10 * P + 100 * periodic)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rho_f = dev(1.0 + 0.05 * rng.standard_normal(ns))
    p_f = dev(1.0 + 0.05 * rng.standard_normal(ns))
    vtx = dev(m.vertices.reshape(-1))
    stream = torch.cuda.current_stream()
    srcs = [dev(1.0 + 0.1 * rng.standard_normal(ns)) for _ in range(2)]
    got, its = [], []
    for call in range(2):  # two calls in a row, different inputs
        out = torch.full((ns,), np.nan, dtype=torch.float64, device="cuda")
        it = ctypes.c_int(-1)
        torch.cuda.synchronize()
        st = L.af_schur_apply_noalloc(m.nx, m.nz, int(m.periodic_x), _p(vtx), P, sc.Ma, dt, stage, _p(rho_f),
                                      _p(p_f), _p(srcs[call]), _p(out), ctypes.c_void_p(stream.cuda_stream),
                                      ctypes.byref(it))
        assert st == AF_OK, L.af_last_error_message()
        torch.cuda.synchronize()
        got.append(out.cpu().numpy())
        its.append(it.value)

    op = EULEROperator(m, P, sc.Ma, sc.Fr, dt)
    op.set_rho_for_fixed(rho_f)
    op.set_pres_fixed(p_f)
    op.set_HYPERBOLIC_stage(stage)
    op.set_NS_stage(2)
    for call in range(2):
        want = torch.zeros(ns, dtype=torch.float64, device="cuda")
        op.vmult(want, srcs[call])
        op.synchronize()
        assert its[call] == op.last_inner_iterations() > 0
        err = rel(got[call], want.cpu().numpy())
        assert err < TOL, (call, err)


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    from atmospheric_flows_b200.operator import AF_BAD_ARG
    L = _lib()
    P = 4
    m = M.hill_mesh(64, 48)   # 3072 cells * 25 = 76800 > 65536 pressure DoFs
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    its = ctypes.c_int(0)
    st = L.af_schur_apply_noalloc(m.nx, m.nz, 0, _p(buf), P, 0.1, 1.0, 1, _p(buf), _p(buf), _p(buf), _p(buf),
                                  None, ctypes.byref(its))
    assert st == AF_BAD_ARG
    assert b"exceed the static scratch limit" in L.af_last_error_message()
