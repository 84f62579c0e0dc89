"""Schur-complement pressure solver (the linear solve of the reference's pressure_fixed_point,
Atmospheric_Flow.cc:544-673) over the C ABI of libaf_gpu.so (af_schur_*).

``SchurSolver(op, preconditioner)`` wraps flexible GMRES in FP64 around the operator's
NS_stage-2 apply with a Jacobi (diag D), geometric-multigrid (FP64 or FP32 levels) or
single-level Chebyshev-polynomial (FP64 or FP32) preconditioner.  Vectors are CUDA float64 tensors in the pressure space; the solver runs on
the operator's stream.
"""
from __future__ import annotations

import ctypes

from .operator import AFError, _ptr, check, lib

JACOBI, MG_FP64, MG_FP32, CHEB_FP64, CHEB_FP32 = 0, 1, 2, 3, 4
NAMES = {"jacobi": JACOBI, "mg_fp64": MG_FP64, "mg_fp32": MG_FP32, "cheb_fp64": CHEB_FP64, "cheb_fp32": CHEB_FP32}


class Options(ctypes.Structure):
    _fields_ = [("preconditioner", ctypes.c_int), ("smoother_degree", ctypes.c_int),
                ("smoothing_range", ctypes.c_double), ("coarse_degree", ctypes.c_int),
                ("max_levels", ctypes.c_int), ("min_coarse_cells", ctypes.c_int),
                ("eig_iterations", ctypes.c_int), ("restart", ctypes.c_int), ("coarse_lmax", ctypes.c_double),
                ("poly_degree", ctypes.c_int), ("reduced_quadrature", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("initial_residual", ctypes.c_double),
                ("final_residual", ctypes.c_double), ("seconds", ctypes.c_double)]


def _bind():
    L = lib()
    if getattr(L, "_schur_bound", False):
        return L
    vp = ctypes.c_void_p
    L.af_schur_default_options.argtypes = [ctypes.POINTER(Options)]
    L.af_schur_solver_create.argtypes = [vp, ctypes.POINTER(Options), ctypes.POINTER(vp)]
    L.af_schur_solver_destroy.argtypes = [vp]
    L.af_schur_solver_setup.argtypes = [vp, ctypes.c_int]
    L.af_schur_solver_levels.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    L.af_schur_solver_precondition.argtypes = [vp, vp, vp]
    L.af_schur_solve.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(Stats)]
    L.af_schur_solve_transpose.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(Stats)]
    L._schur_bound = True
    return L


def default_options():
    opt = Options()
    check(_bind().af_schur_default_options(ctypes.byref(opt)))
    return opt


class SchurSolver:
    """FGMRES for (D - C A^{-1} B) p = b on an EULEROperator (its rho_for_fixed and
    pres_fixed must be set before ``setup``)."""

    def __init__(self, op, preconditioner="cheb_fp32", **options):
        L = _bind()
        opt = default_options()
        opt.preconditioner = NAMES[preconditioner] if isinstance(preconditioner, str) else int(preconditioner)
        for k, v in options.items():
            if not hasattr(opt, k):
                raise TypeError(f"unknown option {k}")
            setattr(opt, k, v)
        h = ctypes.c_void_p()
        check(L.af_schur_solver_create(op._h, ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self._destroy = L.af_schur_solver_destroy  # kept: module globals may be gone at exit
        self.op = op  # keeps the operator alive
        self.options = opt

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._destroy(h)
            self._h = None

    def setup(self, estimate_eigenvalues=False):
        check(_bind().af_schur_solver_setup(self._h, int(estimate_eigenvalues)))

    def levels(self):
        """Per-level eigenvalue estimates lmax of D^{-1} S0 (finest first)."""
        n = ctypes.c_int()
        lm = (ctypes.c_double * 32)()
        check(_bind().af_schur_solver_levels(self._h, ctypes.byref(n), lm))
        return [lm[i] for i in range(n.value)]

    def precondition(self, dst, src):
        check(_bind().af_schur_solver_precondition(self._h, _ptr(dst), _ptr(src)))

    def solve_transpose(self, p, x, b, rel_tol=1e-10, max_iterations=1000, raise_on_failure=True):
        """Adjoint solve J_S(p)^T x = b (x: initial guess in, solution out)."""
        st = Stats()
        r = _bind().af_schur_solve_transpose(self._h, _ptr(p), _ptr(x), _ptr(b), rel_tol, max_iterations,
                                             ctypes.byref(st))
        return self._result(r, st, raise_on_failure)

    def solve(self, x, b, rel_tol=1e-10, max_iterations=1000, raise_on_failure=True):
        """x: initial guess in, solution out.  Returns the stats dict."""
        st = Stats()
        r = _bind().af_schur_solve(self._h, _ptr(x), _ptr(b), rel_tol, max_iterations, ctypes.byref(st))
        return self._result(r, st, raise_on_failure)

    def _result(self, r, st, raise_on_failure):
        out = {"iterations": st.iterations, "initial_residual": st.initial_residual,
               "final_residual": st.final_residual, "seconds": st.seconds, "status": r}
        if r != 0 and raise_on_failure:
            raise AFError(r, lib().af_last_error_message().decode())
        return out
