"""IMEX-DG time stepping on the GPU (the reference's EulerSolver::run time loop,
Atmospheric_Flow.cc:1100-1257) over the C ABI of libaf_gpu.so (af_imex_*)."""
from __future__ import annotations

import ctypes

import numpy as np

from .operator import _MeshDesc, _ptr, check, lib
from .schur import NAMES as SCHUR_NAMES


class Options(ctypes.Structure):
    _fields_ = [("eps", ctypes.c_double), ("max_iterations", ctypes.c_int), ("fixed_point_tol", ctypes.c_double),
                ("fixed_point_max_iterations", ctypes.c_int), ("gmres_restart", ctypes.c_int),
                ("mass_solver", ctypes.c_int), ("schur_inner", ctypes.c_int), ("schur_preconditioner", ctypes.c_int),
                ("schur_poly_degree", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("fixed_point_iterations", ctypes.c_int * 2), ("gmres_iterations", ctypes.c_longlong),
                ("cg_iterations", ctypes.c_longlong), ("last_fixed_point_error", ctypes.c_double)]


def _bind():
    L = lib()
    if getattr(L, "_imex_bound", False):
        return L
    vp = ctypes.c_void_p
    L.af_imex_default_options.argtypes = [ctypes.POINTER(Options)]
    L.af_imex_create.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.POINTER(Options), ctypes.POINTER(vp)]
    L.af_imex_destroy.argtypes = [vp]
    L.af_imex_operator.restype = vp
    L.af_imex_operator.argtypes = [vp]
    L.af_imex_set_state.argtypes = [vp, vp, vp, vp]
    L.af_imex_get_state.argtypes = [vp, vp, vp, vp]
    L.af_imex_step.argtypes = [vp, ctypes.c_int]
    L.af_imex_last_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.af_imex_stage1_forward.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.af_imex_stage1_tangent.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_double]
    L.af_imex_stage1_backward.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_double]
    L.af_imex_step_forward.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.af_imex_step_tangent.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_double]
    L.af_imex_step_backward.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_double]
    L.af_imex_gradient.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp,
                                   ctypes.c_double]
    L._imex_bound = True
    return L


class IMEXStepper:
    """GPU time stepper: set_state(rho, u, p) -> step(n) -> get_state()."""

    def __init__(self, mesh, degree, Ma, Fr, dt, eps=None, max_iterations=None, fixed_point_tol=None,
                 fixed_point_max_iterations=None, gmres_restart=None, mass_solver=None, schur_inner=None,
                 schur_preconditioner=None, schur_poly_degree=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("IMEXStepper needs a CUDA device (no CPU fallback)")
        L = _bind()
        torch.cuda.current_device()
        opt = Options()
        check(L.af_imex_default_options(ctypes.byref(opt)))
        for k, v in (("eps", eps), ("max_iterations", max_iterations), ("fixed_point_tol", fixed_point_tol),
                     ("fixed_point_max_iterations", fixed_point_max_iterations), ("gmres_restart", gmres_restart),
                     ("mass_solver", mass_solver), ("schur_inner", schur_inner),
                     ("schur_preconditioner", SCHUR_NAMES.get(schur_preconditioner, schur_preconditioner)),
                     ("schur_poly_degree", schur_poly_degree)):
            if v is not None:
                setattr(opt, k, v)
        self.mesh, self.degree = mesh, degree
        self._vtx = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
        desc = _MeshDesc(mesh.nx, mesh.nz, int(mesh.periodic_x), self._vtx.ctypes.data, int(mesh.gravity),
                         float(mesh.radial_a))
        h = ctypes.c_void_p()
        check(L.af_imex_create(ctypes.byref(desc), degree, Ma, Fr, dt, ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self._destroy = L.af_imex_destroy  # kept: module globals may be gone when __del__ runs at exit
        self.n_scalar = mesh.n_cells * (degree + 1) ** 2

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._destroy(h)
            self._h = None

    def set_state(self, rho, u, p):
        check(_bind().af_imex_set_state(self._h, _ptr(rho), _ptr(u), _ptr(p)))

    def get_state(self):
        import torch
        rho = torch.empty(self.n_scalar, dtype=torch.float64, device="cuda")
        u = torch.empty(2 * self.n_scalar, dtype=torch.float64, device="cuda")
        p = torch.empty(self.n_scalar, dtype=torch.float64, device="cuda")
        check(_bind().af_imex_get_state(self._h, _ptr(rho), _ptr(u), _ptr(p)))
        return rho, u, p

    def step(self, n=1):
        check(_bind().af_imex_step(self._h, n))

    def set_sponge(self, z_start, z_top, rate_top, x_left, x_right, width_lateral, rate_lateral, u_ref):
        """Rayleigh damping of the momentum (af_set_sponge on the stepper's operator)."""
        from atmospheric_flows_b200.operator import lib as oplib
        L = oplib()
        check(L.af_set_sponge(_bind().af_imex_operator(self._h), z_start, z_top, rate_top, x_left, x_right,
                              width_lateral, rate_lateral, u_ref))

    def _triple(self):
        import torch
        return (torch.empty(self.n_scalar, dtype=torch.float64, device="cuda"),
                torch.empty(2 * self.n_scalar, dtype=torch.float64, device="cuda"),
                torch.empty(self.n_scalar, dtype=torch.float64, device="cuda"))

    def stage1_forward(self, rho0, u0, p0):
        """Stage 1 (density update and pressure fixed point) from (rho0, u0, p0), recording the
        linearisation point of stage1_tangent / stage1_backward; returns (rho2, u2, p2)."""
        r, u, p = self._triple()
        check(_bind().af_imex_stage1_forward(self._h, _ptr(rho0), _ptr(u0), _ptr(p0), _ptr(r), _ptr(u), _ptr(p)))
        return r, u, p

    def stage1_tangent(self, drho0, du0, dp0, rel_tol=1e-13):
        """(drho2, du2, dp2) = J (drho0, du0, dp0) at the last stage1_forward"""
        r, u, p = self._triple()
        check(_bind().af_imex_stage1_tangent(self._h, _ptr(drho0), _ptr(du0), _ptr(dp0), _ptr(r), _ptr(u), _ptr(p),
                                             rel_tol))
        return r, u, p

    def step_forward(self, rho0, u0, p0):
        """One IMEX step from (rho0, u0, p0), recording the linearisation point of step_tangent /
        step_backward; returns the new state (also the stepper's state)."""
        r, u, p = self._triple()
        check(_bind().af_imex_step_forward(self._h, _ptr(rho0), _ptr(u0), _ptr(p0), _ptr(r), _ptr(u), _ptr(p)))
        return r, u, p

    def step_tangent(self, drho0, du0, dp0, rel_tol=1e-13):
        r, u, p = self._triple()
        check(_bind().af_imex_step_tangent(self._h, _ptr(drho0), _ptr(du0), _ptr(dp0), _ptr(r), _ptr(u), _ptr(p),
                                           rel_tol))
        return r, u, p

    def step_backward(self, rho1bar, u1bar, p1bar, rel_tol=1e-13):
        r, u, p = self._triple()
        check(_bind().af_imex_step_backward(self._h, _ptr(rho1bar), _ptr(u1bar), _ptr(p1bar), _ptr(r), _ptr(u),
                                            _ptr(p), rel_tol))
        return r, u, p

    def gradient(self, rho0, u0, p0, nsteps, checkpoint_every, rhobar, ubar, pbar, rel_tol=1e-12):
        """(d state_N / d state_0)^T (rhobar, ubar, pbar) with checkpointed recomputation."""
        r, u, p = self._triple()
        check(_bind().af_imex_gradient(self._h, _ptr(rho0), _ptr(u0), _ptr(p0), nsteps, checkpoint_every,
                                       _ptr(rhobar), _ptr(ubar), _ptr(pbar), _ptr(r), _ptr(u), _ptr(p), rel_tol))
        return r, u, p

    def stage1_backward(self, rho2bar, u2bar, p2bar, rel_tol=1e-13):
        """(rho0bar, u0bar, p0bar) = J^T (rho2bar, u2bar, p2bar) at the last stage1_forward"""
        r, u, p = self._triple()
        check(_bind().af_imex_stage1_backward(self._h, _ptr(rho2bar), _ptr(u2bar), _ptr(p2bar), _ptr(r), _ptr(u),
                                              _ptr(p), rel_tol))
        return r, u, p

    def stats(self):
        s = Stats()
        check(_bind().af_imex_last_stats(self._h, ctypes.byref(s)))
        return {"fixed_point_iterations": tuple(s.fixed_point_iterations), "gmres_iterations": s.gmres_iterations,
                "cg_iterations": s.cg_iterations, "last_fixed_point_error": s.last_fixed_point_error}
