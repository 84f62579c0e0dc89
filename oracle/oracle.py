"""ctypes front end of the CPU restatement in af_oracle.cpp.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs, never by the product package.

``OracleOperator`` mirrors the reference's ``EULEROperator`` surface
(euler_operator.h:24-67): set_dt / set_Mach / set_Froude / set_HYPERBOLIC_stage /
set_NS_stage / set_rho_for_fixed / set_pres_fixed / set_u_fixed / vmult_rhs_rho_update /
vmult_rhs_pressure / vmult_rhs_velocity_fixed / vmult / vmult_pressure / vmult_enthalpy /
compute_diagonal, with numpy vectors in the deal.II DoF layout.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libaf_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp,
                                 ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_params.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_set_stages.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_set_sponge.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 8
        L.orc_set_fixed.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_rhs.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, ctypes.POINTER(dp), ctypes.c_int]
        L.orc_vmult.restype = ctypes.c_int
        L.orc_vmult.argtypes = [ctypes.c_void_p, dp, dp]
        L.orc_vmult_pressure.argtypes = [ctypes.c_void_p, dp, dp]
        L.orc_vmult_enthalpy.argtypes = [ctypes.c_void_p, dp, dp]
        L.orc_inverse_diagonal.argtypes = [ctypes.c_void_p, dp]
        L.orc_tables.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp]
        L.orc_imex_steps.restype = ctypes.c_int
        L.orc_imex_steps.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.c_int, ctypes.c_int]
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        L.orc_get_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_num_threads(n: int):
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return lib().orc_get_num_threads()


def tables(P, NQ):
    nodes = np.zeros(P + 1); qp = np.zeros(NQ); qw = np.zeros(NQ)
    S = np.zeros(NQ * (P + 1)); D = np.zeros(NQ * (P + 1))
    lib().orc_tables(P, NQ, _p(nodes), _p(qp), _p(qw), _p(S), _p(D))
    return nodes, qp, qw, S.reshape(NQ, P + 1), D.reshape(NQ, P + 1)


class OracleOperator:
    """CPU EULEROperator restatement; all vectors are float64 numpy arrays."""

    def __init__(self, mesh, degree, Ma, Fr, dt, n_q_1d=None, long_double=False):
        self.mesh = mesh
        self.P = degree
        self.NQ = n_q_1d if n_q_1d is not None else 2 * degree + 1
        self._vtx = _c(mesh.vertices)
        self.Ma, self.Fr, self.dt = Ma, Fr, dt
        self._h = lib().orc_create(self.P, self.NQ, mesh.nx, mesh.nz, int(mesh.periodic_x), _p(self._vtx),
                                   int(mesh.gravity), float(mesh.radial_a), Ma, Fr, dt, int(long_double))
        self.hyperbolic_stage = 1
        self.ns_stage = 1

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    @property
    def n_scalar(self):
        return self.mesh.n_cells * (self.P + 1) ** 2

    # --- setters (euler_operator.h:243-339) ---
    def _push(self):
        lib().orc_set_params(self._h, self.Ma, self.Fr, self.dt)
        lib().orc_set_stages(self._h, self.hyperbolic_stage, self.ns_stage)

    def set_dt(self, dt):
        self.dt = dt; self._push()

    def set_Mach(self, Ma):
        self.Ma = Ma; self._push()

    def set_Froude(self, Fr):
        self.Fr = Fr; self._push()

    def set_sponge(self, z_start, z_top, rate_top, x_left, x_right, width_lateral, rate_lateral, u_ref):
        """Rayleigh damping of the momentum towards (u_ref, 0) (the hill case's upper sponge and
        lateral relaxation zones, no counterpart in the reference); rates 0 switch it off."""
        on = int(rate_top > 0 or rate_lateral > 0)
        lib().orc_set_sponge(self._h, on, z_start, z_top, rate_top, x_left, x_right, width_lateral, rate_lateral,
                             u_ref)

    def set_HYPERBOLIC_stage(self, s):
        assert 1 <= s <= 3
        self.hyperbolic_stage = s; self._push()

    def set_NS_stage(self, s):
        assert 1 <= s <= 6
        self.ns_stage = s; self._push()

    def set_rho_for_fixed(self, v):
        lib().orc_set_fixed(self._h, 0, _p(_c(v)))

    def set_pres_fixed(self, v):
        lib().orc_set_fixed(self._h, 1, _p(_c(v)))

    def set_u_fixed(self, v):
        lib().orc_set_fixed(self._h, 2, _p(_c(v)))

    # --- explicit right-hand sides ---
    def _rhs(self, kind, src):
        src = [_c(s) for s in src]
        arr = (ctypes.POINTER(ctypes.c_double) * len(src))(*[_p(s) for s in src])
        n = self.n_scalar * (2 if kind == 2 else 1)
        dst = np.zeros(n)
        lib().orc_rhs(self._h, kind, _p(dst), arr, len(src))
        return dst

    def vmult_rhs_rho_update(self, src):
        return self._rhs(0, src)

    def vmult_rhs_pressure(self, src):
        return self._rhs(1, src)

    def vmult_rhs_velocity_fixed(self, src):
        return self._rhs(2, src)

    # --- implicit operators ---
    def vmult(self, src):
        ns = self.ns_stage
        n = self.n_scalar * (2 if ns in (3, 5) else 1)
        dst = np.zeros(n)
        self.last_inner_iterations = lib().orc_vmult(self._h, _p(dst), _p(_c(src)))
        return dst

    def vmult_pressure(self, src):
        dst = np.zeros(2 * self.n_scalar)
        lib().orc_vmult_pressure(self._h, _p(dst), _p(_c(src)))
        return dst

    def vmult_enthalpy(self, src):
        dst = np.zeros(self.n_scalar)
        lib().orc_vmult_enthalpy(self._h, _p(dst), _p(_c(src)))
        return dst

    def inverse_diagonal(self):
        ns = self.ns_stage
        n = self.n_scalar * (2 if ns in (3, 5) else 1)
        dst = np.zeros(n)
        lib().orc_inverse_diagonal(self._h, _p(dst))
        return dst


def imex_steps(op: OracleOperator, rho, u, p, nsteps, eps=1e-8, max_iterations=30000, fixed_point_tol=1e-10,
               fixed_point_max_iterations=100, gmres_restart=28, true_residual=False, exact_inverse=False):
    """EulerSolver::run time steps (Atmospheric_Flow.cc:1110-1251) on the CPU; returns the new
    (rho, u, p) and the fixed-point iteration counts of stages 1 and 2 of the last step.
    true_residual: the pressure GMRES is right-preconditioned and stops on |b - S x| (the
    criterion of the library's af_schur_solve) instead of the reference's |P^{-1} r|.
    exact_inverse: the mass-type systems and the A^{-1} inside the Schur apply are solved by
    dense cell-wise Cholesky factors (the library's default) instead of CG + Jacobi."""
    rho, u, p = _c(rho).copy(), _c(u).copy(), _c(p).copy()
    fp = (ctypes.c_int * 2)()
    r = lib().orc_imex_steps(op._h, _p(rho), _p(u), _p(p), nsteps, eps, max_iterations, fixed_point_tol,
                             fixed_point_max_iterations, gmres_restart, fp, int(bool(true_residual)),
                             int(bool(exact_inverse)))
    assert r == 0
    return rho, u, p, (fp[0], fp[1])


def cpu_port_rhs_fused_stage1(mesh, P, Ma, Fr, dt, src):
    """The tuned CPU port (af_cpu_port.cpp) of the fused stage-1 rhs triple: src = [rho0, u0,
    p0, rho_tmp_2, u_fixed]; returns (rho, u, p).  Gravity e_z only (the hill meshes)."""
    L = lib()
    if not getattr(L, "_port_bound", False):
        dp = ctypes.POINTER(ctypes.c_double)
        L.cpu_rhs_fused_stage1.restype = ctypes.c_int
        L.cpu_rhs_fused_stage1.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.POINTER(dp),
                                           dp, dp, dp]
        L._port_bound = True
    assert mesh.gravity == 0, "the CPU port implements the hill's vertical gravity only"
    src = [_c(s) for s in src]
    ns = mesh.n_cells * (P + 1) ** 2
    out = [np.empty(ns), np.empty(2 * ns), np.empty(ns)]
    arr = (ctypes.POINTER(ctypes.c_double) * 5)(*[_p(s) for s in src])
    vtx = _c(mesh.vertices)
    r = L.cpu_rhs_fused_stage1(P, mesh.nx, mesh.nz, int(mesh.periodic_x), _p(vtx), Ma, Fr, dt, arr,
                               _p(out[0]), _p(out[1]), _p(out[2]))
    assert r == 0, f"degree {P} not supported by the CPU port"
    return out
