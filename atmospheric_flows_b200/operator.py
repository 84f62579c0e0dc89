"""Python mirror of the reference's ``EULEROperator`` (euler_operator.h:24-211) over the
C ABI of libaf_gpu.so (include/af_gpu.h).

Method names, argument meaning and positional source lists follow the reference; vectors
are CUDA float64 torch tensors in deal.II's DoF layout (see atmospheric_flows_b200.mesh).
There is no CPU fallback: constructing an operator without the CUDA library or without a
GPU raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaf_gpu.so")

AF_OK, AF_BAD_ARG, AF_CUDA, AF_NO_CONVERGENCE, AF_NAN, AF_UNSUPPORTED, AF_NO_DEVICE, AF_TIMEOUT = range(8)

_lib = None


class AFError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"libaf_gpu status {status}: {msg}")
        self.status = status


def lib():
    """Load libaf_gpu.so (built by __graft_entry__.build / make -C atmospheric_flows_b200/csrc)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C atmospheric_flows_b200/csrc`")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, ip = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int
        L.af_create.argtypes = [vp, ip, ip, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.POINTER(vp)]
        for name in ("af_destroy", "af_synchronize"):
            getattr(L, name).argtypes = [vp]
        L.af_set_stream.argtypes = [vp, vp]
        for name in ("af_set_dt", "af_set_Mach", "af_set_Froude"):
            getattr(L, name).argtypes = [vp, ctypes.c_double]
        for name in ("af_set_HYPERBOLIC_stage", "af_set_NS_stage"):
            getattr(L, name).argtypes = [vp, ip]
        for name in ("af_set_rho_for_fixed", "af_set_pres_fixed", "af_set_u_fixed"):
            getattr(L, name).argtypes = [vp, dp]
        for name in ("af_vmult_rhs_rho_update", "af_vmult_rhs_velocity_fixed", "af_vmult_rhs_pressure"):
            getattr(L, name).argtypes = [vp, dp, ctypes.POINTER(dp), ip]
        L.af_vmult_rhs_fused.argtypes = [vp, dp, dp, dp, ctypes.POINTER(dp), ip]
        L.af_vmult_rhs_fused_host.argtypes = [vp, dp, dp, dp, ctypes.POINTER(dp), ip]
        L.af_vmult_rhs_fused_backward.argtypes = [vp, ctypes.POINTER(dp), ip, dp, dp, dp, ctypes.POINTER(dp)]
        L.af_vmult_rhs_fused_tangent.argtypes = [vp, ctypes.POINTER(dp), ip, ctypes.POINTER(dp), dp, dp, dp]
        for name in ("af_vmult", "af_vmult_pressure", "af_vmult_enthalpy", "af_vmult_inverse"):
            getattr(L, name).argtypes = [vp, dp, dp]
        L.af_compute_diagonal.argtypes = [vp, dp]
        L.af_set_schur_mode.argtypes = [vp, ip, ctypes.c_double, ip]
        L.af_last_inner_iterations.argtypes = [vp, ctypes.POINTER(ip)]
        L.af_n_dofs.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_longlong)]
        L.af_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        for name in ("af_vmult_pressure_transpose",):
            getattr(L, name).argtypes = [vp, dp, dp]
        for name in ("af_vmult_enthalpy_tangent", "af_vmult_enthalpy_transpose", "af_schur_tangent",
                     "af_schur_transpose", "af_vmult_velocity_mass_rho_transpose",
                     "af_vmult_enthalpy_pf_transpose"):
            getattr(L, name).argtypes = [vp, dp, dp, dp]
        L.af_compute_diagnostics.argtypes = [vp, dp, dp, dp, dp, ctypes.POINTER(Diagnostics)]
        L.af_l2_norm.argtypes = [vp, ip, dp, ctypes.POINTER(ctypes.c_double)]
        L.af_set_stage_wait_test.argtypes = [vp, ip]
        L.af_set_sponge.argtypes = [vp] + [ctypes.c_double] * 8
        L.af_error_string.restype = ctypes.c_char_p
        L.af_error_string.argtypes = [ip]
        L.af_last_error_message.restype = ctypes.c_char_p
        _lib = L
    return _lib


class Diagnostics(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("max_velocity", "min_density", "max_density", "max_celerity",
                                                "min_cell_diameter", "cfl_c", "cfl_u")]


def check(status):
    if status != AF_OK:
        raise AFError(status, lib().af_last_error_message().decode())


class _MeshDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("periodic_x", ctypes.c_int),
                ("vertices", ctypes.c_void_p), ("gravity", ctypes.c_int), ("radial_a", ctypes.c_double)]


def _ptr(t):
    if t is None:
        return None
    import torch
    assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous(), "need contiguous CUDA float64 tensors"
    return ctypes.c_void_p(t.data_ptr())


def _ptr_array(ts):
    arr = (ctypes.c_void_p * len(ts))()
    for k, t in enumerate(ts):
        arr[k] = _ptr(t).value
    return arr


class EULEROperator:
    """GPU EULEROperator.  ``mesh`` is an atmospheric_flows_b200.mesh.Mesh."""

    def __init__(self, mesh, degree, Ma, Fr, dt, n_q_points_1d=None, stream=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("EULEROperator needs a CUDA device (no CPU fallback)")
        self.mesh = mesh
        self.degree = degree
        self.n_q = n_q_points_1d if n_q_points_1d is not None else 2 * degree + 1
        self._vtx = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
        desc = _MeshDesc(mesh.nx, mesh.nz, int(mesh.periodic_x), self._vtx.ctypes.data, int(mesh.gravity),
                         float(mesh.radial_a))
        h = ctypes.c_void_p()
        torch.cuda.current_device()  # make the context current before the library uses it
        check(lib().af_create(ctypes.byref(desc), degree, self.n_q, Ma, Fr, dt, ctypes.byref(h)))
        self._h = h
        self._destroy = lib().af_destroy  # kept: module globals may be gone when __del__ runs at exit
        self.Ma, self.Fr, self.dt = Ma, Fr, dt
        self.HYPERBOLIC_stage, self.NS_stage = 1, 1
        if stream is not None:
            self.set_stream(stream)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._destroy(h)
            self._h = None

    # --- plumbing ---
    def set_stream(self, stream):
        """Run on a torch stream (None: the handle's own stream).  torch's default stream has
        handle 0, which the C ABI reads as "own stream"; it is passed as cudaStreamLegacy (0x1)."""
        if stream is None:
            h = 0
        else:
            h = stream.cuda_stream or 1  # cudaStreamLegacy
        check(lib().af_set_stream(self._h, ctypes.c_void_p(h)))

    def synchronize(self):
        check(lib().af_synchronize(self._h))

    def n_dofs(self, space):
        n = ctypes.c_longlong()
        check(lib().af_n_dofs(self._h, space, ctypes.byref(n)))
        return n.value

    def launch_count(self):
        n = ctypes.c_longlong()
        check(lib().af_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def initialize_dof_vector(self, space):
        import torch
        return torch.zeros(self.n_dofs(space), dtype=torch.float64, device="cuda")

    # --- setters (euler_operator.h:243-339) ---
    def set_dt(self, dt):
        check(lib().af_set_dt(self._h, dt)); self.dt = dt

    def set_Mach(self, Ma):
        check(lib().af_set_Mach(self._h, Ma)); self.Ma = Ma

    def set_Froude(self, Fr):
        check(lib().af_set_Froude(self._h, Fr)); self.Fr = Fr

    def set_HYPERBOLIC_stage(self, s):
        check(lib().af_set_HYPERBOLIC_stage(self._h, s)); self.HYPERBOLIC_stage = s

    def set_NS_stage(self, s):
        check(lib().af_set_NS_stage(self._h, s)); self.NS_stage = s

    def set_rho_for_fixed(self, v):
        check(lib().af_set_rho_for_fixed(self._h, _ptr(v)))

    def set_pres_fixed(self, v):
        check(lib().af_set_pres_fixed(self._h, _ptr(v)))

    def set_u_fixed(self, v):
        check(lib().af_set_u_fixed(self._h, _ptr(v)))

    # --- explicit right-hand sides ---
    def vmult_rhs_rho_update(self, dst, src):
        check(lib().af_vmult_rhs_rho_update(self._h, _ptr(dst), _ptr_array(src), len(src)))

    def vmult_rhs_velocity_fixed(self, dst, src):
        check(lib().af_vmult_rhs_velocity_fixed(self._h, _ptr(dst), _ptr_array(src), len(src)))

    def vmult_rhs_pressure(self, dst, src):
        check(lib().af_vmult_rhs_pressure(self._h, _ptr(dst), _ptr_array(src), len(src)))

    def vmult_rhs_fused(self, dst_rho, dst_u, dst_p, src):
        check(lib().af_vmult_rhs_fused(self._h, _ptr(dst_rho), _ptr(dst_u), _ptr(dst_p), _ptr_array(src), len(src)))

    def vmult_rhs_fused_host(self, dst_rho, dst_u, dst_p, src):
        """numpy (ideally pinned) host arrays in, host arrays out."""
        arr = (ctypes.c_void_p * len(src))(*[s.ctypes.data for s in src])
        p = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)
        check(lib().af_vmult_rhs_fused_host(self._h, p(dst_rho), p(dst_u), p(dst_p), arr, len(src)))

    # --- forward / backward pair of the fused stage-1 rhs (autograd-style) ---
    def vmult_rhs_fused_backward(self, src, ybar_rho, ybar_u, ybar_p, xbar):
        """xbar[k] = (d rhs / d src[k])^T ybar for the sources of the current stage (overwritten)."""
        check(lib().af_vmult_rhs_fused_backward(self._h, _ptr_array(src), len(src), _ptr(ybar_rho), _ptr(ybar_u),
                                                _ptr(ybar_p), _ptr_array(xbar)))

    def vmult_rhs_fused_tangent(self, src, dsrc, d_rho, d_u, d_p):
        """(d_rho, d_u, d_p) = (d rhs / d src) dsrc."""
        check(lib().af_vmult_rhs_fused_tangent(self._h, _ptr_array(src), len(src), _ptr_array(dsrc), _ptr(d_rho),
                                               _ptr(d_u), _ptr(d_p)))

    # --- implicit operators ---
    def vmult(self, dst, src):
        check(lib().af_vmult(self._h, _ptr(dst), _ptr(src)))

    def vmult_inverse(self, dst, src):
        """Exact inverse of the block-diagonal mass-type operator of the current NS_stage."""
        check(lib().af_vmult_inverse(self._h, _ptr(dst), _ptr(src)))

    def vmult_pressure(self, dst, src):
        check(lib().af_vmult_pressure(self._h, _ptr(dst), _ptr(src)))

    def vmult_enthalpy(self, dst, src):
        check(lib().af_vmult_enthalpy(self._h, _ptr(dst), _ptr(src)))

    def compute_diagonal(self, dst):
        check(lib().af_compute_diagonal(self._h, _ptr(dst)))

    # --- tangents and transposes of the implicit operators ---
    def vmult_pressure_transpose(self, pbar, ubar):
        """pbar = B^T ubar"""
        check(lib().af_vmult_pressure_transpose(self._h, _ptr(pbar), _ptr(ubar)))

    def vmult_enthalpy_tangent(self, dst, w, dw):
        """dst = J_C(w) dw"""
        check(lib().af_vmult_enthalpy_tangent(self._h, _ptr(dst), _ptr(w), _ptr(dw)))

    def vmult_enthalpy_transpose(self, wbar, w, pbar):
        """wbar = J_C(w)^T pbar"""
        check(lib().af_vmult_enthalpy_transpose(self._h, _ptr(wbar), _ptr(w), _ptr(pbar)))

    def velocity_mass_rho_transpose(self, rhobar, x, y):
        """rhobar = (d/drho [A(rho) x])^T y  (A = the rho_for_fixed-weighted velocity mass)"""
        check(lib().af_vmult_velocity_mass_rho_transpose(self._h, _ptr(rhobar), _ptr(x), _ptr(y)))

    def enthalpy_pf_transpose(self, pfbar, w, pbar):
        """pfbar = (d/dp_f [C(w; p_f)])^T pbar  (C = vmult_enthalpy, p_f = pres_fixed)"""
        check(lib().af_vmult_enthalpy_pf_transpose(self._h, _ptr(pfbar), _ptr(w), _ptr(pbar)))

    def schur_tangent(self, dst, p, dp):
        """dst = J_S(p) dp"""
        check(lib().af_schur_tangent(self._h, _ptr(dst), _ptr(p), _ptr(dp)))

    def schur_transpose(self, dst, p, pbar):
        """dst = J_S(p)^T pbar"""
        check(lib().af_schur_transpose(self._h, _ptr(dst), _ptr(p), _ptr(pbar)))

    # --- diagnostics (Atmospheric_Flow.cc:925-1087) ---
    def compute_diagnostics(self, rho, u, p, rho_stage=None):
        """max |u|, min/max density, max celerity, min cell diameter and Courant numbers."""
        d = Diagnostics()
        check(lib().af_compute_diagnostics(self._h, _ptr(rho), _ptr(rho_stage), _ptr(u), _ptr(p), ctypes.byref(d)))
        return {k: getattr(d, k) for k, _ in Diagnostics._fields_}

    def l2_norm(self, v, ncomp=1):
        """L2 norm of a field over the mesh by QGauss(p+1) (integrate_difference's norm)."""
        out = ctypes.c_double()
        check(lib().af_l2_norm(self._h, ncomp, _ptr(v), ctypes.byref(out)))
        return out.value

    def set_sponge(self, z_start, z_top, rate_top, x_left, x_right, width_lateral, rate_lateral, u_ref):
        """Rayleigh damping of the momentum towards (u_ref, 0): an upper sponge above z_start and
        relaxation zones of width_lateral at x_left and x_right (no counterpart in the reference;
        the 2D hill configuration's damping layers).  Rates 0 switch it off."""
        check(lib().af_set_sponge(self._h, z_start, z_top, rate_top, x_left, x_right, width_lateral, rate_lateral,
                                  u_ref))

    def set_stage_wait_test(self, polls):
        """Test hook: polls > 0 makes the handle's cell kernels give up a bounded wait (before any
        copy is issued) after that many polls; 0 restores normal operation."""
        check(lib().af_set_stage_wait_test(self._h, polls))

    def set_schur_mode(self, mode=0, rel_tol=1e-12, max_iter=10000):
        check(lib().af_set_schur_mode(self._h, mode, rel_tol, max_iter))

    def last_inner_iterations(self):
        n = ctypes.c_int()
        check(lib().af_last_inner_iterations(self._h, ctypes.byref(n)))
        return n.value
