"""State files and VTU output over the C ABI of libaf_gpu.so (af_io_*; host arrays, no GPU).

``write_vtu`` writes what the reference's output_results (Atmospheric_Flow.cc:886-918)
writes in 2D; ``write_state`` / ``read_state`` are a binary restart format (the reference
has none)."""
from __future__ import annotations

import ctypes

import numpy as np

from .operator import _MeshDesc, check, lib


class StateHeader(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("degree", ctypes.c_int), ("periodic_x", ctypes.c_int),
                ("gravity", ctypes.c_int), ("radial_a", ctypes.c_double), ("time", ctypes.c_double),
                ("step", ctypes.c_longlong)]


def _bind():
    L = lib()
    if getattr(L, "_io_bound", False):
        return L
    vp, cp = ctypes.c_void_p, ctypes.c_char_p
    L.af_io_write_state.argtypes = [cp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_longlong, vp, vp, vp]
    L.af_io_read_state_header.argtypes = [cp, ctypes.POINTER(StateHeader)]
    L.af_io_read_state.argtypes = [cp, vp, vp, vp, vp]
    L.af_io_write_vtu.argtypes = [cp, vp, ctypes.c_int, vp, vp, vp]
    L._io_bound = True
    return L


def _arr(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _desc(mesh):
    vtx = _arr(mesh.vertices)
    d = _MeshDesc(mesh.nx, mesh.nz, int(mesh.periodic_x), vtx.ctypes.data, int(mesh.gravity), float(mesh.radial_a))
    return d, vtx


def write_state(path, mesh, degree, rho, u, p, time=0.0, step=0):
    d, vtx = _desc(mesh)
    r, uu, pp = _arr(rho), _arr(u), _arr(p)
    check(_bind().af_io_write_state(str(path).encode(), ctypes.byref(d), degree, time, step, r.ctypes.data,
                                    uu.ctypes.data, pp.ctypes.data))


def read_state(path):
    """Returns (mesh, degree, time, step, rho, u, p)."""
    from .mesh import Mesh
    h = StateHeader()
    L = _bind()
    check(L.af_io_read_state_header(str(path).encode(), ctypes.byref(h)))
    n = h.nx * h.nz * (h.degree + 1) ** 2
    vtx = np.empty((h.nz + 1, h.nx + 1, 2))
    rho, u, p = np.empty(n), np.empty(2 * n), np.empty(n)
    check(L.af_io_read_state(str(path).encode(), vtx.ctypes.data, rho.ctypes.data, u.ctypes.data, p.ctypes.data))
    mesh = Mesh(h.nx, h.nz, vtx, bool(h.periodic_x), h.gravity, h.radial_a)
    return mesh, h.degree, h.time, h.step, rho, u, p


def write_vtu(path, mesh, degree, rho, u, p):
    d, vtx = _desc(mesh)
    r, uu, pp = _arr(rho), _arr(u), _arr(p)
    check(_bind().af_io_write_vtu(str(path).encode(), ctypes.byref(d), degree, r.ctypes.data, uu.ctypes.data,
                                  pp.ctypes.data))
