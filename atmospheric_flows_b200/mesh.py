"""Host-side problem setup: structured 2D meshes, DoF coordinates and initial states.

The reference builds its mesh with deal.II (``GridGenerator::concentric_hyper_shells``
scaled to the Earth radius, Atmospheric_Flow.cc:283-284) and interpolates analytic
fields at the FE support points (``VectorTools::interpolate``, Atmospheric_Flow.cc:420-422).
This module provides the same services for the structured meshes this library runs on:

* ``hill_mesh``   -- 2D terrain-following mesh over a Witch-of-Agnesi hill (the flat
  terrain extension of the reference; gravity along e_z).
* ``box_mesh``    -- axis-aligned rectangle (affine cells; used by exact tests).
* ``annulus_mesh``-- 2D slice of the reference's spherical shell (radial gravity).

Layout conventions shared with the C ABI (include/af_gpu.h):
  vertices[j, i, :] = (x, z) of mesh vertex (i, j), i = 0..nx, j = 0..nz; cell (i, j) has
  index c = j*nx + i and uses vertices (i,j), (i+1,j), (i,j+1), (i+1,j+1) as deal.II's
  vertices 0..3.  Geometry is bilinear (deal.II MappingQ1).  Scalar DoFs are stored
  cell-major, lexicographic (x fastest) at the p+1 Gauss-Lobatto points per direction;
  velocity DoFs are component-blocked inside each cell.

Non-dimensionalisation follows the reference (runtime_parameters.h:29-33): lengths in
metres and velocities in m/s (L_ref = u_ref = 1), p_ref = 1e5 Pa, rho_ref = p_ref/(R T_ref),
so Ma = sqrt(rho_ref/p_ref) and Fr = 1/sqrt(g).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

GAMMA = 1.4          # equation_data.h:25
R_GAS = 287.0        # equation_data.h:26
CP = GAMMA * R_GAS / (GAMMA - 1.0)   # = 1004.5
G_ACC = 9.81


@dataclasses.dataclass
class Mesh:
    nx: int
    nz: int
    vertices: np.ndarray          # (nz+1, nx+1, 2) float64, C-contiguous
    periodic_x: bool
    gravity: int                  # 0: vertical e_z, 1: radial (reference shell)
    radial_a: float = 0.0         # Earth radius for radial gravity

    @property
    def n_cells(self) -> int:
        return self.nx * self.nz


def box_mesh(nx, nz, x0=0.0, x1=1.0, z0=0.0, z1=1.0, periodic_x=False, gravity=0):
    xs = np.linspace(x0, x1, nx + 1)
    zs = np.linspace(z0, z1, nz + 1)
    v = np.zeros((nz + 1, nx + 1, 2))
    v[:, :, 0] = xs[None, :]
    v[:, :, 1] = zs[:, None]
    return Mesh(nx, nz, np.ascontiguousarray(v), periodic_x, gravity)


def agnesi(x, h0=400.0, a=1000.0):
    return h0 / (1.0 + (x / a) ** 2)


def hill_mesh(nx, nz, x0=-20000.0, x1=20000.0, top=16000.0, h0=400.0, a=1000.0, periodic_x=False):
    """Terrain-following (Gal-Chen) map z = h(x) + zeta (1 - h(x)/top), zeta uniform."""
    xs = np.linspace(x0, x1, nx + 1)
    zeta = np.linspace(0.0, top, nz + 1)
    h = agnesi(xs, h0, a)
    v = np.zeros((nz + 1, nx + 1, 2))
    v[:, :, 0] = xs[None, :]
    v[:, :, 1] = h[None, :] + zeta[:, None] * (1.0 - h[None, :] / top)
    return Mesh(nx, nz, np.ascontiguousarray(v), periodic_x, 0)


def annulus_mesh(nx, nz, r0=0.9 * 6.37122e6, r1=6.37122e6):
    """2D slice of the reference shell (inner radius 0.9 a, outer a), periodic in angle."""
    # angle decreasing along x and radius increasing along z keeps det J > 0
    th = np.linspace(0.0, -2.0 * np.pi, nx + 1)
    th[-1] = 0.0  # the last column coincides with the first
    rs = np.linspace(r0, r1, nz + 1)
    v = np.zeros((nz + 1, nx + 1, 2))
    v[:, :, 0] = rs[:, None] * np.cos(th[None, :])
    v[:, :, 1] = rs[:, None] * np.sin(th[None, :])
    return Mesh(nx, nz, np.ascontiguousarray(v), True, 1, radial_a=6.37122e6)


def jitter_mesh(mesh: Mesh, amplitude: float, seed: int) -> Mesh:
    """Randomly displaced interior vertices (non-affine cells for tests)."""
    rng = np.random.default_rng(seed)
    v = mesh.vertices.copy()
    hx = np.abs(np.diff(v[:, :, 0], axis=1)).min()
    hz = np.abs(np.diff(v[:, :, 1], axis=0)).min()
    d = rng.uniform(-amplitude, amplitude, size=v.shape)
    d[..., 0] *= hx
    d[..., 1] *= hz
    d[0, :, :] = 0
    d[-1, :, :] = 0
    if mesh.periodic_x:
        d[:, -1, :] = d[:, 0, :]
    else:
        d[:, 0, :] = 0
        d[:, -1, :] = 0
    v += d
    return Mesh(mesh.nx, mesh.nz, np.ascontiguousarray(v), mesh.periodic_x, mesh.gravity, mesh.radial_a)


def gll_nodes_01(p: int) -> np.ndarray:
    """Gauss-Lobatto nodes on [0,1] (support points of FE_DGQ)."""
    if p == 1:
        return np.array([0.0, 1.0])
    leg = np.polynomial.legendre.Legendre.basis(p).deriv()
    inner = np.sort(np.real(leg.roots()))
    x = np.concatenate([[-1.0], inner, [1.0]])
    # polish the interior roots with Newton on P'_p
    for _ in range(4):
        d1 = leg(x[1:-1])
        d2 = leg.deriv()(x[1:-1])
        x[1:-1] -= d1 / d2
    return 0.5 * (x + 1.0)


def dof_coordinates(mesh: Mesh, p: int) -> np.ndarray:
    """(n_cells, (p+1)^2, 2) physical coordinates of the scalar DoFs (bilinear map)."""
    s = gll_nodes_01(p)
    xi = np.tile(s, p + 1)            # x fastest
    eta = np.repeat(s, p + 1)
    v = mesh.vertices
    v0 = v[:-1, :-1].reshape(-1, 2)
    v1 = v[:-1, 1:].reshape(-1, 2)
    v2 = v[1:, :-1].reshape(-1, 2)
    v3 = v[1:, 1:].reshape(-1, 2)
    w0 = ((1 - xi) * (1 - eta))[None, :, None]
    w1 = (xi * (1 - eta))[None, :, None]
    w2 = ((1 - xi) * eta)[None, :, None]
    w3 = (xi * eta)[None, :, None]
    return v0[:, None, :] * w0 + v1[:, None, :] * w1 + v2[:, None, :] * w2 + v3[:, None, :] * w3


@dataclasses.dataclass
class Scaling:
    p_ref: float = 1.0e5
    T_ref: float = 300.0

    @property
    def rho_ref(self) -> float:
        return self.p_ref / (R_GAS * self.T_ref)

    @property
    def Ma(self) -> float:
        return math.sqrt(self.rho_ref / self.p_ref)

    @property
    def Fr(self) -> float:
        return 1.0 / math.sqrt(G_ACC)


def hydrostatic_background(z, theta0=300.0, N=0.01, p0=1.0e5, sc: Scaling = Scaling()):
    """Constant Brunt-Vaisala frequency atmosphere; returns non-dimensional (rho, p)."""
    th = theta0 * np.exp(N * N * z / G_ACC)
    exner = 1.0 + G_ACC * G_ACC / (CP * theta0 * N * N) * (np.exp(-N * N * z / G_ACC) - 1.0)
    p = p0 * exner ** (CP / R_GAS)
    T = th * exner
    rho = p / (R_GAS * T)
    return rho / sc.rho_ref, p / sc.p_ref


def _harmonics(theta, modes):
    """cos(k theta), sin(k theta) for k = 1..modes by the angle-addition recurrence."""
    c1, s1 = np.cos(theta), np.sin(theta)
    C = np.empty((theta.size, modes), order="F")  # column k contiguous
    S = np.empty((theta.size, modes), order="F")
    C[:, 0], S[:, 0] = c1, s1
    for k in range(1, modes):
        C[:, k] = C[:, k - 1] * c1 - S[:, k - 1] * s1
        S[:, k] = S[:, k - 1] * c1 + C[:, k - 1] * s1
    return C, S


def fourier_perturbation(xz, seed, modes=16, amplitude=1e-3, box=None):
    """Smooth seeded field: sum_{k,l<=modes} a_kl/(k^2+l^2) cos(2pi k x^ + phi) cos(pi l z^ + psi),
    a_kl ~ N(0,1), scaled to max |.| = amplitude over the given points."""
    rng = np.random.default_rng(seed)
    x, z = xz[..., 0], xz[..., 1]
    if box is None:
        box = (x.min(), x.max(), z.min(), z.max())
    xh = (x - box[0]) / max(box[1] - box[0], 1e-300)
    zh = (z - box[2]) / max(box[3] - box[2], 1e-300)
    a = rng.standard_normal((modes, modes))
    ph = rng.uniform(0, 2 * np.pi, (modes, modes))
    ps = rng.uniform(0, 2 * np.pi, (modes, modes))
    k = np.arange(1, modes + 1)
    c = a / (k[:, None] ** 2 + k[None, :] ** 2)
    # cos(kX + phi) cos(lZ + psi) expanded so the double sum becomes four matrix products;
    # evaluated in cache-sized chunks of points
    Mcc, Mcs = c * np.cos(ph) * np.cos(ps), c * np.cos(ph) * np.sin(ps)
    Msc, Mss = c * np.sin(ph) * np.cos(ps), c * np.sin(ph) * np.sin(ps)
    xr, zr = xh.reshape(-1), zh.reshape(-1)
    f = np.empty(xr.size)
    chunk = 1 << 15
    for b in range(0, xr.size, chunk):
        CX, SX = _harmonics(2 * np.pi * xr[b:b + chunk], modes)
        CZ, SZ = _harmonics(np.pi * zr[b:b + chunk], modes)
        f[b:b + chunk] = (((CX @ Mcc) * CZ).sum(1) - ((CX @ Mcs) * SZ).sum(1)
                          - ((SX @ Msc) * CZ).sum(1) + ((SX @ Mss) * SZ).sum(1))
    f = f.reshape(x.shape)
    m = np.abs(f).max()
    return f * (amplitude / m if m > 0 else 0.0)


@dataclasses.dataclass
class State:
    rho: np.ndarray   # (n_cells*(p+1)^2,)
    u: np.ndarray     # (n_cells*2*(p+1)^2,) component-blocked per cell
    p: np.ndarray


def hill_state(mesh: Mesh, p: int, seed: int = 20261203, amplitude: float = 1e-3, U: float = 10.0,
               modes: int = 16, sc: Scaling = Scaling()) -> State:
    """Hydrostatic background + seeded smooth relative perturbations of each field."""
    xz = dof_coordinates(mesh, p)
    rho_b, p_b = hydrostatic_background(xz[..., 1], sc=sc)
    box = (mesh.vertices[..., 0].min(), mesh.vertices[..., 0].max(),
           mesh.vertices[..., 1].min(), mesh.vertices[..., 1].max())
    d = [fourier_perturbation(xz, seed + 17 * k, modes, amplitude, box) for k in range(4)]
    rho = rho_b * (1.0 + d[0])
    pres = p_b * (1.0 + d[1])
    ux = U * (1.0 + d[2])
    uz = U * d[3]
    u = np.stack([ux, uz], axis=1)  # (n_cells, 2, nd)
    return State(np.ascontiguousarray(rho.reshape(-1)), np.ascontiguousarray(u.reshape(-1)),
                 np.ascontiguousarray(pres.reshape(-1)))


def random_state(mesh: Mesh, p: int, seed: int, rel: float = 0.05) -> State:
    """Positive density/pressure with O(1) random nodal noise (rough inputs for parity tests)."""
    rng = np.random.default_rng(seed)
    n = mesh.n_cells * (p + 1) ** 2
    rho = 1.0 + rel * rng.standard_normal(n)
    pres = 1.0 + rel * rng.standard_normal(n)
    u = 10.0 * rng.standard_normal(2 * n)
    return State(rho, u, pres)
