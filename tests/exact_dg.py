"""Exact (symbolic) evaluation of the reference's weak forms on affine rectangles.

Independent of the oracle's sum-factorised code path: every integral here is taken
analytically with sympy over each rectangle / edge, with the reference's integrands
written from euler_operator.h.  With p = 1, 2 the Gauss-Lobatto support points are
rational and, for polynomial integrands of the tested degrees, QGauss(2p+1) is exact,
so the oracle must reproduce these values to rounding.

Used only by tests/test_oracle_kat.py.
"""
from __future__ import annotations

import itertools

import sympy as sp

x, z = sp.symbols("x z", real=True)

SQ2 = sp.sqrt(2)
GAM = 2 - SQ2
TAB = dict(a21=GAM, a31=sp.Rational(1, 2), a32=sp.Rational(1, 2),
           a21t=GAM / 2, a22t=GAM / 2, a31t=SQ2 / 4, a32t=SQ2 / 4, a33t=1 - SQ2 / 2)
TAB.update(b1=TAB["a31t"], b2=TAB["a32t"], b3=TAB["a33t"])
G = sp.Rational(7, 5)   # Cp_Cv


def gll_rational(p):
    if p == 1:
        return [sp.Integer(0), sp.Integer(1)]
    if p == 2:
        return [sp.Integer(0), sp.Rational(1, 2), sp.Integer(1)]
    raise ValueError("rational GLL nodes only for p <= 2")


def lagrange(nodes, i, s):
    e = sp.Integer(1)
    for j, nj in enumerate(nodes):
        if j != i:
            e *= (s - nj) / (nodes[i] - nj)
    return sp.expand(e)


def poly(e):
    """Polynomial in (x, z) over the rationals; all integrands of the tests are such."""
    if isinstance(e, sp.Poly):
        return e
    return sp.Poly(e, x, z, domain=sp.QQ)


def _int_rect(pl, X0, X1, Z0, Z1):
    tot = sp.Integer(0)
    for (a, b), cf in pl.terms():
        tot += cf * (X1 ** (a + 1) - X0 ** (a + 1)) / (a + 1) * (Z1 ** (b + 1) - Z0 ** (b + 1)) / (b + 1)
    return tot


class Box:
    """nx x nz uniform rectangles on [x0,x1] x [z0,z1] (rational coordinates)."""

    def __init__(self, nx, nz, x0, x1, z0, z1, p, periodic_x=False):
        self.nx, self.nz, self.p = nx, nz, p
        self.periodic_x = periodic_x
        self.xs = [sp.Rational(x0) + (sp.Rational(x1) - sp.Rational(x0)) * i / nx for i in range(nx + 1)]
        self.zs = [sp.Rational(z0) + (sp.Rational(z1) - sp.Rational(z0)) * j / nz for j in range(nz + 1)]
        self.nodes = gll_rational(p)
        self.nd = (p + 1) ** 2

    def cell_rect(self, c):
        i, j = c % self.nx, c // self.nx
        return self.xs[i], self.xs[i + 1], self.zs[j], self.zs[j + 1]

    def basis(self, c):
        X0, X1, Z0, Z1 = self.cell_rect(c)
        sx = (x - X0) / (X1 - X0)
        sz = (z - Z0) / (Z1 - Z0)
        P1 = self.p + 1
        out = []
        for iz in range(P1):
            for ix in range(P1):
                out.append(poly(lagrange(self.nodes, ix, sx) * lagrange(self.nodes, iz, sz)))
        return out

    def nodal(self, c, f):
        """Nodal values of expression f in cell c (lexicographic, x fastest)."""
        X0, X1, Z0, Z1 = self.cell_rect(c)
        vals = []
        for iz in range(self.p + 1):
            for ix in range(self.p + 1):
                xv = X0 + (X1 - X0) * self.nodes[ix]
                zv = Z0 + (Z1 - Z0) * self.nodes[iz]
                vals.append(poly(f).as_expr().subs({x: xv, z: zv}))
        return vals

    def cell_int(self, c, e):
        X0, X1, Z0, Z1 = self.cell_rect(c)
        return _int_rect(poly(e), X0, X1, Z0, Z1)

    def faces(self):
        """Interior faces as (cell_plus, cell_minus, normal, param) with n the outward
        normal of the + (left/lower) cell; param = ('x', X) vertical or ('z', Z) horizontal."""
        out = []
        for j in range(self.nz):
            for i in range(1, self.nx):
                out.append((j * self.nx + i - 1, j * self.nx + i, (1, 0), ("x", self.xs[i], self.zs[j], self.zs[j + 1])))
            if self.periodic_x:
                raise NotImplementedError
        for j in range(1, self.nz):
            for i in range(self.nx):
                out.append(((j - 1) * self.nx + i, j * self.nx + i, (0, 1), ("z", self.zs[j], self.xs[i], self.xs[i + 1])))
        return out

    def bfaces(self):
        out = []
        for i in range(self.nx):
            out.append((i, (0, -1), ("z", self.zs[0], self.xs[i], self.xs[i + 1])))
            c = (self.nz - 1) * self.nx + i
            out.append((c, (0, 1), ("z", self.zs[-1], self.xs[i], self.xs[i + 1])))
        for j in range(self.nz):
            out.append((j * self.nx, (-1, 0), ("x", self.xs[0], self.zs[j], self.zs[j + 1])))
            out.append((j * self.nx + self.nx - 1, (1, 0), ("x", self.xs[-1], self.zs[j], self.zs[j + 1])))
        return out


def face_int(param, e):
    kind, v, a, b = param
    pl = poly(e)
    tot = sp.Integer(0)
    for (ex, ez), cf in pl.terms():
        if kind == "x":   # vertical edge x = v, z in [a, b]
            tot += cf * v ** ex * (b ** (ez + 1) - a ** (ez + 1)) / (ez + 1)
        else:             # horizontal edge z = v, x in [a, b]
            tot += cf * v ** ez * (b ** (ex + 1) - a ** (ex + 1)) / (ex + 1)
    return tot


def to_float(vals):
    return [float(sp.N(v, 30)) for v in vals]
