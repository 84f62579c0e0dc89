"""Tangent-linear and adjoint of IMEX stage 1 (af_imex_stage1_*): the density update and the
pressure fixed point with its Schur solves, differentiated through the recorded iterations.

1. Dot-product test: <J dx, ybar> = <dx, J^T ybar> for seeded random directions.
2. The tangent against central finite differences of the forward stage (solves and the fixed
   point converged tightly, so the differences carry little solver noise at the step used).
Measured on a 16x8 periodic hill, p = 2 and 3: dot products agree to 1e-15 of their scale.
"""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _stepper(P, eps):
    from atmospheric_flows_b200.imex import IMEXStepper
    sc = M.Scaling()
    m = M.hill_mesh(16, 8, periodic_x=True)
    st = M.hill_state(m, P, seed=20261203, modes=4)
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, 2.0, eps=eps, fixed_point_tol=1e-12, schur_preconditioner="cheb_fp32")
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return m, g, (d(st.rho), d(st.u), d(st.p))


def _dirs(x, seed, scale):
    rng = np.random.default_rng(seed)
    return tuple(torch.from_numpy(scale * float(v.abs().max()) * rng.standard_normal(v.numel())).cuda() for v in x)


def _dot(a, b):
    return sum(float(torch.dot(p, q)) for p, q in zip(a, b))


@pytest.mark.parametrize("P", [2, 3])
def test_stage1_dot_product(P):
    m, g, x = _stepper(P, 1e-13)
    g.stage1_forward(*x)
    dx = _dirs(x, 1, 1.0)
    yb = _dirs(x, 2, 1.0)
    dy = g.stage1_tangent(*dx, rel_tol=1e-13)
    xb = g.stage1_backward(*yb, rel_tol=1e-13)
    torch.cuda.synchronize()
    lhs, rhs = _dot(dy, yb), _dot(dx, xb)
    scale = sum(float((a.abs() * b.abs()).sum()) for a, b in zip(dy, yb))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)


@pytest.mark.parametrize("P", [2, 3])
def test_stage1_tangent_matches_differences(P):
    """Central differences along a smooth direction (a second seeded hill perturbation, so that
    no face flips its Rusanov wave-speed branch) at step 1e-3: 1e-10..2e-9 measured."""
    m, g, x = _stepper(P, 1e-13)
    base = M.hill_state(m, P, seed=20261203, modes=4)
    other = M.hill_state(m, P, seed=99, modes=4, amplitude=1e-2)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dx = (d(other.rho - base.rho), d(other.u - base.u), d(other.p - base.p))
    g.stage1_forward(*x)
    dy = g.stage1_tangent(*dx, rel_tol=1e-13)
    h = 1e-3
    yp = g.stage1_forward(*(a + h * b for a, b in zip(x, dx)))
    ym = g.stage1_forward(*(a - h * b for a, b in zip(x, dx)))
    torch.cuda.synchronize()
    for a, b, t in zip(yp, ym, dy):
        err = float(torch.linalg.norm((a - b) / (2 * h) - t) / torch.linalg.norm(t))
        assert err < 1e-8, err
