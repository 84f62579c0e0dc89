"""Tangent-linear and adjoint of IMEX stage 1 (af_imex_stage1_*) and of a whole IMEX step
(af_imex_step_*, af_imex_gradient): the density updates and the pressure fixed points with their
Schur solves, differentiated through the recorded iterations, and checkpointed gradients.

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


def _stepper(P, eps, m=None):
    from atmospheric_flows_b200.imex import IMEXStepper
    sc = M.Scaling()
    m = m or M.hill_mesh(16, 8, periodic_x=True)
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


def _smooth_direction(m, P):
    base = M.hill_state(m, P, seed=20261203, modes=4)
    other = M.hill_state(m, P, seed=99, modes=4, amplitude=1e-2)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return (d(other.rho - base.rho), d(other.u - base.u), d(other.p - base.p))


@pytest.mark.parametrize("P", [2, 3, 4])
def test_step_dot_product(P):
    """A whole IMEX step (both fixed points, stage 3): dot product to 1e-12 of its scale
    (5.6e-16 measured at p = 2)."""
    m, g, x = _stepper(P, 1e-13)
    g.step_forward(*x)
    dx = _dirs(x, 4, 1.0)
    yb = _dirs(x, 5, 1.0)
    dy = g.step_tangent(*dx, rel_tol=1e-13)
    xb = g.step_backward(*yb, rel_tol=1e-13)
    torch.cuda.synchronize()
    lhs, rhs = _dot(dy, yb), _dot(dx, xb)
    scale = sum(float((a.abs() * b.abs()).sum()) for a, b in zip(dy, yb))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)


def test_step_tangent_matches_differences():
    """Central differences of the step along a smooth direction at step 1e-4 (1e-9 measured)."""
    P = 2
    m, g, x = _stepper(P, 1e-13)
    dx = _smooth_direction(m, P)
    g.step_forward(*x)
    dy = g.step_tangent(*dx, rel_tol=1e-13)
    h = 1e-4
    yp = g.step_forward(*(a + h * b for a, b in zip(x, dx)))
    ym = g.step_forward(*(a - h * b for a, b in zip(x, dx)))
    torch.cuda.synchronize()
    for a, b, t in zip(yp, ym, dy):
        err = float(torch.linalg.norm((a - b) / (2 * h) - t) / torch.linalg.norm(t))
        assert err < 1e-7, err


def test_gradient_with_checkpointing():
    """Gradient of J = |u_N|^2 / 2 after 4 steps with respect to the initial state: the same with
    a checkpoint every 1, 2 or 4 steps, and against central differences of J along a smooth
    direction (step 1e-4)."""
    P, N = 2, 4
    m, g, x = _stepper(P, 1e-13)

    def J(x0):
        g.set_state(*x0)
        g.step(N)
        r, u, p = g.get_state()
        return 0.5 * float(torch.dot(u, u)), u
    _, uN = J(x)
    zr = torch.zeros(m.n_cells * (P + 1) ** 2, dtype=torch.float64, device="cuda")
    grads = {K: g.gradient(*x, N, K, zr, uN, zr, rel_tol=1e-13) for K in (1, 2, 4)}
    for K in (2, 4):
        for a, b in zip(grads[K], grads[1]):
            assert float(torch.linalg.norm(a - b)) <= 1e-13 * float(torch.linalg.norm(b)), K
    dx = _smooth_direction(m, P)
    dJ = _dot(grads[2], dx)
    h = 1e-4
    jp, _ = J(tuple(a + h * b for a, b in zip(x, dx)))
    jm, _ = J(tuple(a - h * b for a, b in zip(x, dx)))
    assert abs((jp - jm) / (2 * h) - dJ) <= 1e-5 * abs(dJ), ((jp - jm) / (2 * h), dJ)


def test_step_adjoint_and_gradient_with_odd_field_lengths():
    """3 x 3 periodic cells at degree 4: 225 DoFs per scalar field, so the checkpoint buffer
    of af_imex_gradient and the solver's Krylov vectors use padded strides.  The step's dot
    product holds, and the gradient is the same for a checkpoint every 1 or 2 steps."""
    P, N = 4, 2
    m, g, x = _stepper(P, 1e-13, M.hill_mesh(3, 3, periodic_x=True))
    assert (m.n_cells * (P + 1) ** 2) % 2 == 1
    g.step_forward(*x)
    dx = _dirs(x, 4, 1.0)
    yb = _dirs(x, 5, 1.0)
    dy = g.step_tangent(*dx, rel_tol=1e-13)
    xb = g.step_backward(*yb, rel_tol=1e-13)
    torch.cuda.synchronize()
    lhs, rhs = _dot(dy, yb), _dot(dx, xb)
    scale = sum(float((a.abs() * b.abs()).sum()) for a, b in zip(dy, yb))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)
    g.set_state(*x)
    g.step(N)
    _, uN, _ = g.get_state()
    zr = torch.zeros_like(x[0])
    g1 = g.gradient(*x, N, 1, zr, uN, zr, rel_tol=1e-13)
    g2 = g.gradient(*x, N, 2, zr, uN, zr, rel_tol=1e-13)
    for a, b in zip(g2, g1):
        assert torch.isfinite(a).all()
        assert float(torch.linalg.norm(a - b)) <= 1e-13 * float(torch.linalg.norm(b))


def test_tangent_needs_a_recorded_forward():
    """The tangent / backward of a step refuse to run before the recorded forward, and after
    af_imex_step moved the state (the linearisation point is gone)."""
    from atmospheric_flows_b200.operator import AFError
    m, g, x = _stepper(2, 1e-10)
    dx = _dirs(x, 6, 1.0)
    with pytest.raises(AFError):
        g.step_tangent(*dx)
    g.step_forward(*x)
    g.step_tangent(*dx)  # fine now
    g.step(1)
    with pytest.raises(AFError):
        g.step_backward(*dx)


def _oracle_steps(m, P, nsteps):
    """The oracle's restatement of the time loop with accurate solves (GMRES on the true residual
    to 1e-13, exact cell-wise mass inverses, fixed point to 1e-12): the function whose
    differences check the GPU's tangent and gradient."""
    from oracle.oracle import OracleOperator, imex_steps
    sc = M.Scaling()
    o = OracleOperator(m, P, sc.Ma, sc.Fr, 2.0)

    def run(x):
        r, u, p, _ = imex_steps(o, *x, nsteps, eps=1e-13, fixed_point_tol=1e-12, true_residual=True,
                                exact_inverse=True)
        return r, u, p
    return run


def test_step_tangent_matches_oracle_differences():
    """The GPU tangent of one IMEX step against central differences of the ORACLE's step at step
    h = 1e-6 (the adjoint check's finite-difference step), along a smooth direction of the size
    of the state: the differences carry the oracle's solver noise, about 1e-12 / h (1.2e-9 to
    6.1e-9 measured)."""
    P = 2
    m, g, x = _stepper(P, 1e-13)
    dx = tuple(100.0 * v for v in _smooth_direction(m, P))
    g.step_forward(*x)
    dy = g.step_tangent(*dx, rel_tol=1e-13)
    step = _oracle_steps(m, P, 1)
    xh = [v.cpu().numpy() for v in x]
    dxh = [v.cpu().numpy() for v in dx]
    h = 1e-6
    yp = step([a + h * b for a, b in zip(xh, dxh)])
    ym = step([a - h * b for a, b in zip(xh, dxh)])
    errs = []
    for a, b, t in zip(yp, ym, dy):
        t = t.cpu().numpy()
        errs.append(float(np.linalg.norm((a - b) / (2 * h) - t) / np.linalg.norm(t)))
    print("step tangent vs oracle central differences (h = 1e-6):", errs)
    assert max(errs) < 1e-7, errs


def test_gradient_matches_oracle_differences():
    """The checkpointed GPU gradient of J = |u_N|^2 / 2 after 4 steps against central differences
    of J computed with the oracle's time loop, step h = 1e-6 along a smooth direction (9.6e-7
    relative measured)."""
    P, N = 2, 4
    m, g, x = _stepper(P, 1e-13)
    g.set_state(*x)
    g.step(N)
    _, uN, _ = g.get_state()
    zr = torch.zeros(m.n_cells * (P + 1) ** 2, dtype=torch.float64, device="cuda")
    grad = g.gradient(*x, N, 2, zr, uN, zr, rel_tol=1e-13)
    dx = tuple(100.0 * v for v in _smooth_direction(m, P))
    dJ = _dot(grad, dx)
    run = _oracle_steps(m, P, N)
    xh = [v.cpu().numpy() for v in x]
    dxh = [v.cpu().numpy() for v in dx]
    h = 1e-6
    up = run([a + h * b for a, b in zip(xh, dxh)])[1]
    um = run([a - h * b for a, b in zip(xh, dxh)])[1]
    fd = (0.5 * float(np.dot(up, up)) - 0.5 * float(np.dot(um, um))) / (2 * h)
    print("gradient . dx vs oracle central differences of J (h = 1e-6):", dJ, fd, abs(fd - dJ) / abs(dJ))
    assert abs(fd - dJ) <= 1e-5 * abs(dJ), (fd, dJ)
