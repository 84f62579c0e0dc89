"""Forward / tangent / backward of the fused stage-1 right-hand side on the GPU.

1. Dot-product test: <ybar, J dx> (af_vmult_rhs_fused_tangent) equals <J^T ybar, dx>
   (af_vmult_rhs_fused_backward) to 1e-12 relative, on walled, periodic and radial-gravity
   meshes, smooth and rough states (the wave-speed branch is frozen the same way in both).
2. The tangent against tangent-linear differences of the oracle's restatement of the
   reference operators: a 5-point central difference (exact for the cubic integrands away
   from the wave-speed kink) evaluated in long double, on rough states whose two face traces
   differ, so that no kink lies within the stencil: 1e-8 relative.
"""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _case(name, P, rough):
    sc = M.Scaling()
    Ma, Fr = sc.Ma, sc.Fr
    if name == "hill":
        m = M.jitter_mesh(M.hill_mesh(10, 5), 0.15, seed=11)
    elif name == "hill_periodic":
        m = M.hill_mesh(9, 4, periodic_x=True)
    else:
        m = M.annulus_mesh(24, 3, r0=6.37122e6, r1=6.37122e6 + 16e3)
        Ma, Fr = (1.0 / (287.0 * 273.0)) ** 0.5, 1.0 / 9.80616 ** 0.5
        rough = True
    if rough:
        st = [M.random_state(m, P, seed=30 + k) for k in range(2)]
    else:
        st = [M.hill_state(m, P, seed=30 + k, amplitude=0.05) for k in range(2)]
    src = [st[0].rho, st[0].u, st[0].p, st[1].rho, st[1].u]
    return m, Ma, Fr, src


@pytest.mark.parametrize("P", [2, 3, 4])
@pytest.mark.parametrize("name,rough", [("hill", False), ("hill", True), ("hill_periodic", False), ("annulus", True)])
def test_dot_product(P, name, rough):
    from atmospheric_flows_b200.operator import EULEROperator
    m, Ma, Fr, src = _case(name, P, rough)
    op = EULEROperator(m, P, Ma, Fr, 2.0)
    op.set_HYPERBOLIC_stage(1)
    rng = np.random.default_rng(7)
    ns = m.n_cells * (P + 1) ** 2
    sizes = [ns, 2 * ns, ns, ns, 2 * ns]
    dx = [rng.standard_normal(n) for n in sizes]
    yb = [rng.standard_normal(n) for n in (ns, 2 * ns, ns)]
    s = [_d(a) for a in src]
    dy = [torch.empty(n, dtype=torch.float64, device="cuda") for n in (ns, 2 * ns, ns)]
    op.vmult_rhs_fused_tangent(s, [_d(a) for a in dx], *dy)
    xb = [torch.full((n,), np.nan, dtype=torch.float64, device="cuda") for n in sizes]
    op.vmult_rhs_fused_backward(s, *[_d(a) for a in yb], xb)
    torch.cuda.synchronize()
    lhs = sum(float(np.dot(a, b.cpu().numpy())) for a, b in zip(yb, dy))
    terms = [float(np.dot(b.cpu().numpy(), a)) for a, b in zip(dx, xb)]
    rhs = sum(terms)
    scale = sum(abs(t) for t in terms)
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)


@pytest.mark.parametrize("P", [2, 4])
@pytest.mark.parametrize("name", ["hill", "annulus"])
def test_tangent_matches_oracle_differences(P, name):
    from atmospheric_flows_b200.operator import EULEROperator
    from oracle.oracle import OracleOperator
    m, Ma, Fr, src = _case(name, P, True)
    dt = 2.0
    op = EULEROperator(m, P, Ma, Fr, dt)
    op.set_HYPERBOLIC_stage(1)
    o = OracleOperator(m, P, Ma, Fr, dt, long_double=True)
    o.set_HYPERBOLIC_stage(1)
    rng = np.random.default_rng(9)
    dx = [1e-5 * np.abs(a).mean() * rng.standard_normal(a.size) for a in src]

    def F(t):
        x = [a + t * d for a, d in zip(src, dx)]
        return np.concatenate([o.vmult_rhs_rho_update(x[:2]), o.vmult_rhs_velocity_fixed(x[:4]),
                               o.vmult_rhs_pressure(x)])
    fd = (8.0 * (F(1.0) - F(-1.0)) - (F(2.0) - F(-2.0))) / 12.0
    ns = m.n_cells * (P + 1) ** 2
    dy = [torch.empty(n, dtype=torch.float64, device="cuda") for n in (ns, 2 * ns, ns)]
    op.vmult_rhs_fused_tangent([_d(a) for a in src], [_d(a) for a in dx], *dy)
    torch.cuda.synchronize()
    got = np.concatenate([t.cpu().numpy() for t in dy])
    err = np.linalg.norm(got - fd) / np.linalg.norm(fd)
    assert err < 1e-8, err


# ------------------------------------------------------------------ implicit operators
def _implicit_setup(name, P):
    from atmospheric_flows_b200.operator import EULEROperator
    m, Ma, Fr, src = _case(name, P, True)
    op = EULEROperator(m, P, Ma, Fr, 2.0)
    op.set_stream(torch.cuda.current_stream())
    op.set_schur_mode(1)
    op.set_HYPERBOLIC_stage(1)
    op.set_rho_for_fixed(_d(src[0]))
    op.set_pres_fixed(_d(src[2]))
    return m, op, src


def _dot(a, b):
    return float(torch.dot(a, b))


@pytest.mark.parametrize("P", [2, 4])
@pytest.mark.parametrize("name", ["hill", "hill_periodic"])
def test_implicit_dot_products(P, name):
    """B^T, J_C^T and J_S^T against B, J_C and J_S: dot-product tests to 1e-12."""
    m, op, src = _implicit_setup(name, P)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(21)
    rnd = lambda n: _d(rng.standard_normal(n))
    q, pbar, p = rnd(ns), rnd(ns), _d(src[2])
    ubar, w, dw = rnd(2 * ns), _d(src[1]), rnd(2 * ns)
    Bq = torch.empty(2 * ns, dtype=torch.float64, device="cuda")
    op.vmult_pressure(Bq, q)
    BTu = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.vmult_pressure_transpose(BTu, ubar)
    Jdw = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.vmult_enthalpy_tangent(Jdw, w, dw)
    JTp = torch.empty(2 * ns, dtype=torch.float64, device="cuda")
    op.vmult_enthalpy_transpose(JTp, w, pbar)
    Sq = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.schur_tangent(Sq, p, q)
    STp = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.schur_transpose(STp, p, pbar)
    torch.cuda.synchronize()
    for lhs, rhs, scale in ((_dot(ubar, Bq), _dot(BTu, q), float((ubar.abs() * Bq.abs()).sum())),
                            (_dot(pbar, Jdw), _dot(JTp, dw), float((pbar.abs() * Jdw.abs()).sum())),
                            (_dot(pbar, Sq), _dot(STp, q), float((pbar.abs() * Sq.abs()).sum()))):
        assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)


@pytest.mark.parametrize("P", [2, 4])
@pytest.mark.parametrize("name", ["hill", "hill_periodic"])
def test_coefficient_derivative_dot_products(P, name):
    """A is linear in rho_for_fixed and C in pres_fixed, so their coefficient tangents are the
    operators with the perturbation as coefficient; the transposed kernels pass the
    dot-product test against them to 1e-12."""
    m, op, src = _implicit_setup(name, P)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(23)
    rnd = lambda n: _d(rng.standard_normal(n))
    x, y, drho = rnd(2 * ns), rnd(2 * ns), rnd(ns)
    w, pbar, dpf = _d(src[1]), rnd(ns), rnd(ns)
    rhobar = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.velocity_mass_rho_transpose(rhobar, x, y)
    pfbar = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.enthalpy_pf_transpose(pfbar, w, pbar)
    Ax = torch.empty(2 * ns, dtype=torch.float64, device="cuda")
    op.set_rho_for_fixed(drho)  # A(drho) x
    op.set_NS_stage(3)
    op.vmult(Ax, x)
    Cw = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.set_pres_fixed(dpf)  # C(w; dpf)
    op.vmult_enthalpy(Cw, w)
    torch.cuda.synchronize()
    for lhs, rhs, scale in ((_dot(y, Ax), _dot(rhobar, drho), float((y.abs() * Ax.abs()).sum())),
                            (_dot(pbar, Cw), _dot(pfbar, dpf), float((pbar.abs() * Cw.abs()).sum()))):
        assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)


@pytest.mark.parametrize("P", [2, 3])
def test_implicit_tangents_match_differences(P):
    """J_C and J_S against 5-point differences of the forward C and Schur applies (rough
    states, no wave-speed kink inside the stencil; C is piecewise linear in w, S in p)."""
    m, op, src = _implicit_setup("hill", P)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(5)
    w, p = _d(src[1]), _d(src[2])
    dw = _d(1e-4 * float(w.abs().mean()) * rng.standard_normal(2 * ns))
    # the wave speed of C acts on w = A^{-1} B p, whose face traces on rough data are closer
    # together than those of u: a smaller step keeps the branches of the stencil fixed
    dp = _d(1e-7 * float(p.abs().mean()) * rng.standard_normal(ns))

    def fd(F, x, dx):
        out = []
        for t in (1.0, -1.0, 2.0, -2.0):
            y = torch.empty(ns, dtype=torch.float64, device="cuda")
            F(y, x + t * dx)
            out.append(y)
        torch.cuda.synchronize()
        return (8.0 * (out[0] - out[1]) - (out[2] - out[3])) / 12.0
    want = fd(op.vmult_enthalpy, w, dw)
    got = torch.empty(ns, dtype=torch.float64, device="cuda")
    op.vmult_enthalpy_tangent(got, w, dw)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(got - want) / torch.linalg.norm(want)) < 1e-8
    op.set_NS_stage(2)
    want = fd(op.vmult, p, dp)
    op.schur_tangent(got, p, dp)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(got - want) / torch.linalg.norm(want)) < 1e-7


@pytest.mark.parametrize("pc", ["jacobi", "cheb_fp32"])
def test_adjoint_pressure_solve(pc):
    """J_S(p)^T x = b solved to 1e-12 (checked with the transpose apply); and J_S(p) p = S p
    (the Schur apply is positively homogeneous of degree 1 in p, Euler's identity), which ties
    the linearisation to the forward operator."""
    from atmospheric_flows_b200.schur import SchurSolver
    P = 3
    m, op, src = _implicit_setup("hill", P)
    op.set_NS_stage(2)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(8)
    p = _d(src[2])
    b = _d(rng.standard_normal(ns))
    s = SchurSolver(op, pc)
    s.setup()
    x = torch.zeros(ns, dtype=torch.float64, device="cuda")
    out = s.solve_transpose(p, x, b, rel_tol=1e-12, max_iterations=5000)
    assert out["iterations"] > 0
    r = torch.empty_like(x)
    op.schur_transpose(r, p, x)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(r - b) / torch.linalg.norm(b)) < 1e-11
    Sp, Jp = torch.empty_like(x), torch.empty_like(x)
    op.vmult(Sp, p)
    op.schur_tangent(Jp, p, p)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(Jp - Sp) / torch.linalg.norm(Sp)) < 1e-12


def _stage_sources(m, P, stage, rough):
    """The fused rhs sources of a stage: rho, u, p of each explicit stage, then rho_c, u_fixed."""
    mk = (lambda k: M.random_state(m, P, seed=40 + k)) if rough else (lambda k: M.hill_state(m, P, seed=40 + k,
                                                                                               amplitude=0.05))
    st = [mk(k) for k in range(stage + 1)]
    src = []
    for j in range(stage):
        src += [st[j].rho, st[j].u, st[j].p]
    return src + [st[stage].rho, st[stage].u]


@pytest.mark.parametrize("P", [2, 3])
@pytest.mark.parametrize("stage", [2, 3])
@pytest.mark.parametrize("name,rough", [("hill", True), ("hill_periodic", False), ("annulus", True)])
def test_dot_product_stages_2_3(P, stage, name, rough):
    """Stages 2 and 3 (dual-number kernels): <ybar, J dx> = <J^T ybar, dx> to 1e-12."""
    from atmospheric_flows_b200.operator import EULEROperator
    m, Ma, Fr, _ = _case(name, P, rough)
    src = _stage_sources(m, P, stage, rough or name == "annulus")
    op = EULEROperator(m, P, Ma, Fr, 2.0)
    op.set_HYPERBOLIC_stage(stage)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(9)
    dx = [rng.standard_normal(a.size) for a in src]
    yb = [rng.standard_normal(n) for n in (ns, 2 * ns, ns)]
    s = [_d(a) for a in src]
    dy = [torch.empty(n, dtype=torch.float64, device="cuda") for n in (ns, 2 * ns, ns)]
    op.vmult_rhs_fused_tangent(s, [_d(a) for a in dx], *dy)
    xb = [torch.full((a.size,), np.nan, dtype=torch.float64, device="cuda") for a in src]
    op.vmult_rhs_fused_backward(s, *[_d(a) for a in yb], xb)
    torch.cuda.synchronize()
    lhs = sum(float(np.dot(a, b.cpu().numpy())) for a, b in zip(yb, dy))
    terms = [float(np.dot(b.cpu().numpy(), a)) for a, b in zip(dx, xb)]
    assert abs(lhs - sum(terms)) <= 1e-12 * sum(abs(t) for t in terms), (lhs, sum(terms))


@pytest.mark.parametrize("stage", [1, 2, 3])
def test_tangent_matches_forward_differences(stage):
    """The tangent (hand-written at stage 1, dual numbers at 2 and 3) against central differences
    of the forward rhs on a rough state (face traces differ, so no wave-speed branch flips
    within the step): 1e-7 relative."""
    from atmospheric_flows_b200.operator import EULEROperator
    P = 3
    m, Ma, Fr, _ = _case("hill", P, True)
    src = _stage_sources(m, P, stage, True)
    op = EULEROperator(m, P, Ma, Fr, 2.0)
    op.set_HYPERBOLIC_stage(stage)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(13)
    dx = [1e-2 * np.abs(a).max() * rng.standard_normal(a.size) for a in src]
    dy = [torch.empty(n, dtype=torch.float64, device="cuda") for n in (ns, 2 * ns, ns)]
    op.vmult_rhs_fused_tangent([_d(a) for a in src], [_d(a) for a in dx], *dy)

    def fwd(sign, h):
        out = [torch.empty(n, dtype=torch.float64, device="cuda") for n in (ns, 2 * ns, ns)]
        op.vmult_rhs_fused(*out, [_d(a + sign * h * b) for a, b in zip(src, dx)])
        return out
    h = 1e-4
    yp, ym = fwd(1, h), fwd(-1, h)
    torch.cuda.synchronize()
    for a, b, t in zip(yp, ym, dy):
        err = float(torch.linalg.norm((a - b) / (2 * h) - t) / torch.linalg.norm(t))
        assert err < 1e-7, (stage, err)
