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
