"""GPU parity: every EULEROperator entry point of libaf_gpu.so (through the C ABI) against
the CPU oracle on the same seeded inputs.  Tolerances: 1e-12 relative L2 for the operator
applies; 1e-10 for the Schur complement, whose inner A^{-1} is an
iterative solve to 1e-12 in both implementations."""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12
DEGREES = [1, 2, 3, 4, 5, 6]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _meshes():
    return {
        "hill": M.jitter_mesh(M.hill_mesh(10, 5), 0.15, seed=11),
        "hill_periodic": M.hill_mesh(9, 4, periodic_x=True),
        "annulus": M.annulus_mesh(24, 3, r0=6.37122e6, r1=6.37122e6 + 16e3),
        # edge cases: a single cell; one column (both lateral faces are walls); one column
        # that is its own periodic neighbour; two periodic cells (both lateral neighbours are
        # the other cell); every block of cells per CTA is a partial one
        "box_1x1": M.box_mesh(1, 1, -500.0, 500.0, 0.0, 1000.0),
        "column_1x3": M.hill_mesh(1, 3),
        "self_periodic_1x2": M.hill_mesh(1, 2, periodic_x=True),
        "periodic_2x1": M.hill_mesh(2, 1, periodic_x=True),
    }

TINY = ["box_1x1", "column_1x3", "self_periodic_1x2", "periodic_2x1"]


def _setup(name, P, seed=5):
    from atmospheric_flows_b200.operator import EULEROperator
    from oracle.oracle import OracleOperator
    m = _meshes()[name]
    sc = M.Scaling()
    Ma, Fr, dt = sc.Ma, sc.Fr, 3.0
    if name == "annulus":
        Ma, Fr = (1.0 / (287.0 * 273.0)) ** 0.5, 1.0 / 9.80616 ** 0.5
    g = EULEROperator(m, P, Ma, Fr, dt)
    o = OracleOperator(m, P, Ma, Fr, dt)
    if name == "annulus":  # rough positive states; the hill background needs heights, not radii
        states = [M.random_state(m, P, seed=seed + k) for k in range(4)]
    else:
        states = [M.hill_state(m, P, seed=seed + k, amplitude=0.05) for k in range(4)]
    return m, g, o, states


def _d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _h(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _srcs(states, stage, kind):
    s0, s1, s2, s3 = states
    trip = [(s0.rho, s0.u, s0.p), (s1.rho, s1.u, s1.p), (s2.rho, s2.u, s2.p)]
    if kind == "rho":
        return sum(([trip[j][0], trip[j][1]] for j in range(stage)), [])
    base = sum(([*trip[j]] for j in range(stage)), [])
    if kind == "vel":
        return base + ([s3.rho] if stage < 3 else [])
    return base + [s3.rho, s3.u]


@pytest.mark.parametrize("P", DEGREES)
@pytest.mark.parametrize("name", ["hill", "hill_periodic", "annulus"] + TINY)
def test_rhs_parity(P, name):
    m, g, o, states = _setup(name, P)
    ns = m.n_cells * (P + 1) ** 2
    for stage in (1, 2, 3):
        g.set_HYPERBOLIC_stage(stage)
        o.set_HYPERBOLIC_stage(stage)
        for kind, n, gfun, ofun in (("rho", ns, g.vmult_rhs_rho_update, o.vmult_rhs_rho_update),
                                    ("vel", 2 * ns, g.vmult_rhs_velocity_fixed, o.vmult_rhs_velocity_fixed),
                                    ("pres", ns, g.vmult_rhs_pressure, o.vmult_rhs_pressure)):
            src = _srcs(states, stage, kind)
            want = ofun(src)
            dst = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
            gfun(dst, [_d(s) for s in src])
            err = rel(_h(dst), want)
            assert err < TOL, (stage, kind, err)


@pytest.mark.parametrize("P,name", [(2, "hill"), (4, "hill"), (6, "hill")] + [(P, t) for t in TINY for P in (1, 4)])
def test_fused_triple_and_host_path(P, name):
    m, g, o, states = _setup(name, P)
    ns = m.n_cells * (P + 1) ** 2
    for stage in (1, 2, 3):
        g.set_HYPERBOLIC_stage(stage)
        o.set_HYPERBOLIC_stage(stage)
        src = _srcs(states, stage, "pres")
        dr, du, dp = (torch.zeros(k * ns, dtype=torch.float64, device="cuda") for k in (1, 2, 1))
        g.vmult_rhs_fused(dr, du, dp, [_d(s) for s in src])
        assert rel(_h(dr), o.vmult_rhs_rho_update(_srcs(states, stage, "rho"))) < TOL
        assert rel(_h(du), o.vmult_rhs_velocity_fixed(_srcs(states, stage, "vel"))) < TOL
        assert rel(_h(dp), o.vmult_rhs_pressure(src)) < TOL
        hr, hu, hp = np.zeros(ns), np.zeros(2 * ns), np.zeros(ns)
        g.vmult_rhs_fused_host(hr, hu, hp, [np.ascontiguousarray(s) for s in src])
        assert np.array_equal(hr, _h(dr)) and np.array_equal(hu, _h(du)) and np.array_equal(hp, _h(dp))


@pytest.mark.parametrize("P", DEGREES)
@pytest.mark.parametrize("name", ["hill", "annulus"] + TINY)
def test_implicit_parity(P, name):
    m, g, o, states = _setup(name, P)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(3)
    rho_f = states[0].rho
    p_f = states[1].p
    for op in (g, o):
        op.set_rho_for_fixed(_d(rho_f) if op is g else rho_f)
        op.set_pres_fixed(_d(p_f) if op is g else p_f)
    for hs in (1, 2):
        g.set_HYPERBOLIC_stage(hs)
        o.set_HYPERBOLIC_stage(hs)
        for ns_stage, n in ((1, ns), (4, ns), (6, ns), (3, 2 * ns), (5, 2 * ns)):
            g.set_NS_stage(ns_stage)
            o.set_NS_stage(ns_stage)
            x = rng.standard_normal(n)
            dst = torch.zeros(n, dtype=torch.float64, device="cuda")
            g.vmult(dst, _d(x))
            assert rel(_h(dst), o.vmult(x)) < TOL, ns_stage
            inv = torch.zeros(n, dtype=torch.float64, device="cuda")
            g.compute_diagonal(inv)
            assert rel(_h(inv), o.inverse_diagonal()) < TOL, ("diag", ns_stage)
        p = states[2].p
        dst = torch.zeros(2 * ns, dtype=torch.float64, device="cuda")
        g.vmult_pressure(dst, _d(p))
        assert rel(_h(dst), o.vmult_pressure(p)) < TOL
        w = states[2].u
        dst = torch.zeros(ns, dtype=torch.float64, device="cuda")
        g.vmult_enthalpy(dst, _d(w))
        assert rel(_h(dst), o.vmult_enthalpy(w)) < TOL
        g.set_NS_stage(2)
        o.set_NS_stage(2)
        dst = torch.zeros(ns, dtype=torch.float64, device="cuda")
        g.vmult(dst, _d(p))
        assert g.last_inner_iterations() > 0
        assert rel(_h(dst), o.vmult(p)) < 1e-10


@pytest.mark.parametrize("P,name", [(1, "hill"), (2, "hill"), (4, "hill"), (6, "hill")] + [(P, t) for t in TINY for P in (1, 4)])
def test_exact_inverse_and_schur_mode(P, name):
    """af_vmult_inverse inverts the mass-type operators to rounding (checked against the
    oracle's forward operators), and the Schur apply with the exact cell-wise A^{-1} agrees
    with the reference's nested-CG form."""
    m, g, o, states = _setup(name, P)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(11)
    for op in (g, o):
        op.set_rho_for_fixed(_d(states[0].rho) if op is g else states[0].rho)
        op.set_pres_fixed(_d(states[1].p) if op is g else states[1].p)
    for ns_stage, n in ((1, ns), (6, ns), (3, 2 * ns), (5, 2 * ns)):
        o.set_NS_stage(ns_stage)
        g.set_NS_stage(ns_stage)
        x = rng.standard_normal(n)
        b = o.vmult(x)
        dst = torch.zeros(n, dtype=torch.float64, device="cuda")
        g.vmult_inverse(dst, _d(b))
        assert rel(_h(dst), x) < 1e-11, ns_stage
    for hs in (1, 2):
        g.set_HYPERBOLIC_stage(hs)
        o.set_HYPERBOLIC_stage(hs)
        g.set_NS_stage(2)
        o.set_NS_stage(2)
        g.set_schur_mode(1)
        p = states[2].p
        dst = torch.zeros(ns, dtype=torch.float64, device="cuda")
        g.vmult(dst, _d(p))
        assert g.last_inner_iterations() == 0
        assert rel(_h(dst), o.vmult(p)) < 1e-10
        g.set_schur_mode(0)
