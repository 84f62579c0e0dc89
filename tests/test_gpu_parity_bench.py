"""GPU parity at the sizes the benchmark times, against the CPU oracle on the same inputs.

* The explicit apply on the benchmark's 512x256 hill mesh (the 2D terrain-following
  operator microbenchmark: hydrostatic background plus the seeded 16x16-mode perturbation,
  seed 20261203), at degree 4 and at the odd degree 3: the fused stage-1 triple that
  bench.py times and the three separate right-hand sides of every stage; at degrees 2, 5 (the
  layout with padded per-cell bulk slots) and 6, the rest of the benchmark's degree sweep, the
  stage-1 launches.  1e-12 relative L2.
* The implicit operators on the same mesh at degree 4: the mass-type operators, B
  (vmult_pressure), C (vmult_enthalpy), the inverse diagonals, and the NS-stage-2 Schur apply
  D p - C A^{-1} B p with the nested CG to 1e-12 on both sides (1e-10).
* IMEX steps on the 40x16 hill mesh at degree 4 (the plain FP64 hill case, periodic lateral
  boundaries, dt = 2 s, exact cell-wise inverses of the mass-type systems on both sides):
  - 100 steps with the library's default pressure solve, the reference's left-Jacobi GMRES
    stopping on |D^-1 r| <= eps |b| at eps = 1e-12.  That criterion leaves each solve far
    less accurate than eps: D^-1 scales the residual by about 1e-4 on this mesh, and the
    oracle's own states after 10 steps lie 5e-6 (velocity) from those of accurate solves.
    Two implementations that round differently stop at different iterates inside that
    band, so the stated tolerance after 100 steps is 1e-6 relative L2 per field.
  - 10 steps with accurate solves (GMRES stopping on the true residual |b - S p| <= 1e-12
    |b| on both sides): stated tolerance 1e-9.
"""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12
SEED = 20261203


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _h(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _bench_setup(P):
    from atmospheric_flows_b200.operator import EULEROperator
    from oracle.oracle import OracleOperator
    m = M.hill_mesh(512, 256)
    sc = M.Scaling()
    st = M.hill_state(m, P, seed=SEED, modes=16)
    st2 = M.hill_state(m, P, seed=SEED + 1, modes=4)
    st3 = M.hill_state(m, P, seed=SEED + 2, modes=4)
    g = EULEROperator(m, P, sc.Ma, sc.Fr, 2.0)
    o = OracleOperator(m, P, sc.Ma, sc.Fr, 2.0)
    return m, g, o, (st, st2, st3)


def _stage_sources(states, stage):
    """Pressure-list sources of a stage: (rho, u, p) per explicit stage, then rho_c, u_fix."""
    st, st2, st3 = states
    trip = [(st.rho, st.u, st.p), (st2.rho, st2.u, st2.p), (st3.rho, st3.u, st3.p)]
    src = sum(([*trip[j]] for j in range(stage)), [])
    cur = [st2, st3, st][stage - 1]
    return src + [cur.rho, cur.u]


@pytest.mark.parametrize("P", [4, 3, 5, 2, 6])
def test_rhs_parity_on_the_bench_mesh(P):
    m, g, o, states = _bench_setup(P)
    ns = m.n_cells * (P + 1) ** 2
    stages = (1, 2, 3) if P == 4 else (1,)
    for stage in stages:
        g.set_HYPERBOLIC_stage(stage)
        o.set_HYPERBOLIC_stage(stage)
        src = _stage_sources(states, stage)
        want_r = o.vmult_rhs_rho_update(sum(([src[3 * j], src[3 * j + 1]] for j in range(stage)), []))
        vel_src = src[:3 * stage] + ([src[3 * stage]] if stage < 3 else [])
        want_u = o.vmult_rhs_velocity_fixed(vel_src)
        want_p = o.vmult_rhs_pressure(src)
        dsrc = [_d(s) for s in src]
        if stage == 1:  # the benchmark's fused launch
            dr, du, dp = (torch.full((k * ns,), np.nan, dtype=torch.float64, device="cuda") for k in (1, 2, 1))
            g.vmult_rhs_fused(dr, du, dp, dsrc)
            for got, want, name in ((dr, want_r, "rho"), (du, want_u, "u"), (dp, want_p, "p")):
                err = rel(_h(got), want)
                assert err < TOL, ("fused", stage, name, err)
        for n, fn, s, want, name in ((ns, g.vmult_rhs_rho_update,
                                      [dsrc[k] for j in range(stage) for k in (3 * j, 3 * j + 1)], want_r, "rho"),
                                     (2 * ns, g.vmult_rhs_velocity_fixed, [_d(a) for a in vel_src], want_u, "u"),
                                     (ns, g.vmult_rhs_pressure, dsrc, want_p, "p")):
            dst = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
            fn(dst, s)
            err = rel(_h(dst), want)
            assert err < TOL, ("separate", stage, name, err)


def test_implicit_parity_on_the_bench_mesh():
    P = 4
    m, g, o, (st, st2, st3) = _bench_setup(P)
    ns = m.n_cells * (P + 1) ** 2
    rng = np.random.default_rng(3)
    for op in (g, o):
        op.set_rho_for_fixed(_d(st.rho) if op is g else st.rho)
        op.set_pres_fixed(_d(st2.p) if op is g else st2.p)
    for hs in (1, 2):
        g.set_HYPERBOLIC_stage(hs)
        o.set_HYPERBOLIC_stage(hs)
        if hs == 1:
            for ns_stage, n in ((1, ns), (6, ns), (3, 2 * ns)):
                g.set_NS_stage(ns_stage)
                o.set_NS_stage(ns_stage)
                x = rng.standard_normal(n)
                dst = torch.zeros(n, dtype=torch.float64, device="cuda")
                g.vmult(dst, _d(x))
                assert rel(_h(dst), o.vmult(x)) < TOL, ns_stage
                inv = torch.zeros(n, dtype=torch.float64, device="cuda")
                g.compute_diagonal(inv)
                assert rel(_h(inv), o.inverse_diagonal()) < TOL, ("diag", ns_stage)
        dst = torch.zeros(2 * ns, dtype=torch.float64, device="cuda")
        g.vmult_pressure(dst, _d(st3.p))
        assert rel(_h(dst), o.vmult_pressure(st3.p)) < TOL, ("B", hs)
        dst = torch.zeros(ns, dtype=torch.float64, device="cuda")
        g.vmult_enthalpy(dst, _d(st3.u))
        assert rel(_h(dst), o.vmult_enthalpy(st3.u)) < TOL, ("C", hs)
        g.set_NS_stage(2)
        o.set_NS_stage(2)
        dst = torch.zeros(ns, dtype=torch.float64, device="cuda")
        g.vmult(dst, _d(st3.p))
        assert g.last_inner_iterations() > 0
        assert rel(_h(dst), o.vmult(st3.p)) < 1e-10, ("Schur", hs)


def _imex_40x16(nsteps, eps, accurate):
    from atmospheric_flows_b200.imex import IMEXStepper
    from oracle.oracle import OracleOperator, imex_steps
    P, dt = 4, 2.0
    m = M.hill_mesh(40, 16, periodic_x=True)
    sc = M.Scaling()
    st = M.hill_state(m, P, amplitude=1e-3)
    o = OracleOperator(m, P, sc.Ma, sc.Fr, dt)
    ref = imex_steps(o, st.rho, st.u, st.p, nsteps, eps=eps, exact_inverse=True, true_residual=accurate)
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, dt, eps=eps, schur_preconditioner="jacobi" if accurate else None)
    g.set_state(_d(st.rho), _d(st.u), _d(st.p))
    g.step(nsteps)
    got = [t.cpu().numpy() for t in g.get_state()]
    errs = {k: rel(a, b) for k, a, b in zip(("rho", "u", "p"), got, ref[:3])}
    print(f"imex 40x16 p=4, {nsteps} steps, eps {eps}, accurate solves {accurate}: state errors vs oracle {errs}, "
          f"fixed point {g.stats()['fixed_point_iterations']} / {ref[3]}")
    assert np.abs(ref[1]).max() > 10.0  # the flow has moved over the hill (not a trivial state)
    return errs


def test_imex_100_steps_on_the_40x16_hill():
    for k, e in _imex_40x16(100, 1e-12, False).items():
        assert e < 1e-6, (k, e)


def test_imex_10_accurate_steps_on_the_40x16_hill():
    for k, e in _imex_40x16(10, 1e-12, True).items():
        assert e < 1e-9, (k, e)


# Rayleigh damping layers of the 2D hill case (no counterpart in the reference): the upper
# sponge above 10 km and relaxation zones 4 km wide at the lateral boundaries, towards the
# inflow velocity (10 m/s, 0).
SPONGE = dict(z_start=10000.0, z_top=16000.0, rate_top=0.05, x_left=-20000.0, x_right=20000.0,
              width_lateral=4000.0, rate_lateral=0.02, u_ref=10.0)


@pytest.mark.parametrize("P", [2, 4])
def test_rhs_parity_with_sponge(P):
    from atmospheric_flows_b200.operator import EULEROperator
    from oracle.oracle import OracleOperator
    m = M.jitter_mesh(M.hill_mesh(10, 5, periodic_x=True), 0.1, seed=4)
    sc = M.Scaling()
    g = EULEROperator(m, P, sc.Ma, sc.Fr, 3.0)
    o = OracleOperator(m, P, sc.Ma, sc.Fr, 3.0)
    g.set_sponge(**SPONGE)
    o.set_sponge(**SPONGE)
    states = [M.hill_state(m, P, seed=5 + k, amplitude=0.05) for k in range(3)]
    ns = m.n_cells * (P + 1) ** 2
    o0 = OracleOperator(m, P, sc.Ma, sc.Fr, 3.0)  # without the sponge: the term must matter
    for stage in (1, 2, 3):
        g.set_HYPERBOLIC_stage(stage)
        o.set_HYPERBOLIC_stage(stage)
        o0.set_HYPERBOLIC_stage(stage)
        src = _stage_sources(tuple(states), stage)
        vel_src = src[:3 * stage] + ([src[3 * stage]] if stage < 3 else [])
        want = o.vmult_rhs_velocity_fixed(vel_src)
        assert rel(want, o0.vmult_rhs_velocity_fixed(vel_src)) > 1e-6
        dst = torch.full((2 * ns,), np.nan, dtype=torch.float64, device="cuda")
        g.vmult_rhs_velocity_fixed(dst, [_d(a) for a in vel_src])
        assert rel(_h(dst), want) < TOL, ("separate", stage)
        dr, du, dp = (torch.zeros(k * ns, dtype=torch.float64, device="cuda") for k in (1, 2, 1))
        g.vmult_rhs_fused(dr, du, dp, [_d(a) for a in src])
        assert rel(_h(du), want) < TOL, ("fused", stage)
        assert rel(_h(dp), o.vmult_rhs_pressure(src)) < TOL, ("pressure unaffected", stage)


def _imex_40x16_sponge(nsteps, accurate):
    from atmospheric_flows_b200.imex import IMEXStepper
    from oracle.oracle import OracleOperator, imex_steps
    P, dt, eps = 4, 2.0, 1e-12
    m = M.hill_mesh(40, 16, periodic_x=True)
    sc = M.Scaling()
    st = M.hill_state(m, P, amplitude=1e-3)
    o = OracleOperator(m, P, sc.Ma, sc.Fr, dt)
    o.set_sponge(**SPONGE)
    ref = imex_steps(o, st.rho, st.u, st.p, nsteps, eps=eps, exact_inverse=True, true_residual=accurate)
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, dt, eps=eps, schur_preconditioner="jacobi" if accurate else None)
    g.set_sponge(**SPONGE)
    g.set_state(_d(st.rho), _d(st.u), _d(st.p))
    g.step(nsteps)
    got = [t.cpu().numpy() for t in g.get_state()]
    errs = {k: rel(a, b) for k, a, b in zip(("rho", "u", "p"), got, ref[:3])}
    print(f"imex 40x16 p=4 with sponge, {nsteps} steps, accurate solves {accurate}: state errors vs oracle {errs}")
    return errs


def test_imex_100_steps_with_sponge_on_the_40x16_hill():
    """The plain FP64 hill case with its damping layers: Rayleigh sponge above 10 km and
    lateral relaxation zones (periodic lateral boundaries), 100 steps at the reference's
    criterion (stated tolerance 1e-6, as above)."""
    for k, e in _imex_40x16_sponge(100, False).items():
        assert e < 1e-6, (k, e)


def test_imex_10_accurate_steps_with_sponge_on_the_40x16_hill():
    for k, e in _imex_40x16_sponge(10, True).items():
        assert e < 1e-9, (k, e)
