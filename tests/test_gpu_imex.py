"""Full IMEX steps on the GPU (af_imex_*) against the oracle's restatement of
EulerSolver::run (Atmospheric_Flow.cc:1110-1251) on the same mesh and state.

Both sides solve every linear system to eps = 1e-12 relative and stop the pressure fixed
point at 1e-10 (the reference's criterion); their iterates differ in rounding and in the
mass-system preconditioners, so the states after N steps agree to a stated tolerance of
1e-9 relative L2 (checked with the fixed-point iteration counts)."""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

STATE_TOL = 1e-9


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("P,nsteps,mesh,exact", [(2, 3, "hill", 1), (3, 2, "hill_periodic", 1), (4, 2, "hill", 1),
                                                 (3, 2, "hill", 0), (4, 2, "column_1x3", 1),
                                                 (4, 2, "self_periodic_1x2", 1), (2, 2, "periodic_2x1", 0)])
def test_imex_steps_match_oracle(P, nsteps, mesh, exact):
    """exact = 1: cell-wise exact inverses for the mass systems and inside the Schur apply
    (the default); exact = 0: CG + Jacobi and the nested CG as in the reference."""
    from atmospheric_flows_b200.imex import IMEXStepper
    from oracle.oracle import OracleOperator, imex_steps
    m = {"hill": M.hill_mesh(10, 5), "hill_periodic": M.hill_mesh(12, 4, periodic_x=True),
         "column_1x3": M.hill_mesh(1, 3), "self_periodic_1x2": M.hill_mesh(1, 2, periodic_x=True),
         "periodic_2x1": M.hill_mesh(2, 1, periodic_x=True)}[mesh]
    sc = M.Scaling()
    dt = 2.0
    st = M.hill_state(m, P, amplitude=1e-3)
    o = OracleOperator(m, P, sc.Ma, sc.Fr, dt)
    r_ref, u_ref, p_ref, fp_ref = imex_steps(o, st.rho, st.u, st.p, nsteps, eps=1e-12)
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, dt, eps=1e-12, mass_solver=exact, schur_inner=exact)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g.set_state(d(st.rho), d(st.u), d(st.p))
    g.step(nsteps)
    r, u, p = (t.cpu().numpy() for t in g.get_state())
    s = g.stats()
    assert s["fixed_point_iterations"][0] >= 1 and s["gmres_iterations"] > 0
    assert abs(s["fixed_point_iterations"][0] - fp_ref[0]) <= 1
    assert rel(r, r_ref) < STATE_TOL
    assert rel(u, u_ref) < STATE_TOL
    assert rel(p, p_ref) < STATE_TOL


@pytest.mark.parametrize("pc,odd", [(pc, False) for pc in ("jacobi", "mg_fp64", "mg_fp32", "cheb_fp64", "cheb_fp32")]
                         + [("cheb_fp32", True), ("jacobi", True)])
def test_imex_schur_solver_options_match_oracle(pc, odd):
    """The pressure system solved by af_schur_solve (FGMRES on the true residual, Jacobi or
    multigrid preconditioning with FP64 or FP32 levels) instead of the reference's
    left-Jacobi GMRES, against the oracle run with the same true-residual criterion (its
    GMRES right-preconditioned): same states after two steps to the stated tolerance.
    odd: 3 x 3 cells at degree 4, 225 DoFs per scalar field, so that the solver's stored
    Krylov vectors need a padded stride to stay 16-byte aligned."""
    from atmospheric_flows_b200.imex import IMEXStepper
    from oracle.oracle import OracleOperator, imex_steps
    P, nsteps, dt = (4, 2, 2.0) if odd else (3, 2, 2.0)
    m = M.hill_mesh(3, 3) if odd else M.hill_mesh(16, 8)
    sc = M.Scaling()
    st = M.hill_state(m, P, amplitude=1e-3)
    o = OracleOperator(m, P, sc.Ma, sc.Fr, dt)
    r_ref, u_ref, p_ref, fp_ref = imex_steps(o, st.rho, st.u, st.p, nsteps, eps=1e-12, true_residual=True)
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, dt, eps=1e-12, schur_preconditioner=pc)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g.set_state(d(st.rho), d(st.u), d(st.p))
    g.step(nsteps)
    r, u, p = (t.cpu().numpy() for t in g.get_state())
    s = g.stats()
    assert s["gmres_iterations"] > 0
    assert abs(s["fixed_point_iterations"][0] - fp_ref[0]) <= 1
    assert rel(r, r_ref) < STATE_TOL
    assert rel(u, u_ref) < STATE_TOL
    assert rel(p, p_ref) < STATE_TOL


def test_imex_rest_state_stays_balanced():
    """An isothermal atmosphere at rest on a flat box is a discrete steady state up to the
    hydrostatic discretisation residual: velocities stay tiny after a few steps."""
    from atmospheric_flows_b200.imex import IMEXStepper
    P = 3
    m = M.box_mesh(8, 6, -4000.0, 4000.0, 0.0, 6000.0, periodic_x=True)
    sc = M.Scaling()
    xz = M.dof_coordinates(m, P)
    rho, p = M.hydrostatic_background(xz[..., 1], sc=sc)
    u = np.zeros(2 * rho.size)
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, 5.0, eps=1e-12)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a.ravel())).cuda()
    g.set_state(d(rho), d(u), d(p))
    g.step(3)
    r2, u2, p2 = (t.cpu().numpy() for t in g.get_state())
    assert np.abs(u2).max() < 1e-2          # m/s, after 15 s
    assert rel(p2, p.ravel()) < 1e-6
