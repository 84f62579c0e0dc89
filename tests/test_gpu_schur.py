"""Schur-complement pressure solver on the GPU (af_schur_*).

1. The multigrid V-cycle against a dense CPU restatement of the same cycle built from the
   oracle's operator matrices (box mesh, constant coefficients, so the wave-speed term of C
   vanishes and the operator is linear): FP64 levels agree to 1e-12 relative, FP32 levels to
   1e-4.
2. FGMRES with each preconditioner (Jacobi, FP64 and FP32 multigrid, FP64 and FP32 Chebyshev
   polynomial, the latter with reduced and full quadrature) solves S x = S x_true
   on a hill mesh to a true residual of 1e-10; the solution matches x_true and its residual,
   recomputed by the oracle's Schur apply on the CPU, is below 1e-9.
"""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _lag(nd, j, s):
    v = 1.0
    for k in range(len(nd)):
        if k != j:
            v *= (s - nd[k]) / (nd[j] - nd[k])
    return v


def _prolongation(P, nx, nz):
    """Fine (nx x nz) <- coarse (nx/2 x nz/2) embedding of DG(P) nodal vectors."""
    nd = M.gll_nodes_01(P)
    Pm = np.array([[[_lag(nd, j, (o + nd[i]) / 2) for j in range(P + 1)] for i in range(P + 1)] for o in range(2)])
    ND = (P + 1) ** 2
    nxc, nzc = nx // 2, nz // 2
    Pr = np.zeros((nx * nz * ND, nxc * nzc * ND))
    for jc in range(nzc):
        for ic in range(nxc):
            cc = jc * nxc + ic
            for oz in range(2):
                for ox in range(2):
                    cf = (2 * jc + oz) * nx + 2 * ic + ox
                    Pr[cf * ND:(cf + 1) * ND, cc * ND:(cc + 1) * ND] = np.kron(Pm[oz], Pm[ox])
    return Pr


def _dense_schur(P, nx, nz, dt):
    from oracle.oracle import OracleOperator
    sc = M.Scaling()
    m = M.box_mesh(nx, nz, -20000.0, 20000.0, 0.0, 16000.0)
    n = nx * nz * (P + 1) ** 2
    o = OracleOperator(m, P, sc.Ma, sc.Fr, dt)
    o.set_HYPERBOLIC_stage(1)
    o.set_rho_for_fixed(np.ones(n))
    o.set_pres_fixed(np.ones(n))
    o.set_NS_stage(2)

    def dense():
        S = np.zeros((n, n))
        for j in range(n):
            e = np.zeros(n)
            e[j] = 1.0
            S[:, j] = o.vmult(e)
        return S
    S = dense()
    o.set_dt(1e-30)  # D = M/(gamma-1) alone
    D = dense()
    return S, D


def _cheb(S, Dinv, b, x0, deg, lo, hi, zero_init, final_res):
    theta, delta = (hi + lo) / 2, (hi - lo) / 2
    sigma = theta / delta
    r = b.copy() if zero_init else b - S @ x0
    d = Dinv @ r / theta
    x = d.copy() if zero_init else x0 + d
    ro = 1 / sigma
    for _ in range(1, deg):
        r = r - S @ d
        rho = 1 / (2 * sigma - ro)
        d = rho * ro * d + 2 * rho / delta * (Dinv @ r)
        x = x + d
        ro = rho
    if final_res:
        r = r - S @ d
    return x, r


@pytest.mark.parametrize("precision,tol", [("mg_fp64", 1e-12), ("mg_fp32", 1e-4)])
def test_vcycle_matches_dense_restatement(precision, tol):
    from atmospheric_flows_b200.operator import EULEROperator
    from atmospheric_flows_b200.schur import SchurSolver
    P, nx, nz, dt = 2, 8, 4, 60.0
    sc = M.Scaling()
    n = nx * nz * (P + 1) ** 2
    op = EULEROperator(M.box_mesh(nx, nz, -20000.0, 20000.0, 0.0, 16000.0), P, sc.Ma, sc.Fr, dt)
    op.set_stream(torch.cuda.current_stream())
    op.set_schur_mode(1)
    op.set_HYPERBOLIC_stage(1)
    one = torch.ones(n, dtype=torch.float64, device="cuda")
    op.set_rho_for_fixed(one)
    op.set_pres_fixed(one)
    op.set_NS_stage(2)
    b = np.random.default_rng(3).standard_normal(n)
    s = SchurSolver(op, precision, max_levels=2, coarse_degree=60, smoother_degree=3, coarse_lmax=0.0)
    s.setup()
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    s.precondition(z, torch.from_numpy(b).cuda())
    torch.cuda.synchronize()
    lmax = s.levels()
    assert len(lmax) == 2
    Sf, Df = _dense_schur(P, nx, nz, dt)
    Sc, Dc = _dense_schur(P, nx // 2, nz // 2, dt)
    true_lmax = np.abs(np.linalg.eigvals(np.linalg.solve(Df, Sf))).max()
    assert abs(lmax[0] / true_lmax - 1) < 0.1  # power-iteration estimate
    Pr = _prolongation(P, nx, nz)
    rng = s.options.smoothing_range
    hi0, hi1 = 1.2 * lmax[0], 1.2 * lmax[1]
    Dfi, Dci = np.linalg.inv(Df), np.linalg.inv(Dc)
    x, r = _cheb(Sf, Dfi, b, None, 3, hi0 / rng, hi0, True, True)
    xc, _ = _cheb(Sc, Dci, Pr.T @ r, None, 60, min(0.9, hi1 / rng), hi1, True, False)
    want, _ = _cheb(Sf, Dfi, b, x + Pr @ xc, 3, hi0 / rng, hi0, False, False)
    assert rel(z.cpu().numpy(), want) < tol


def test_schur_solve_all_preconditioners():
    from atmospheric_flows_b200.operator import EULEROperator
    from atmospheric_flows_b200.schur import SchurSolver
    from oracle.oracle import OracleOperator
    P, dt = 3, 2.0
    m = M.hill_mesh(32, 16)
    sc = M.Scaling()
    st = M.hill_state(m, P, modes=4)
    xt = M.hill_state(m, P, seed=99, modes=8, amplitude=1e-2).p
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    op = EULEROperator(m, P, sc.Ma, sc.Fr, dt)
    op.set_stream(torch.cuda.current_stream())
    op.set_schur_mode(1)
    op.set_HYPERBOLIC_stage(1)
    op.set_rho_for_fixed(d(st.rho))
    op.set_pres_fixed(d(st.p))
    op.set_NS_stage(2)
    b = torch.empty_like(d(xt))
    op.vmult(b, d(xt))
    torch.cuda.synchronize()
    bh = b.cpu().numpy()
    o = OracleOperator(m, P, sc.Ma, sc.Fr, dt)
    o.set_HYPERBOLIC_stage(1)
    o.set_rho_for_fixed(st.rho)
    o.set_pres_fixed(st.p)
    o.set_NS_stage(2)
    its = {}
    cases = {"jacobi": {}, "mg_fp64": {}, "mg_fp32": {}, "cheb_fp64": {}, "cheb_fp32": {},
             "cheb_fp32_full_quadrature": {"reduced_quadrature": 0},
             "cheb_fp32_nodal": {"reduced_quadrature": 1}}
    for pc, kw in cases.items():
        s = SchurSolver(op, pc.replace("_full_quadrature", "").replace("_nodal", ""), **kw)
        s.setup()
        x = torch.zeros_like(b)
        out = s.solve(x, b, rel_tol=1e-10, max_iterations=5000)
        torch.cuda.synchronize()
        xh = x.cpu().numpy()
        its[pc] = out["iterations"]
        assert out["final_residual"] <= 1e-10 * np.linalg.norm(bh) * (1 + 1e-6)
        assert rel(xh, xt) < 1e-8, pc
        assert rel(o.vmult(xh), bh) < 1e-9, pc
    # the multigrid and polynomial preconditioners take far fewer iterations than Jacobi
    for pc in ("mg_fp64", "mg_fp32", "cheb_fp64", "cheb_fp32", "cheb_fp32_full_quadrature", "cheb_fp32_nodal"):
        assert its[pc] * 2 < its["jacobi"], its
    # the Gauss-point smoother (the default) is the nodal reduced-quadrature one in another basis
    assert abs(its["cheb_fp32"] - its["cheb_fp32_nodal"]) <= 1, its


def test_reduced_quadrature_preconditioner_is_exact_on_affine_cells():
    """With P+1 Gauss points the FP32 level operators integrate B and D exactly on bilinear
    cells, and C0 and A too when rho_for_fixed and pres_fixed are constant, so on a box mesh
    with constant coefficients the reduced and the full-quadrature preconditioners agree to FP32
    rounding; with the hill state's varying coefficients they differ (the reduced one is an
    approximation)."""
    from atmospheric_flows_b200.operator import EULEROperator
    from atmospheric_flows_b200.schur import SchurSolver
    P, dt = 4, 2.0
    sc = M.Scaling()
    out = {}
    for name, m in (("box", M.box_mesh(16, 8, -20000.0, 20000.0, 0.0, 16000.0)), ("hill", M.hill_mesh(16, 8))):
        n = m.n_cells * (P + 1) ** 2
        op = EULEROperator(m, P, sc.Ma, sc.Fr, dt)
        op.set_stream(torch.cuda.current_stream())
        op.set_HYPERBOLIC_stage(1)
        if name == "box":
            op.set_rho_for_fixed(torch.full((n,), 1.3, dtype=torch.float64, device="cuda"))
            op.set_pres_fixed(torch.full((n,), 0.9, dtype=torch.float64, device="cuda"))
        else:
            st = M.hill_state(m, P, modes=4)
            op.set_rho_for_fixed(torch.from_numpy(st.rho).cuda())
            op.set_pres_fixed(torch.from_numpy(st.p).cuda())
        op.set_NS_stage(2)
        b = torch.from_numpy(np.random.default_rng(5).standard_normal(n)).cuda()
        z = {}
        for rq in (0, 1):
            s = SchurSolver(op, "cheb_fp32", reduced_quadrature=rq)
            s.setup()
            z[rq] = torch.zeros(n, dtype=torch.float64, device="cuda")
            s.precondition(z[rq], b)
        torch.cuda.synchronize()
        out[name] = rel(z[1].cpu().numpy(), z[0].cpu().numpy())
    assert out["box"] < 1e-4, out
    assert out["hill"] > 10 * out["box"], out


@pytest.mark.parametrize("P", [2, 4])
def test_fp32_chebyshev_on_the_preconditioned_residual_matches_fp64(P):
    """The FP32 Chebyshev preconditioner carries z = D^{-1} r (its step kernel has no D term:
    z' = z + D^{-1} C0 w - d), the FP64 one the residual r itself (r' = r + C0 w - D d, then
    D^{-1} r').  With the same quadrature (2P+1 points, reduced_quadrature = 0) and degree the
    two are the same polynomial in D^{-1} S0.  rho_for_fixed is constant, so that the FP32
    levels' change-of-basis A^{-1} (exact for a constant rho) and the FP64 levels' packed
    A^{-1} invert the same A; pres_fixed is the hill state's.  The outputs then agree to FP32
    rounding, amplified by the recurrence with the degree (degree 2: one z-step, 1e-5;
    degree 16: 1e-3)."""
    from atmospheric_flows_b200.operator import EULEROperator
    from atmospheric_flows_b200.schur import SchurSolver
    dt = 2.0
    sc = M.Scaling()
    m = M.hill_mesh(16, 8)
    n = m.n_cells * (P + 1) ** 2
    op = EULEROperator(m, P, sc.Ma, sc.Fr, dt)
    op.set_stream(torch.cuda.current_stream())
    op.set_HYPERBOLIC_stage(1)
    st = M.hill_state(m, P, modes=4)
    op.set_rho_for_fixed(torch.full((n,), 1.3, dtype=torch.float64, device="cuda"))
    op.set_pres_fixed(torch.from_numpy(st.p).cuda())
    op.set_NS_stage(2)
    b = torch.from_numpy(np.random.default_rng(9).standard_normal(n)).cuda()
    errs = {}
    for degree, tol in ((2, 1e-5), (16, 1e-3)):
        z = {}
        for pc, opts in (("cheb_fp64", {}), ("cheb_fp32", {"reduced_quadrature": 0})):
            s = SchurSolver(op, pc, poly_degree=degree, **opts)
            s.setup()
            z[pc] = torch.zeros(n, dtype=torch.float64, device="cuda")
            s.precondition(z[pc], b)
        torch.cuda.synchronize()
        errs[degree] = rel(z["cheb_fp32"].cpu().numpy(), z["cheb_fp64"].cpu().numpy())
        assert errs[degree] < tol, errs
    print("fp32 z-form vs fp64 r-form, relative difference by degree:", errs)


@pytest.mark.parametrize("P,periodic", [(1, False), (2, True), (3, False), (4, False), (4, True), (5, True), (6, False)])
def test_gauss_point_smoother_matches_the_nodal_one(P, periodic):
    """reduced_quadrature = 2 runs the FP32 Chebyshev polynomial in the basis of the Lagrange
    polynomials of the P+1 Gauss points, where the cell inverses of A and D are diagonal; it is
    the same polynomial in D^{-1} S0 as the nodal reduced-quadrature smoother
    (reduced_quadrature = 1), so the two preconditioner outputs agree to FP32 rounding amplified
    by the recurrence (degree 2: one step; degree 16).  Hill state coefficients, walled and
    x-periodic meshes, every compiled degree."""
    from atmospheric_flows_b200.operator import EULEROperator
    from atmospheric_flows_b200.schur import SchurSolver
    dt = 2.0
    sc = M.Scaling()
    m = M.hill_mesh(16, 8, periodic_x=periodic)
    n = m.n_cells * (P + 1) ** 2
    op = EULEROperator(m, P, sc.Ma, sc.Fr, dt)
    op.set_stream(torch.cuda.current_stream())
    op.set_HYPERBOLIC_stage(1)
    st = M.hill_state(m, P, modes=4)
    op.set_rho_for_fixed(torch.from_numpy(st.rho).cuda())
    op.set_pres_fixed(torch.from_numpy(st.p).cuda())
    op.set_NS_stage(2)
    b = torch.from_numpy(np.random.default_rng(11).standard_normal(n)).cuda()
    errs = {}
    for degree, tol in ((2, 2e-5), (16, 1e-3)):
        z = {}
        for rq in (1, 2):
            s = SchurSolver(op, "cheb_fp32", poly_degree=degree, reduced_quadrature=rq)
            s.setup()
            z[rq] = torch.zeros(n, dtype=torch.float64, device="cuda")
            s.precondition(z[rq], b)
        torch.cuda.synchronize()
        errs[degree] = rel(z[2].cpu().numpy(), z[1].cpu().numpy())
        assert errs[degree] < tol, errs
    print(f"P={P} periodic={periodic}: Gauss-point vs nodal smoother, relative difference by degree:", errs)
