"""Time-loop diagnostics and the L2 norm on the GPU (af_compute_diagnostics, af_l2_norm)
against numpy restatements of the reference's definitions (Atmospheric_Flow.cc:925-1087,
1224-1235)."""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_diagnostics_match_nodal_reductions():
    from atmospheric_flows_b200.operator import EULEROperator
    P, dt = 3, 1.5
    m = M.jitter_mesh(M.hill_mesh(20, 8), 0.2, seed=5)
    sc = M.Scaling()
    st = M.hill_state(m, P, amplitude=0.05)
    st2 = M.hill_state(m, P, seed=77, amplitude=0.05)
    op = EULEROperator(m, P, sc.Ma, sc.Fr, dt)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    got = op.compute_diagnostics(d(st.rho), d(st.u), d(st.p), rho_stage=d(st2.rho))
    nd = (P + 1) ** 2
    u = st.u.reshape(m.n_cells, 2, nd)
    vmax = np.sqrt(u[:, 0] ** 2 + u[:, 1] ** 2).max()
    cel = np.sqrt(1.4 * st.p / st.rho).max()
    v = m.vertices
    d1 = np.hypot(*(v[1:, 1:] - v[:-1, :-1]).transpose(2, 0, 1))
    d2 = np.hypot(*(v[1:, :-1] - v[:-1, 1:]).transpose(2, 0, 1))
    dmin = np.maximum(d1, d2).min()
    want = {"max_velocity": vmax, "min_density": st2.rho.min(), "max_density": np.abs(st2.rho).max(),
            "max_celerity": cel, "min_cell_diameter": dmin,
            "cfl_c": dt * cel / sc.Ma * P * np.sqrt(2) / dmin, "cfl_u": dt * vmax * P * np.sqrt(2) / dmin}
    for k, w in want.items():
        assert abs(got[k] - w) <= 1e-13 * abs(w), (k, got[k], w)
    # without rho_stage the density extrema come from rho
    got2 = op.compute_diagnostics(d(st.rho), d(st.u), d(st.p))
    assert got2["min_density"] == st.rho.min()


@pytest.mark.parametrize("P", [1, 3, 4])
def test_l2_norm_is_exact_for_polynomials(P):
    """|f|_L2 over a box for f of degree <= P is integrated exactly by QGauss(P+1)."""
    from atmospheric_flows_b200.operator import EULEROperator
    Lx, Lz = 3.0, 2.0
    m = M.box_mesh(6, 4, 0.0, Lx, 0.0, Lz)
    sc = M.Scaling()
    op = EULEROperator(m, P, sc.Ma, sc.Fr, 1.0)
    xz = M.dof_coordinates(m, P)
    f = (xz[..., 0] + 2.0 * xz[..., 1]).ravel()  # degree 1
    want = np.sqrt(Lx ** 3 * Lz / 3 + 2 * Lx ** 2 * Lz ** 2 / 2 + 4 * Lx * Lz ** 3 / 3)  # int (x+2z)^2
    got = op.l2_norm(torch.from_numpy(f).cuda())
    assert abs(got - want) < 1e-13 * want
    # two components: |(f, f)| = sqrt(2) |f|
    ff = np.stack([f.reshape(m.n_cells, -1)] * 2, axis=1).ravel()
    assert abs(op.l2_norm(torch.from_numpy(ff).cuda(), ncomp=2) - np.sqrt(2) * want) < 1e-13 * want
