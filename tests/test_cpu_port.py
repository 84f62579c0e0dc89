"""The tuned CPU port of the fused stage-1 rhs (oracle/af_cpu_port.cpp, the timed CPU
baseline) against the oracle's three stage-1 right-hand sides: 1e-12 relative L2 on walled,
periodic and distorted hill meshes at degrees 2..6, including meshes narrower than one SIMD
batch of cells."""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M
from oracle.oracle import OracleOperator, cpu_port_rhs_fused_stage1

TOL = 1e-12


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("P,name", [(2, "hill"), (3, "periodic"), (4, "hill"), (4, "periodic"), (4, "jitter"),
                                    (5, "jitter"), (6, "hill"), (4, "tiny")])
def test_cpu_port_matches_oracle(P, name):
    m = {"hill": M.hill_mesh(9, 5), "periodic": M.hill_mesh(10, 4, periodic_x=True),
         "jitter": M.jitter_mesh(M.hill_mesh(7, 6, periodic_x=True), 0.15, seed=3),
         "tiny": M.hill_mesh(1, 3)}[name]
    sc = M.Scaling()
    st = M.hill_state(m, P, seed=5, amplitude=0.05)
    st2 = M.hill_state(m, P, seed=6, amplitude=0.05)
    src = [st.rho, st.u, st.p, st2.rho, st2.u]
    o = OracleOperator(m, P, sc.Ma, sc.Fr, 2.0)
    o.set_HYPERBOLIC_stage(1)
    r, u, p = cpu_port_rhs_fused_stage1(m, P, sc.Ma, sc.Fr, 2.0, src)
    assert rel(r, o.vmult_rhs_rho_update(src[:2])) < TOL
    assert rel(u, o.vmult_rhs_velocity_fixed(src[:4])) < TOL
    assert rel(p, o.vmult_rhs_pressure(src)) < TOL
