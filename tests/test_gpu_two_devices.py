"""Handles on two devices in one process (skipped with fewer than two visible GPUs): the cell
kernels' shared-memory attribute is per device, so the second device's first launch must
configure it again."""
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_fused_apply_on_two_devices_agrees():
    if not torch.cuda.is_available() or torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    from atmospheric_flows_b200.operator import EULEROperator
    P = 4
    m = M.hill_mesh(16, 8)
    sc = M.Scaling()
    st = M.hill_state(m, P)
    ns = m.n_cells * (P + 1) ** 2
    outs = []
    for d in (0, 1):
        with torch.cuda.device(d):
            op = EULEROperator(m, P, sc.Ma, sc.Fr, 2.0)
            op.set_HYPERBOLIC_stage(1)
            src = [torch.from_numpy(a).cuda(d) for a in (st.rho, st.u, st.p, st.rho, st.u)]
            o = [torch.zeros(n, dtype=torch.float64, device=f"cuda:{d}") for n in (ns, 2 * ns, ns)]
            op.vmult_rhs_fused(*o, src)
            op.synchronize()
            outs.append([t.cpu() for t in o])
            del op
    for a, b in zip(*outs):
        assert torch.equal(a, b)
