"""Failure detection of the cell kernels' bounded waits.

A cell kernel waits for its bulk copies with a bounded number of polls.  When a wait gives
up, the kernel leaves a code in the handle's status word and returns without writing its
outputs; the library must then report AF_TIMEOUT instead of AF_OK over stale memory.  The
wait is made to run out by the handle's test hook: each CTA first waits on a barrier phase
that nothing completes, with a poll limit of a few iterations, before it issues any copy.
Nothing here faults, traps or hangs the GPU.
"""
import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = 4
POLLS = 4


def _setup():
    from atmospheric_flows_b200.operator import EULEROperator
    m = M.hill_mesh(16, 8)
    sc = M.Scaling()
    st = M.hill_state(m, P)
    op = EULEROperator(m, P, sc.Ma, sc.Fr, 2.0)
    op.set_HYPERBOLIC_stage(1)
    src = [torch.from_numpy(a).cuda() for a in (st.rho, st.u, st.p, st.rho, st.u)]
    ns = m.n_cells * (P + 1) ** 2
    return op, src, ns, st


def _outs(ns, fill):
    mk = lambda n: torch.full((n,), fill, dtype=torch.float64, device="cuda")
    return mk(ns), mk(2 * ns), mk(ns)


def test_timed_out_apply_reports_at_synchronize_and_writes_nothing():
    from atmospheric_flows_b200.operator import AFError, AF_TIMEOUT
    op, src, ns, _ = _setup()
    ref = _outs(ns, 0.0)
    op.vmult_rhs_fused(*ref, src)
    op.synchronize()
    op.set_stage_wait_test(POLLS)
    out = _outs(ns, 12345.0)
    op.vmult_rhs_fused(*out, src)  # queued: the launching call cannot know yet
    with pytest.raises(AFError) as e:
        op.synchronize()
    assert e.value.status == AF_TIMEOUT
    for t in out:  # every CTA left before writing
        assert bool(torch.all(t == 12345.0))
    op.synchronize()  # reported once, then cleared
    op.set_stage_wait_test(0)
    op.vmult_rhs_fused(*out, src)
    op.synchronize()
    for a, b in zip(out, ref):
        assert torch.equal(a, b)


def test_timeout_is_reported_by_the_next_call_that_queues_work():
    from atmospheric_flows_b200.operator import AFError, AF_TIMEOUT
    op, src, ns, _ = _setup()
    op.set_stage_wait_test(POLLS)
    out = _outs(ns, 0.0)
    op.vmult_rhs_fused(*out, src)
    torch.cuda.synchronize()  # the kernel has finished (outside the library)
    op.set_stage_wait_test(0)
    with pytest.raises(AFError) as e:
        op.vmult_rhs_pressure(out[2], src)
    assert e.value.status == AF_TIMEOUT
    op.vmult_rhs_pressure(out[2], src)  # the word was cleared by the report
    op.synchronize()


def test_calls_that_synchronize_return_the_timeout_themselves():
    from atmospheric_flows_b200.operator import AFError, AF_TIMEOUT
    op, src, ns, st = _setup()
    # the Schur apply (NS 2) with the inner CG: B and the CG's mass applies are cell kernels and
    # the CG reads its state back every 8 iterations
    rho_f = src[0]
    p_f = src[2]
    op.set_rho_for_fixed(rho_f)
    op.set_pres_fixed(p_f)
    op.set_NS_stage(2)
    op.set_stage_wait_test(POLLS)
    dst = torch.zeros(ns, dtype=torch.float64, device="cuda")
    with pytest.raises(AFError) as e:
        op.vmult(dst, p_f)
    assert e.value.status == AF_TIMEOUT
    # the host-buffer apply synchronizes before it returns
    hsrc = [np.ascontiguousarray(a) for a in (st.rho, st.u, st.p, st.rho, st.u)]
    hout = [np.zeros(ns), np.zeros(2 * ns), np.zeros(ns)]
    with pytest.raises(AFError) as e:
        op.vmult_rhs_fused_host(*hout, hsrc)
    assert e.value.status == AF_TIMEOUT
    op.set_stage_wait_test(0)
    op.vmult(dst, p_f)
    op.synchronize()
    assert bool(torch.isfinite(dst).all())


def test_imex_step_reports_the_timeout():
    """A time step whose kernels give up their waits returns AF_TIMEOUT from af_imex_step (the
    stepper synchronises inside its solves), and the next steps run normally."""
    import ctypes
    from atmospheric_flows_b200.imex import IMEXStepper, _bind
    from atmospheric_flows_b200.operator import AFError, AF_TIMEOUT, lib
    m = M.hill_mesh(8, 4, periodic_x=True)
    sc = M.Scaling()
    st = M.hill_state(m, P)
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, 2.0)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g.set_state(d(st.rho), d(st.u), d(st.p))
    op = ctypes.c_void_p(_bind().af_imex_operator(g._h))
    assert lib().af_set_stage_wait_test(op, POLLS) == 0
    with pytest.raises(AFError) as e:
        g.step(1)
    assert e.value.status == AF_TIMEOUT
    assert lib().af_set_stage_wait_test(op, 0) == 0
    g.set_state(d(st.rho), d(st.u), d(st.p))
    g.step(2)
    r, u, p = g.get_state()
    assert bool(torch.isfinite(u).all())
