"""GPU run of the reference's "Channel" test (examples/navierstokes.c:252, examples/channel.yaml): degree 1 with q_extra 2 on
5 x 5 x 1 faces, body force, no-slip walls and symmetry planes as essential DOFs, 5 backward-Euler steps through the time
loop (hb_ts_* with hb_ts_set_essential), FP64 and mixed precision, point Jacobi and point-block Jacobi, in conservative
variables and as "Channel, Primitive" (examples/navierstokes.c:253).  The final state must meet the reference's own regression
bound against tests/output/channel.bin / channel-prim.bin (max |Q - Q_ref| / max |Q_ref| <= 2e-11, over the free DOFs as a
sorted multiset), and the fused operators at this (P, Q) = (2, 4) must equal the oracle."""
import importlib

import numpy as np
import pytest

from helpers import O, oracle_ifunction, oracle_mesh, prob, rel_l2
from test_channel import channel_case, free_state_error

pytestmark = pytest.mark.gpu

K = importlib.import_module("honee-4aiad_b200.kernels")
S = importlib.import_module("honee-4aiad_b200.solver")


def _dev():
    import torch
    return torch.device("cuda:0")


def test_channel_operators_match_oracle():
    import torch
    G, mesh, basis, ch, q, idx = channel_case()
    ctx = ch.newt_ctx
    ctx.dt, ctx.ijacobian_time_shift = 5e-6, 2e5
    qd = q * 1e-3 * np.random.default_rng(0).uniform(-1, 1, q.shape)
    v_ref, jd_ref, qdata, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    op = K.ElemOp(mesh, basis)
    cb = prob.context_bytes(ctx)
    tq, tqd, tqdata = (torch.from_numpy(a).to(_dev()) for a in (q, qd, qdata))
    v = torch.zeros_like(tq)
    jd = torch.zeros(jd_ref.size, dtype=torch.float64, device=_dev())
    op.ifunction(cb, tq, tqd, tqdata, v, jac_data=jd)
    assert rel_l2(v.cpu().numpy(), v_ref) < 1e-12
    dq = q * 1e-4 * np.random.default_rng(1).normal(size=q.shape)
    jv = torch.zeros_like(tq)
    op.ijacobian(cb, tqdata, jd, torch.from_numpy(dq).to(_dev()), jv)
    assert rel_l2(jv.cpu().numpy(), O.apply_ijacobian(m, cb, dq, qdata, jd_ref)) < 1e-12


@pytest.mark.parametrize("golden,fp32,pc", [("channel_be5.npz", 0, 1), ("channel_be5.npz", 1, 1), ("channel_be5.npz", 0, 2), ("channel_be5.npz", 1, 2),
                                             ("channel_prim_be5.npz", 0, 2), ("channel_prim_be5.npz", 1, 2)])
def test_channel_run_reproduces_reference(fp32, pc, golden):
    """Conservative ("Channel") and primitive ("Channel, Primitive", tests/output/channel-prim.bin) variables.  In primitive
    variables the rate term couples the five components of every node (dU/dY is a full 5 x 5 block), so point Jacobi leaves
    GMRES stagnating (10000 iterations per Newton step without reaching rtol 1e-5); the point-block Jacobi (-pc_type
    vpbjacobi) inverts that coupling and converges in 2 Newton / 14 GMRES iterations per step."""
    import torch
    G, mesh, basis, ch, q, idx = channel_case(golden)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    dt = float(G["dt"])
    ts = S.TimeStepper(op, prob.context_bytes(ch.newt_ctx), qdata, dt=dt, bdf_order=1, newton_rtol=1e-8, jacobian_fp32=fp32, pc_jacobi=pc)
    ts.set_essential(idx)
    tq = torch.from_numpy(q).to(_dev())
    ts.set_state(tq, 0.0)
    for _ in range(int(G["steps"])):
        st = ts.step()
        assert st.converged_reason == 1, st
    out = torch.empty_like(tq)
    assert abs(ts.get_state(out) - float(G["final_time"])) < 1e-18
    qf = out.cpu().numpy()
    assert np.all(qf[idx] == 0.0)
    assert free_state_error(qf, idx, G) <= float(G["compare_atol"])


def test_checkpoint_and_resume_through_a_honee_file(tmp_path):
    """3 steps, a HONEE solution file (free DOFs, step, time), a fresh stepper resumed from it for 2 more steps: the same
    state as 5 uninterrupted steps (backward Euler carries no history) and as the reference's channel.bin."""
    import torch
    HF = importlib.import_module("honee-4aiad_b200.honee_file")
    G, mesh, basis, ch, q, idx = channel_case()
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    dt = float(G["dt"])

    def stepper():
        ts = S.TimeStepper(op, prob.context_bytes(ch.newt_ctx), qdata, dt=dt, bdf_order=1, newton_rtol=1e-8)
        ts.set_essential(idx)
        return ts

    ts = stepper()
    tq = torch.from_numpy(q).to(_dev())
    ts.set_state(tq, 0.0)
    for _ in range(5):
        ts.step()
    full = torch.empty_like(tq)
    ts.get_state(full)
    ts = stepper()
    ts.set_state(tq, 0.0)
    for _ in range(3):
        ts.step()
    mid = torch.empty_like(tq)
    t = ts.get_state(mid)
    path = str(tmp_path / "channel-3.bin")
    HF.write(path, HF.free_values(mid.cpu().numpy(), idx), step=3, time=t)
    f = HF.read(path)
    ts2 = stepper()
    ts2.set_state(torch.from_numpy(HF.expand(f.values, mesh.l_size, idx)).to(_dev()), f.time)
    for _ in range(2):
        ts2.step()
    out = torch.empty_like(tq)
    assert abs(ts2.get_state(out) - 5 * dt) < 1e-18
    np.testing.assert_array_equal(out.cpu().numpy(), full.cpu().numpy())
    assert free_state_error(out.cpu().numpy(), idx, G) <= float(G["compare_atol"])
