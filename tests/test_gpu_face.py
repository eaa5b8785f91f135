"""GPU tests of the free-stream boundary operator (face geometric factors, HLL/HLLC residual and Jacobian) against the
CPU oracle (oracle/face_oracle.py, pinned to the reference QFunctions by tests/test_face_oracle.py): FP64, 1e-12."""
import importlib
import os
import sys

import numpy as np
import pytest

from helpers import case, prob, rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import face_oracle as FO  # noqa: E402

K = importlib.import_module("honee-4aiad_b200.kernels")


@pytest.mark.parametrize("P,Q,flux", [(3, 3, 1), (4, 5, 1), (3, 4, 0)])
def test_freestream_residual_and_jacobian_match_oracle(P, Q, flux):
    import torch
    mesh, basis, ctx, q, _ = case(n=(2, 3, 2), P=P, Q=Q, state="pulse")
    off, xn, names = prob.box_faces(mesh, basis)
    fop = K.FaceOp(off, mesh.l_size, basis, xn)
    qd_ref = FO.face_qdata(basis.interp1d, basis.grad1d, basis.qweight1d, P, Q, xn)
    np.testing.assert_allclose(fop.qdata.cpu().numpy().reshape(qd_ref.shape), qd_ref, rtol=1e-13, atol=1e-14 * np.abs(qd_ref).max())
    # exterior state moving at an angle through the box, so faces see inflow and outflow
    u_inf = np.array([60.0, -25.0, 10.0])
    cb = prob.freestream_context(ctx, 101325.0 * 1.02, u_inf, 290.0)
    gas = ctx.gas
    rho = 101325.0 * 1.02 / ((gas.cp - gas.cv) * 290.0)
    U = np.array([rho, *(rho * u_inf), rho * (gas.cv * 290.0 + 0.5 * u_inf @ u_inf)])
    Y = np.array([101325.0 * 1.02, *u_inf, 290.0])
    tq = torch.from_numpy(q).to("cuda:0")
    v = torch.zeros_like(tq)
    fop.freestream(cb, tq, v, flux_type=flux)
    ref = FO.freestream_apply(off, basis.interp1d, P, Q, qd_ref, q, U, Y, gas.cv, gas.cp, hllc=flux == 1)
    assert rel_l2(v.cpu().numpy(), ref) < 1e-12
    jac = fop.jac.cpu().numpy().reshape(len(names), 5, Q * Q)
    dq = q * 1e-3 * np.random.default_rng(2).uniform(-1, 1, q.shape)
    dv = torch.zeros_like(tq)
    fop.freestream_jacobian(cb, torch.from_numpy(dq).to("cuda:0"), dv, flux_type=flux)
    dref = FO.freestream_apply(off, basis.interp1d, P, Q, qd_ref, q, U, Y, gas.cv, gas.cp, hllc=flux == 1, dq=dq, jac=jac)
    assert rel_l2(dv.cpu().numpy(), dref) < 1e-11
    # the tangent is the derivative of the residual (away from branch switches): finite differences of the GPU residual
    eps = 1e-6
    vp, vm = torch.zeros_like(tq), torch.zeros_like(tq)
    fop.freestream(cb, torch.from_numpy(q + eps * dq).to("cuda:0"), vp, flux_type=flux)
    fop.freestream(cb, torch.from_numpy(q - eps * dq).to("cuda:0"), vm, flux_type=flux)
    fd = (vp - vm).cpu().numpy() / (2 * eps)
    assert rel_l2(dv.cpu().numpy(), fd) < 1e-5


@pytest.mark.parametrize("fp32", [0, 1])
def test_gaussian_pulse_with_freestream_faces_ten_bdf2_steps(fp32):
    """The small configuration: Gaussian pulse, 8^3 elements, degree 2 (P=3, Q=3), SUPG, free-stream faces on all sides,
    10 BDF2 steps at dt = 1e-5.  Every step converges, and the final state satisfies the BDF2 equations (volume plus
    boundary residual) when the CPU oracle evaluates them."""
    import torch
    S = importlib.import_module("honee-4aiad_b200.solver")
    from helpers import O, oracle_mesh
    dt = 1e-5
    mesh, basis, ctx, q0, _ = case(n=(8, 8, 8), P=3, Q=3, state="pulse", dt=dt)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to("cuda:0")
    qdata = torch.zeros(mesh.num_elem * 10 * 27, dtype=torch.float64, device="cuda:0")
    op.setup_qdata(x, qdata)
    off, xn, names = prob.box_faces(mesh, basis)
    fop = K.FaceOp(off, mesh.l_size, basis, xn)
    cb_face = prob.freestream_context(ctx, 101325.0, (10.0, 0.0, 0.0), 288.0)
    ts = S.TimeStepper(op, prob.context_bytes(ctx), qdata, dt=dt, bdf_order=2, newton_rtol=1e-9, jacobian_fp32=fp32)
    ts.set_freestream(fop, cb_face, flux_type=1)
    tq = torch.from_numpy(q0).to("cuda:0")
    ts.set_state(tq, 0.0)
    states = [q0]
    for k in range(10):
        st = ts.step()
        assert st.converged_reason == 1, (k, st)
        out = torch.empty_like(tq)
        ts.get_state(out)
        states.append(out.cpu().numpy())
    q2, q1, qn = states[-3], states[-2], states[-1]
    qdot = (3 * qn - 4 * q1 + q2) / (2 * dt)
    ctx.dt, ctx.ijacobian_time_shift, ctx.time = dt, 1.5 / dt, 10 * dt
    m = oracle_mesh(mesh, basis)
    qd_o = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    jd = np.zeros(mesh.num_elem * 14 * 27)
    r_vol = O.apply_ifunction(m, prob.context_bytes(ctx), qn, qdot, qd_o, jd)
    gas = ctx.gas
    rho = 101325.0 / ((gas.cp - gas.cv) * 288.0)
    U = np.array([rho, rho * 10.0, 0, 0, rho * (gas.cv * 288.0 + 50.0)])
    Y = np.array([101325.0, 10.0, 0, 0, 288.0])
    qd_f = FO.face_qdata(basis.interp1d, basis.grad1d, basis.qweight1d, 3, 3, xn)
    r_face = FO.freestream_apply(off, basis.interp1d, 3, 3, qd_f, qn, U, Y, gas.cv, gas.cp, hllc=True)
    r = r_vol + r_face
    # scale: the residual of the step's initial guess (q_n itself)
    r_first = O.apply_ifunction(m, prob.context_bytes(ctx), q1, (3 * q1 - 4 * q1 + q2) / (2 * dt), qd_o, jd) + \
        FO.freestream_apply(off, basis.interp1d, 3, 3, qd_f, q1, U, Y, gas.cv, gas.cp, hllc=True)
    assert np.linalg.norm(r) <= 2e-9 * np.linalg.norm(r_first), np.linalg.norm(r) / np.linalg.norm(r_first)
