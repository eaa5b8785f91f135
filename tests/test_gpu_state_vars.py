"""GPU parity of the fused operators in primitive and entropy state variables (IFunction_Newtonian_Prim/_Entropy and
IJacobian_Newtonian_Prim/_Entropy, qfunctions/newtonian.h:263-269, 317-323; the state algebra of newtonian_state.h:64-423)
against the oracle's QFunctions of the same state variable (oracle/honee_oracle.c, pinned bit for bit to the reference's).

Tolerances: residual, stored Jacobian data, Jacobian action, diagonal and point blocks 1e-12 relative L2 in FP64, or 10x the
change the oracle itself shows when the state is perturbed by one ulp, whichever is larger.  That floor matters for entropy
variables only: pressure and density are rebuilt through exp(log(...)) of arguments of size ~10, so the last-bit differences
between the device's and the C library's exp/log reach the residual, amplified where its flux terms nearly cancel (a
periodic multi-mode state).  The FP32 Jacobian action: 1e-6 for primitive variables; 2e-5 for entropy variables (the
same rebuild in FP32: ~10 FP32 ulp in pressure and density)."""
import importlib

import numpy as np
import pytest

from helpers import O, case, prob, rel_l2

import face_oracle as FO  # noqa: E402
import filter_oracle as FIL  # noqa: E402

pytestmark = pytest.mark.gpu

K = importlib.import_module("honee-4aiad_b200.kernels")
NAMES = {prob.STATEVAR_PRIMITIVE: "prim", prob.STATEVAR_ENTROPY: "entropy"}

CASES = {
    "prim_P3Q3_supg": (prob.STATEVAR_PRIMITIVE, dict(n=(3, 3, 2), P=3, Q=3)),
    "prim_P2Q4_none_gravity": (prob.STATEVAR_PRIMITIVE, dict(n=(3, 2, 2), P=2, Q=4, stab=prob.STAB_NONE, g=(0.0, -9.81, 0.0))),
    "prim_P4Q5_su_idl_modes": (prob.STATEVAR_PRIMITIVE, dict(n=(2, 2, 2), P=4, Q=5, stab=prob.STAB_SU, idl=(2e-3, 0.2, 0.5, 101000.0),
                                                              state="modes")),
    "entropy_P3Q4_supg": (prob.STATEVAR_ENTROPY, dict(n=(3, 2, 2), P=3, Q=4)),
    "entropy_P2Q3_none_idl": (prob.STATEVAR_ENTROPY, dict(n=(3, 3, 2), P=2, Q=3, stab=prob.STAB_NONE, idl=(2e-3, 0.2, 0.5, 101000.0))),
    "entropy_P4Q5_supg_modes_periodic": (prob.STATEVAR_ENTROPY, dict(n=(2, 2, 2), P=4, Q=5, periodic=(1, 1, 1), state="modes")),
}


def _dev():
    import torch
    return torch.device("cuda:0")


def sv_case(sv, **kw):
    mesh, basis, ctx, q, _ = case(**kw)
    ctx.state_var = sv
    qv = prob.state_to_q(ctx.gas, q, sv)
    qdv = qv * 1e-3 * np.random.default_rng(7).uniform(-1, 1, qv.shape)
    return mesh, basis, ctx, qv, qdv


def _oracle_mesh(mesh, basis):
    return O.Mesh(mesh.num_elem, basis.P, basis.Q, mesh.offsets, basis.interp1d, basis.grad1d, basis.qweight1d, colors=mesh.colors)


def _oracle_all(mesh, basis, ctx, q, qd, dq):
    """Residual, stored data, Jacobian action, diagonal and point blocks of the oracle for the state q."""
    tag = NAMES[ctx.state_var]
    cb = prob.context_bytes(ctx)
    m = _oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    njd = 15 if ctx.idl_enable else 14
    jd = np.zeros(mesh.num_elem * njd * basis.Q ** 3)
    xq = O.coords_at_qpts(mesh.num_elem, basis.Q, mesh.x_elem)
    v = O.apply_ifunction(m, cb, q, qd, qdata, jd, num_jd=njd, x_q=xq, qf_name=f"oracle_qf_ifunction_{tag}")
    jv = O.apply_ijacobian(m, cb, dq, qdata, jd, num_jd=njd, qf_name=f"oracle_qf_ijacobian_{tag}")
    d = O.assemble_diagonal(m, cb, qdata, jd, mesh.l_size, num_jd=njd, qf_name=f"oracle_qf_ijacobian_{tag}")
    pb = O.assemble_point_block(m, cb, qdata, jd, mesh.l_size, num_jd=njd, qf_name=f"oracle_qf_ijacobian_{tag}")
    return dict(v=v, jd=jd, jv=jv, d=d, pb=pb, qdata=qdata)


@pytest.mark.parametrize("name", list(CASES))
def test_operators_match_oracle(name):
    import torch
    sv, kw = CASES[name]
    mesh, basis, ctx, q, qd = sv_case(sv, **kw)
    cb = prob.context_bytes(ctx)
    dq = q * 1e-4 * np.random.default_rng(1).normal(size=q.shape)
    ref = _oracle_all(mesh, basis, ctx, q, qd, dq)
    # the oracle's own sensitivity to a one-ulp perturbation of the state
    q1 = q * (1 + np.finfo(np.float64).eps * np.random.default_rng(3).uniform(-1, 1, q.shape))
    ref1 = _oracle_all(mesh, basis, ctx, q1, qd, dq)
    bound = {k: max(1e-12, 10 * rel_l2(ref1[k], ref[k])) for k in ("v", "jd", "jv", "d", "pb")}
    op = K.ElemOp(mesh, basis)
    if ctx.idl_enable:
        op.set_vertex_coords(np.ascontiguousarray(mesh.x_elem))
    dev = _dev()
    tq, tqd, tqdata = (torch.from_numpy(a).to(dev) for a in (q, qd, ref["qdata"]))
    v = torch.zeros_like(tq)
    jd = torch.zeros(ref["jd"].size, dtype=torch.float64, device=dev)
    op.ifunction(cb, tq, tqd, tqdata, v, jac_data=jd)
    assert rel_l2(v.cpu().numpy(), ref["v"]) < bound["v"], bound
    assert rel_l2(jd.cpu().numpy(), ref["jd"]) < bound["jd"], bound
    # Jacobian action, FP64 and FP32
    jv = torch.zeros_like(tq)
    tdq = torch.from_numpy(dq).to(dev)
    op.ijacobian(cb, tqdata, jd, tdq, jv)
    assert rel_l2(jv.cpu().numpy(), ref["jv"]) < bound["jv"], bound
    jv32 = torch.zeros(q.size, dtype=torch.float32, device=dev)
    op.ijacobian(cb, tqdata, jd.float(), tdq.float(), jv32, fp32=True)
    assert rel_l2(jv32.double().cpu().numpy(), ref["jv"]) < (2e-5 if sv == prob.STATEVAR_ENTROPY else 1e-6)
    # diagonal and point blocks
    d = torch.zeros_like(tq)
    op.diagonal(cb, tqdata, jd, d)
    assert rel_l2(d.cpu().numpy(), ref["d"]) < bound["d"], bound
    pb = torch.zeros(5 * mesh.l_size, dtype=torch.float64, device=dev)
    op.point_block_diagonal(cb, tqdata, jd, pb)
    assert rel_l2(pb.cpu().numpy(), ref["pb"]) < bound["pb"], bound


def test_state_variable_outside_the_compiled_bases_is_refused():
    import torch
    mesh, basis, ctx, q, qd = sv_case(prob.STATEVAR_PRIMITIVE, n=(2, 1, 1), P=5, Q=6)
    op = K.ElemOp(mesh, basis)
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    tq = torch.from_numpy(q).to(_dev())
    with pytest.raises(K.HbError):
        op.ifunction(prob.context_bytes(ctx), tq, tq, qdata, torch.zeros_like(tq))


@pytest.mark.parametrize("resource", ["/gpu/b200", "/gpu/b200/mixed"])
def test_primitive_operators_through_the_ceed_api(resource):
    """HONEE's operator set-up with -state_var primitive (IFunction_Newtonian_Prim / IJacobian_Newtonian_Prim) through the
    libCEED API: residual and Jacobi diagonal equal the oracle's."""
    ce = importlib.import_module("honee-4aiad_b200.ceed")
    hon = importlib.import_module("honee-4aiad_b200.honee")
    mesh, basis, ctx, q, qd = sv_case(prob.STATEVAR_PRIMITIVE, n=(3, 2, 2), P=3, Q=4)
    ceed = ce.Ceed(resource)
    ops = hon.NewtonianOperators(ceed, mesh, basis, ctx)
    qv = ce.Vector(ceed, mesh.l_size)
    qv.set_array_host(q)
    ops.q_dot.set_array_host(qd)
    out = ce.Vector(ceed, mesh.l_size)
    ops.ifunction(qv, ops.q_dot, out)
    cb = prob.context_bytes(ctx)
    m = _oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    jd_ref = np.zeros(mesh.num_elem * 14 * basis.Q ** 3)
    xq = O.coords_at_qpts(mesh.num_elem, basis.Q, mesh.x_elem)
    v_ref = O.apply_ifunction(m, cb, q, qd, qdata, jd_ref, x_q=xq, qf_name="oracle_qf_ifunction_prim")
    assert rel_l2(out.to_numpy(), v_ref) < 1e-12
    d = ce.Vector(ceed, mesh.l_size)
    ops.diagonal(d)
    d_ref = O.assemble_diagonal(m, cb, qdata, jd_ref, mesh.l_size, qf_name="oracle_qf_ijacobian_prim")
    assert rel_l2(d.to_numpy(), d_ref) < (1e-12 if resource == "/gpu/b200" else 2e-6)


@pytest.mark.parametrize("sv,hllc", [(prob.STATEVAR_PRIMITIVE, True), (prob.STATEVAR_ENTROPY, False)])
def test_freestream_faces_match_oracle(sv, hllc):
    """Free-stream face operator in primitive / entropy variables (Freestream_Prim_*, Freestream_Entropy_*): residual,
    stored face state, tangent and point blocks against oracle/face_oracle.py with the same state variable."""
    import torch
    mesh, basis, ctx, q, qd = sv_case(sv, n=(2, 3, 2), P=3, Q=4)
    off, xn, names = prob.box_faces(mesh, basis)
    fop = K.FaceOp(off, mesh.l_size, basis, xn)
    gas = ctx.gas
    P_inf, u_inf, T_inf = 101325.0 * 1.02, np.array([60.0, -25.0, 10.0]), 290.0
    cb = prob.freestream_context(ctx, P_inf, u_inf, T_inf)
    rho = P_inf / ((gas.cp - gas.cv) * T_inf)
    U = np.array([rho, *(rho * u_inf), rho * (gas.cv * T_inf + 0.5 * u_inf @ u_inf)])
    Y = np.array([P_inf, *u_inf, T_inf])
    flux_type = 1 if hllc else 0
    dev = _dev()
    tq = torch.from_numpy(q).to(dev)
    v = torch.zeros_like(tq)
    fop.freestream(cb, tq, v, flux_type=flux_type)
    qd_sur = FO.face_qdata(basis.interp1d, basis.grad1d, basis.qweight1d, basis.P, basis.Q, xn)
    ref = FO.freestream_apply(off, basis.interp1d, basis.P, basis.Q, qd_sur, q, U, Y, gas.cv, gas.cp, hllc=hllc, l_size=mesh.l_size, sv=sv)
    assert rel_l2(v.cpu().numpy(), ref) < 1e-12
    jac = fop.jac.cpu().numpy().reshape(len(names), 5, basis.Q ** 2)
    B = np.asarray(basis.interp1d).reshape(basis.Q, basis.P)
    Bq = np.einsum("jb,ia->jiba", B, B).reshape(basis.Q ** 2, basis.P ** 2)
    jac_ref = np.stack([(Bq @ q.reshape(-1, 5)[off[f] // 5]).T for f in range(len(names))])
    assert rel_l2(jac, jac_ref) < 1e-14
    dq = q * 1e-4 * np.random.default_rng(2).normal(size=q.shape)
    jv = torch.zeros_like(tq)
    fop.freestream_jacobian(cb, torch.from_numpy(dq).to(dev), jv, flux_type=flux_type)
    jv_ref = FO.freestream_apply(off, basis.interp1d, basis.P, basis.Q, qd_sur, q, U, Y, gas.cv, gas.cp, hllc=hllc, dq=dq, jac=jac,
                                 l_size=mesh.l_size, sv=sv)
    assert rel_l2(jv.cpu().numpy(), jv_ref) < 1e-12
    pb = torch.zeros(5 * mesh.l_size, dtype=torch.float64, device=dev)
    fop.freestream_point_block(cb, pb, flux_type=flux_type)
    pb_ref = FO.freestream_point_block(off, basis.interp1d, basis.P, basis.Q, qd_sur, jac, U, Y, gas.cv, gas.cp, hllc=hllc, l_size=mesh.l_size,
                                       sv=sv)
    assert rel_l2(pb.cpu().numpy(), pb_ref) < 1e-12


def test_bdf2_with_freestream_faces_in_primitive_variables():
    """The small configuration's box with free-stream faces, 4 BDF2 steps in conservative and in primitive variables
    (point-block Jacobi).  Every step converges; in primitive variables the mixed-precision run reaches the FP64 run's
    state to the Newton tolerance.  Conservative and primitive runs are different discretisations (a polynomial in U is
    not one in Y), so they agree only to discretisation error: here 1.4e-3 of the state change over the 4 steps."""
    import torch
    S = importlib.import_module("honee-4aiad_b200.solver")
    mesh, basis, ctx, q, _ = case(n=(4, 4, 4), P=3, Q=3, dt=1e-5)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    off, xn, _ = prob.box_faces(mesh, basis)
    fop = K.FaceOp(off, mesh.l_size, basis, xn)
    finals = {}
    for sv in (prob.STATEVAR_CONSERVATIVE, prob.STATEVAR_PRIMITIVE):
        for fp32 in (0, 1):
            ctx.state_var = sv
            cb = prob.freestream_context(ctx, 101325.0, np.array([10.0, 0.0, 0.0]), 288.0)
            ts = S.TimeStepper(op, prob.context_bytes(ctx), qdata, dt=1e-5, bdf_order=2, newton_rtol=1e-10, jacobian_fp32=fp32, pc_jacobi=2)
            ts.set_freestream(fop, cb, flux_type=1)
            tq = torch.from_numpy(prob.state_to_q(ctx.gas, q, sv)).to(_dev())
            ts.set_state(tq, 0.0)
            stats = [ts.step() for _ in range(4)]
            assert all(s.converged_reason == 1 for s in stats), (sv, fp32, stats)
            out = torch.empty_like(tq)
            ts.get_state(out)
            finals[(sv, fp32)] = out.cpu().numpy()
    y0 = prob.state_to_q(ctx.gas, q, prob.STATEVAR_PRIMITIVE)
    prim64, prim32 = finals[(prob.STATEVAR_PRIMITIVE, 0)], finals[(prob.STATEVAR_PRIMITIVE, 1)]
    assert rel_l2(prim32 - y0, prim64 - y0) < 1e-6
    cons_as_prim = prob.state_to_q(ctx.gas, finals[(prob.STATEVAR_CONSERVATIVE, 0)], prob.STATEVAR_PRIMITIVE)
    assert rel_l2(prim64 - y0, cons_as_prim - y0) < 1e-2


def test_monitors_read_the_state_variable():
    """MonitorTotalKineticEnergy / MonitorCFL in all three variables (qfunctions/monitor_totalkineticenergy.h:41-51,
    monitor_cfl.h:48-58).  A uniform-pressure, uniform-temperature shear u = (a + b y, 0, 0) is exactly quadratic in each
    representation, so at degree 2 every monitor integral is exact: kinetic energy 1/2 rho int (a + b y)^2, strain
    dissipation -mu b^2 V, vorticity mu b^2 V, divergence terms 0; the CFL extremes are those of |u| on the quadrature grid."""
    import torch
    S = importlib.import_module("honee-4aiad_b200.solver")
    n, P, Q = (2, 3, 2), 3, 4
    mesh = prob.box_mesh(n, P, hi=(1.0, 2.0, 0.5))
    basis = prob.tensor_basis(P, Q)
    ctx = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-2)
    X = prob.node_coordinates(mesh, basis)
    a, b, Pr, T = 3.0, 4.0, 1.0e5, 300.0
    u = np.stack([a + b * X[1], 0 * X[1], 0 * X[1]])
    q_cons = prob.conservative_from_primitive(ctx.gas, Pr + 0 * X[1], u, T + 0 * X[1]).T.reshape(-1)
    rho = Pr / ((ctx.gas.cp - ctx.gas.cv) * T)
    V = 1.0 * 2.0 * 0.5
    ke = 0.5 * rho * 1.0 * 0.5 * ((a + 2 * b) ** 3 - a ** 3) / (3 * b)
    expect = np.array([ke, -ctx.gas.mu * b * b * V, 0.0, 0.0, ctx.gas.mu * b * b * V])
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    scratch = torch.zeros(5 * mesh.num_elem, dtype=torch.float64, device=_dev())
    cfl = {}
    for sv in (prob.STATEVAR_CONSERVATIVE, prob.STATEVAR_PRIMITIVE, prob.STATEVAR_ENTROPY):
        ctx.state_var = sv
        cb = prob.context_bytes(ctx)
        tq = torch.from_numpy(prob.state_to_q(ctx.gas, q_cons, sv)).to(_dev())
        sums = S.monitor_ke(op, cb, tq, qdata, scratch)
        np.testing.assert_allclose(sums[[0, 1, 4]], expect[[0, 1, 4]], rtol=1e-11)
        assert abs(sums[2]) < 1e-10 * abs(expect[1]) and abs(sums[3]) < 1e-10 * Pr * V
        cfl[sv] = S.monitor_cfl(op, cb, tq, qdata, 1e-3, scratch)
    for sv in (prob.STATEVAR_PRIMITIVE, prob.STATEVAR_ENTROPY):
        np.testing.assert_allclose(cfl[sv], cfl[prob.STATEVAR_CONSERVATIVE], rtol=1e-12)
    ctx.state_var = 9
    with pytest.raises(K.HbError):
        S.monitor_ke(op, prob.context_bytes(ctx), tq, qdata, scratch)


@pytest.mark.parametrize("sv", [prob.STATEVAR_PRIMITIVE, prob.STATEVAR_ENTROPY])
def test_filter_rhs_and_filtered_state_in_other_variables(sv):
    """The differential filter's right-hand side from a primitive / entropy state (DifferentialFilter_RHS_Prim/_Entropy)
    against the oracle, and the state rebuilt from filtered (P, u, T) fields in that variable."""
    import torch
    F = importlib.import_module("honee-4aiad_b200.filter")
    mesh, basis, ctx, q, _ = sv_case(sv, n=(3, 3, 2), P=3, Q=4, state="modes")
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    filt = F.DifferentialFilter(op, qdata, prob.context_bytes(ctx), grid_based_width=True, width_scaling=(1.0, 1.0, 1.0), kernel_scaling=0.1)
    b = torch.empty(mesh.num_nodes * 11, dtype=torch.float64, device=_dev())
    filt.rhs(torch.from_numpy(q).to(_dev()), b)
    assert rel_l2(b.cpu().numpy(), FIL.rhs(mesh, basis, qdata.cpu().numpy(), q, ctx.gas, sv=sv)) < 1e-12
    rng = np.random.default_rng(9)
    n = mesh.num_nodes
    Pn, Tn, un = 101325 * (1 + 0.01 * rng.uniform(-1, 1, n)), 288 * (1 + 0.01 * rng.uniform(-1, 1, n)), rng.uniform(-20, 20, (3, n))
    fields = np.zeros((n, 11))
    fields[:, 0], fields[:, 1:4], fields[:, 4] = Pn, un.T, Tn
    out = torch.empty(5 * n, dtype=torch.float64, device=_dev())
    filt.conservative(torch.from_numpy(fields.reshape(-1)).to(_dev()), out)
    expect = prob.state_to_q(ctx.gas, prob.conservative_from_primitive(ctx.gas, Pn, un, Tn).T.reshape(-1), sv)
    assert rel_l2(out.cpu().numpy(), expect) < 1e-14


@pytest.mark.parametrize("sv", [prob.STATEVAR_PRIMITIVE, prob.STATEVAR_ENTROPY])
def test_fused_closure_in_other_state_variables(sv):
    """The learned closure fused into the residual with the state in primitive / entropy variables (the reference's
    data-driven SGS runs use -state_var primitive): its residual contribution against the oracle's, which rebuilds
    density, velocity and velocity gradient through StateFromQ and its tangent; 1e-5 (FP32 network)."""
    import math
    import torch
    SG = importlib.import_module("honee-4aiad_b200.sgs")
    import sgs_oracle as SO
    import os
    L = 2 * math.pi
    mesh = prob.box_mesh((3, 3, 3), 3, periodic=(1, 1, 1), hi=(L, L, L))
    basis = prob.tensor_basis(3, 4)
    tg = prob.taylor_green_context(2)
    tg.u[0], tg.u[1], tg.u[2] = 0.2, 0.1, 0.3
    q = prob.taylor_green_state(mesh, basis, tg)
    ctx = tg.newt_ctx
    ctx.dt, ctx.ijacobian_time_shift = 0.01, 150.0
    ctx.state_var = sv
    qv = prob.state_to_q(ctx.gas, q, sv)
    cb = prob.context_bytes(ctx)
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "sgs_points.npz"))
    d, w = SG.desc(20, 0, 0.0, g["bounds"]), g["weights"].astype(np.float32)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    tq = torch.from_numpy(qv).to(_dev())
    tqd = torch.zeros_like(tq)
    v0, v1 = torch.empty_like(tq), torch.empty_like(tq)
    op.ifunction(cb, tq, tqd, qdata, v0)
    op.ifunction_sgs(cb, tq, tqd, qdata, v1, d, w)
    torch.cuda.synchronize()
    got = (v1 - v0).cpu().numpy()
    ref = SO.residual_contribution(mesh, basis, qdata.cpu().numpy(), qv, ctx.gas, w, d.hidden1, d.hidden2, np.array(d.out_bounds[:]), sv=sv)
    assert np.linalg.norm(ref) > 0
    assert rel_l2(got, ref) < 1e-5, rel_l2(got, ref)
