"""GPU tests of the implicit time loop around the fused operators and of the device monitors.

The time loop restates HONEE's TSBDF + Newton + GMRES + Jacobi solve (src/setupts.c:333-480).  Its parity bar is the
equations themselves: the state a step returns must satisfy the BDF residual F(t, q, alpha q + z) = 0 to the Newton
tolerance when that residual is evaluated by the CPU oracle, and the mixed-precision solve (FP32 Krylov, Jacobian data and
diagonal) must reach the same FP64 tolerance and the same state as the FP64 solve.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

from helpers import O, case, oracle_mesh, prob, rel_l2

pytestmark = pytest.mark.gpu

K = importlib.import_module("honee-4aiad_b200.kernels")
S = importlib.import_module("honee-4aiad_b200.solver")


def _dev():
    import torch
    return torch.device("cuda:0")


def _problem(n=(5, 5, 5), P=3, Q=3, dt=5e-5, state="pulse", stab=prob.STAB_SUPG, periodic=(1, 1, 1)):
    """Periodic boxes: without boundary operators a non-periodic box has an unbalanced pressure force on its faces, which
    makes the implicit step violently nonlinear at CFL-sized time steps."""
    import torch
    mesh, basis, ctx, q, _ = case(n=n, P=P, Q=Q, dt=dt, state=state, stab=stab, periodic=periodic)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    torch.cuda.synchronize()
    return mesh, basis, ctx, q, op, qdata


def _run(op, ctx, qdata, q0, steps, **opts):
    import torch
    ts = S.TimeStepper(op, prob.context_bytes(ctx), qdata, **opts)
    tq = torch.from_numpy(q0).to(_dev())
    ts.set_state(tq, 0.0)
    stats = [ts.step() for _ in range(steps)]
    out = torch.empty_like(tq)
    t = ts.get_state(out)
    torch.cuda.synchronize()
    return out.cpu().numpy(), t, stats, ts


def _oracle_bdf1_residual(mesh, basis, ctx, q1, q0, dt):
    """F(t, q1, (q1 - q0)/dt) from the CPU oracle, with the context fields the step sets."""
    ctx.dt = dt
    ctx.ijacobian_time_shift = 1.0 / dt
    ctx.time = dt
    m = oracle_mesh(mesh, basis)
    qd = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    jd = np.zeros(mesh.num_elem * 14 * basis.Q ** 3)
    return O.apply_ifunction(m, prob.context_bytes(ctx), q1, (q1 - q0) / dt, qd, jd)


@pytest.mark.parametrize("name,kw", [("pulse_P3Q3", dict()), ("modes_P4Q5", dict(n=(3, 3, 3), P=4, Q=5, state="modes")),
                                     ("pulse_open_box", dict(periodic=(0, 0, 0)))])
def test_bdf1_step_solves_the_equations_fp64_and_mixed(name, kw):
    mesh, basis, ctx, q0, op, qdata = _problem(**kw)
    dt = ctx.dt
    rtol = 1e-9
    res = {}
    for fp32 in (0, 1):
        q1, t, (st,), _ = _run(op, ctx, qdata, q0, 1, dt=dt, bdf_order=1, newton_rtol=rtol, jacobian_fp32=fp32)
        assert st.converged_reason == 1, st
        assert st.res_final <= rtol * st.res0
        assert st.newton_its >= 1 and st.ksp_its >= 1
        assert t == pytest.approx(dt)
        # the returned state satisfies the BDF1 equations when the oracle evaluates them
        r = _oracle_bdf1_residual(mesh, basis, ctx, q1, q0, dt)
        assert np.linalg.norm(r) <= 2 * rtol * st.res0, (fp32, np.linalg.norm(r) / st.res0)
        res[fp32] = (q1, st)
    (q64, s64), (q32, s32) = res[0], res[1]
    # the mixed solve converges to the same FP64 tolerance, so the two states agree to well below the step's change
    assert rel_l2(q32 - q0, q64 - q0) < 1e-6, rel_l2(q32 - q0, q64 - q0)
    assert s32.newton_its <= s64.newton_its + 2


def test_bdf2_steps_fp64_and_mixed_agree():
    mesh, basis, ctx, q0, op, qdata = _problem(n=(4, 4, 4), dt=1e-4)
    out = {}
    for fp32 in (0, 1):
        q, t, stats, ts = _run(op, ctx, qdata, q0, 4, dt=1e-4, bdf_order=2, newton_rtol=1e-10, jacobian_fp32=fp32)
        assert all(s.converged_reason == 1 for s in stats), stats
        assert t == pytest.approx(4e-4)
        c = ts.context_bytes()
        nc = prob.NewtonianContext.from_buffer_copy(c)
        assert nc.ijacobian_time_shift == pytest.approx(1.5 / 1e-4)  # BDF2 after the BDF1 start
        assert nc.time == pytest.approx(4e-4)
        out[fp32] = q
    assert rel_l2(out[1] - q0, out[0] - q0) < 1e-6


def test_gmres_without_preconditioner_and_with_short_restarts():
    mesh, basis, ctx, q0, op, qdata = _problem(n=(3, 3, 3), dt=2e-4)
    kw = dict(dt=2e-4, bdf_order=1, newton_rtol=1e-9, ksp_max_it=400)
    q_a, _, (sa,), _ = _run(op, ctx, qdata, q0, 1, pc_jacobi=0, **kw)
    q_b, _, (sb,), _ = _run(op, ctx, qdata, q0, 1, gmres_restart=12, pc_every_newton=1, **kw)
    q_c, _, (sc,), _ = _run(op, ctx, qdata, q0, 1, **kw)
    assert sa.converged_reason == 1 and sb.converged_reason == 1 and sc.converged_reason == 1, (sa, sb, sc)
    assert sa.ksp_its > sc.ksp_its  # Jacobi helps (about 2x on this case)
    assert rel_l2(q_a - q0, q_c - q0) < 1e-6 and rel_l2(q_b - q0, q_c - q0) < 1e-6


def test_invalid_options_rejected():
    mesh, basis, ctx, q0, op, qdata = _problem(n=(2, 2, 2))
    with pytest.raises(K.HbError):
        S.TimeStepper(op, prob.context_bytes(ctx), qdata, gmres_restart=40)
    with pytest.raises(K.HbError):
        S.TimeStepper(op, prob.context_bytes(ctx), qdata, bdf_order=3)


def test_monitor_ke_matches_oracle_and_golden():
    import json
    import os

    import torch
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "taylorgreen_ke_step0.json")))
    L = gold["box"][1]
    mesh = prob.box_mesh(gold["faces"], gold["P"], periodic=(1, 1, 1), hi=(L, L, L))
    basis = prob.tensor_basis(gold["P"], gold["Q"])
    tg = prob.TaylorGreenContext()
    tg.reference = prob.StatePrimitive(gold["reference_pressure"], (C.c_double * 3)(*gold["reference_velocity"]), gold["reference_temperature"])
    tg.newt_ctx = prob.newtonian_context(gold["degree"], cv=gold["cv"], cp=gold["cp"], mu=gold["mu"], k=gold["k"])
    tg.lx = tg.ly = tg.lz = L
    X = prob.node_coordinates(mesh, basis)
    qn = np.zeros((5, X.shape[1]))
    O.call_qf(O.lib().oracle_qf_ics_taylorgreen, bytes(memoryview(tg)), X.shape[1], [np.ascontiguousarray(X)], [qn])
    q = np.ascontiguousarray(qn.T.reshape(-1))
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    scratch = torch.empty(5 * mesh.num_elem, dtype=torch.float64, device=_dev())
    cb = bytes(memoryview(tg.newt_ctx))
    sums = S.monitor_ke(op, cb, torch.from_numpy(q).to(_dev()), qdata, scratch)
    ref = O.monitor_ke(oracle_mesh(mesh, basis), cb, q, O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem))
    np.testing.assert_allclose(sums, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    names = ["TotalKineticEnergy", "StrainDissipation", "DivergenceDissipation", "VolumeExpansion", "MuVorticity2"]
    for s, name in zip(sums / L ** 3, names):
        assert abs(s - gold[name]) <= max(gold["csv_rtol"] * abs(gold[name]), gold["csv_ztol"]), (name, s, gold[name])


def test_monitor_cfl_uniform_flow_on_anisotropic_box():
    import torch
    n = (4, 6, 8)
    mesh, basis, ctx, _, op, qdata = _problem(n=n, P=3, Q=4, periodic=(0, 0, 0))
    X = prob.node_coordinates(mesh, basis)
    u = np.array([10.0, -5.0, 2.0])
    qn = prob.conservative_from_primitive(ctx.gas, 101325.0 * np.ones(X.shape[1]), u[:, None] * np.ones((1, X.shape[1])), 288.0 * np.ones(X.shape[1]))
    q = np.ascontiguousarray(qn.T.reshape(-1))
    scratch = torch.empty(2 * mesh.num_elem, dtype=torch.float64, device=_dev())
    dt = 1e-3
    mn, mx = S.monitor_cfl(op, prob.context_bytes(ctx), torch.from_numpy(q).to(_dev()), qdata, dt, scratch)
    expect = dt * np.sqrt(np.sum((u * np.array(n)) ** 2))  # element size 1/n_i, metric 0.25 dXdx^T dXdx = diag(n_i^2)
    assert mn == pytest.approx(expect, rel=1e-12) and mx == pytest.approx(expect, rel=1e-12)


def test_taylor_green_driver_fp64_and_mixed_monitors_agree():
    """Short Taylor-Green run through the time-stepping driver: Newton converges every step in both precisions, the
    kinetic energy decays, and the mixed-precision monitors follow the FP64 ones."""
    NS = importlib.import_module("honee-4aiad_b200.navierstokes")
    r64 = NS.run("taylor_green", faces=4, degree=3, steps=4, cfl=1.0, mixed=False)
    r32 = NS.run("taylor_green", faces=4, degree=3, steps=4, cfl=1.0, mixed=True)
    ke = [row["TotalKineticEnergy"] for row in r64.rows]
    assert all(b < a for a, b in zip(ke, ke[1:])), ke
    assert abs(ke[0] - 0.125) < 0.01  # V0^2/8 for the Taylor-Green velocity field, up to discretisation error
    d = NS.compare(r64, r32)
    assert d["TotalKineticEnergy"] < 1e-8 and d["StrainDissipation"] < 1e-6, d
    assert r64.rows[-1]["maxcfl"] > 0


@pytest.mark.parametrize("fp32", [0, 1])
def test_cgs_refinement_gives_the_same_step(fp32):
    mesh, basis, ctx, q0, op, qdata = _problem(n=(3, 3, 3), dt=1e-4)
    kw = dict(dt=1e-4, bdf_order=1, newton_rtol=1e-9, jacobian_fp32=fp32)
    qa, _, (sa,), _ = _run(op, ctx, qdata, q0, 1, cgs_refine=0, **kw)
    qb, _, (sb,), _ = _run(op, ctx, qdata, q0, 1, cgs_refine=1, **kw)
    assert sa.converged_reason == 1 and sb.converged_reason == 1
    assert rel_l2(qa - q0, qb - q0) < 1e-6


def test_matrix_free_jacobian_newton_reaches_the_same_state():
    mesh, basis, ctx, q0, op, qdata = _problem(n=(3, 3, 3), dt=1e-4)
    kw = dict(dt=1e-4, bdf_order=1, newton_rtol=1e-9)
    qa, _, (sa,), _ = _run(op, ctx, qdata, q0, 1, **kw)
    qb, _, (sb,), _ = _run(op, ctx, qdata, q0, 1, jfnk=1, **kw)
    assert sa.converged_reason == 1 and sb.converged_reason == 1, (sa, sb)
    assert rel_l2(qb - q0, qa - q0) < 1e-6
    with pytest.raises(K.HbError):
        S.TimeStepper(op, prob.context_bytes(ctx), qdata, jfnk=1, jacobian_fp32=1)


@pytest.mark.parametrize("P,Q,n", [(2, 2, (3, 2, 2)), (4, 5, (2, 2, 1)), (6, 7, (2, 1, 1)), (8, 8, (1, 1, 2))])
def test_monitors_tabulate_every_basis_size(P, Q, n):
    """The monitors tabulate q and its gradient by sum factorisation in shared memory sized from P and Q (205 KB at the
    largest basis the library accepts, P = Q = 8): the kinetic-energy sums equal the oracle's direct evaluation to 1e-12,
    and the CFL monitor of a uniform flow is exact, at the smallest, the benchmarked and the largest bases."""
    import torch
    mesh = prob.box_mesh(n, P)
    basis = prob.tensor_basis(P, Q)
    ctx = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)
    cb = prob.context_bytes(ctx)
    q = prob.multimode_state(mesh, basis, ctx.gas, seed=P)
    op = K.ElemOp(mesh, basis)
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev()), qdata)
    scratch = torch.empty(5 * mesh.num_elem, dtype=torch.float64, device=_dev())
    sums = S.monitor_ke(op, cb, torch.from_numpy(q).to(_dev()), qdata, scratch)
    ref = O.monitor_ke(oracle_mesh(mesh, basis), cb, q, O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem))
    np.testing.assert_allclose(sums, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    X = prob.node_coordinates(mesh, basis)
    u = np.array([10.0, -5.0, 2.0])
    qn = prob.conservative_from_primitive(ctx.gas, 101325.0 * np.ones(X.shape[1]), u[:, None] * np.ones((1, X.shape[1])), 288.0 * np.ones(X.shape[1]))
    mn, mx = S.monitor_cfl(op, cb, torch.from_numpy(np.ascontiguousarray(qn.T.reshape(-1))).to(_dev()), qdata, 1e-3, scratch)
    expect = 1e-3 * np.sqrt(np.sum((u * np.array(n)) ** 2))
    assert mn == pytest.approx(expect, rel=1e-12) and mx == pytest.approx(expect, rel=1e-12)
