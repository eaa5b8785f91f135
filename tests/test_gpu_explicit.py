"""GPU tests of the explicit path (hb_mass_*, hb_explicit_*): the fused mass operator and its diagonal against the CPU
oracle (1e-14), the right-hand side M^-1 RHS(q) with lumped and GMRES mass solves (1e-12), other RK tableaux against the
oracle's loop, and the reference's own explicit run (examples/navierstokes.c:222) reproduced on the GPU: kinetic-energy rows
of tests/output/taylorgreen_totalke.csv and the final state tests/output/taylor-green.bin, through
tests/golden/taylorgreen_rk4.npz."""
import importlib
import os

import numpy as np
import pytest

from helpers import O, case, oracle_mesh, prob, rel_l2
from test_explicit_oracle import GOLD, ke_rows_match, state_matches, taylor_green_rk4_case

import explicit_oracle as X  # noqa: E402

pytestmark = pytest.mark.gpu

K = importlib.import_module("honee-4aiad_b200.kernels")
S = importlib.import_module("honee-4aiad_b200.solver")


def _dev():
    import torch
    return torch.device("cuda:0")


def _setup(mesh, basis):
    import torch
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    torch.cuda.synchronize()
    return op, qdata


@pytest.mark.parametrize("n,P,Q,periodic", [((3, 2, 2), 3, 3, (0, 0, 0)), ((2, 3, 2), 4, 5, (1, 0, 1)), ((2, 2, 2), 5, 6, (1, 1, 1)),
                                           ((2, 2, 1), 6, 7, (0, 0, 0))])
def test_mass_and_diagonal_match_oracle(n, P, Q, periodic):
    import torch
    mesh, basis, ctx, q, _ = case(n, P, Q, periodic=periodic)
    op, qdata = _setup(mesh, basis)
    m = oracle_mesh(mesh, basis)
    qd = qdata.cpu().numpy()
    u = np.random.default_rng(1).normal(size=mesh.l_size)
    v = torch.zeros(mesh.l_size, dtype=torch.float64, device=_dev())
    op.mass(qdata, torch.from_numpy(u).to(_dev()), v)
    assert rel_l2(v.cpu().numpy(), O.apply_mass(m, u, qd)) < 1e-14
    d = torch.zeros_like(v)
    op.mass_diagonal(qdata, d)
    assert rel_l2(d.cpu().numpy(), X.mass_diagonal(m, P, Q, qd, mesh.l_size)) < 1e-14
    # add mode accumulates
    op.mass(qdata, torch.from_numpy(u).to(_dev()), v, add=True)
    assert rel_l2(v.cpu().numpy(), 2 * O.apply_mass(m, u, qd)) < 1e-14


@pytest.mark.parametrize("mass_ksp,pc", [("preonly", "rowsum"), ("gmres", "diagonal"), ("gmres", "rowsum")])
def test_explicit_rhs_matches_oracle(mass_ksp, pc):
    import torch
    mesh, basis, ctx, q, _ = case((3, 3, 2), 4, 5, periodic=(1, 1, 0), g=(0.0, -9.81, 0.0))
    op, qdata = _setup(mesh, basis)
    dt = 1e-5
    ex = S.ExplicitStepper(op, prob.context_bytes(ctx), qdata, dt=dt, mass_ksp=mass_ksp, pc_jacobi=pc)
    g = torch.zeros(mesh.l_size, dtype=torch.float64, device=_dev())
    its, reason = ex.rhs(torch.from_numpy(q).to(_dev()), g, 0.0)
    assert reason == 1
    ox = X.Explicit(oracle_mesh(mesh, basis), 4, 5, prob.context_bytes(ctx), qdata.cpu().numpy(), mesh.l_size, dt=dt,
                    mass_ksp=mass_ksp, pc_jacobi=pc)
    ref = ox.rhs(q, 0.0)
    assert rel_l2(g.cpu().numpy(), ref) < 1e-12
    if mass_ksp == "gmres":
        assert its == ox.mass_its[-1]


@pytest.mark.parametrize("rk,mass_ksp", [("3bs", "preonly"), ("2a", "gmres"), ("1fe", "preonly")])
def test_other_tableaux_track_the_oracle_loop(rk, mass_ksp):
    import torch
    mesh, basis, ctx, q, _ = case((3, 3, 3), 3, 3, periodic=(1, 1, 1))
    op, qdata = _setup(mesh, basis)
    dt = 2e-6
    ex = S.ExplicitStepper(op, prob.context_bytes(ctx), qdata, dt=dt, rk_type=rk, mass_ksp=mass_ksp, pc_jacobi="diagonal")
    ex.set_state(torch.from_numpy(q).to(_dev()), 0.0)
    ox = X.Explicit(oracle_mesh(mesh, basis), 3, 3, prob.context_bytes(ctx), qdata.cpu().numpy(), mesh.l_size, dt=dt, tableau=rk,
                    mass_ksp=mass_ksp, pc_jacobi="diagonal")
    qo, t = q.copy(), 0.0
    for _ in range(3):
        st = ex.step()
        assert st.converged_reason == 1
        qo = ox.step(qo, t)
        t += dt
    out = torch.empty(mesh.l_size, dtype=torch.float64, device=_dev())
    assert abs(ex.get_state(out) - 3 * dt) < 1e-18
    assert rel_l2(out.cpu().numpy(), qo) < 1e-14
    # the change over the three steps (about 1e-6 of the state, so state round-off alone is ~1e-10 of it)
    assert rel_l2(out.cpu().numpy() - q, qo - q) < 1e-9


def test_taylor_green_rk4_reproduces_reference_run():
    """examples/navierstokes.c:222 on the GPU: TSRK4, dt 2e-3, GMRES + Jacobi-diagonal mass solves, 3 steps."""
    import torch
    G = np.load(os.path.join(GOLD, "taylorgreen_rk4.npz"))
    mesh, basis, tg, q, L = taylor_green_rk4_case()
    op, qdata = _setup(mesh, basis)
    cb = bytes(memoryview(tg.newt_ctx))
    ex = S.ExplicitStepper(op, cb, qdata, dt=float(G["dt"]), rk_type=str(G["tableau"]), mass_ksp=str(G["mass_ksp"]),
                           pc_jacobi=str(G["mass_pc_jacobi"]))
    tq = torch.from_numpy(q).to(_dev())
    ex.set_state(tq, 0.0)
    scratch = torch.zeros(5 * mesh.num_elem, dtype=torch.float64, device=_dev())
    rows = {0: S.monitor_ke(op, cb, tq, qdata, scratch) / L ** 3}
    its = []
    for step in (1, 2, 3):
        st = ex.step()
        assert st.converged_reason == 1
        its.append(st.mass_its)
        ex.get_state(tq)
        rows[step] = S.monitor_ke(op, cb, tq, qdata, scratch) / L ** 3
    ke_rows_match(rows, G)
    assert state_matches(tq.cpu().numpy(), G) < 1e-10
    assert all(4 <= i <= 4 * 29 for i in its)


def test_explicit_operators_through_the_ceed_api():
    """RHSFunction_Newtonian and Mass_5 operators built as SetupLibceed / CreateKSPMass build them, applied through the
    libCEED C API (FP64 in both resources), against the oracle; the mass diagonal through CeedOperatorLinearAssembleDiagonal."""
    ce = importlib.import_module("honee-4aiad_b200.ceed")
    hon = importlib.import_module("honee-4aiad_b200.honee")
    mesh, basis, ctx, q, _ = case((3, 2, 2), 4, 5, periodic=(1, 0, 0), idl=(2e-3, 0.2, 0.5, 101000.0), g=(0.0, -9.81, 0.0))
    m = oracle_mesh(mesh, basis)
    qd_ref = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    xq = O.coords_at_qpts(mesh.num_elem, basis.Q, mesh.x_elem)
    r_ref = O.apply_rhs(m, prob.context_bytes(ctx), q, qd_ref, xq)
    u = np.random.default_rng(2).normal(size=q.shape)
    for resource in ("/gpu/b200", "/gpu/b200/mixed"):
        ceed = ce.Ceed(resource)
        ops = hon.NewtonianOperators(ceed, mesh, basis, ctx)
        ops.add_explicit()
        qv, g = ce.Vector(ceed, mesh.l_size), ce.Vector(ceed, mesh.l_size)
        qv.set_array_host(q)
        ops.rhs(qv, g)
        assert rel_l2(g.to_numpy(), r_ref) < 1e-12
        uv, mv, dv = ce.Vector(ceed, mesh.l_size), ce.Vector(ceed, mesh.l_size), ce.Vector(ceed, mesh.l_size)
        uv.set_array_host(u)
        ops.op_mass.apply(uv, mv)
        assert rel_l2(mv.to_numpy(), O.apply_mass(m, u, qd_ref)) < 1e-14
        ops.op_mass.assemble_diagonal(dv)
        assert rel_l2(dv.to_numpy(), X.mass_diagonal(m, 4, 5, qd_ref, mesh.l_size)) < 1e-14
