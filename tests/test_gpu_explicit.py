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


@pytest.mark.parametrize("mass_ksp,pc,stab", [("preonly", "rowsum", prob.STAB_NONE), ("gmres", "diagonal", prob.STAB_SUPG),
                                             ("gmres", "rowsum", prob.STAB_NONE), ("gmres", "diagonal", prob.STAB_SU)])
def test_explicit_rhs_matches_oracle(mass_ksp, pc, stab):
    """M^-1 RHS(q) against the oracle's loop: Mass_5 (none, SU) or the SUPG-stabilized mass (SUPG) by GMRES, Mass_5 lumped.
    (The stabilized mass has row sums close to zero: lumped, the quotient amplifies their round-off, and as a Jacobi
    preconditioner they stall GMRES; its row sums are checked directly in test_stabilized_mass_row_sums_match_oracle.)"""
    import torch
    mesh, basis, ctx, q, _ = case((3, 3, 2), 4, 5, periodic=(1, 1, 0), g=(0.0, -9.81, 0.0), stab=stab)
    op, qdata = _setup(mesh, basis)
    dt = 1e-5
    ex = S.ExplicitStepper(op, prob.context_bytes(ctx), qdata, dt=dt, mass_ksp=mass_ksp, pc_jacobi=pc)
    g = torch.zeros(mesh.l_size, dtype=torch.float64, device=_dev())
    its, reason = ex.rhs(torch.from_numpy(q).to(_dev()), g, 0.0)
    assert reason == 1
    ox = X.Explicit(oracle_mesh(mesh, basis), 4, 5, prob.context_bytes(ctx), qdata.cpu().numpy(), mesh.l_size, dt=dt,
                    mass_ksp=mass_ksp, pc_jacobi=pc)
    assert ox.stab_mass == (stab == prob.STAB_SUPG)
    ref = ox.rhs(q, 0.0)
    assert rel_l2(g.cpu().numpy(), ref) < 1e-12
    if mass_ksp == "gmres":
        assert its == ox.mass_its[-1]


def test_stabilized_mass_row_sums_match_oracle():
    """The lumped stabilized mass's row sums M_stab(q) 1, entry by entry against the largest (they cancel to near zero)."""
    import torch
    mesh, basis, ctx, q, _ = case((3, 3, 2), 4, 5, periodic=(1, 1, 0))
    op, qdata = _setup(mesh, basis)
    m = oracle_mesh(mesh, basis)
    cb = prob.context_bytes(ctx)
    ones = np.ones(mesh.l_size)
    tq = torch.from_numpy(q).to(_dev())
    v = torch.zeros_like(tq)
    op.mass_stab(cb, qdata, tq, torch.from_numpy(ones).to(_dev()), v)
    ref = O.apply_mass_stab(m, cb, ones, q, qdata.cpu().numpy())
    assert np.abs(v.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


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


@pytest.mark.parametrize("stab", [prob.STAB_SUPG, prob.STAB_NONE])
def test_explicit_operators_through_the_ceed_api(stab):
    """RHSFunction_Newtonian and the mass operator (MassFunction_Newtonian for SUPG, Mass_5 otherwise) built as SetupLibceed /
    CreateKSPMass build them, applied through the libCEED C API (FP64 in both resources), against the oracle; the mass
    diagonal through CeedOperatorLinearAssembleDiagonal."""
    ce = importlib.import_module("honee-4aiad_b200.ceed")
    hon = importlib.import_module("honee-4aiad_b200.honee")
    mesh, basis, ctx, q, _ = case((3, 2, 2), 4, 5, periodic=(1, 0, 0), idl=(2e-3, 0.2, 0.5, 101000.0), g=(0.0, -9.81, 0.0), stab=stab)
    m = oracle_mesh(mesh, basis)
    qd_ref = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    xq = O.coords_at_qpts(mesh.num_elem, basis.Q, mesh.x_elem)
    cb = prob.context_bytes(ctx)
    r_ref = O.apply_rhs(m, cb, q, qd_ref, xq)
    u = np.random.default_rng(2).normal(size=q.shape)
    if stab == prob.STAB_SUPG:
        m_ref, d_ref = O.apply_mass_stab(m, cb, u, q, qd_ref), O.mass_stab_diagonal(m, cb, q, qd_ref, mesh.l_size)
    else:
        m_ref, d_ref = O.apply_mass(m, u, qd_ref), X.mass_diagonal(m, 4, 5, qd_ref, mesh.l_size)
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
        assert rel_l2(mv.to_numpy(), m_ref) < 1e-13
        ops.op_mass.assemble_diagonal(dv)
        assert rel_l2(dv.to_numpy(), d_ref) < 1e-13


@pytest.mark.parametrize("n,P,Q,periodic", [((3, 2, 2), 3, 3, (0, 0, 0)), ((2, 3, 2), 4, 5, (1, 0, 1)), ((2, 2, 2), 5, 6, (1, 1, 1)),
                                           ((2, 2, 1), 6, 7, (0, 0, 0)), ((3, 2, 1), 2, 4, (0, 0, 0))])
def test_stabilized_mass_and_diagonal_match_oracle(n, P, Q, periodic):
    import torch
    mesh, basis, ctx, q, _ = case(n, P, Q, periodic=periodic)
    op, qdata = _setup(mesh, basis)
    m = oracle_mesh(mesh, basis)
    qd = qdata.cpu().numpy()
    cb = prob.context_bytes(ctx)
    u = q * np.random.default_rng(3).uniform(-1, 1, q.shape)
    tq, tu = torch.from_numpy(q).to(_dev()), torch.from_numpy(u).to(_dev())
    v = torch.zeros_like(tq)
    op.mass_stab(cb, qdata, tq, tu, v)
    assert rel_l2(v.cpu().numpy(), O.apply_mass_stab(m, cb, u, q, qd)) < 1e-13
    d = torch.zeros_like(tq)
    op.mass_stab_diagonal(cb, qdata, tq, d)
    assert rel_l2(d.cpu().numpy(), O.mass_stab_diagonal(m, cb, q, qd, mesh.l_size)) < 1e-13


def test_gaussian_wave_explicit_reproduces_reference_run():
    """examples/navierstokes.c:233 on the GPU: TSRK5F, free-stream faces, symmetry planes, IDL, SUPG with the stabilized mass
    solved by GMRES + Jacobi diagonal (set up at the first solve); the reference's own bound 1e-8 on the final state."""
    import torch
    from test_explicit_oracle import gaussian_wave_explicit_case
    G, mesh, basis, newt, gw, q, ess, off, xn, fs, U, Y, FO = gaussian_wave_explicit_case()
    op, qdata = _setup(mesh, basis)
    op.set_vertex_coords(np.ascontiguousarray(mesh.x_elem))
    fop = K.FaceOp(off, mesh.l_size, basis, xn)
    ex = S.ExplicitStepper(op, prob.context_bytes(newt), qdata, dt=float(G["dt"]), rk_type=str(G["rk_type"]), mass_ksp=str(G["mass_ksp"]),
                           pc_jacobi=str(G["mass_pc_jacobi"]))
    ex.set_essential(ess)
    ex.set_freestream(fop, fs, flux_type=1)
    tq = torch.from_numpy(q).to(_dev())
    ex.set_state(tq, 0.0)
    for _ in range(int(G["steps"])):
        st = ex.step()
        assert st.converged_reason == 1 and st.mass_its > 0
    ex.get_state(tq)
    qf = tq.cpu().numpy()
    free = np.setdiff1d(np.arange(mesh.l_size), ess)
    ref = G["free_state"]
    err = np.abs(np.sort(qf[free]) - np.sort(ref)).max() / np.abs(ref).max()
    assert err <= float(G["compare_atol"]), err
