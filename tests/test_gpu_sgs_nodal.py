"""HONEE's nodal data-driven SGS pipeline through the drop-in libCEED library on /gpu/b200: the operators SgsDDSetup and
SgsDDApplyIFunction build (problems/sgs_dd_model.c:98-200, 508-560, 645-737; src/velocity_gradient_projection.c:44-152;
src/grid_anisotropy_tensor.c:10-118; src/inverse_multiplicity.c:24-80), made with the same QFunction names, fields,
evaluation modes and restrictions, and compared with the CPU oracle (oracle/sgs_nodal_oracle.py) on the same inputs.
The two L2 projections' solvers are PETSc's in the reference (CG + Jacobi for the anisotropy tensor, one row-sum Jacobi
step for the velocity gradient); here numpy plays PETSc on the host, with every operator apply and the diagonal taken
from the library.

Tolerances: each operator against the oracle on identical inputs, 1e-12 relative L2 (1e-10 for the closure, whose
eigen-solver and network amplify rounding; exact for the inverse multiplicity); the chained pipeline (projections
solved to 1e-12) against the chained oracle, 1e-9."""
import ctypes as C
import importlib

import numpy as np
import pytest

from helpers import O, rel_l2
import sgs_nodal_oracle as SN

pytestmark = pytest.mark.gpu
prob = importlib.import_module("honee-4aiad_b200.problem")
CE = importlib.import_module("honee-4aiad_b200.ceed")
sgs = importlib.import_module("honee-4aiad_b200.sgs")
SV_NAME = {0: "Conserv", 1: "Prim", 2: "Entropy"}
GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "sgs_points.npz"))

CASES = [((3, 2, 2), 3, 4, (False, False, False), 0), ((2, 2, 2), 4, 5, (True, True, True), 1), ((2, 2, 1), 3, 3, (False, True, False), 2)]


class _Setup:
    """The objects SgsDDSetup creates, on one box mesh."""

    def __init__(self, n, P, Q, periodic, sv):
        self.mesh = m = prob.box_mesh(n, P, periodic=periodic)
        self.basis = b = prob.tensor_basis(P, Q)
        self.sv = sv
        ctx = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, state_var=sv)
        self.gas = ctx.gas
        self.ceed = ce = CE.Ceed("/gpu/b200")
        E, P3, Q3 = m.num_elem, P ** 3, Q ** 3
        self.E, self.P3, self.Q3, self.nodes = E, P3, Q3, m.num_nodes
        # restrictions (DMPlexCeedElemRestrictionCreate on the solution DM and its 9-, 7- and 6-field clones), qdata
        self.r = {nc: CE.ElemRestriction(ce, E, P3, nc, 1, m.num_nodes * nc, offsets=(m.offsets // 5) * nc) for nc in (5, 6, 7, 9)}
        self.r_qd = CE.ElemRestriction(ce, E, Q3, 10, None, E * Q3 * 10)
        self.r_inv = CE.ElemRestriction(ce, E, P3, 1, None, E * P3)   # DMPlexCeedElemRestrictionCollocatedCreate
        self.bas = {nc: CE.Basis(ce, 3, nc, P, Q, b.interp1d, b.grad1d, b.qref1d, b.qweight1d) for nc in (5, 6, 7, 9)}
        # the trilinear coordinate field and its projection onto the solution nodes (problems/sgs_dd_model.c:162-165)
        xb = prob.tensor_basis(2, Q)
        self.r_x = CE.ElemRestriction(ce, E, 8, 3, None, E * 24, strides=(1, 8, 24))
        self.b_x = CE.Basis(ce, 3, 3, 2, Q, xb.interp1d, xb.grad1d, xb.qref1d, xb.qweight1d)
        self.b_x_to_q = CE.Basis.__new__(CE.Basis)
        CE._Obj.__init__(self.b_x_to_q, ce)
        ce.chk(CE.L().CeedBasisCreateProjection(self.b_x.ptr, self.bas[5].ptr, C.byref(self.b_x_to_q.ptr)))
        self.x = self._vec(m.x_elem.reshape(-1))
        self.qdata = O.setup_qdata(E, Q, m.x_elem)
        self.v_qd = self._vec(self.qdata)
        self.newt = (C.c_char * 184).from_buffer_copy(prob.context_bytes(ctx))
        self.c_newt = CE.QFunctionContext(ce, self.newt)
        self.sgs_blob = sgs.sgs_dd_context(prob.context_bytes(ctx), GOLD["weights"], GOLD["bounds"])
        self.c_sgs = CE.QFunctionContext(ce, self.sgs_blob)
        self.net = SN.Net(GOLD["weights"], GOLD["bounds"])

    def _vec(self, a):
        v = CE.Vector(self.ceed, a.size)
        v.set_array_host(np.ascontiguousarray(a, dtype=np.float64))
        return v

    def qf(self, name, ins, outs, ctx=None):
        q = CE.QFunction(self.ceed, f"qfunctions/sgs.h:{name}")
        for nm, size, em in ins:
            q.add_input(nm, size, em)
        for nm, size, em in outs:
            q.add_output(nm, size, em)
        if ctx is not None:
            q.set_context(ctx)
        return q

    def op(self, qf, fields):
        o = CE.Operator(self.ceed, qf)
        for nm, r, bs, v in fields:
            o.set_field(nm, r, bs, v)
        o._keep = (qf, fields)
        return o


def _generic_state(mesh, basis, gas, seed):
    """The seeded multimode state with all three velocity components perturbed at every node.  The closure is evaluated in
    the strain-rate eigenframe oriented by the vorticity: at a degenerate state (v = w = 0 makes the strain rate's
    eigenvalues repeat and the frame's orientation test read exact zeros) the reference's own result depends on rounding,
    so parity is checked on generic states."""
    q = prob.multimode_state(mesh, basis, gas, seed=seed).reshape(-1, 5).copy()
    rng = np.random.default_rng(100 + seed)
    rho, m_old = q[:, 0], q[:, 1:4].copy()
    q[:, 1:4] += rho[:, None] * rng.normal(0, 2.0, (q.shape[0], 3))
    q[:, 4] += 0.5 * ((q[:, 1:4] ** 2).sum(1) - (m_old ** 2).sum(1)) / rho  # the internal energy is kept
    return q.reshape(-1)


def _mass(S, nc):
    """HoneeMassQFunctionCreate (src/honee-mass.c:20-60) + the operator of the projection's KSP"""
    qf = S.qf(f"Mass_{nc}", [("u", nc, CE.CEED_EVAL_INTERP), ("qdata", 10, CE.CEED_EVAL_NONE)], [("v", nc, CE.CEED_EVAL_INTERP)])
    a = S.ceed.active
    return S.op(qf, [("u", S.r[nc], S.bas[nc], a), ("qdata", S.r_qd, S.ceed.basis_none, S.v_qd), ("v", S.r[nc], S.bas[nc], a)])


def _apply(S, op, x, n_out, add_to=None):
    out = CE.Vector(S.ceed, n_out)
    if add_to is None:
        out.set_value(0.0)
    else:
        out.set_array_host(np.ascontiguousarray(add_to))
    inp = S._vec(x) if x is not None else None
    op.apply(inp, out, add=add_to is not None)
    return out.to_numpy()


def _cg(apply, dinv, b, rtol=1e-12, max_it=2000):
    x = np.zeros_like(b)
    r = b.copy()
    z = dinv * r
    p = z.copy()
    rz = rz0 = float(r @ z)
    for _ in range(max_it):
        if rz <= rtol * rtol * rz0:
            break
        Ap = apply(p)
        a = rz / float(p @ Ap)
        x += a * p
        r -= a * Ap
        z = dinv * r
        rz_new = float(r @ z)
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x


@pytest.mark.parametrize("n,P,Q,periodic,sv", CASES)
def test_nodal_sgs_pipeline_matches_oracle(n, P, Q, periodic, sv):
    S = _Setup(n, P, Q, periodic, sv)
    m, b, a, none_b = S.mesh, S.basis, S.ceed.active, S.ceed.basis_none
    cv, cp, mu = S.gas.cv, S.gas.cp, S.gas.mu
    N = S.nodes
    q_cons = _generic_state(m, b, S.gas, 3 + sv)
    q = prob.state_to_q(S.gas, q_cons, sv)

    # ---- GridAnisotropyTensorProjectionSetupApply: right-hand side, Mass_7 + diagonal, CG + Jacobi
    qf_a = S.qf("AnisotropyTensorProjection", [("qdata", 10, CE.CEED_EVAL_NONE)], [("v", 7, CE.CEED_EVAL_INTERP)])
    op_a = S.op(qf_a, [("qdata", S.r_qd, none_b, S.v_qd), ("v", S.r[7], S.bas[7], a)])
    rhs7 = _apply(S, op_a, None, N * 7)
    rhs7_o = SN.aniso_rhs(m, b, S.qdata)
    assert rel_l2(rhs7, rhs7_o) < 1e-12
    op_m7 = _mass(S, 7)
    d7 = CE.Vector(S.ceed, N * 7)
    op_m7.assemble_diagonal(d7)
    assert rel_l2(d7.to_numpy(), SN.mass_diagonal(m, b, S.qdata, 7)) < 1e-13
    u7 = np.random.default_rng(1).normal(size=N * 7)
    assert rel_l2(_apply(S, op_m7, u7, N * 7), SN.mass_apply(m, b, S.qdata, u7, 7)) < 1e-13
    A7 = _cg(lambda p: _apply(S, op_m7, p, N * 7), 1.0 / d7.to_numpy(), rhs7)
    A7_o = SN.project_cg(m, b, S.qdata, rhs7_o, 7, rtol=1e-12)
    assert rel_l2(A7, A7_o) < 1e-9

    # ---- GetInverseMultiplicity (local): CeedElemRestrictionGetMultiplicity + InverseMultiplicity
    mult = CE.Vector(S.ceed, N * 6)
    S.ceed.chk(CE.L().CeedElemRestrictionGetMultiplicity(S.r[6].ptr, mult.ptr))
    qf_im = S.qf("InverseMultiplicity", [("multiplicity", 6, CE.CEED_EVAL_NONE)], [("inverse multiplicity", 1, CE.CEED_EVAL_NONE)])
    op_im = S.op(qf_im, [("multiplicity", S.r[6], none_b, a), ("inverse multiplicity", S.r_inv, none_b, a)])
    inv = CE.Vector(S.ceed, S.E * S.P3)
    op_im.apply(mult, inv)
    inv_o = SN.inverse_multiplicity(m)
    np.testing.assert_array_equal(inv.to_numpy(), inv_o.reshape(-1))

    # ---- VelocityGradientProjectionApply: right-hand side, Mass_9 row sums, one Jacobi step
    qf_g = S.qf(f"VelocityGradientProjectionRHS_{SV_NAME[sv]}", [("q", 5, CE.CEED_EVAL_INTERP), ("Grad_q", 15, CE.CEED_EVAL_GRAD),
                                                                ("qdata", 10, CE.CEED_EVAL_NONE), ("x", 3, CE.CEED_EVAL_INTERP)],
                [("velocity gradient", 9, CE.CEED_EVAL_INTERP)], S.c_newt)
    op_g = S.op(qf_g, [("q", S.r[5], S.bas[5], a), ("Grad_q", S.r[5], S.bas[5], a), ("qdata", S.r_qd, none_b, S.v_qd),
                       ("x", S.r_x, S.b_x, S.x), ("velocity gradient", S.r[9], S.bas[9], a)])
    rhs9 = _apply(S, op_g, q, N * 9)
    rhs9_o = SN.velgrad_rhs(m, b, S.qdata, q, sv, cv, cp)
    assert rel_l2(rhs9, rhs9_o) < (1e-12 if sv != 2 else 1e-10)
    op_m9 = _mass(S, 9)
    G9 = rhs9 / _apply(S, op_m9, np.ones(N * 9), N * 9)
    G9_o = SN.project_rowsum(m, b, S.qdata, rhs9_o, 9)
    assert rel_l2(G9, G9_o) < (1e-12 if sv != 2 else 1e-10)

    # ---- SgsDDNodalStressEval_Fused: ComputeSgsDDNodal_* on identical inputs
    qf_s = S.qf(f"ComputeSgsDDNodal_{SV_NAME[sv]}", [("q", 5, CE.CEED_EVAL_NONE), ("x", 3, CE.CEED_EVAL_INTERP),
                                                     ("gradient velocity", 9, CE.CEED_EVAL_NONE), ("anisotropy tensor", 7, CE.CEED_EVAL_NONE),
                                                     ("inverse multiplicity", 1, CE.CEED_EVAL_NONE)],
                [("km_sgs", 6, CE.CEED_EVAL_NONE)], S.c_sgs)
    v_q, v_A = S._vec(q), S._vec(A7_o)
    op_s = S.op(qf_s, [("q", S.r[5], none_b, v_q), ("x", S.r_x, S.b_x_to_q, S.x), ("gradient velocity", S.r[9], none_b, a),
                       ("anisotropy tensor", S.r[7], none_b, v_A), ("inverse multiplicity", S.r_inv, none_b, inv), ("km_sgs", S.r[6], none_b, a)])
    km = _apply(S, op_s, G9_o, N * 6)
    km_o = SN.sgs_nodal(m, S.net, q, G9_o, A7_o, inv_o, sv, mu, cv, cp)
    assert rel_l2(km, km_o) < 1e-10

    # ---- SgsDDApplyIFunction: IFunction_NodalSgs_* added to an existing residual, on identical inputs
    qf_i = S.qf(f"IFunction_NodalSgs_{SV_NAME[sv]}", [("q", 5, CE.CEED_EVAL_INTERP), ("qdata", 10, CE.CEED_EVAL_NONE), ("km_sgs", 6, CE.CEED_EVAL_INTERP)],
                [("Grad_v", 15, CE.CEED_EVAL_GRAD)], S.c_newt)
    v_km = S._vec(km_o)
    op_i = S.op(qf_i, [("q", S.r[5], S.bas[5], a), ("qdata", S.r_qd, none_b, S.v_qd), ("km_sgs", S.r[6], S.bas[6], v_km),
                       ("Grad_v", S.r[5], S.bas[5], a)])
    g0 = np.random.default_rng(2).normal(size=N * 5)
    g = _apply(S, op_i, q, N * 5, add_to=g0)
    g_o = SN.sgs_ifunction(m, b, S.qdata, q, km_o, sv, cv, cp)
    assert rel_l2(g - g0, g_o) < 1e-12

    # ---- the chained pipeline: every stage from the library's own previous outputs
    v_A.set_array_host(np.ascontiguousarray(A7))
    km_chain = _apply(S, op_s, G9, N * 6)
    v_km.set_array_host(np.ascontiguousarray(km_chain))
    g_chain = _apply(S, op_i, q, N * 5)
    assert rel_l2(g_chain, g_o) < 1e-9


def test_honee_operators_add_the_nodal_sgs_term_to_the_residual():
    """NewtonianOperators.add_sgs_dd (the Python mirror of SgsDDSetup) makes ifunction() add SgsDDApplyIFunction's term:
    the residual with the model minus the residual without it equals the oracle's nodal pipeline on the same state."""
    hon = importlib.import_module("honee-4aiad_b200.honee")
    mesh = prob.box_mesh((3, 2, 2), 3, periodic=(True, True, False))
    basis = prob.tensor_basis(3, 3)
    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=prob.STAB_SUPG, state_var=prob.STATEVAR_PRIMITIVE, dt=1e-4)
    ceed = CE.Ceed("/gpu/b200")
    ops = hon.NewtonianOperators(ceed, mesh, basis, ctx)
    q_h = prob.state_to_q(ctx.gas, _generic_state(mesh, basis, ctx.gas, 9), prob.STATEVAR_PRIMITIVE)
    q, q_dot, g = CE.Vector(ceed, mesh.l_size), CE.Vector(ceed, mesh.l_size), CE.Vector(ceed, mesh.l_size)
    q.set_array_host(q_h)
    q_dot.set_array_host(q_h * 1e-3)
    ops.ifunction(q, q_dot, g)
    g_plain = g.to_numpy()
    ops.add_sgs_dd(GOLD["weights"], GOLD["bounds"], aniso_rtol=1e-12)
    ops.ifunction(q, q_dot, g)
    term = g.to_numpy() - g_plain
    qdata = ops.host_inputs()
    cv, cp, mu = ctx.gas.cv, ctx.gas.cp, ctx.gas.mu
    A7 = SN.project_cg(mesh, basis, qdata, SN.aniso_rhs(mesh, basis, qdata), 7, rtol=1e-12)
    G9 = SN.project_rowsum(mesh, basis, qdata, SN.velgrad_rhs(mesh, basis, qdata, q_h, 1, cv, cp), 9)
    km = SN.sgs_nodal(mesh, SN.Net(GOLD["weights"], GOLD["bounds"]), q_h, G9, A7, SN.inverse_multiplicity(mesh), 1, mu, cv, cp)
    term_o = SN.sgs_ifunction(mesh, basis, qdata, q_h, km, 1, cv, cp)
    assert np.abs(term_o).max() > 0
    assert rel_l2(term, term_o) < 1e-8


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_nodal_closure_kernel_matches_reference_points(sv):
    """hb_sgs_nodal_closure on the seeded points of tests/golden/sgs_nodal_points.npz against the reference's own
    ComputeSgsDDNodal_* (inverse multiplicity as the node weight)."""
    import os
    import torch
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "sgs_nodal_points.npz"))
    name = SV_NAME[sv]
    ctx = prob.newtonian_context(2, cv=float(gold["cv"]), cp=float(gold["cp"]), mu=float(gold["mu"]), k=0.0257, state_var=sv)
    blob = sgs.sgs_dd_context(prob.context_bytes(ctx), GOLD["weights"], GOLD["bounds"])
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    q, G = t(gold[f"q_{name}"].T), t(gold["G"].reshape(-1, 9))
    A, w = t(gold["Aij_delta"].T), t(gold["inv_mult"])
    km = torch.zeros(q.shape[0], 6, dtype=torch.float64, device=dev)
    sgs.nodal_closure(blob, sv, q, G, A, w, km)
    torch.cuda.synchronize()
    ref = gold[f"km_sgs_{name}"].T
    np.testing.assert_allclose(km.cpu().numpy(), ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
