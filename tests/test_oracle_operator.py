"""Operator-level oracle checks on the CPU: libCEED semantics restated in oracle/honee_oracle.c.

* tabulation: Gauss-Lobatto nodes / Gauss-Legendre points / Lagrange matrices (src/dm-utils.c:594-735, PETSc defaults)
* qdata of affine boxes against the closed form (qfunctions/setupgeo.h:42-56)
* the reference's Taylor-Green kinetic-energy golden row (tests/output/taylorgreen_totalke.csv, rtol 1e-9 / ztol 3e-10
  as tests/junit.py:55 and tests/junit_common.py:141 diff it) -- pins basis, quadrature, qdata, IC and monitor together
* the oracle operator driven by the restated QFunctions equals the one driven by the reference's own QFunctions
* IJacobian: linearity and, without stabilisation, agreement with a finite difference of the IFunction
* diagonal assembly against the brute-force diagonal e_i^T J e_i
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from helpers import O, case, oracle_ifunction, oracle_mesh, prob, rel_l2

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("P,Q", [(2, 2), (3, 3), (4, 5), (5, 6), (6, 7)])
def test_tabulation_matches_numpy(P, Q):
    x, w = O.gauss_legendre(Q)
    xn, wn = prob.gauss_legendre(Q)
    np.testing.assert_allclose(x, xn, atol=2e-16)
    np.testing.assert_allclose(w, wn, rtol=2e-15)
    assert abs(w.sum() - 2) < 1e-14
    nodes = O.gauss_lobatto(P)
    np.testing.assert_allclose(nodes, prob.gauss_lobatto(P), atol=2e-16)
    B, G = O.lagrange_tabulate(nodes, x)
    b = prob.tensor_basis(P, Q)
    np.testing.assert_allclose(B, b.interp1d, atol=1e-15)
    np.testing.assert_allclose(G, b.grad1d, atol=1e-13)
    np.testing.assert_allclose(B.sum(axis=1), 1, atol=1e-14)        # partition of unity
    np.testing.assert_allclose(G.sum(axis=1), 0, atol=1e-13)
    np.testing.assert_allclose(B @ nodes, x, atol=1e-14)             # reproduces linears
    np.testing.assert_allclose(G @ nodes, 1, atol=1e-13)


def test_degree2_nodes_are_unambiguous():
    """For degree 2 Gauss-Lobatto and equispaced nodes coincide ({-1, 0, 1}), so P=3 workloads do not depend on the
    PETSc node family."""
    np.testing.assert_allclose(O.gauss_lobatto(3), [-1, 0, 1], atol=1e-16)


def test_qdata_affine_box():
    n = (3, 2, 4)
    mesh = prob.box_mesh(n, 3, lo=(0, 0, 0), hi=(0.6, 1.0, 2.0))
    Q = 4
    qd = O.setup_qdata(mesh.num_elem, Q, mesh.x_elem).reshape(mesh.num_elem, 10, Q ** 3)
    h = np.array([0.2, 0.5, 0.5])
    x, w = O.gauss_legendre(Q)
    W = np.einsum("i,j,k->kji", w, w, w).reshape(-1)
    np.testing.assert_allclose(qd[:, 0, :], np.broadcast_to(W[None, :] * np.prod(h / 2), qd[:, 0, :].shape), rtol=1e-14)
    for a in range(3):
        for b in range(3):
            np.testing.assert_allclose(qd[:, 1 + 3 * a + b, :], np.full(qd[:, 0, :].shape, (2 / h[a]) if a == b else 0.), atol=1e-13)


def test_restriction_roundtrip():
    mesh = prob.box_mesh((3, 2, 2), 4, periodic=(1, 0, 1))
    rng = np.random.default_rng(3)
    l = rng.normal(size=mesh.l_size)
    e = np.zeros(mesh.num_elem * 5 * 64)
    O.lib().oracle_restrict(mesh.num_elem, 64, 5, 1, O.ptr(mesh.offsets), O.ptr(l), O.ptr(e))
    off = mesh.offsets.reshape(mesh.num_elem, 64)
    ref = np.stack([l[off + c] for c in range(5)], axis=1).reshape(-1)
    np.testing.assert_array_equal(e, ref)
    lt = np.zeros_like(l)
    O.lib().oracle_restrict_t(mesh.num_elem, 64, 5, 1, O.ptr(mesh.offsets), O.ptr(e), O.ptr(lt))
    mult = np.zeros(mesh.l_size)
    np.add.at(mult, (off[:, :, None] + np.arange(5)).reshape(-1), 1)
    np.testing.assert_allclose(lt, l * mult, rtol=1e-15)


def test_taylor_green_ke_golden():
    g = json.load(open(os.path.join(GOLD, "taylorgreen_ke_step0.json")))
    L = g["box"][1]
    mesh = prob.box_mesh(g["faces"], g["P"], periodic=(1, 1, 1), hi=(L, L, L))
    basis = prob.tensor_basis(g["P"], g["Q"])
    tg = prob.TaylorGreenContext()
    tg.reference = prob.StatePrimitive(g["reference_pressure"], (C.c_double * 3)(*g["reference_velocity"]), g["reference_temperature"])
    tg.newt_ctx = prob.newtonian_context(g["degree"], cv=g["cv"], cp=g["cp"], mu=g["mu"], k=g["k"])
    tg.lx = tg.ly = tg.lz = L
    X = prob.node_coordinates(mesh, basis)
    q = np.zeros((5, X.shape[1]))
    O.call_qf(O.lib().oracle_qf_ics_taylorgreen, bytes(memoryview(tg)), X.shape[1], [np.ascontiguousarray(X)], [q])
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    sums = O.monitor_ke(oracle_mesh(mesh, basis), bytes(memoryview(tg.newt_ctx)), np.ascontiguousarray(q.T.reshape(-1)), qdata) / L ** 3
    names = ["TotalKineticEnergy", "StrainDissipation", "DivergenceDissipation", "VolumeExpansion", "MuVorticity2"]
    for s, name in zip(sums, names):
        ref = g[name]
        assert abs(s - ref) <= max(g["csv_rtol"] * abs(ref), g["csv_ztol"]), (name, s, ref)
    assert abs(sums[0] - g["TotalKineticEnergy"]) < 1e-14 * g["TotalKineticEnergy"] * 10


@pytest.mark.parametrize("P,Q,periodic", [(3, 3, (0, 0, 0)), (4, 5, (1, 0, 0))])
def test_operator_restatement_equals_reference_qfunctions(P, Q, periodic):
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    mesh, basis, ctx, q, qd = case((2, 2, 2), P, Q, periodic=periodic)
    v_o, jd_o, qdata, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    v_r, jd_r, _, _ = oracle_ifunction(mesh, basis, ctx, q, qd, use_ref=True)
    np.testing.assert_array_equal(v_o, v_r)
    np.testing.assert_array_equal(jd_o, jd_r)
    dq = np.random.default_rng(5).normal(size=q.shape) * np.abs(q) * 1e-3
    cb = prob.context_bytes(ctx)
    j_o = O.apply_ijacobian(m, cb, dq, qdata, jd_o)
    j_r = O.apply_ijacobian(m, cb, dq, qdata, jd_o, use_ref=True)
    np.testing.assert_array_equal(j_o, j_r)


def test_ijacobian_linear_and_matches_fd_without_stabilisation():
    mesh, basis, ctx, q, qd = case((2, 2, 2), 3, 3, stab=prob.STAB_NONE, dt=1e-4)
    v0, jd, qdata, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    cb = prob.context_bytes(ctx)
    rng = np.random.default_rng(11)
    x = rng.normal(size=q.shape) * np.abs(q) * 1e-6
    y = rng.normal(size=q.shape) * np.abs(q) * 1e-6
    Jx = O.apply_ijacobian(m, cb, x, qdata, jd)
    Jy = O.apply_ijacobian(m, cb, y, qdata, jd)
    Jxy = O.apply_ijacobian(m, cb, np.ascontiguousarray(2 * x - 3 * y), qdata, jd)
    assert rel_l2(Jxy, 2 * Jx - 3 * Jy) < 1e-12
    # F(q + eps x, q_dot + shift eps x) - F(q, q_dot) ~ eps J x  (BDF: q_dot = shift q + history)
    shift = ctx.ijacobian_time_shift
    for eps in (1.0,):
        v1, _, _, _ = oracle_ifunction(mesh, basis, ctx, np.ascontiguousarray(q + eps * x), np.ascontiguousarray(qd + shift * eps * x))
        assert rel_l2((v1 - v0) / eps, Jx) < 1e-5


def test_diagonal_matches_brute_force():
    mesh, basis, ctx, q, qd = case((1, 1, 1), 3, 3)
    _, jd, qdata, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    cb = prob.context_bytes(ctx)
    d = O.assemble_diagonal(m, cb, qdata, jd, mesh.l_size)
    brute = np.zeros(mesh.l_size)
    for i in range(mesh.l_size):
        e = np.zeros(mesh.l_size); e[i] = 1
        brute[i] = O.apply_ijacobian(m, cb, e, qdata, jd)[i]
    assert rel_l2(d, brute) < 1e-13


@pytest.mark.parametrize("n,periodic", [((5, 5, 5), (1, 1, 1)), ((3, 4, 5), (1, 0, 1)), ((2, 3, 2), (0, 0, 0)), ((4, 4, 4), (1, 1, 1))])
def test_box_colouring_is_conflict_free(n, periodic):
    """The oracle's threaded scatter relies on the colouring: elements of one colour share no L-vector node."""
    mesh = prob.box_mesh(n, 3, periodic=periodic)
    ptr_, order = mesh.colors
    off = mesh.offsets.reshape(mesh.num_elem, -1)
    assert sorted(order.tolist()) == list(range(mesh.num_elem))
    for c in range(len(ptr_) - 1):
        nodes = off[order[ptr_[c]:ptr_[c + 1]]]
        per_elem = [np.unique(r) for r in nodes]
        allnodes = np.concatenate(per_elem)
        assert len(np.unique(allnodes)) == len(allnodes), (c, n, periodic)


def test_taylor_green_state_matches_reference_initial_condition():
    """The product's nodal TG initial state equals the reference ICsTaylorGreen QFunction run by the oracle."""
    L = 2 * np.pi
    mesh = prob.box_mesh((3, 3, 3), 5, periodic=(1, 1, 1), hi=(L, L, L))
    basis = prob.tensor_basis(5, 6)
    tg = prob.taylor_green_context(4)
    tg.u[0], tg.u[1], tg.u[2] = 0.1, -0.2, 0.05
    X = prob.node_coordinates(mesh, basis)
    qn = np.zeros((5, X.shape[1]))
    O.call_qf(O.lib().oracle_qf_ics_taylorgreen, bytes(memoryview(tg)), X.shape[1], [np.ascontiguousarray(X)], [qn])
    np.testing.assert_allclose(prob.taylor_green_state(mesh, basis, tg), qn.T.reshape(-1), rtol=1e-14, atol=0)
