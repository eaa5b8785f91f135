"""GPU parity of the free-stream boundary sub-operators reached through the libCEED C API, the way HONEE builds them
(QDataBoundaryGet with ``SetupBoundary``; HoneeBCAddIFunctionOp / HoneeBCAddIJacobianOp with the
``Freestream_[Jacobian_]Conserv_HLL[C]`` QFunctions), against the CPU oracle (oracle/face_oracle.py, pinned to the
reference QFunctions by tests/test_face_oracle.py).

Tolerances: surface geometric factors 1e-14 relative L2; FP64 residual, Jacobian action and diagonal of the face
sub-operators 1e-12; composites equal the sum of their sub-operators to 1e-14; the mixed-precision composite Jacobian
(FP32 volume, FP64 faces) within 2e-6 of the FP64 one.
"""
import importlib
import os
import sys

import numpy as np
import pytest

from helpers import case, rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import face_oracle as FO  # noqa: E402

ce = importlib.import_module("honee-4aiad_b200.ceed")
hon = importlib.import_module("honee-4aiad_b200.honee")

P_INF, U_INF, T_INF = 101325.0 * 1.02, np.array([60.0, -25.0, 10.0]), 290.0

CASES = {
    "P3Q3_hllc": dict(n=(3, 2, 2), P=3, Q=3, riemann="hllc"),
    "P4Q5_hll": dict(n=(2, 3, 2), P=4, Q=5, riemann="hll", state="modes"),
    "P3Q4_hllc_periodic_x": dict(n=(3, 3, 2), P=3, Q=4, riemann="hllc", periodic=(1, 0, 0)),
}


def _exterior(gas):
    rho = P_INF / ((gas.cp - gas.cv) * T_INF)
    U = np.array([rho, *(rho * U_INF), rho * (gas.cv * T_INF + 0.5 * U_INF @ U_INF)])
    Y = np.array([P_INF, *U_INF, T_INF])
    return U, Y


def _setup(name, resource="/gpu/b200"):
    kw = dict(CASES[name])
    riemann = kw.pop("riemann")
    mesh, basis, ctx, q, qd = case(**kw)
    ceed = ce.Ceed(resource)
    ops = hon.NewtonianOperators(ceed, mesh, basis, ctx)
    bc = ops.add_freestream(P_INF, U_INF, T_INF, riemann=riemann)
    qv = ce.Vector(ceed, mesh.l_size)
    qv.set_array_host(q)
    ops.q_dot.set_array_host(qd)
    return mesh, basis, ctx, q, ceed, ops, bc, qv


def _face_interp(basis, off, q):
    """q at the face points [F][5][Q^2] (what the IFunction face operator stores as surface jacobian data)."""
    P, Q = basis.P, basis.Q
    B = np.asarray(basis.interp1d).reshape(Q, P)
    Bq = np.einsum("jb,ia->jiba", B, B).reshape(Q * Q, P * P)
    nodes = off // 5
    return np.stack([(Bq @ q.reshape(-1, 5)[nodes[f]]).T for f in range(off.shape[0])])


@pytest.mark.parametrize("name", list(CASES))
def test_freestream_subops_match_oracle(name):
    mesh, basis, ctx, q, ceed, ops, bc, qv = _setup(name)
    P, Q = basis.P, basis.Q
    off = bc["offsets"]
    F = off.shape[0]
    gas = ctx.gas
    U, Y = _exterior(gas)
    # surface geometric factors from the bilinear face coordinates (SetupBoundary)
    Bx, Gx = hon.linear_coordinate_basis(Q, basis.qref1d, basis.qweight1d)
    corners = [0, P - 1, P * (P - 1), P * P - 1]
    qd_ref = FO.face_qdata(Bx.reshape(-1), Gx.reshape(-1), basis.qweight1d, 2, Q, bc["x_nodes"][:, :, corners])
    qd = bc["q_data"].to_numpy().reshape(F, 10, Q * Q)
    assert rel_l2(qd, qd_ref) < 1e-14
    # residual of the face sub-operator and its surface jacobian data
    v = ce.Vector(ceed, mesh.l_size)
    bc["op_ifunction"].apply(qv, v)
    ref = FO.freestream_apply(off, basis.interp1d, P, Q, qd_ref, q, U, Y, gas.cv, gas.cp, hllc=bc["hllc"])
    assert rel_l2(v.to_numpy(), ref) < 1e-12
    jac_ref = _face_interp(basis, off, q)
    assert rel_l2(bc["jac_data"].to_numpy().reshape(jac_ref.shape), jac_ref) < 1e-14
    # Jacobian action
    dq = q * 1e-3 * np.random.default_rng(4).uniform(-1, 1, q.shape)
    dqv = ce.Vector(ceed, mesh.l_size)
    dqv.set_array_host(dq)
    dv = ce.Vector(ceed, mesh.l_size)
    bc["op_ijacobian"].apply(dqv, dv)
    dref = FO.freestream_apply(off, basis.interp1d, P, Q, qd_ref, q, U, Y, gas.cv, gas.cp, hllc=bc["hllc"], dq=dq, jac=jac_ref)
    assert rel_l2(dv.to_numpy(), dref) < 1e-12
    # diagonal
    d = ce.Vector(ceed, mesh.l_size)
    bc["op_ijacobian"].assemble_diagonal(d)
    d_ref = FO.freestream_diagonal(off, basis.interp1d, P, Q, qd_ref, jac_ref, U, Y, gas.cv, gas.cp, hllc=bc["hllc"], l_size=mesh.l_size)
    assert rel_l2(d.to_numpy(), d_ref) < 1e-12


def test_freestream_diagonal_is_the_jacobian_diagonal():
    """e_i^T J e_i from the face Jacobian action equals the assembled diagonal, on a sample of boundary DOFs."""
    mesh, basis, ctx, q, ceed, ops, bc, qv = _setup("P3Q3_hllc")
    ops.ifunction(qv, ops.q_dot, ce.Vector(ceed, mesh.l_size))
    d = ce.Vector(ceed, mesh.l_size)
    bc["op_ijacobian"].assemble_diagonal(d)
    dn = d.to_numpy()
    nodes = np.unique(bc["offsets"].reshape(-1))
    rng = np.random.default_rng(7)
    dofs = rng.choice(nodes, 30, replace=False) + rng.integers(0, 5, 30)
    e, out = ce.Vector(ceed, mesh.l_size), ce.Vector(ceed, mesh.l_size)
    for i in dofs:
        h = np.zeros(mesh.l_size)
        h[i] = 1.0
        e.set_array_host(h)
        bc["op_ijacobian"].apply(e, out)
        assert abs(out.to_numpy()[i] - dn[i]) <= 1e-12 * max(1.0, np.abs(dn).max())


@pytest.mark.parametrize("name", ["P3Q3_hllc", "P3Q4_hllc_periodic_x"])
def test_composites_are_volume_plus_faces(name):
    mesh, basis, ctx, q, ceed, ops, bc, qv = _setup(name)
    n = mesh.l_size
    g, gv, gf = (ce.Vector(ceed, n) for _ in range(3))
    ops.ifunction(qv, ops.q_dot, g)
    ops.op_ifunction_volume.apply(qv, gv)
    bc["op_ifunction"].apply(qv, gf)
    assert rel_l2(g.to_numpy(), gv.to_numpy() + gf.to_numpy()) < 1e-14
    dq = q * 1e-3 * np.random.default_rng(5).uniform(-1, 1, q.shape)
    dqv = ce.Vector(ceed, n)
    dqv.set_array_host(dq)
    ops.set_ijacobian_shift(1.5 / 1e-5)
    j, jv, jf = (ce.Vector(ceed, n) for _ in range(3))
    ops.ijacobian(dqv, j)
    ops.op_ijacobian_volume.apply(dqv, jv)
    bc["op_ijacobian"].apply(dqv, jf)
    assert rel_l2(j.to_numpy(), jv.to_numpy() + jf.to_numpy()) < 1e-14
    d, dv, df = (ce.Vector(ceed, n) for _ in range(3))
    ops.diagonal(d)
    ops.op_ijacobian_volume.assemble_diagonal(dv)
    bc["op_ijacobian"].assemble_diagonal(df)
    assert rel_l2(d.to_numpy(), dv.to_numpy() + df.to_numpy()) < 1e-14
    # the mixed-precision resource: FP32 volume Jacobian and diagonal, FP64 faces
    mesh, basis, ctx, q, ceed32, ops32, bc32, qv32 = _setup(name, "/gpu/b200/mixed")
    ops32.ifunction(qv32, ops32.q_dot, ce.Vector(ceed32, n))
    ops32.set_ijacobian_shift(1.5 / 1e-5)
    dq32, j32, d32 = ce.Vector(ceed32, n), ce.Vector(ceed32, n), ce.Vector(ceed32, n)
    dq32.set_array_host(dq)
    ops32.ijacobian(dq32, j32)
    ops32.diagonal(d32)
    assert rel_l2(j32.to_numpy(), j.to_numpy()) < 2e-6
    assert rel_l2(d32.to_numpy(), d.to_numpy()) < 2e-6
