"""CPU checks of the point-block oracle (oracle_assemble_point_block, face_oracle.freestream_point_block): each 5 x 5 node
block is the corresponding block of the operator's matrix, e_(node,i)^T J e_(node,j) from the oracle's Jacobian action
(itself pinned to the reference's IJacobian / Freestream_Jacobian QFunctions), and its diagonal is the oracle's diagonal."""
import os

import numpy as np
import pytest

from helpers import O, case, oracle_ifunction, oracle_mesh, prob

import face_oracle as FO  # noqa: E402


@pytest.mark.parametrize("P,Q,periodic,idl", [(3, 3, (0, 0, 0), None), (3, 4, (1, 0, 0), (2e-3, 0.2, 0.5, 101000.0))])
def test_volume_point_blocks_are_jacobian_blocks(P, Q, periodic, idl):
    mesh, basis, ctx, q, qd = case((2, 1, 2), P, Q, periodic=periodic, idl=idl)
    v, jd, qdata, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    njd = 15 if ctx.idl_enable else 14
    cb = prob.context_bytes(ctx)
    pb = O.assemble_point_block(m, cb, qdata, jd, mesh.l_size, num_jd=njd)
    d = O.assemble_diagonal(m, cb, qdata, jd, mesh.l_size, num_jd=njd)
    np.testing.assert_array_equal(pb.reshape(-1, 5, 5)[:, np.arange(5), np.arange(5)].reshape(-1), d)
    scale = np.abs(pb).max()
    for node in np.random.default_rng(0).choice(mesh.l_size // 5, 6, replace=False):
        for j in range(5):
            e = np.zeros(mesh.l_size)
            e[node * 5 + j] = 1.0
            col = O.apply_ijacobian(m, cb, e, qdata, jd, num_jd=njd)
            np.testing.assert_allclose(pb[node * 25 + np.arange(5) * 5 + j], col[node * 5:node * 5 + 5], rtol=0, atol=1e-13 * scale)


@pytest.mark.parametrize("hllc", [False, True])
def test_face_point_blocks_are_jacobian_blocks(hllc):
    G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "face_points.npz"))
    cv, cp = float(G["cv"]), float(G["cp"])
    u = G["u_inf"]
    rho = float(G["P_inf"]) / ((cp - cv) * float(G["T_inf"]))
    U = np.array([rho, *(rho * u), rho * (cv * float(G["T_inf"]) + 0.5 * u @ u)])
    Y = np.array([float(G["P_inf"]), *u, float(G["T_inf"])])
    mesh = prob.box_mesh((2, 1, 1), 3)
    basis = prob.tensor_basis(3, 3)
    q = prob.gaussian_pulse_state(mesh, basis, prob.GasProperties(cv=cv, cp=cp), seed=2)
    off, xn, _ = prob.box_faces(mesh, basis)
    qd = FO.face_qdata(basis.interp1d, basis.grad1d, basis.qweight1d, 3, 3, xn)
    B = np.asarray(basis.interp1d).reshape(3, 3)
    Bq = np.einsum("jb,ia->jiba", B, B).reshape(9, 9)
    jac = np.stack([(Bq @ q.reshape(-1, 5)[off[f] // 5]).T for f in range(off.shape[0])])
    pb = FO.freestream_point_block(off, basis.interp1d, 3, 3, qd, jac, U, Y, cv, cp, hllc=hllc, l_size=mesh.l_size)
    d = FO.freestream_diagonal(off, basis.interp1d, 3, 3, qd, jac, U, Y, cv, cp, hllc=hllc, l_size=mesh.l_size)
    np.testing.assert_allclose(pb.reshape(-1, 5, 5)[:, np.arange(5), np.arange(5)].reshape(-1), d, rtol=1e-14, atol=1e-14 * np.abs(d).max())
    for node in np.random.default_rng(1).choice(np.unique(off.reshape(-1)) // 5, 5, replace=False):
        for j in range(5):
            e = np.zeros(mesh.l_size)
            e[node * 5 + j] = 1.0
            col = FO.freestream_apply(off, basis.interp1d, 3, 3, qd, q, U, Y, cv, cp, hllc=hllc, dq=e, jac=jac)
            np.testing.assert_allclose(pb[node * 25 + np.arange(5) * 5 + j], col[node * 5:node * 5 + 5], rtol=0, atol=1e-12 * np.abs(pb).max())
