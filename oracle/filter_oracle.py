"""CPU restatement of the differential filter and of the SGS training pairs on a box mesh (TEST INFRASTRUCTURE ONLY:
the checker for k_filter.cu).

Point-wise forms follow qfunctions/differential_filter.h:29-58 (DifferentialFilter_RHS: wdetJ * (P, u, T, u_i u_j)) and
:66-128 (DifferentialFilter_LHS_N without wall damping: v = wdetJ q, Grad_v = wdetJ alpha (dXdx grad q), alpha =
kernel_scaling (S Delta)(S Delta)), and qfunctions/sgs_dd_training.h:22-56 for the training pairs; the operator is the
libCEED element assembly (restriction, tensor basis, transpose, sum) written with numpy.  Pinned by
tests/test_sgs_oracle.py against the reference's QFunctions compiled in oracle/_ref.
"""
from __future__ import annotations

import numpy as np

import face_oracle as FaceO
import sgs_oracle as SO


def tensor_ops(interp1d, grad1d, P, Q):
    """Q^3 x P^3 interpolation and the three reference-derivative matrices, x fastest in both index orders."""
    B = np.asarray(interp1d).reshape(Q, P)
    G = np.asarray(grad1d).reshape(Q, P)
    Bq = np.einsum("ka,jb,ic->kjiabc", B, B, B).reshape(Q ** 3, P ** 3)
    D0 = np.einsum("ka,jb,ic->kjiabc", B, B, G).reshape(Q ** 3, P ** 3)
    D1 = np.einsum("ka,jb,ic->kjiabc", B, G, B).reshape(Q ** 3, P ** 3)
    D2 = np.einsum("ka,jb,ic->kjiabc", G, B, B).reshape(Q ** 3, P ** 3)
    return Bq, (D0, D1, D2)


def alpha_at(X, grid_based, width_scaling, kernel_scaling):
    if grid_based:
        kmA, delta = SO.anisotropy(X)
        D = SO.km_unpack(kmA * delta)
    else:
        D = np.eye(3)
    SD = np.diag(width_scaling) @ D
    return kernel_scaling * SD @ SD


def lhs_point(q, grad_ref, X, w, al):
    """q [nc], grad_ref [3][nc] -> v [nc], Grad_v [3][nc]"""
    dq = np.einsum("rc,rk->kc", grad_ref, X)      # physical gradient
    dqx = X @ dq                                  # dXdx . grad
    return w * q, w * (al @ dqx)


def alpha_field(mesh, basis, qdata, grid_based=False, width_scaling=(1, 1, 1), kernel_scaling=0.1):
    """alpha [E][Q3][3][3] at every quadrature point."""
    Q3 = basis.Q ** 3
    qd = np.asarray(qdata).reshape(mesh.num_elem, 10, Q3)
    ws = np.asarray(width_scaling, dtype=np.float64)
    return np.array([[alpha_at(qd[e, 1:, q].reshape(3, 3), grid_based, ws, kernel_scaling) for q in range(Q3)] for e in range(mesh.num_elem)])


def apply(mesh, basis, qdata, x, nc, grid_based=False, width_scaling=(1, 1, 1), kernel_scaling=0.1, alphas=None):
    """y = (M + K_alpha) x, x and y node-interleaved [node][nc]; `alphas` from alpha_field (computed if not given)."""
    P, Q = basis.P, basis.Q
    Q3 = Q ** 3
    if alphas is None:
        alphas = alpha_field(mesh, basis, qdata, grid_based, width_scaling, kernel_scaling)
    Bq, D = tensor_ops(basis.interp1d, basis.grad1d, P, Q)
    nodes = mesh.offsets.reshape(mesh.num_elem, -1) // 5
    xe = np.asarray(x).reshape(-1, nc)[nodes]                                   # [E][P3][nc]
    V = np.einsum("qp,epc->eqc", Bq, xe)
    Gr = np.stack([np.einsum("qp,epc->eqc", Dr, xe) for Dr in D], axis=2)      # [E][Q3][3][nc]
    qd = np.asarray(qdata).reshape(mesh.num_elem, 10, Q3)
    w = qd[:, 0, :]
    X = qd[:, 1:, :].transpose(0, 2, 1).reshape(mesh.num_elem, Q3, 3, 3)
    dq = np.einsum("eqrc,eqrk->eqkc", Gr, X)                                    # physical gradient
    dqx = np.einsum("eqak,eqkc->eqac", X, dq)                                   # dXdx . grad
    gv = w[..., None, None] * np.einsum("eqab,eqbc->eqac", alphas, dqx)
    v = w[..., None] * V
    ye = np.einsum("qp,eqc->epc", Bq, v) + sum(np.einsum("qp,eqc->epc", D[r], gv[:, :, r, :]) for r in range(3))
    y = np.zeros((mesh.num_nodes, nc))
    np.add.at(y, nodes, ye)
    return y.reshape(-1)


def rhs(mesh, basis, qdata, q, gas, sv=0):
    """[node][11] = int phi (P, u, T, u_i u_j) of the state q, given in the state variable sv (0 conservative)."""
    P, Q = basis.P, basis.Q
    Q3 = Q ** 3
    Bq, _ = tensor_ops(basis.interp1d, basis.grad1d, P, Q)
    nodes = mesh.offsets.reshape(mesh.num_elem, -1) // 5
    qe = np.asarray(q).reshape(-1, 5)[nodes]
    U = np.einsum("qp,epc->eqc", Bq, qe)                          # [E][Q3][5]
    R, cv = gas.cp - gas.cv, gas.cv
    if sv == 0:
        rho, m, E = U[..., 0], U[..., 1:4], U[..., 4]
        u = m / rho[..., None]
        T = (E / rho - 0.5 * (u ** 2).sum(-1)) / cv
        Pr = rho * R * T
    else:  # StateFromQ (newtonian_state.h:393-407) at every point
        s = FaceO.state_from_q(U.reshape(-1, 5).T, sv, cv, gas.cp)
        shp = U.shape[:2]
        Pr, T = s.P.reshape(shp), s.T.reshape(shp)
        u = np.moveaxis(s.u, 0, -1).reshape(shp + (3,))
    f = np.stack([Pr, u[..., 0], u[..., 1], u[..., 2], T, u[..., 0] ** 2, u[..., 1] ** 2, u[..., 2] ** 2, u[..., 1] * u[..., 2],
                  u[..., 0] * u[..., 2], u[..., 0] * u[..., 1]], -1)
    w = np.asarray(qdata).reshape(mesh.num_elem, 10, Q3)[:, 0, :]
    out = np.zeros((mesh.num_nodes, 11))
    contrib = np.einsum("qp,eqc->epc", Bq, w[..., None] * f)
    for e in range(mesh.num_elem):
        np.add.at(out, nodes[e], contrib[e])
    return out.reshape(-1)


def training_pairs(mesh, basis, qdata, filtered, mu, R, width_scale):
    """X, Y [E*Q3][6] at every quadrature point from filtered fields [node][11]."""
    P, Q = basis.P, basis.Q
    Q3 = Q ** 3
    Bq, D = tensor_ops(basis.interp1d, basis.grad1d, P, Q)
    nodes = mesh.offsets.reshape(mesh.num_elem, -1) // 5
    fe = np.asarray(filtered).reshape(-1, 11)[nodes]
    V = np.einsum("qp,epc->eqc", Bq, fe)
    Gr = np.stack([np.einsum("qp,epc->eqc", Dr, fe[..., 1:4]) for Dr in D], axis=2)  # [E][Q3][3 dirs][3 comps]
    qd = np.asarray(qdata).reshape(mesh.num_elem, 10, Q3)
    Xs, Ys = [], []
    for e in range(mesh.num_elem):
        for q in range(Q3):
            X = qd[e, 1:, q].reshape(3, 3)
            G = Gr[e, q].T @ X                    # G[i][j] = sum_r d u_i / d xi_r * dxi_r / dx_j
            kmA, delta = SO.anisotropy(X)
            delta *= width_scale
            v = V[e, q]
            rho = v[0] / (R * v[4])
            x, E, g = SO.inputs(G, kmA, delta, mu / rho)
            u = v[1:4]
            tau = np.array([v[5] - u[0] ** 2, v[6] - u[1] ** 2, v[7] - u[2] ** 2, v[8] - u[1] * u[2], v[9] - u[0] * u[2], v[10] - u[0] * u[1]])
            Xs.append(x)
            Ys.append(SO.stress_to_sframe(tau, delta, E, g))
    return np.array(Xs), np.array(Ys)
