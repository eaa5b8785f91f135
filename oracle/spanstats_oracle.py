"""CPU restatement of HONEE's spanwise turbulence statistics (TEST INFRASTRUCTURE ONLY: the checker for k_stats.cu and
hb_stats.c).

Follows the reference step by step, without the GPU's column structure:
  stats_point        ChildStatsCollection (qfunctions/spanstats/turbulence.h:41-79) with StateFromU
                     (qfunctions/newtonian_state.h:64-73); pinned bit for bit by tests/test_spanstats_oracle.py against
                     the reference's ChildStatsCollection_Conserv compiled in oracle/_ref
  collect_child      the collection operator (src/spanstats/turbulence.c:19-108): interpolate the state to every child
                     quadrature point, w detJ * (t - t_prev) * stats, added into the child array [E][Q^3][22]
  star_forest        PetscSFSetGraphFromCoordinates on the (x, y) of the child and parent quadrature points with
                     tolerance 1e-12 (src/spanstats/spanstats.c:253-289), then the MPI_SUM reduction (:425-443)
  process            scale by 1 / (duration * span width), B^T onto the parent nodes, solve with the parent mass matrix
                     (:445-455; solved directly here, the reference's CG stops at rtol 1e-10)
"""
from __future__ import annotations

import numpy as np

import face_oracle as FaceO
import filter_oracle as FO
import oracle as O

NS = 22


def stats_point(U, cv, cp):
    """U [5][n] -> v [22][n] unweighted statistics (the reference multiplies by w detJ * dt first; see stats_weighted)."""
    return stats_weighted(U, np.ones(np.asarray(U).shape[1]), cv, cp)


def stats_weighted(U, w, cv, cp):
    """turbulence.h:51-77 with wdetJ = w, products associated left to right as written there."""
    U = np.asarray(U, dtype=np.float64)
    rho = U[0]
    u = U[1:4] / rho
    e_kinetic = .5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
    e_internal = U[4] / rho - e_kinetic
    T = e_internal / cv
    p = (cp / cv - 1) * rho * e_internal
    v = np.empty((NS, U.shape[1]))
    v[0] = w * rho
    v[1] = w * p
    v[2] = w * (p * p)
    for i in range(3):
        v[3 + i] = w * p * u[i]
    v[6] = w * rho * T
    for i in range(3):
        v[7 + i] = w * rho * T * u[i]
        v[10 + i] = w * U[1 + i]
    v[13] = w * U[1] * u[0]
    v[14] = w * U[2] * u[1]
    v[15] = w * U[3] * u[2]
    v[16] = w * U[2] * u[2]
    v[17] = w * U[1] * u[2]
    v[18] = w * U[1] * u[1]
    for i in range(3):
        v[19 + i] = w * u[i]
    return v


def stats_state(s, w):
    """ChildStatsCollection_Prim / _Entropy (turbulence.h:85-91): the statistics of a state already converted (StateFromQ)."""
    v = np.empty((NS, np.asarray(s.rho).size))
    v[0] = w * s.rho
    v[1] = w * s.P
    v[2] = w * (s.P * s.P)
    for i in range(3):
        v[3 + i] = w * s.P * s.u[i]
    v[6] = w * s.rho * s.T
    for i in range(3):
        v[7 + i] = w * s.rho * s.T * s.u[i]
        v[10 + i] = w * s.m[i]
    v[13] = w * s.m[0] * s.u[0]
    v[14] = w * s.m[1] * s.u[1]
    v[15] = w * s.m[2] * s.u[2]
    v[16] = w * s.m[1] * s.u[2]
    v[17] = w * s.m[0] * s.u[2]
    v[18] = w * s.m[0] * s.u[1]
    for i in range(3):
        v[19 + i] = w * s.u[i]
    return v


def collect_child(mesh, basis, qdata, q, cv, cp, dt, child=None, sv=0):
    """child [E][Q^3][22] (+)= w detJ * dt * stats(B q_e) (the collocated child restriction is [elem][qpt][comp]); q in the
    state variable sv."""
    P, Q = basis.P, basis.Q
    Q3 = Q ** 3
    Bq, _ = FO.tensor_ops(basis.interp1d, basis.grad1d, P, Q)
    nodes = np.asarray(mesh.offsets).reshape(mesh.num_elem, -1) // 5
    qd = np.asarray(qdata).reshape(mesh.num_elem, 10, Q3)
    qn = np.asarray(q).reshape(-1, 5)
    if child is None:
        child = np.zeros((mesh.num_elem, Q3, NS))
    for e in range(mesh.num_elem):
        Uq = Bq @ qn[nodes[e]]                # [Q3][5]
        wdt = qd[e, 0] * dt
        if sv == 0:
            child[e] += stats_weighted(Uq.T, wdt, cv, cp).T
        else:
            child[e] += stats_state(FaceO.state_from_q(Uq.T, sv, cv, cp), wdt).T
    return child


def parent_points(parent_x, Q, qref1d, qweight1d):
    """Bilinear map of the parent elements: (x, y) of the points [E2][Q^2][2] and w detJ [E2][Q^2] (point qi + Q qj)."""
    E2 = parent_x.shape[0]
    xi = np.asarray(qref1d)
    XI, ETA = np.meshgrid(xi, xi, indexing="xy")
    XI, ETA = XI.reshape(-1), ETA.reshape(-1)
    W = np.outer(qweight1d, qweight1d).reshape(-1)  # [qj][qi] order: w_qj * w_qi
    N = np.stack([(1 - XI) * (1 - ETA), (1 + XI) * (1 - ETA), (1 - XI) * (1 + ETA), (1 + XI) * (1 + ETA)]) / 4  # [4][Q2]
    dNx = np.stack([-(1 - ETA), (1 - ETA), -(1 + ETA), (1 + ETA)]) / 4
    dNe = np.stack([-(1 - XI), -(1 + XI), (1 - XI), (1 + XI)]) / 4
    xy = np.einsum("ecv,vq->eqc", parent_x[:, :2], N)
    Jx = np.einsum("ecv,vq->eqc", parent_x, dNx)
    Je = np.einsum("ecv,vq->eqc", parent_x, dNe)
    wdetJ = W[None, :] * np.linalg.norm(np.cross(Jx, Je), axis=-1)
    return xy, wdetJ


def star_forest(child_xy, parent_xy, tol=1e-12):
    """Index of the parent point each child point sums into, matched on (x, y) within tol (every child must match one)."""
    cx = np.asarray(child_xy).reshape(-1, 2)
    px = np.asarray(parent_xy).reshape(-1, 2)
    match = np.full(cx.shape[0], -1, dtype=np.int64)
    for s in range(0, cx.shape[0], 4096):
        d = np.abs(cx[s:s + 4096, None, :] - px[None, :, :]).max(axis=-1)
        hit = d <= tol
        n_hit = hit.sum(axis=1)
        if np.any(n_hit != 1):
            raise ValueError("child quadrature point without exactly one parent point")
        match[s:s + 4096] = hit.argmax(axis=1)
    return match


def reduce_to_parent(child, match, num_parent_points):
    out = np.zeros((num_parent_points, NS))
    np.add.at(out, match, np.asarray(child).reshape(-1, NS))
    return out


def plane_operators(parent_offsets, num_nodes, interp1d, P, Q, wdetJ):
    """Dense-free parent operators: Bt (B^T assembly matrix [nodes][E2*Q^2]) and the mass matrix M [nodes][nodes]."""
    import scipy.sparse as sp
    B = np.asarray(interp1d).reshape(Q, P)
    B2 = np.einsum("jb,ia->jiba", B, B).reshape(Q * Q, P * P)  # point qi + Q qj, node a + P b: B[qj][b] B[qi][a]
    E2 = parent_offsets.shape[0]
    rows, cols, vals = [], [], []
    for e in range(E2):
        for qp in range(Q * Q):
            rows.append(parent_offsets[e])
            cols.append(np.full(P * P, e * Q * Q + qp))
            vals.append(B2[qp])
    Bt = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(num_nodes, E2 * Q * Q))
    Wd = sp.diags(np.asarray(wdetJ).reshape(-1))
    M = (Bt @ Wd @ Bt.T).tocsc()
    return Bt, M


def process(parent_sums, duration, span_width, parent_offsets, num_nodes, interp1d, P, Q, wdetJ):
    """stats [nodes][22] = M^{-1} B^T (parent_sums / (duration * span_width))."""
    import scipy.sparse.linalg as spla
    Bt, M = plane_operators(parent_offsets, num_nodes, interp1d, P, Q, wdetJ)
    rhs = Bt @ (np.asarray(parent_sums).reshape(-1, NS) / (duration * span_width))
    lu = spla.splu(M)
    return np.stack([lu.solve(rhs[:, c]) for c in range(NS)], axis=1)


def child_points_xy(mesh, Q):
    """(x, y) of every child quadrature point [E][Q^3][2] (trilinear coordinate field)."""
    xq = O.coords_at_qpts(mesh.num_elem, Q, mesh.x_elem).reshape(mesh.num_elem, 3, Q ** 3)
    return np.transpose(xq[:, :2], (0, 2, 1))
