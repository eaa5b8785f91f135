"""CPU restatement of HONEE's nodal data-driven SGS pipeline (TEST INFRASTRUCTURE ONLY: the checker for k_sgs_nodal.cu
and for the nodal SGS operators of libceed_b200.so).

Point-wise functions, float64, vectorised over points where the reference's arithmetic allows:
  velgrad_points     VelocityGradientProjectionRHS_* (qfunctions/velocity_gradient_projection.h:9-37):
                     wdetJ du_a/dx_j of StateFromQ_fwd along the physical gradient (newtonian_state.h:511-521, 581-593)
  aniso_points       AnisotropyTensorProjection (qfunctions/grid_anisotropy_tensor.h:35-55): wdetJ (km A_ij, delta)
  closure_point      ComputeSgsDDNodal_* without the multiplicity weight (qfunctions/sgs_dd_model.h:55-96):
                     inputs (sgs_dd_utils.h:58-96), DataDrivenInference (sgs_dd_model.h:38-53), outputs (:107-127)
  sgs_flux_points    IFunction_NodalSgs_* (qfunctions/sgs_dd_model.h:205-243): -wdetJ dXdx F_sgs

Operators, restating the libCEED semantics of the operators HONEE builds (restriction gather, tensor-product basis with
the reference's interp1d / grad1d, point function, transposes, sum into the L-vector):
  velgrad_rhs        src/velocity_gradient_projection.c:61-103
  aniso_rhs          src/grid_anisotropy_tensor.c:49-69
  mass_apply / mass_diagonal   Mass_N (src/honee-mass.c:20-60, qfunctions/mass.h)
  inverse_multiplicity         src/inverse_multiplicity.c:24-80 (local multiplicity, as problems/sgs_dd_model.c:146 asks)
  sgs_nodal          problems/sgs_dd_model.c:113-200: the closure at every element node times the inverse multiplicity,
                     summed into the node
  sgs_ifunction      problems/sgs_dd_model.c:508-556
  project_cg / project_rowsum  the two L2 projections' solvers (CG + Jacobi to a natural-norm rtol,
                     src/grid_anisotropy_tensor.c:84-95; PREONLY + row-sum Jacobi, src/velocity_gradient_projection.c:118-127)
Pinned by tests/test_sgs_nodal_oracle.py against the reference QFunctions (tests/golden/sgs_nodal_points.npz, made by
tests/golden/make_sgs_nodal_golden.py).
"""
from __future__ import annotations

import numpy as np

import face_oracle as FaceO
import filter_oracle as FO
import sgs_oracle as SO


def _nodes(mesh):
    return (np.asarray(mesh.offsets).reshape(mesh.num_elem, -1) // 5).astype(np.int64)


def _qd(qdata, E, Q3):
    qd = np.asarray(qdata).reshape(E, 10, Q3)
    return qd[:, 0], qd[:, 1:].reshape(E, 3, 3, Q3)


def _gather(l, nodes, nc):
    """[E][nc][P3] from a node-interleaved L-vector of nc fields"""
    return np.asarray(l).reshape(-1, nc)[nodes].transpose(0, 2, 1)


def _scatter(e_vec, nodes, nc, num_nodes):
    """node-interleaved L-vector of nc fields = the sum of e_vec [E][nc][P3] over element nodes"""
    out = np.zeros((num_nodes, nc))
    for c in range(nc):
        np.add.at(out[:, c], nodes.reshape(-1), e_vec[:, c, :].reshape(-1))
    return out.reshape(-1)


# ---- point-wise -------------------------------------------------------------------------------------------------------

def velgrad_points(q, grad_ref, w, X, sv, cv, cp):
    """q [5][n], grad_ref [3][5][n] (reference directions), w [n], X [3][3][n] = dXdx -> v [9][n], v[a*3+j] = w du_a/dx_j"""
    s = FaceO.state_from_q(q, sv, cv, cp)
    v = np.zeros((9, q.shape[1]))
    for j in range(3):
        dq = grad_ref[0] * X[0, j] + grad_ref[1] * X[1, j] + grad_ref[2] * X[2, j]
        ds = FaceO.state_from_q_fwd(s, dq, sv, cv, cp)
        for a in range(3):
            v[a * 3 + j] = w * ds.u[a]
    return v


def aniso_points(w, X):
    """w [n], X [3][3][n] -> [7][n] = w (km A_ij (6), delta)"""
    n = w.shape[0]
    out = np.zeros((7, n))
    for i in range(n):
        kmA, delta = SO.anisotropy(X[:, :, i])
        out[:6, i] = w[i] * kmA
        out[6, i] = w[i] * delta
    return out


class Net:
    """The network of SgsDDContext_: W1 [20][6], b1, W2 [6][20], b2 (FP64) and the output bounds [6][2]."""

    def __init__(self, flat_params, bounds, alpha=0.0):
        self.params = np.asarray(flat_params, dtype=np.float64)  # flat layout W1 | b1 | W2 | b2 (sgs_oracle)
        self.bounds = np.asarray(bounds, dtype=np.float64).reshape(6, 2)
        self.alpha = float(alpha)


def closure_point(net: Net, qi, G, A7, sv, mu, cv, cp):
    """ComputeSgsDD_Fused at one node: q (5) in sv, velocity gradient G [3][3], anisotropy (km A (6), delta) -> km tau (6)"""
    s = FaceO.state_from_q(np.asarray(qi, dtype=np.float64).reshape(5, 1), sv, cv, cp)
    x, E, g = SO.inputs(np.asarray(G), np.asarray(A7[:6]), A7[6], mu / s.rho[0])
    y, _, _ = SO.forward(net.params, 20, 0, x[None, :], net.alpha)
    return SO.outputs_to_stress(y[0], A7[6], E, net.bounds, g)


def sgs_flux_points(q, km, w, X, sv, cv, cp):
    """q [5][n], km [6][n], w [n], X [3][3][n] -> Grad_v [3][5][n] = -w sum_j X[k][j] F[c][j]"""
    s = FaceO.state_from_q(q, sv, cv, cp)
    n = q.shape[1]
    r2 = 1 / np.sqrt(2.)
    tau = np.empty((3, 3, n))
    tau[0, 0], tau[1, 1], tau[2, 2] = km[0], km[1], km[2]
    tau[1, 2] = tau[2, 1] = r2 * km[3]
    tau[0, 2] = tau[2, 0] = r2 * km[4]
    tau[0, 1] = tau[1, 0] = r2 * km[5]
    F = np.zeros((5, 3, n))
    for j in range(3):
        for k in range(3):
            F[k + 1, j] = tau[k, j]
        F[4, j] = s.u[0] * tau[0, j] + s.u[1] * tau[1, j] + s.u[2] * tau[2, j]
    gv = np.zeros((3, 5, n))
    for k in range(3):
        for c in range(5):
            gv[k, c] = -w * (X[k, 0] * F[c, 0] + X[k, 1] * F[c, 1] + X[k, 2] * F[c, 2])
    return gv


# ---- operators ----------------------------------------------------------------------------------------------------------

def _ops(basis):
    return FO.tensor_ops(basis.interp1d, basis.grad1d, basis.P, basis.Q)


def velgrad_rhs(mesh, basis, qdata, q, sv, cv, cp):
    """[node][9] right-hand side of the velocity-gradient projection"""
    Bq, D = _ops(basis)
    nodes, E, Q3 = _nodes(mesh), mesh.num_elem, basis.Q ** 3
    w, X = _qd(qdata, E, Q3)
    qe = _gather(q, nodes, 5)                                            # [E][5][P3]
    qq = np.einsum("qp,ecp->ceq", Bq, qe).reshape(5, -1)
    gr = np.stack([np.einsum("qp,ecp->ceq", Dd, qe).reshape(5, -1) for Dd in D])
    v = velgrad_points(qq, gr, w.reshape(-1), X.transpose(1, 2, 0, 3).reshape(3, 3, -1), sv, cv, cp)
    ve = np.einsum("qp,ceq->ecp", Bq, v.reshape(9, E, Q3))
    return _scatter(ve, nodes, 9, mesh.num_nodes)


def aniso_rhs(mesh, basis, qdata):
    Bq, _ = _ops(basis)
    nodes, E, Q3 = _nodes(mesh), mesh.num_elem, basis.Q ** 3
    w, X = _qd(qdata, E, Q3)
    v = aniso_points(w.reshape(-1), X.transpose(1, 2, 0, 3).reshape(3, 3, -1))
    ve = np.einsum("qp,ceq->ecp", Bq, v.reshape(7, E, Q3))
    return _scatter(ve, nodes, 7, mesh.num_nodes)


def mass_apply(mesh, basis, qdata, u, nc):
    Bq, _ = _ops(basis)
    nodes, E, Q3 = _nodes(mesh), mesh.num_elem, basis.Q ** 3
    w, _ = _qd(qdata, E, Q3)
    ue = _gather(u, nodes, nc)
    uq = np.einsum("qp,ecp->ecq", Bq, ue) * w[:, None, :]
    return _scatter(np.einsum("qp,ecq->ecp", Bq, uq), nodes, nc, mesh.num_nodes)


def mass_diagonal(mesh, basis, qdata, nc):
    Bq, _ = _ops(basis)
    nodes, E, Q3 = _nodes(mesh), mesh.num_elem, basis.Q ** 3
    w, _ = _qd(qdata, E, Q3)
    d = np.einsum("qp,eq->ep", Bq * Bq, w)
    return _scatter(np.repeat(d[:, None, :], nc, axis=1), nodes, nc, mesh.num_nodes)


def inverse_multiplicity(mesh):
    """[E][P3] = 1 / (number of element nodes at the node): CeedElemRestrictionGetMultiplicity, then InverseMultiplicity"""
    nodes = _nodes(mesh)
    mult = np.bincount(nodes.reshape(-1), minlength=mesh.num_nodes).astype(np.float64)
    return 1.0 / mult[nodes]


def sgs_nodal(mesh, net: Net, q, G9, A7, inv_mult_e, sv, mu, cv, cp):
    """[node][6] = sum over element nodes of inv_mult * closure(node values) (the reference evaluates the closure at every
    element node; the values of one node are the same in every element, so they are computed once per node here)"""
    nodes = _nodes(mesh)
    q5, g9, a7 = np.asarray(q).reshape(-1, 5), np.asarray(G9).reshape(-1, 9), np.asarray(A7).reshape(-1, 7)
    cache = {}
    out = np.zeros((mesh.num_nodes, 6))
    for e in range(mesh.num_elem):
        for i, n in enumerate(nodes[e]):
            if n not in cache:
                cache[n] = closure_point(net, q5[n], g9[n].reshape(3, 3), a7[n], sv, mu, cv, cp)
            out[n] += inv_mult_e[e, i] * cache[n]
    return out.reshape(-1)


def sgs_ifunction(mesh, basis, qdata, q, km, sv, cv, cp):
    """[node][5] residual contribution of the nodal stress km [node][6]"""
    Bq, D = _ops(basis)
    nodes, E, Q3 = _nodes(mesh), mesh.num_elem, basis.Q ** 3
    w, X = _qd(qdata, E, Q3)
    qq = np.einsum("qp,ecp->ceq", Bq, _gather(q, nodes, 5)).reshape(5, -1)
    kq = np.einsum("qp,ecp->ceq", Bq, _gather(km, nodes, 6)).reshape(6, -1)
    gv = sgs_flux_points(qq, kq, w.reshape(-1), X.transpose(1, 2, 0, 3).reshape(3, 3, -1), sv, cv, cp).reshape(3, 5, E, Q3)
    ve = sum(np.einsum("qp,ceq->ecp", D[k], gv[k]) for k in range(3))
    return _scatter(ve, nodes, 5, mesh.num_nodes)


def project_rowsum(mesh, basis, qdata, rhs, nc):
    """KSPPREONLY with PC_JACOBI_ROWSUM: x = rhs / (M 1)"""
    return rhs / mass_apply(mesh, basis, qdata, np.ones(mesh.num_nodes * nc), nc)


def project_cg(mesh, basis, qdata, rhs, nc, rtol=1e-10, max_it=1000):
    """CG with the point-Jacobi preconditioner, stopped on the natural norm sqrt(r . z) relative to the first one"""
    dinv = 1.0 / mass_diagonal(mesh, basis, qdata, nc)
    x = np.zeros_like(rhs)
    r = rhs.copy()
    z = dinv * r
    p = z.copy()
    rz = float(r @ z)
    rz0 = rz
    for _ in range(max_it):
        if rz <= rtol * rtol * rz0:
            break
        Ap = mass_apply(mesh, basis, qdata, p, nc)
        a = rz / float(p @ Ap)
        x += a * p
        r -= a * Ap
        z = dinv * r
        rz_new = float(r @ z)
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x
