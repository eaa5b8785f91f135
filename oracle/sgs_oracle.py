"""CPU restatement of the learned subgrid-stress closure (TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels).

Follows, point by point:
  * qfunctions/utils_eigensolver_jacobi.h:26-173  max-pivot Jacobi eigen-solver (Diagonalize3), descending sort
  * qfunctions/grid_anisotropy_tensor.h:14-32     AnisotropyTensor (A_ij = Delta_ij / |Delta|, delta = 2 |Delta|)
  * qfunctions/sgs_dd_utils.h:58-96               ComputeSgsDDInputs, OrientBasisWithVector, VelocityGradientMagnitude
  * qfunctions/sgs_dd_utils.h:38-44, 107-127      DenormalizeDDOutputs, ComputeSgsDDOutputs
  * qfunctions/sgs_dd_model.h:38-53               DataDrivenInference (V = b1 + W1 x, leaky ReLU, out = b2 + W2 V)
  * qfunctions/sgs_dd_training.h:22-56            training pairs: model inputs and filtered u_i u_j - u_i u_j
and, for training (which the reference does outside HONEE), the published algorithms the CUDA kernels implement:
mean-squared-error back-propagation through the network and Adam (Kingma & Ba, 2015).  float64 throughout.
Pinned by tests/test_sgs_oracle.py against the reference QFunctions compiled in oracle/_ref and against the committed
golden fixture tests/golden/sgs_points.npz.
"""
from __future__ import annotations

import math

import numpy as np

EPS = 2.220446049250313e-16


def km_unpack(v):
    w = 1 / math.sqrt(2.)
    return np.array([[v[0], w * v[5], w * v[4]], [w * v[5], v[1], w * v[3]], [w * v[4], w * v[3], v[2]]])


def km_pack(A):
    w = math.sqrt(2.)
    return np.array([A[0, 0], A[1, 1], A[2, 2], A[2, 1] * w, A[2, 0] * w, A[1, 0] * w])


def eig3(A, max_sweeps):
    """Max-pivot Jacobi on a symmetric 3x3 matrix; eigenvalues descending, eigenvectors as rows."""
    A = np.array(A, dtype=np.float64, copy=True)
    E = np.eye(3)
    pairs = [(0, 1), (0, 2), (1, 2)]
    for _ in range(max_sweeps * 3):
        # pivot: largest |A_ij|, i < j; ties keep the earlier pair
        i, j = pairs[0]
        m = abs(A[0, 1])
        for (a, b) in pairs[1:]:
            if abs(A[a, b]) > m:
                i, j, m = a, b, abs(A[a, b])
        if A[i, i] + A[i, j] == A[i, i] and A[j, j] + A[i, j] == A[j, j]:
            A[i, j] = 0.0
        if A[i, j] == 0.0:
            break
        t = 1.0
        d = A[j, j] - A[i, i]
        if d != 0.0:
            kappa = d / (2.0 * A[i, j])
            t = 1.0 / (math.sqrt(1 + kappa * kappa) + abs(kappa))
            if kappa < 0:
                t = -t
        c = 1.0 / math.sqrt(1 + t * t)
        s = c * t
        A[i, i] -= t * A[i, j]
        A[j, j] += t * A[i, j]
        A[i, j] = 0.0
        w = 3 - i - j
        wi, wj = (min(w, i), max(w, i)), (min(w, j), max(w, j))
        a_wi, a_wj = A[wi], A[wj]
        A[wi] = c * a_wi - s * a_wj
        A[wj] = s * a_wi + c * a_wj
        ei = E[i].copy()
        E[i] = c * ei - s * E[j]
        E[j] = s * ei + c * E[j]
    ev = np.array([A[0, 0], A[1, 1], A[2, 2]])
    for a in range(2):  # selection sort, descending
        am = a
        for b in range(a + 1, 3):
            if ev[b] > ev[am]:
                am = b
        ev[[a, am]] = ev[[am, a]]
        E[[a, am]] = E[[am, a]]
    return ev, E


def anisotropy(dXdx):
    g = km_unpack(km_pack(dXdx.T @ dXdx))
    ev, E = eig3(g, 15)
    ev = 1 / np.sqrt(ev)
    A = E.T @ (ev[:, None] * E)
    delta = math.sqrt(float(ev @ ev))
    A = A * (1 / delta)
    return km_pack(A), 2 * delta


def inputs(G, km_A, delta, nu):
    """Model inputs (6), eigenframe E (rows) and |G A|."""
    Gi = G @ km_unpack(km_A)
    w = 1 / math.sqrt(2.)
    km_s = np.array([Gi[0, 0], Gi[1, 1], Gi[2, 2], w * (Gi[1, 2] + Gi[2, 1]), w * (Gi[0, 2] + Gi[2, 0]), w * (Gi[0, 1] + Gi[1, 0])])
    sf, E = eig3(km_unpack(km_s), 5)
    R = 0.5 * (Gi - Gi.T)
    vort = np.array([-2 * R[1, 2], 2 * R[0, 2], -2 * R[0, 1]])
    al = E @ vort
    if al[0] < 0:
        E[0] = -E[0]
    if al[2] < 0:
        E[2] = -E[2]
    if np.cross(E[2], E[0]) @ E[1] < 0:
        E[1] = -E[1]
    wf = E @ vort
    gmag = math.sqrt(float(sf @ sf + 0.5 * wf @ wf))
    x = np.array([sf[0], sf[1], sf[2], wf[0], wf[1], nu / delta ** 2]) / (gmag + EPS)
    return x, E, gmag


def outputs_to_stress(out_n, delta, E, bounds, gmag):
    b = np.asarray(bounds, dtype=np.float64).reshape(6, 2)
    o = (b[:, 1] - b[:, 0]) * (np.asarray(out_n) - 1) + b[:, 1]
    o = o * delta ** 2 * gmag ** 2
    S = np.array([[o[0], o[3], o[4]], [o[3], o[1], o[5]], [o[4], o[5], o[2]]])
    return km_pack(E.T @ S @ E)


def stress_to_sframe(tau6, delta, E, gmag):
    tau = np.array([[tau6[0], tau6[5], tau6[4]], [tau6[5], tau6[1], tau6[3]], [tau6[4], tau6[3], tau6[2]]])
    S = E @ tau @ E.T / (delta ** 2 * gmag ** 2 + 1e-300)
    return np.array([S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[0, 2], S[1, 2]])


# ---- network: flat parameters, per layer W [out][in] row-major then b [out]

def shapes(h1, h2):
    dims = [6, h1] + ([h2] if h2 else []) + [6]
    return list(zip(dims[:-1], dims[1:]))


def unpack(params, h1, h2):
    out, o = [], 0
    for (nin, nout) in shapes(h1, h2):
        W = params[o:o + nin * nout].reshape(nout, nin)
        o += nin * nout
        b = params[o:o + nout]
        o += nout
        out.append((W, b))
    assert o == len(params)
    return out


def forward(params, h1, h2, X, alpha=0.0):
    """X [n][6] -> Y [n][6]; also the pre-activations and activations of every layer."""
    layers = unpack(np.asarray(params, dtype=np.float64), h1, h2)
    acts, zs = [np.asarray(X, dtype=np.float64)], []
    for k, (W, b) in enumerate(layers):
        z = acts[-1] @ W.T + b
        zs.append(z)
        acts.append(z if k == len(layers) - 1 else np.where(z < 0, alpha * z, z))
    return acts[-1], acts, zs


def loss_and_grad(params, h1, h2, X, Y, alpha=0.0):
    """MSE over samples and the 6 outputs and its gradient with respect to the flat parameters."""
    y, acts, zs = forward(params, h1, h2, X, alpha)
    n = X.shape[0]
    e = y - Y
    loss = float((e ** 2).sum() / (6 * n))
    d = 2 * e / (6 * n)
    layers = unpack(np.asarray(params, dtype=np.float64), h1, h2)
    grads = [None] * len(layers)
    for k in range(len(layers) - 1, -1, -1):
        W, _ = layers[k]
        grads[k] = (d.T @ acts[k], d.sum(0))
        if k > 0:
            d = (d @ W) * np.where(zs[k - 1] < 0, alpha, 1.0)
    flat = np.concatenate([np.concatenate([gW.reshape(-1), gb]) for gW, gb in grads])
    return loss, flat


def adam_step(params, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v


def reference_layout_to_flat(b1, b2, w1_file, w2_file):
    """The reference's weight files (w1.dat [6][20], w2.dat [20][6], problems/sgs_dd_model.c:631-644 transposes them) to
    the flat layout W1 [20][6], b1, W3 [6][20], b2."""
    W1 = np.asarray(w1_file).reshape(6, 20).T
    W2 = np.asarray(w2_file).reshape(20, 6).T
    return np.concatenate([W1.reshape(-1), np.asarray(b1)[:20], W2.reshape(-1), np.asarray(b2)[:6]])


def residual_contribution(mesh, basis, qdata, q, gas, params, h1, h2, bounds, alpha=0.0, float32_net=True, sv=0):
    """Nodal residual contribution of the closure's flux (IFunction_NodalSgs, sgs_dd_model.h:219-241, with the stress of
    ComputeSgsDD_Fused evaluated at the quadrature points).  float32_net rounds the network's inputs, weights and
    outputs to float32 the way the CUDA kernel evaluates it (FP64 everywhere else).  q in the state variable sv
    (StateFromQ and its tangent give the density, velocity and velocity gradient at each point)."""
    import face_oracle as FaceO
    import filter_oracle as FO
    P, Q = basis.P, basis.Q
    Q3 = Q ** 3
    Bq, D = FO.tensor_ops(basis.interp1d, basis.grad1d, P, Q)
    nodes = mesh.offsets.reshape(mesh.num_elem, -1) // 5
    qe = np.asarray(q).reshape(-1, 5)[nodes]
    U = np.einsum("qp,epc->eqc", Bq, qe)
    Gr = np.stack([np.einsum("qp,epc->eqc", Dr, qe) for Dr in D], axis=2)      # [E][Q3][3 dirs][5]
    qd = np.asarray(qdata).reshape(mesh.num_elem, 10, Q3)
    w32 = np.asarray(params, dtype=np.float32).astype(np.float64) if float32_net else np.asarray(params, dtype=np.float64)
    out = np.zeros((mesh.num_nodes, 5))
    for e in range(mesh.num_elem):
        gv = np.zeros((Q3, 3, 5))
        for k in range(Q3):
            X = qd[e, 1:, k].reshape(3, 3)
            if sv == 0:
                rho, m = U[e, k, 0], U[e, k, 1:4]
                u = m / rho
                du_ref = (Gr[e, k][:, 1:4] - np.outer(Gr[e, k][:, 0], u)) / rho   # [dir][comp] d u / d xi
            else:
                st = FaceO.state_from_q(U[e, k][:, None], sv, gas.cv, gas.cp)
                rho, u = st.rho[0], st.u[:, 0]
                du_ref = np.stack([FaceO.state_from_q_fwd(st, Gr[e, k][r][:, None], sv, gas.cv, gas.cp).u[:, 0] for r in range(3)])
            G = du_ref.T @ X
            kmA, delta = anisotropy(X)
            x, E, g = inputs(G, kmA, delta, gas.mu / rho)
            if float32_net:
                x = x.astype(np.float32).astype(np.float64)
            y, _, _ = forward(w32, h1, h2, x[None, :], alpha)
            if float32_net:
                y = y.astype(np.float32).astype(np.float64)
            km = outputs_to_stress(y[0], delta, E, np.asarray(bounds, dtype=np.float32).astype(np.float64), g)
            tau = km_unpack(km)
            F = np.zeros((5, 3))
            F[1:4] = tau
            F[4] = u @ tau
            gv[k] = -qd[e, 0, k] * (X @ F.T)          # [dir][comp]
        ye = sum(D[r].T @ gv[:, r, :] for r in range(3))
        np.add.at(out, nodes[e], ye)
    return out.reshape(-1)
