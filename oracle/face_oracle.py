"""CPU restatement of the free-stream boundary condition and of the face operator (TEST INFRASTRUCTURE ONLY: the checker
for k_face.cu).

Point-wise: qfunctions/riemann_solver.h (HLL / HLLC fluxes with Roe-averaged wave speeds and their forward tangents,
:22-338), qfunctions/bc_freestream.h:14-114 (v = wdetJb F, Jacobian wdetJb dF with the exterior state fixed),
qfunctions/setupgeo.h:100-117 (face qdata: w detJb, unit normal, Moore-Penrose dX/dx).  The face operator is the
libCEED face assembly (restriction of the face nodes, 2D tensor basis, transpose, sum) in numpy.  float64, vectorised over
points.  Pinned by tests/test_face_oracle.py against those reference QFunctions (tests/golden/face_points.npz).
"""
from __future__ import annotations

import numpy as np


class St:
    """Conservative state with its primitive variables, arrays over points."""

    def __init__(self, rho, m, E, P, u, T):
        self.rho, self.m, self.E, self.P, self.u, self.T = rho, m, E, P, u, T


def state_from_U(U, cv, cp):
    rho, m, E = U[0], U[1:4], U[4]
    u = m / rho
    e = E / rho - 0.5 * (u * u).sum(0)
    return St(rho, m, E, (cp / cv - 1) * rho * e, u, e / cv)


def state_from_U_fwd(s, dU, cv, cp):
    drho, dm, dE = dU[0], dU[1:4], dU[4]
    du = (dm - s.u * drho) / s.rho
    etot = s.E / s.rho
    detot = (dE - etot * drho) / s.rho
    dek = (du * s.u).sum(0)
    e = etot - 0.5 * (s.u * s.u).sum(0)
    de = detot - dek
    return St(drho, dm, dE, (cp / cv - 1) * (drho * e + s.rho * de), du, de / cv)


def state_from_q(q, sv, cv, cp):
    """StateFromQ (newtonian_state.h:393-407) over points: conservative U, primitive Y = (P, u, T) (StateFromY, :159-168),
    entropy V (StateFromV: StatePrimitiveFromEntropy :122-132, StateConservativeFromEntropy :222-238)."""
    q = np.asarray(q, dtype=np.float64)
    if sv == 0:
        return state_from_U(q, cv, cp)
    R, g = cp - cv, cp / cv
    if sv == 1:
        P, u, T = q[0], q[1:4], q[4]
        rho = P / (R * T)
        return St(rho, rho * u, rho * (cv * T + 0.5 * (u * u).sum(0)), P, u, T)
    V = q
    u = -V[1:4] / V[4]
    T = -1 / (R * V[4])
    ke = 0.5 * (u * u).sum(0)
    ent = g - (g - 1) * (V[0] - ke * V[4])
    P = np.exp(-(ent + g * np.log(-V[4])) / (g - 1))
    rho = np.exp(-(ent + np.log(-V[4])) / (g - 1))
    return St(rho, rho * u, rho * (-cv / (R * V[4]) + ke), P, u, T)


def state_from_q_fwd(s, dq, sv, cv, cp):
    """StateFromQ_fwd (newtonian_state.h:409-423) over points for the state variable sv."""
    dq = np.asarray(dq, dtype=np.float64)
    if sv == 0:
        return state_from_U_fwd(s, dq, cv, cp)
    R, g = cp - cv, cp / cv
    ke = 0.5 * (s.u * s.u).sum(0)
    if sv == 1:  # StateFromY_fwd (:170-184)
        dP, du, dT = dq[0], dq[1:4], dq[4]
        drho = (dP * s.T - s.P * dT) / (R * s.T * s.T)
        dke = (du * s.u).sum(0)
        return St(drho, drho * s.u + s.rho * du, drho * (cv * s.T + ke) + s.rho * (cv * dT + dke), dP, du, dT)
    V4 = -1 / (R * s.T)  # the entropy variable V4 of the state (StateEntropyFromPrimitive, :91-103)
    du = (-dq[1:4] - s.u * dq[4]) / V4
    dke = (du * s.u).sum(0)
    dent = -(g - 1) * (dq[0] - (dke * V4 + ke * dq[4]))
    drho = -s.rho / (g - 1) * (dent + dq[4] / V4)
    deint = cv * dq[4] / (R * V4 * V4)
    dE = drho * (-cv / (R * V4) + ke) + s.rho * (deint + dke)
    dT = dq[4] / (R * V4 * V4)
    dP = s.P * (-dent - g * dq[4] / V4) / (g - 1)
    return St(drho, drho * s.u + s.rho * du, dE, dP, du, dT)


def flux_n(s, n):
    mn = (s.m * n).sum(0)
    un = (s.u * n).sum(0)
    return np.concatenate([mn[None], mn[None] * s.u + s.P[None] * n, ((s.E + s.P) * un)[None]])


def flux_n_fwd(s, ds, n):
    mn, dmn = (s.m * n).sum(0), (ds.m * n).sum(0)
    un, dun = (s.u * n).sum(0), (ds.u * n).sum(0)
    return np.concatenate([dmn[None], dmn[None] * s.u + mn[None] * ds.u + ds.P[None] * n, ((ds.E + ds.P) * un + (s.E + s.P) * dun)[None]])


def _H(s, cv):
    return cv * s.T + 0.5 * (s.u * s.u).sum(0) + s.P / s.rho


def _dH(s, ds, cv):
    return cv * ds.T + (ds.u * s.u).sum(0) + ds.P / s.rho - s.P / s.rho ** 2 * ds.rho


def speeds(L, uL, R, uR, cv, gamma):
    ql, qr = np.sqrt(L.rho), np.sqrt(R.rho)
    wl, wr = ql / (ql + qr), qr / (ql + qr)
    u = wl * uL + wr * uR
    H = wl * _H(L, cv) + wr * _H(R, cv)
    a = np.sqrt((gamma - 1) * (H - 0.5 * u * u))
    return u - a, u + a


def speeds_fwd(L, dL, uL, duL, R, dR, uR, duR, cv, gamma):
    ql, qr = np.sqrt(L.rho), np.sqrt(R.rho)
    wl, wr = ql / (ql + qr), qr / (ql + qr)
    sq = (ql + qr) ** 2
    dwr = (ql / (2 * qr * sq)) * dR.rho - (qr / (2 * ql * sq)) * dL.rho
    dwl = (qr / (2 * ql * sq)) * dL.rho - (ql / (2 * qr * sq)) * dR.rho
    u = wl * uL + wr * uR
    du = uR * dwr + uL * dwl + wr * duR + wl * duL
    Hl, Hr = _H(L, cv), _H(R, cv)
    H = wl * Hl + wr * Hr
    dH = Hr * dwr + Hl * dwl + wr * _dH(R, dR, cv) + wl * _dH(L, dL, cv)
    a = np.sqrt((gamma - 1) * (H - 0.5 * u * u))
    da = 0.5 * np.sqrt((gamma - 1) / (H - 0.5 * u * u)) * dH - 0.5 * np.sqrt(gamma - 1) * u / np.sqrt(H - 0.5 * u * u) * du
    return u - a, du - da, u + a, du + da


def _U(s):
    return np.concatenate([s.rho[None], s.m, s.E[None]])


def _star(S, Fs, n, us, ss, sst):
    fact = S.rho * (ss - us) / (ss - sst)
    denom = S.rho * (ss - us)
    star = np.concatenate([np.ones_like(S.rho)[None], S.u + (sst - us)[None] * n, (S.E / S.rho + (sst - us) * (sst + S.P / denom))[None]])
    return Fs + (ss * fact)[None] * star - ss[None] * _U(S)


def _star_fwd(S, dS, Fs, dFs, n, us, dus, ss, dss, sst, dsst):
    fact = S.rho * (ss - us) / (ss - sst)
    dfact = (S.rho * (dss - dus) + dS.rho * (ss - us)) / (ss - sst) - fact / (ss - sst) * (dss - dsst)
    denom = S.rho * (ss - us)
    ddenom = S.rho * (dss - dus) + dS.rho * (ss - us)
    star = np.concatenate([np.ones_like(S.rho)[None], S.u + (sst - us)[None] * n, (S.E / S.rho + (sst - us) * (sst + S.P / denom))[None]])
    dstar = np.concatenate([np.zeros_like(S.rho)[None], dS.u + (dsst - dus)[None] * n,
                            (dS.E / S.rho - S.E / S.rho ** 2 * dS.rho + (dsst - dus) * (sst + S.P / denom)
                             + (sst - us) * (dsst + dS.P / denom - S.P / denom ** 2 * ddenom))[None]])
    return dFs + (dss * fact + ss * dfact)[None] * star + (ss * fact)[None] * dstar - dss[None] * _U(S) - ss[None] * _U(dS)


def riemann(L, R, n, cv, cp, hllc=True, dL=None, dR=None):
    """Flux F (and, with dL/dR, its tangent dF) through normal n between interior L and exterior R."""
    gamma = cp / cv
    Fl, Fr = flux_n(L, n), flux_n(R, n)
    uL, uR = (L.u * n).sum(0), (R.u * n).sum(0)
    tangent = dL is not None
    if tangent:
        dFl, dFr = flux_n_fwd(L, dL, n), flux_n_fwd(R, dR, n)
        duL, duR = (dL.u * n).sum(0), (dR.u * n).sum(0)
        sl, dsl, sr, dsr = speeds_fwd(L, dL, uL, duL, R, dR, uR, duR, cv, gamma)
    else:
        sl, sr = speeds(L, uL, R, uR, cv, gamma)
    out = np.zeros_like(Fl)
    if not hllc:
        Ul, Ur = _U(L), _U(R)
        mid = (sr - sl)
        if not tangent:
            hllv = (sr * Fl - sl * Fr + sl * sr * (Ur - Ul)) / mid
            return np.where(0 <= sl, Fl, np.where(sr <= 0, Fr, hllv))
        dUl, dUr = _U(dL), _U(dR)
        v = (sl * (-Fl + Fr + sl * Ul - sl * Ur) / mid ** 2) * dsr + (sr * (Fl - Fr - sr * Ul + sr * Ur) / mid ** 2) * dsl \
            + (sr * dFl - sl * dFr + sr * sl * (dUr - dUl)) / mid
        return np.where(0 <= sl, dFl, np.where(sr <= 0, dFr, v))
    rl, rr = L.rho * uL, R.rho * uR
    numer = R.P - L.P + rl * (sl - uL) - rr * (sr - uR)
    denom = L.rho * (sl - uL) - R.rho * (sr - uR)
    sst = numer / denom
    if not tangent:
        starL = _star(L, Fl, n, uL, sl, sst)
        starR = _star(R, Fr, n, uR, sr, sst)
        return np.where(0 <= sl, Fl, np.where(0 <= sst, starL, np.where(0 <= sr, starR, Fr)))
    drl, drr = L.rho * duL + dL.rho * uL, R.rho * duR + dR.rho * uR
    dnumer = dR.P - dL.P + rl * (dsl - duL) + drl * (sl - uL) - rr * (dsr - duR) - drr * (sr - uR)
    ddenom = L.rho * (dsl - duL) + dL.rho * (sl - uL) - R.rho * (dsr - duR) - dR.rho * (sr - uR)
    dsst = dnumer / denom - numer / denom ** 2 * ddenom
    dstarL = _star_fwd(L, dL, Fl, dFl, n, uL, duL, sl, dsl, sst, dsst)
    dstarR = _star_fwd(R, dR, Fr, dFr, n, uR, duR, sr, dsr, sst, dsst)
    return np.where(0 <= sl, dFl, np.where(0 <= sst, dstarL, np.where(0 <= sr, dstarR, dFr)))


def exterior(U_inf, Y_inf, npts):
    U = np.asarray(U_inf, dtype=np.float64)[:, None] * np.ones(npts)
    Y = np.asarray(Y_inf, dtype=np.float64)[:, None] * np.ones(npts)
    return St(U[0], U[1:4], U[4], Y[0], Y[1:4], Y[4])


def face_qdata(interp1d, grad1d, qweight1d, P, Q, x_nodes):
    """[F][10][Q^2] from face node coordinates [F][3][P^2]."""
    B = np.asarray(interp1d).reshape(Q, P)
    G = np.asarray(grad1d).reshape(Q, P)
    D0 = np.einsum("jb,ia->jiba", B, G).reshape(Q * Q, P * P)   # d/dX0 (X0 fastest in both orders)
    D1 = np.einsum("jb,ia->jiba", G, B).reshape(Q * Q, P * P)
    w = np.outer(qweight1d, qweight1d).reshape(-1)
    F = x_nodes.shape[0]
    J0 = np.einsum("qp,fdp->fdq", D0, x_nodes)
    J1 = np.einsum("qp,fdp->fdq", D1, x_nodes)
    N = np.cross(J0, J1, axis=1)
    detJb = np.linalg.norm(N, axis=1)
    out = np.zeros((F, 10, Q * Q))
    out[:, 0] = w[None] * detJb
    out[:, 1:4] = N / detJb[:, None]
    a, c, b = (J0 * J0).sum(1), (J1 * J1).sum(1), (J0 * J1).sum(1)
    det = a * c - b * b
    inv = np.array([[c / det, -b / det], [-b / det, a / det]])       # [2][2][F][Q2]
    for i in range(2):
        for j in range(3):
            out[:, 4 + i * 3 + j] = inv[i, 0] * J0[:, j] + inv[i, 1] * J1[:, j]
    return out


def freestream_apply(offsets, interp1d, P, Q, qdata_sur, q, U_inf, Y_inf, cv, cp, hllc=True, dq=None, jac=None, l_size=None, sv=0):
    """Residual contribution (dq None) or Jacobian action (dq given, jac = q at the face points) as an L-vector; q, dq and
    jac in the state variable sv (Freestream_{Conserv,Prim,Entropy}, bc_freestream.h:54-76)."""
    B = np.asarray(interp1d).reshape(Q, P)
    Bq = np.einsum("jb,ia->jiba", B, B).reshape(Q * Q, P * P)
    F = offsets.shape[0]
    qv = np.asarray(q).reshape(-1, 5)
    out = np.zeros(l_size if l_size is not None else qv.size)
    nodes = offsets // 5
    for f in range(F):
        src = np.asarray(dq).reshape(-1, 5)[nodes[f]] if dq is not None else qv[nodes[f]]
        Uq = (Bq @ src).T                                                 # [5][Q2]
        n = qdata_sur[f, 1:4]
        if dq is None:
            s = state_from_q(Uq, sv, cv, cp)
            flux = riemann(s, exterior(U_inf, Y_inf, Q * Q), n, cv, cp, hllc)
        else:
            s = state_from_q(jac[f], sv, cv, cp)
            ds = state_from_q_fwd(s, Uq, sv, cv, cp)
            zero = St(*(np.zeros(Q * Q) if k not in (1, 4) else np.zeros((3, Q * Q)) for k in range(6)))
            flux = riemann(s, exterior(U_inf, Y_inf, Q * Q), n, cv, cp, hllc, dL=ds, dR=zero)
        v = qdata_sur[f, 0][None] * flux
        contrib = (Bq.T @ v.T)                                            # [P2][5]
        for p in range(P * P):
            out[offsets[f, p]:offsets[f, p] + 5] += contrib[p]
    return out


def freestream_diagonal(offsets, interp1d, P, Q, qdata_sur, jac, U_inf, Y_inf, cv, cp, hllc=True, l_size=None, sv=0):
    """Diagonal of the free-stream Jacobian as an L-vector: for face node p and component c, the sum over the face's
    points of B_p^2 wdetJb dF_c/dU_c, the column of the point Jacobian taken by the forward tangent with dU = e_c (the
    libCEED diagonal assembly of the Freestream_Jacobian operator, bc_freestream.h:75-114, summed over faces)."""
    B = np.asarray(interp1d).reshape(Q, P)
    Bq = np.einsum("jb,ia->jiba", B, B).reshape(Q * Q, P * P)
    F = offsets.shape[0]
    out = np.zeros(l_size if l_size is not None else int(offsets.max()) + 5)
    zero = St(*(np.zeros(Q * Q) if k not in (1, 4) else np.zeros((3, Q * Q)) for k in range(6)))
    for f in range(F):
        s = state_from_q(jac[f], sv, cv, cp)
        n = qdata_sur[f, 1:4]
        D = np.zeros((5, Q * Q))
        for c in range(5):
            dU = np.zeros((5, Q * Q))
            dU[c] = 1.0
            ds = state_from_q_fwd(s, dU, sv, cv, cp)
            D[c] = qdata_sur[f, 0] * riemann(s, exterior(U_inf, Y_inf, Q * Q), n, cv, cp, hllc, dL=ds, dR=zero)[c]
        contrib = (Bq.T ** 2) @ D.T                                          # [P2][5]
        for p in range(P * P):
            out[offsets[f, p]:offsets[f, p] + 5] += contrib[p]
    return out


def freestream_point_block(offsets, interp1d, P, Q, qdata_sur, jac, U_inf, Y_inf, cv, cp, hllc=True, l_size=None, sv=0):
    """5 x 5 point blocks of the free-stream Jacobian, out[(node * 5 + i) * 5 + j] = sum over a node's face points of
    B_p^2 wdetJb dF_i/dU_j (the point-block assembly of the Freestream_Jacobian operator, summed over faces)."""
    B = np.asarray(interp1d).reshape(Q, P)
    Bq = np.einsum("jb,ia->jiba", B, B).reshape(Q * Q, P * P)
    n_l = l_size if l_size is not None else int(offsets.max()) + 5
    out = np.zeros(5 * n_l)
    zero = St(*(np.zeros(Q * Q) if k not in (1, 4) else np.zeros((3, Q * Q)) for k in range(6)))
    for f in range(offsets.shape[0]):
        s = state_from_q(jac[f], sv, cv, cp)
        n = qdata_sur[f, 1:4]
        D = np.zeros((5, 5, Q * Q))                                             # [i][j][point]
        for j in range(5):
            dU = np.zeros((5, Q * Q))
            dU[j] = 1.0
            ds = state_from_q_fwd(s, dU, sv, cv, cp)
            D[:, j] = qdata_sur[f, 0] * riemann(s, exterior(U_inf, Y_inf, Q * Q), n, cv, cp, hllc, dL=ds, dR=zero)
        contrib = np.einsum("kp,ijk->pij", Bq ** 2, D)                          # [P2][5][5]
        for p in range(P * P):
            o = offsets[f, p] * 5
            out[o:o + 25] += contrib[p].reshape(-1)
    return out
