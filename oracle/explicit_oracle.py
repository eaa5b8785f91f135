"""CPU restatement of HONEE's explicit time loop (TEST INFRASTRUCTURE ONLY: the checker for hb_explicit.c).

RHS_NS (src/setupts.c:31-75): G = M^-1 RHS(q), RHS from the RHSFunction_Newtonian operator (oracle.apply_rhs), M the
Mass_5 operator (oracle.apply_mass) inverted by the "mass_" KSP of CreateKSPMass (src/setuplibceed.c:55-93): KSPPREONLY
with PCJacobi row sums ("lumped", the default) or KSPGMRES with PCJacobi; PETSc's defaults for GMRES are restated here
(left preconditioning, preconditioned residual norm, zero initial guess, classical Gram-Schmidt, restart 30, rtol 1e-5,
atol 1e-50).  PETSc's TSRK tableaux (TSRK1FE, TSRK2A, TSRK3, TSRK3BS, TSRK4, TSRK5F) are the published Butcher tables (5F: Fehlberg's pair with
its fifth-order weights).  Essential DOFs are removed from the system as DMPlex constraints do (values in the state, zero rows
in the right-hand side, the mass solved on the free DOFs); free-stream faces add -wdetJb F (the explicit Freestream QFunction,
bc_freestream.h:45-48).

PETSc itself is not present here; the restatement is pinned by the reference's own run of this path:
tests/output/taylorgreen_totalke.csv (kinetic-energy rows at steps 0, 2, 3) and tests/output/taylor-green.bin (the
final state), both made by examples/navierstokes.c:222 and carried in tests/golden/taylorgreen_rk4.npz.
"""
from __future__ import annotations

import numpy as np

import oracle as O

TABLEAUX = {  # name -> (A, b, c)
    "1fe": ([[0.0]], [1.0], [0.0]),
    "2a": ([[0, 0], [1.0, 0]], [0.5, 0.5], [0, 1.0]),
    "3": ([[0, 0, 0], [0.5, 0, 0], [-1.0, 2.0, 0]], [1 / 6, 2 / 3, 1 / 6], [0, 0.5, 1.0]),
    "3bs": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.75, 0, 0], [2 / 9, 1 / 3, 4 / 9, 0]], [2 / 9, 1 / 3, 4 / 9, 0], [0, 0.5, 0.75, 1.0]),
    "4": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.5, 0, 0], [0, 0, 1.0, 0]], [1 / 6, 1 / 3, 1 / 3, 1 / 6], [0, 0.5, 0.5, 1.0]),
    "5f": ([[0, 0, 0, 0, 0, 0], [1 / 4, 0, 0, 0, 0, 0], [3 / 32, 9 / 32, 0, 0, 0, 0], [1932 / 2197, -7200 / 2197, 7296 / 2197, 0, 0, 0],
            [439 / 216, -8, 3680 / 513, -845 / 4104, 0, 0], [-8 / 27, 2, -3544 / 2565, 1859 / 4104, -11 / 40, 0]],
           [16 / 135, 0, 6656 / 12825, 28561 / 56430, -9 / 50, 2 / 55], [0, 1 / 4, 3 / 8, 12 / 13, 1, 1 / 2]),
}


def mass_diagonal(mesh: O.Mesh, P, Q, qdata, l_size):
    """diag(M): sum over each element's points of (B3[q, p])^2 w detJ_q, the same for the five components."""
    B = np.asarray(mesh.interp1d).reshape(Q, P)
    B3 = np.einsum("ka,jb,ic->kjicba", B, B, B).reshape(Q ** 3, P ** 3)  # x fastest in both orders
    E = mesh.offsets.size // P ** 3
    w = np.asarray(qdata).reshape(E, 10, Q ** 3)[:, 0]
    de = w @ (B3 ** 2)                                                   # [E][P3]
    d = np.zeros(l_size)
    off = mesh.offsets.reshape(E, P ** 3)
    for c in range(5):
        np.add.at(d, off + c, de)
    return d


def gmres_left(apply_A, dinv, b, rtol=1e-5, atol=1e-50, restart=30, max_it=10000):
    """KSPGMRES with left preconditioning by dinv (PETSc defaults).  Returns (x, its, reason)."""
    x = np.zeros_like(b)
    r = dinv * b
    beta = np.linalg.norm(r)
    ttol = max(rtol * beta, atol)
    its = 0
    if beta <= ttol or beta == 0:
        return x, 0, 1
    while True:
        m = restart
        V = np.zeros((m + 1, b.size))
        H = np.zeros((m + 1, m))
        cs, sn, g = np.zeros(m), np.zeros(m), np.zeros(m + 1)
        V[0] = r / beta
        g[0] = beta
        k, done, reason = 0, False, -2
        while k < m and its < max_it:
            w = dinv * apply_A(V[k])
            h = V[:k + 1] @ w
            w = w - V[:k + 1].T @ h
            hn = np.linalg.norm(w)
            H[:k + 1, k] = h
            H[k + 1, k] = hn
            if hn > 0:
                V[k + 1] = w / hn
            for i in range(k):
                a, c = H[i, k], H[i + 1, k]
                H[i, k], H[i + 1, k] = cs[i] * a + sn[i] * c, -sn[i] * a + cs[i] * c
            a, c = H[k, k], H[k + 1, k]
            rr = np.hypot(a, c)
            cs[k], sn[k] = (a / rr, c / rr) if rr > 0 else (1.0, 0.0)
            H[k, k], H[k + 1, k] = rr, 0.0
            g[k + 1], g[k] = -sn[k] * g[k], cs[k] * g[k]
            k += 1
            its += 1
            if abs(g[k]) <= ttol or hn == 0:
                done, reason = True, 1
                break
        y = np.zeros(k)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1:k] @ y[i + 1:k]) / H[i, i]
        x = x + V[:k].T @ y
        if done or its >= max_it:
            return x, its, reason
        r = dinv * (b - apply_A(x))
        beta = np.linalg.norm(r)
        if beta <= ttol:
            return x, its, 1


class Explicit:
    """The explicit loop on one box: q_{n+1} from an explicit RK tableau with G = M^-1 RHS(q)."""

    def __init__(self, mesh: O.Mesh, P, Q, ctx_bytes: bytes, qdata, l_size, *, dt, tableau="4", mass_ksp="preonly",
                 pc_jacobi="rowsum", rtol=1e-5, atol=1e-50, restart=30, x_q=None, essential=None, faces=None, mass="auto"):
        """faces: optional callable q -> wdetJb F through the free-stream faces (face_oracle.freestream_apply).  mass "auto":
        the SUPG-stabilized mass (MassFunction_Newtonian, linearised at each right-hand side's state) when the context's
        stabilization is SUPG, as problems/newtonian.c:795 chooses, else Mass_5; the Jacobi preconditioner is set up at the
        first solve and kept (PCSetUp runs once: the MatCEED object never changes state)."""
        self.mesh, self.qdata, self.l_size, self.dt, self.x_q = mesh, qdata, l_size, dt, x_q
        self.ess = np.asarray(essential if essential is not None else [], dtype=np.int64)
        self.faces = faces
        self.ctx = bytearray(ctx_bytes)
        self.ctx[168:176] = np.float64(dt).tobytes()  # "timestep size" (RHS_NS, src/setupts.c:44-46)
        self.A, self.b, self.c = (np.asarray(v, dtype=np.float64) for v in TABLEAUX[tableau])
        self.mass_ksp, self.rtol, self.atol, self.restart = mass_ksp, rtol, atol, restart
        stab = int(np.frombuffer(bytes(self.ctx)[88:92], dtype=np.int32)[0])  # NewtonianIdealGasContext_.stabilization (offset 88)
        self.stab_mass = mass == "auto" and stab == 2
        self.state = None

        def M(u):
            if self.stab_mass:
                v = O.apply_mass_stab(mesh, bytes(self.ctx), np.ascontiguousarray(u), self.state, qdata)
            else:
                v = O.apply_mass(mesh, np.ascontiguousarray(u), qdata)
            v[self.ess] = 0.0
            return v
        self.M = M
        self.P, self.Q, self.pc_jacobi = P, Q, pc_jacobi
        self.dinv = None
        self.mass_its = []

    def rhs(self, q, t):
        self.ctx[64:72] = np.float64(t).tobytes()  # "solution time"
        R = O.apply_rhs(self.mesh, bytes(self.ctx), np.ascontiguousarray(q), self.qdata, self.x_q)
        if self.faces is not None:
            R = R - self.faces(q)
        R[self.ess] = 0.0
        self.state = np.ascontiguousarray(q)
        if self.dinv is None:  # PCSetUp at the first solve
            if self.pc_jacobi == "rowsum":
                ones = np.ones(self.l_size)
                ones[self.ess] = 0.0
                d = self.M(ones)
            elif self.stab_mass:
                d = O.mass_stab_diagonal(self.mesh, bytes(self.ctx), self.state, self.qdata, self.l_size)
            else:
                d = mass_diagonal(self.mesh, self.P, self.Q, self.qdata, self.l_size)
            d[self.ess] = 1.0
            self.dinv = 1.0 / d
        if self.mass_ksp == "preonly":
            return self.dinv * R
        G, its, reason = gmres_left(self.M, self.dinv, R, self.rtol, self.atol, self.restart)
        assert reason == 1
        self.mass_its.append(its)
        return G

    def step(self, q, t):
        K = []
        for i in range(len(self.b)):
            Y = q + self.dt * sum(self.A[i, j] * K[j] for j in range(i) if self.A[i, j] != 0) if i else q
            K.append(self.rhs(Y, t + self.c[i] * self.dt))
        return q + self.dt * sum(bi * Ki for bi, Ki in zip(self.b, K))
