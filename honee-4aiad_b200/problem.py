"""Caller-side problem set-up: what HONEE's L2/L4 layers hand to the operator backend.

HONEE builds its QFunction context in ``NS_NEWTONIAN_IG`` (problems/newtonian.c:573-760), its mesh with PETSc DMPlex and
its tensor basis with PetscFE (src/dm-utils.c:387-879).  PETSc is not part of this project, so this module supplies the
same inputs for structured hex boxes: the 184-byte ``NewtonianIdealGasContext_`` with the reference defaults, int32
restriction offsets into a node-interleaved L-vector, the element coordinate field, and the 1D Lagrange tabulation on
Gauss-Lobatto nodes with Gauss-Legendre quadrature.  The operator backend itself never depends on this module: it takes
whatever offsets, bases and contexts a caller passes through the libCEED API.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

# --------------------------------------------------------------------------------------------------------------------
# QFunction context structs (byte-identical to qfunctions/newtonian_types.h:20-75)

STATEVAR_CONSERVATIVE, STATEVAR_PRIMITIVE, STATEVAR_ENTROPY = 0, 1, 2
STAB_NONE, STAB_SU, STAB_SUPG = 0, 1, 2


class GasProperties(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("mu", C.c_double), ("k", C.c_double), ("cv", C.c_double), ("cp", C.c_double)]


class TauCoefficients(C.Structure):
    _fields_ = [("Ctau_t", C.c_double), ("Ctau_v", C.c_double), ("Ctau_C", C.c_double), ("Ctau_M", C.c_double), ("Ctau_E", C.c_double)]


class NewtonianContext(C.Structure):
    """struct NewtonianIdealGasContext_ (qfunctions/newtonian_types.h:28-47)."""
    _fields_ = [("gas", GasProperties), ("g", C.c_double * 3), ("time", C.c_double), ("ijacobian_time_shift", C.c_double),
                ("is_implicit", C.c_bool), ("state_var", C.c_int), ("stabilization", C.c_int), ("idl_enable", C.c_bool),
                ("idl_pressure", C.c_double), ("idl_amplitude", C.c_double), ("idl_start", C.c_double), ("idl_length", C.c_double),
                ("tau_coeffs", TauCoefficients), ("dt", C.c_double), ("divFdiff_method", C.c_int)]


class StatePrimitive(C.Structure):
    _fields_ = [("pressure", C.c_double), ("velocity", C.c_double * 3), ("temperature", C.c_double)]


class TaylorGreenContext(C.Structure):
    """struct TaylorGreenContext_ (qfunctions/taylorgreen.h:12-20)."""
    _fields_ = [("reference", StatePrimitive), ("newt_ctx", NewtonianContext), ("lx", C.c_double), ("ly", C.c_double),
                ("lz", C.c_double), ("u", C.c_double * 3)]


class ICBoundaryLayer(C.Structure):
    _fields_ = [("wall", StatePrimitive), ("height", C.c_double)]


class SetupContext(C.Structure):
    """struct SetupContext_ (qfunctions/newtonian_types.h:66-75): the context of ICsNewtonianIG_*, with "evaluation time"."""
    _fields_ = [("reference", StatePrimitive), ("ic_boundary_layer", ICBoundaryLayer), ("newt_ctx", NewtonianContext), ("lx", C.c_double),
                ("ly", C.c_double), ("lz", C.c_double), ("time", C.c_double)]


def setup_context(newt, P, u, T, lengths=(1.0, 1.0, 1.0)):
    """A SetupContext with the reference (P, u, T), as NS_NEWTONIAN_IG fills it (problems/newtonian.c:660-700)."""
    ctx = SetupContext()
    ctx.reference = StatePrimitive(P, (C.c_double * 3)(*u), T)
    ctx.newt_ctx = newt
    ctx.lx, ctx.ly, ctx.lz = lengths
    return ctx


assert C.sizeof(NewtonianContext) == 184
assert C.sizeof(SetupContext) == 304
assert NewtonianContext.time.offset == 64 and NewtonianContext.ijacobian_time_shift.offset == 72 and NewtonianContext.dt.offset == 168

# Field offsets HONEE registers with CeedQFunctionContextRegisterDouble (problems/newtonian.c:747-753)
CONTEXT_LABELS = {"timestep size": NewtonianContext.dt.offset,
                  "ijacobian time shift": NewtonianContext.ijacobian_time_shift.offset,
                  "solution time": NewtonianContext.time.offset}


def newtonian_context(degree: int, *, cv=717., cp=1004., lambda_=-2. / 3., mu=1.8e-5, k=0.02638, g=(0., 0., 0.), stab=STAB_NONE,
                      state_var=STATEVAR_CONSERVATIVE, implicit=True, dt=1.0, ijacobian_time_shift=0.0, time=0.0,
                      Ctau_t=1.0, Ctau_v=None, Ctau_C=None, Ctau_M=None, Ctau_E=0.125, idl=None) -> NewtonianContext:
    """Context with the defaults of problems/newtonian.c:588-613, overridable like the -cv/-cp/-mu/-k/-stab/-Ctau_* options."""
    cv_func = (36, 60, 128)
    ctx = NewtonianContext()
    ctx.gas = GasProperties(lambda_, mu, k, cv, cp)
    ctx.g[:] = list(g)
    ctx.time = time
    ctx.ijacobian_time_shift = ijacobian_time_shift
    ctx.is_implicit = bool(implicit)
    ctx.state_var = state_var
    ctx.stabilization = stab
    ctx.tau_coeffs = TauCoefficients(Ctau_t, cv_func[min(3, degree) - 1] if Ctau_v is None else Ctau_v,
                                     0.25 / degree if Ctau_C is None else Ctau_C, 0.25 / degree if Ctau_M is None else Ctau_M, Ctau_E)
    ctx.dt = dt
    ctx.divFdiff_method = 0
    if idl is not None:  # (decay_time, start, length, pressure), problems/newtonian.c:656-677, 722
        decay, start, length, pressure = idl
        ctx.idl_enable = True
        ctx.idl_amplitude = 1.0 / decay
        ctx.idl_start, ctx.idl_length, ctx.idl_pressure = start, length, pressure
    return ctx


def context_bytes(ctx) -> bytes:
    return bytes(memoryview(ctx))


# --------------------------------------------------------------------------------------------------------------------
# ideal-gas state conversion used by initial conditions (qfunctions/newtonian_state.h:159-168)

def conservative_from_primitive(gas: GasProperties, P, u, T):
    R = gas.cp - gas.cv
    rho = P / (R * T)
    u = np.asarray(u)
    E = rho * (gas.cv * T + 0.5 * np.sum(u * u, axis=0))
    return np.stack([rho, rho * u[0], rho * u[1], rho * u[2], E])


def state_to_q(gas: GasProperties, q_cons, state_var: int) -> np.ndarray:
    """Node-interleaved conservative states -> the same states in `state_var` (StateToQ, newtonian_state.h:371-391):
    primitive Y = (P, u, T) (StatePrimitiveFromConservative, :64-73), entropy V (StateEntropyFromPrimitive, :91-103)."""
    U = np.asarray(q_cons, dtype=np.float64).reshape(-1, 5)
    if state_var == STATEVAR_CONSERVATIVE:
        return U.reshape(-1).copy()
    rho = U[:, 0]
    u = U[:, 1:4] / rho[:, None]
    ke = 0.5 * np.sum(u * u, axis=1)
    eint = U[:, 4] / rho - ke
    T = eint / gas.cv
    P = (gas.cp / gas.cv - 1) * rho * eint
    if state_var == STATEVAR_PRIMITIVE:
        return np.column_stack([P, u, T]).reshape(-1)
    if state_var != STATEVAR_ENTROPY:
        raise ValueError(f"unknown state variable {state_var}")
    g, R = gas.cp / gas.cv, gas.cp - gas.cv
    rho_y = P / (R * T)
    ent = np.log(P) - g * np.log(rho_y)
    rho_p = rho_y / P
    return np.column_stack([(g - ent) / (g - 1) - rho_p * ke, rho_p[:, None] * u, -rho_p]).reshape(-1)


# --------------------------------------------------------------------------------------------------------------------
# 1D tabulation

def _legendre(n, x):
    p0, p1 = np.ones_like(x), x.copy()
    if n == 0:
        return p0, np.zeros_like(x)
    for kk in range(2, n + 1):
        p0, p1 = p1, ((2 * kk - 1) * x * p1 - (kk - 1) * p0) / kk
    dp = n * (x * p1 - p0) / (x * x - 1)
    return p1, dp


def gauss_legendre(Q: int):
    x = -np.cos(np.pi * (np.arange(Q) + 0.75) / (Q + 0.5))
    for _ in range(100):
        p, dp = _legendre(Q, x)
        dx = p / dp
        x = x - dx
        if np.max(np.abs(dx)) < 1e-16:
            break
    p, dp = _legendre(Q, x)
    return x, 2.0 / ((1 - x * x) * dp * dp)


def gauss_lobatto(P: int):
    N = P - 1
    x = -np.cos(np.pi * np.arange(P) / N)
    inner = x[1:-1].copy()
    for _ in range(100):
        p, dp = _legendre(N, inner)
        ddp = (2 * inner * dp - N * (N + 1) * p) / (1 - inner * inner)
        dx = dp / ddp
        inner = inner - dx
        if inner.size == 0 or np.max(np.abs(dx)) < 1e-16:
            break
    x[1:-1] = inner
    x[0], x[-1] = -1.0, 1.0
    return x


def lagrange_tabulate(nodes, pts):
    P, Q = len(nodes), len(pts)
    B = np.zeros((Q, P))
    G = np.zeros((Q, P))
    for q in range(Q):
        for j in range(P):
            l, dl = 1.0, 0.0
            for m in range(P):
                if m == j:
                    continue
                f = (pts[q] - nodes[m]) / (nodes[j] - nodes[m])
                dl = dl * f + l / (nodes[j] - nodes[m])
                l *= f
            B[q, j], G[q, j] = l, dl
    return B, G


@dataclass
class TensorBasis:
    """Arguments of CeedBasisCreateTensorH1 (src/dm-utils.c:766-879): 1D interp/grad [Q][P], q_ref, q_weight."""
    P: int
    Q: int
    interp1d: np.ndarray
    grad1d: np.ndarray
    qref1d: np.ndarray
    qweight1d: np.ndarray
    nodes1d: np.ndarray


def tensor_basis(P: int, Q: int) -> TensorBasis:
    nodes = gauss_lobatto(P)
    qx, qw = gauss_legendre(Q)
    B, G = lagrange_tabulate(nodes, qx)
    return TensorBasis(P, Q, B, G, qx, qw, nodes)


# --------------------------------------------------------------------------------------------------------------------
# structured hex box

@dataclass
class BoxMesh:
    n: tuple
    P: int
    periodic: tuple
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    num_elem: int = 0
    num_nodes: int = 0
    offsets: np.ndarray = field(default=None, repr=False)   # int32 [E][P^3], node*5
    x_elem: np.ndarray = field(default=None, repr=False)    # [E][3][8] vertex coordinates (E-vector of the P=2 field)
    colors: tuple = field(default=None, repr=False)         # (color_ptr, color_elem) CSR
    node_dims: tuple = ()

    @property
    def l_size(self):
        return 5 * self.num_nodes


def _nodes_dim(n, P, periodic):
    return n * (P - 1) + (0 if periodic else 1)


def box_mesh(n, P, periodic=(False, False, False), lo=(0., 0., 0.), hi=(1., 1., 1.), planes=None, ncomp=5) -> BoxMesh:
    """Lexicographic hex box with node-interleaved L-vector; `planes` optionally gives the vertex planes per direction."""
    n = tuple(int(v) for v in n)
    periodic = tuple(bool(p) for p in periodic)
    if planes is None:
        planes = [np.linspace(lo[d], hi[d], n[d] + 1) for d in range(3)]
    N = tuple(_nodes_dim(n[d], P, periodic[d]) for d in range(3))
    ex, ey, ez = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    ex, ey, ez = (a.transpose(2, 1, 0).reshape(-1) for a in (ex, ey, ez))  # x fastest
    a = np.arange(P)
    A, Bb, Cc = np.meshgrid(a, a, a, indexing="ij")
    A, Bb, Cc = (t.transpose(2, 1, 0).reshape(-1) for t in (A, Bb, Cc))     # local node a fastest
    i = (ex[:, None] * (P - 1) + A[None, :]) % N[0]
    j = (ey[:, None] * (P - 1) + Bb[None, :]) % N[1]
    k = (ez[:, None] * (P - 1) + Cc[None, :]) % N[2]
    node = i.astype(np.int64) + N[0] * (j.astype(np.int64) + N[1] * k.astype(np.int64))
    num_nodes = N[0] * N[1] * N[2]
    assert num_nodes * ncomp < 2 ** 31, "int32 offsets overflow"
    offsets = (node * ncomp).astype(np.int32).reshape(-1)
    E = n[0] * n[1] * n[2]
    x_elem = np.zeros((E, 3, 8))
    for v in range(8):
        va, vb, vc = v & 1, (v >> 1) & 1, (v >> 2) & 1
        x_elem[:, 0, v] = planes[0][ex + va]
        x_elem[:, 1, v] = planes[1][ey + vb]
        x_elem[:, 2, v] = planes[2][ez + vc]
    m = BoxMesh(n, P, periodic, np.asarray(planes[0]), np.asarray(planes[1]), np.asarray(planes[2]), E, num_nodes, offsets,
                x_elem.reshape(-1), None, N)
    m.colors = parity_colors(n, periodic)
    return m


def parity_colors(n, periodic=(False, False, False)):
    """Parity colouring of a lexicographic box: elements of one colour share no node.  Per direction the colour is the
    element index mod 2; along a periodic direction with an odd element count the last element touches the first, so it
    takes a third colour there (up to 3x3x3 classes)."""
    ex, ey, ez = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    idx = [a.transpose(2, 1, 0).reshape(-1) for a in (ex, ey, ez)]
    per = []
    for d in range(3):
        c = idx[d] % 2
        if periodic[d] and n[d] % 2 == 1 and n[d] > 1:
            c = np.where(idx[d] == n[d] - 1, 2, c)
        per.append(c)
    color = per[0] + 3 * (per[1] + 3 * per[2])
    _, color = np.unique(color, return_inverse=True)
    order = np.argsort(color, kind="stable").astype(np.int32)
    counts = np.bincount(color)
    ptr_ = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return ptr_, order


def node_coordinates(mesh: BoxMesh, basis: TensorBasis):
    """Physical coordinates [3][num_nodes] of the Lagrange nodes (for nodal initial conditions)."""
    coords = []
    for d, planes in enumerate((mesh.xs, mesh.ys, mesh.zs)):
        nd = mesh.n[d]
        Nd = mesh.node_dims[d]
        x = np.zeros(Nd)
        for e in range(nd):
            h0, h1 = planes[e], planes[e + 1]
            loc = h0 + (basis.nodes1d + 1) * 0.5 * (h1 - h0)
            for a in range(mesh.P):
                idx = e * (mesh.P - 1) + a
                if idx < Nd:
                    x[idx] = loc[a]
        coords.append(x)
    X, Y, Z = np.meshgrid(coords[0], coords[1], coords[2], indexing="ij")
    return np.stack([t.transpose(2, 1, 0).reshape(-1) for t in (X, Y, Z)])


# --------------------------------------------------------------------------------------------------------------------
# workloads (synthetic stand-ins with the shapes and value distributions of the benchmark configurations)

def gaussian_pulse_state(mesh: BoxMesh, basis: TensorBasis, gas: GasProperties, *, P0=101325., T0=288., u0=(10., 0., 0.), amp=0.01,
                         sigma=0.1, center=(0.5, 0.5, 0.5), noise=1e-4, seed=0):
    """3D Gaussian pressure pulse on a uniform background plus seeded uniform relative noise on all conservative fields."""
    X = node_coordinates(mesh, basis)
    r2 = sum((X[d] - center[d]) ** 2 for d in range(3))
    P = P0 * (1 + amp * np.exp(-r2 / (2 * sigma ** 2)))
    u = np.array(u0)[:, None] * np.ones_like(P)[None, :]
    q = conservative_from_primitive(gas, P, u, T0 * np.ones_like(P))
    rng = np.random.default_rng(seed)
    q = q * (1 + noise * rng.uniform(-1, 1, size=q.shape))
    return np.ascontiguousarray(q.T.reshape(-1))


def multimode_state(mesh: BoxMesh, basis: TensorBasis, gas: GasProperties, *, P0=101325., T0=288., u0=(10., 0., 0.), modes=8,
                    amp=1e-3, kmax=8, seed=0):
    """Background state plus `modes` seeded sinusoidal perturbations (|k| <= kmax * 2pi) with relative amplitude `amp`."""
    X = node_coordinates(mesh, basis)
    rng = np.random.default_rng(seed)
    q0 = conservative_from_primitive(gas, P0 * np.ones(X.shape[1]), np.array(u0)[:, None] * np.ones((1, X.shape[1])),
                                     T0 * np.ones(X.shape[1]))
    pert = np.zeros_like(q0)
    for _ in range(modes):
        kvec = rng.uniform(-1, 1, 3)
        kvec *= rng.uniform(0, kmax) / max(np.linalg.norm(kvec), 1e-12)
        phase = rng.uniform(0, 2 * np.pi, 5)
        arg = 2 * np.pi * (kvec[0] * X[0] + kvec[1] * X[1] + kvec[2] * X[2])
        pert += np.sin(arg[None, :] + phase[:, None])
    q = q0 * (1 + amp * pert)
    return np.ascontiguousarray(q.T.reshape(-1))


def taylor_green_state(mesh: BoxMesh, basis: TensorBasis, tg: "TaylorGreenContext") -> np.ndarray:
    """Nodal Taylor-Green vortex initial state (conservative, node-interleaved), as ICsTaylorGreen computes it
    (qfunctions/taylorgreen.h:23-50): coordinates scaled by 2 pi / L, pressure with its cos(2 z + 2) factor, velocity
    amplitude |reference velocity| plus the context's mean velocity u, uniform reference temperature."""
    X = node_coordinates(mesh, basis)
    gas = tg.newt_ctx.gas
    R = gas.cp - gas.cv
    ref = tg.reference
    V0 = math.sqrt(sum(ref.velocity[i] ** 2 for i in range(3)))
    rho0 = ref.pressure / (ref.temperature * R)
    x = X[0] * (2 * math.pi / tg.lx)
    y = X[1] * (2 * math.pi / tg.ly)
    z = X[2] * (2 * math.pi / tg.lz)
    P = ref.pressure + (rho0 * V0 * V0 / 16) * (np.cos(2 * x) + np.cos(2 * y)) * np.cos(2 * z + 2)
    u = np.stack([tg.u[0] + V0 * np.sin(x) * np.cos(y) * np.cos(z), tg.u[1] - V0 * np.cos(x) * np.sin(y) * np.cos(z),
                  tg.u[2] + 0 * x])
    q = conservative_from_primitive(gas, P, u, ref.temperature * np.ones_like(P))
    return np.ascontiguousarray(q.T.reshape(-1))


def taylor_green_context(degree: int, *, L=2 * math.pi, Re=1600., Ma=0.1, rho0=1.0, V0=1.0, stab=STAB_SUPG):
    """Taylor-Green vortex parameters in the form of examples/taylor_green_vortex.yaml (Re=1600, Ma=0.1)."""
    cv, cp = 717., 1003.8
    gamma = cp / cv
    R = cp - cv
    c = V0 / Ma
    T0 = c * c / (gamma * R)
    P0 = rho0 * R * T0
    mu = rho0 * V0 * (L / (2 * math.pi)) / Re
    Pr = 0.71
    k = cp * mu / Pr
    ctx = TaylorGreenContext()
    ctx.reference = StatePrimitive(P0, (C.c_double * 3)(V0, 0., 0.), T0)
    ctx.newt_ctx = newtonian_context(degree, cv=cv, cp=cp, mu=mu, k=k, stab=stab, Ctau_v=60, Ctau_C=0.5, Ctau_M=0.5, Ctau_E=0.5)
    ctx.lx = ctx.ly = ctx.lz = L
    return ctx


# --------------------------------------------------------------------------------------------------------------------
# Gaussian wave (problems/gaussianwave.c, qfunctions/gaussianwave.h)

class StateC(C.Structure):
    """struct State (qfunctions/newtonian_types.h): conservative U then primitive Y."""
    _fields_ = [("U", C.c_double * 5), ("Y", C.c_double * 5)]


class GaussianWaveContext(C.Structure):
    """struct GaussianWaveContext_ (qfunctions/gaussianwave.h:12-18)."""
    _fields_ = [("epicenter", C.c_double * 3), ("width", C.c_double), ("amplitude", C.c_double), ("S_infty", StateC),
                ("newt_ctx", NewtonianContext)]


def state_from_primitive(gas: GasProperties, P, u, T):
    """StateFromPrimitive: (U, Y) of an ideal gas at pressure P, velocity u, temperature T."""
    U = conservative_from_primitive(gas, np.array([P]), np.asarray(u, dtype=np.float64).reshape(3, 1), np.array([T]))[:, 0]
    return U, np.array([P, *np.asarray(u, dtype=np.float64), T])


def gaussian_wave_context(newt: NewtonianContext, P, u, T, *, epicenter=(0.0, 0.0, 0.0), width=0.002, amplitude=0.1):
    U, Y = state_from_primitive(newt.gas, P, u, T)
    ctx = GaussianWaveContext()
    ctx.epicenter[:] = list(epicenter)
    ctx.width, ctx.amplitude = width, amplitude
    ctx.S_infty.U[:] = list(U)
    ctx.S_infty.Y[:] = list(Y)
    ctx.newt_ctx = newt
    return ctx


def gaussian_wave_state(mesh: BoxMesh, basis: TensorBasis, gw: GaussianWaveContext) -> np.ndarray:
    """IC_GaussianWave (qfunctions/gaussianwave.h:20-58) at the nodes: the free-stream density and pressure scaled by
    1 + amplitude exp(-r^2 / (2 width^2)) in the x-y plane around the epicentre, the free-stream velocity, kinetic energy of the
    free stream."""
    X = node_coordinates(mesh, basis)
    gas = gw.newt_ctx.gas
    gamma = gas.cp / gas.cv
    rho_inf, Pinf = gw.S_infty.U[0], gw.S_infty.Y[0]
    u = np.array(gw.S_infty.Y[1:4])
    pert = 1 + gw.amplitude * np.exp(-((X[0] - gw.epicenter[0]) ** 2 + (X[1] - gw.epicenter[1]) ** 2) / (2 * gw.width ** 2))
    q = np.empty((5, X.shape[1]))
    q[0] = rho_inf * pert
    q[1:4] = u[:, None] * q[0]
    q[4] = Pinf / (gamma - 1) * pert + 0.5 * rho_inf * (u @ u)
    return np.ascontiguousarray(q.T.reshape(-1))


# --------------------------------------------------------------------------------------------------------------------
# channel flow (problems/channel.c:73-150, qfunctions/channel.h): Poiseuille initial state, body force, no-slip walls

class ChannelContext(C.Structure):
    """struct ChannelContext_ (qfunctions/channel.h:13-22)."""
    _fields_ = [("implicit", C.c_bool), ("theta0", C.c_double), ("P0", C.c_double), ("umax", C.c_double), ("center", C.c_double),
                ("H", C.c_double), ("B", C.c_double), ("newt_ctx", NewtonianContext)]


def channel_context(newt: NewtonianContext, lo, hi, *, umax=10.0, theta0=300.0, P0=1.0e5, body_force_scale=1.0, implicit=True):
    """NS_CHANNEL (problems/channel.c:73-137): half-height H and centre from the box's y extent, body force
    B = scale * 2 umax mu / H^2 applied as the gravity g = (B / rho0, 0, 0) of the Newtonian context (rho0 = P0 / (R theta0))."""
    H = 0.5 * (hi[1] - lo[1])
    center = H + lo[1]
    gas = newt.gas
    B = body_force_scale * 2 * umax * gas.mu / (H * H)
    rho = P0 / ((gas.cp - gas.cv) * theta0)
    newt.g[:] = [B / rho, 0.0, 0.0]
    return ChannelContext(bool(implicit), theta0, P0, umax, center, H, B, newt)


def channel_state(mesh: BoxMesh, basis: TensorBasis, ch: ChannelContext) -> np.ndarray:
    """ICsChannel (qfunctions/channel.h:24-73) at the nodes: pressure P0, velocity umax (1 - ((y - c)/H)^2) along x, temperature
    theta0 (1 + Pr Ec / 3 (1 - ((y - c)/H)^4)) with Pr = mu / (cp k) and Ec = umax^2 / (cp theta0) as the reference writes them."""
    X = node_coordinates(mesh, basis)
    gas = ch.newt_ctx.gas
    eta = (X[1] - ch.center) / ch.H
    Pr = gas.mu / (gas.cp * gas.k)
    Ec = ch.umax ** 2 / (gas.cp * ch.theta0)
    theta = ch.theta0 * (1 + (Pr * Ec / 3) * (1 - eta ** 4))
    u = np.stack([ch.umax * (1 - eta ** 2), 0 * eta, 0 * eta])
    q = conservative_from_primitive(gas, ch.P0 * np.ones_like(eta), u, theta)
    return np.ascontiguousarray(q.T.reshape(-1))


def tanh_planes(n: int, lo: float, hi: float, beta: float) -> np.ndarray:
    """n + 1 vertex planes on [lo, hi] clustered towards both ends: y = c + h tanh(beta (2 j / n - 1)) / tanh(beta) with
    c, h the centre and half-width (the usual wall-resolved channel grading; beta = 0 gives uniform planes)."""
    eta = 2 * np.arange(n + 1) / n - 1
    c, h = 0.5 * (lo + hi), 0.5 * (hi - lo)
    if beta == 0:
        return c + h * eta
    y = c + h * np.tanh(beta * eta) / math.tanh(beta)
    y[0], y[-1] = lo, hi
    return y


def perturbed_channel_state(mesh: BoxMesh, basis: TensorBasis, ch: ChannelContext, amplitude=0.05, seed=0) -> np.ndarray:
    """channel_state with seeded uniform velocity perturbations of +-amplitude * umax in every component at every node
    (the essential DOFs take their wall values when the state is set on a stepper with them)."""
    X = node_coordinates(mesh, basis)
    gas = ch.newt_ctx.gas
    eta = (X[1] - ch.center) / ch.H
    Pr = gas.mu / (gas.cp * gas.k)
    Ec = ch.umax ** 2 / (gas.cp * ch.theta0)
    theta = ch.theta0 * (1 + (Pr * Ec / 3) * (1 - eta ** 4))
    u = np.stack([ch.umax * (1 - eta ** 2), 0 * eta, 0 * eta])
    u = u + amplitude * ch.umax * np.random.default_rng(seed).uniform(-1, 1, u.shape)
    q = conservative_from_primitive(gas, ch.P0 * np.ones_like(eta), u, theta)
    return np.ascontiguousarray(q.T.reshape(-1))


def box_essential(mesh: BoxMesh, sides: dict):
    """Essential DOFs of box sides: {"y-": (1, 2, 3), ...} -> sorted unique L-vector indices node * 5 + component (the
    bc_*_essential_comps of HONEE's options; PETSc's box face sets 1/2 are z-/z+, 3/4 y-/y+, 5/6 x+/x-)."""
    N = mesh.node_dims
    ijk = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), np.arange(N[2]), indexing="ij"), axis=-1).reshape(-1, 3)
    node = ijk[:, 0] + N[0] * (ijk[:, 1] + N[1] * ijk[:, 2])
    idx = []
    for side, comps in sides.items():
        ax = "xyz".index(side[0])
        if mesh.periodic[ax]:
            raise ValueError(f"side {side} is periodic")
        at = ijk[:, ax] == (N[ax] - 1 if side[1] == "+" else 0)
        for c in comps:
            idx.append(node[at] * 5 + c)
    return np.unique(np.concatenate(idx)).astype(np.int32)


# --------------------------------------------------------------------------------------------------------------------
# boundary faces of a box mesh and the free-stream context

_FACE_AXES = {  # side -> (normal axis, at upper end, tangent axis X0, tangent axis X1) with cross(X0, X1) outward
    "x-": (0, False, 2, 1), "x+": (0, True, 1, 2),
    "y-": (1, False, 0, 2), "y+": (1, True, 2, 0),
    "z-": (2, False, 1, 0), "z+": (2, True, 0, 1),
}


def box_faces(mesh: BoxMesh, basis: TensorBasis, sides=None):
    """Boundary faces of the non-periodic sides: offsets [F][P^2] (node * 5, face-tensor order, X0 fastest), node
    coordinates [F][3][P^2] and the side name of each face.  The face parameterisation makes the normal of
    cross(dx/dX0, dx/dX1) point out of the box."""
    if sides is None:
        sides = [s for s, (ax, _, _, _) in _FACE_AXES.items() if not mesh.periodic[ax]]
    P, n, N = mesh.P, mesh.n, mesh.node_dims
    X = node_coordinates(mesh, basis)
    offs, xs, names = [], [], []
    a = np.arange(P)
    for side in sides:
        ax, upper, t0, t1 = _FACE_AXES[side]
        if mesh.periodic[ax]:
            raise ValueError(f"side {side} is periodic")
        e_ax = n[ax] - 1 if upper else 0
        l_ax = P - 1 if upper else 0
        for e1 in range(n[t1]):
            for e0 in range(n[t0]):
                idx = [None, None, None]
                idx[ax] = np.full((P, P), e_ax * (P - 1) + l_ax)
                idx[t0] = (e0 * (P - 1) + a)[None, :] * np.ones((P, 1), dtype=int)   # [b][a], a along X0 (fastest)
                idx[t1] = (e1 * (P - 1) + a)[:, None] * np.ones((1, P), dtype=int)
                idx = [(np.asarray(v) % N[d]).reshape(-1) for d, v in enumerate(idx)]
                node = idx[0] + N[0] * (idx[1] + N[1] * idx[2])
                offs.append(node * 5)
                xs.append(X[:, node])
                names.append(side)
    return np.ascontiguousarray(np.array(offs, dtype=np.int32)), np.ascontiguousarray(np.array(xs)), names


def freestream_context(newt: NewtonianContext, P, u, T) -> bytes:
    """FreestreamContext_ bytes (bc_freestream_type.h): the Newtonian context and the exterior State (U, Y)."""
    gas = newt.gas
    R = gas.cp - gas.cv
    rho = P / (R * T)
    u = np.asarray(u, dtype=np.float64)
    U = np.array([rho, rho * u[0], rho * u[1], rho * u[2], rho * (gas.cv * T + 0.5 * u @ u)])
    Y = np.array([P, u[0], u[1], u[2], T])
    return bytes(memoryview(newt)) + U.tobytes() + Y.tobytes()
