"""CPU checks of the channel problem (problems/channel.c, qfunctions/channel.h, examples/channel.yaml) and of essential
boundary conditions: the Poiseuille initial state equals the reference's ICsChannel QFunction (when oracle/_ref is built), and
the oracle, run as the reference's "Channel" test runs (examples/navierstokes.c:252: 5 x 5 x 1 faces, degree 1, q_extra 2,
5 backward-Euler steps, no-slip walls and symmetry planes as essential DOFs), reproduces tests/output/channel.bin
(tests/golden/channel_be5.npz) under the reference's regression criterion (src/misc.c:111-118), comparing the free DOFs as
a sorted multiset because DMPlex orders them differently.  The Newton solve here is exact (dense Jacobian from the oracle's
Jacobian action), converged like PETSc's SNES default (relative residual 1e-8)."""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import O, oracle_mesh, prob

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
WALLS = {"y-": (1, 2, 3), "y+": (1, 2, 3), "z-": (3,), "z+": (3,)}


def channel_case(golden="channel_be5.npz"):
    """The "Channel" run (channel_be5.npz) or "Channel, Primitive" (channel_prim_be5.npz: the same in primitive variables)."""
    G = np.load(os.path.join(GOLD, golden))
    hi = tuple(float(v) for v in G["box_hi"])
    P = int(G["degree"]) + 1
    Q = P + int(G["q_extra"])
    mesh = prob.box_mesh(tuple(int(v) for v in G["faces"]), P, periodic=(1, 0, 0), hi=hi)
    basis = prob.tensor_basis(P, Q)
    newt = prob.newtonian_context(int(G["degree"]), mu=float(G["mu"]), implicit=True)
    ch = prob.channel_context(newt, (0.0, 0.0, 0.0), hi, umax=float(G["umax"]))
    q = prob.channel_state(mesh, basis, ch)
    sv = int(G["state_var"]) if "state_var" in G else prob.STATEVAR_CONSERVATIVE
    if sv != prob.STATEVAR_CONSERVATIVE:  # ICsChannel returns the state in the problem's variables (qfunctions/channel.h:68)
        ch.newt_ctx.state_var = sv
        q = prob.state_to_q(newt.gas, q, sv)
    idx = prob.box_essential(mesh, WALLS)
    return G, mesh, basis, ch, q, idx


def free_state_error(q, idx, G):
    """max |sorted(free DOFs) - sorted(reference)| / max |reference| (the reference's criterion on a permutation)."""
    free = np.setdiff1d(np.arange(q.size), idx)
    ref = G["free_state"]
    assert free.size == ref.size
    return np.abs(np.sort(q[free]) - np.sort(ref)).max() / np.abs(ref).max()


def test_channel_initial_state_equals_reference():
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    G, mesh, basis, ch, q, idx = channel_case()
    assert O.ref().ref_channel_ctx_size() == C.sizeof(ch)
    X = prob.node_coordinates(mesh, basis)
    qr = np.zeros((5, X.shape[1]))
    O.call_qf(O.ref().ref_ICsChannel, bytes(memoryview(ch)), X.shape[1], [np.ascontiguousarray(X)], [qr])
    np.testing.assert_allclose(q, qr.T.reshape(-1), rtol=1e-15, atol=0)


def test_essential_dofs_match_the_reference_global_vector():
    G, mesh, basis, ch, q, idx = channel_case()
    assert mesh.l_size - idx.size == G["free_state"].size
    # no-slip walls: all three momentum components; symmetry planes: the normal one (every node here, one element thick)
    assert np.all(q[idx] == 0.0)


@pytest.mark.parametrize("golden", ["channel_be5.npz", "channel_prim_be5.npz"])
def test_oracle_reproduces_reference_channel_run(golden):
    G, mesh, basis, ch, q, idx = channel_case(golden)
    tag = ("conserv", "prim", "entropy")[ch.newt_ctx.state_var]
    free = np.setdiff1d(np.arange(mesh.l_size), idx)
    m = oracle_mesh(mesh, basis)
    Q = basis.Q
    qdata = O.setup_qdata(mesh.num_elem, Q, mesh.x_elem)
    ctx = ch.newt_ctx
    dt = float(G["dt"])
    ctx.dt, ctx.ijacobian_time_shift = dt, 1.0 / dt
    jd = np.zeros(mesh.num_elem * 14 * Q ** 3)
    qn = q.copy()
    for step in range(int(G["steps"])):
        ctx.time = (step + 1) * dt
        cb = prob.context_bytes(ctx)
        qk = qn.copy()
        for it in range(10):
            qdot = (qk - qn) / dt
            qdot[idx] = 0.0
            r = O.apply_ifunction(m, cb, qk, qdot, qdata, jd, qf_name=f"oracle_qf_ifunction_{tag}")
            r[idx] = 0.0
            rn = np.linalg.norm(r)
            r0 = rn if it == 0 else r0
            if rn <= 1e-8 * r0:
                break
            J = np.zeros((free.size, free.size))
            for k, j in enumerate(free):
                e = np.zeros(mesh.l_size)
                e[j] = 1.0
                J[:, k] = O.apply_ijacobian(m, cb, e, qdata, jd, qf_name=f"oracle_qf_ijacobian_{tag}")[free]
            qk[free] += np.linalg.solve(J, -r[free])
        assert rn <= 1e-8 * r0
        qn = qk
    assert free_state_error(qn, idx, G) <= float(G["compare_atol"])
