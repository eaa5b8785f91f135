"""CPU checks of the free-stream boundary oracle (oracle/face_oracle.py) against the reference's own QFunctions: the
golden fixture tests/golden/face_points.npz (made by make_face_golden.py from oracle/_ref) covering every HLL / HLLC
branch, the face geometric factors, and finite differences of the restated flux."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import face_oracle as FO  # noqa: E402

G = np.load(os.path.join(ROOT, "tests", "golden", "face_points.npz"))
U_INF = None


def _ext():
    cv, cp = float(G["cv"]), float(G["cp"])
    u = G["u_inf"]
    rho = float(G["P_inf"]) / ((cp - cv) * float(G["T_inf"]))
    U = np.array([rho, rho * u[0], rho * u[1], rho * u[2], rho * (cv * float(G["T_inf"]) + 0.5 * u @ u)])
    Y = np.array([float(G["P_inf"]), u[0], u[1], u[2], float(G["T_inf"])])
    return U, Y, cv, cp


@pytest.mark.parametrize("name", ["HLL", "HLLC"])
def test_flux_and_jacobian_match_reference(name):
    U, Y, cv, cp = _ext()
    q, qd = G["q"], G["qdata"]
    n = q.shape[1]
    s = FO.state_from_U(q, cv, cp)
    F = FO.riemann(s, FO.exterior(U, Y, n), qd[1:4], cv, cp, hllc=name == "HLLC")
    np.testing.assert_allclose(qd[0] * F, G[f"v_{name}"], rtol=1e-11, atol=1e-9)
    np.testing.assert_array_equal(G[f"jac_{name}"], q)
    ds = FO.state_from_U_fwd(s, G[f"dq_{name}"], cv, cp)
    zero = FO.St(np.zeros(n), np.zeros((3, n)), np.zeros(n), np.zeros(n), np.zeros((3, n)), np.zeros(n))
    dF = FO.riemann(s, FO.exterior(U, Y, n), qd[1:4], cv, cp, hllc=name == "HLLC", dL=ds, dR=zero)
    np.testing.assert_allclose(qd[0] * dF, G[f"dv_{name}"], rtol=1e-9, atol=1e-7 * np.abs(G[f"dv_{name}"]).max())


def test_riemann_branches_all_exercised():
    U, Y, cv, cp = _ext()
    q, qd = G["q"], G["qdata"]
    s = FO.state_from_U(q, cv, cp)
    R = FO.exterior(U, Y, q.shape[1])
    uL, uR = (s.u * qd[1:4]).sum(0), (R.u * qd[1:4]).sum(0)
    sl, sr = FO.speeds(s, uL, R, uR, cv, cp / cv)
    assert (sl >= 0).any() and (sr <= 0).any() and ((sl < 0) & (sr > 0)).any()


@pytest.mark.parametrize("name", ["HLL", "HLLC"])
def test_flux_tangent_matches_finite_differences(name):
    U, Y, cv, cp = _ext()
    q, qd = G["q"], G["qdata"]
    n = q.shape[1]
    dq = G[f"dq_{name}"] * 1e-3
    s = FO.state_from_U(q, cv, cp)
    zero = FO.St(np.zeros(n), np.zeros((3, n)), np.zeros(n), np.zeros(n), np.zeros((3, n)), np.zeros(n))
    dF = FO.riemann(s, FO.exterior(U, Y, n), qd[1:4], cv, cp, hllc=name == "HLLC", dL=FO.state_from_U_fwd(s, dq, cv, cp), dR=zero)
    Fp = FO.riemann(FO.state_from_U(q + dq, cv, cp), FO.exterior(U, Y, n), qd[1:4], cv, cp, hllc=name == "HLLC")
    Fm = FO.riemann(FO.state_from_U(q - dq, cv, cp), FO.exterior(U, Y, n), qd[1:4], cv, cp, hllc=name == "HLLC")
    fd = (Fp - Fm) / 2
    ok = np.abs(fd - dF).max(0) <= 1e-4 * (np.abs(fd).max(0) + 1e-6)
    assert ok.mean() > 0.95  # points sitting on a branch switch are not differentiable there


def test_face_qdata_matches_reference():
    J, w = G["J"], G["w"]
    n = w.size
    # one "face" per point: P = Q = 1 style evaluation via the formula on dx/dX directly
    J0, J1 = J[0], J[1]
    N = np.cross(J0.T, J1.T).T
    detJb = np.linalg.norm(N, axis=0)
    ref = G["qdata_sur"]
    np.testing.assert_allclose(ref[0], w * detJb, rtol=1e-13)
    np.testing.assert_allclose(ref[1:4], N / detJb, rtol=1e-12, atol=1e-14)
    a, c, b = (J0 * J0).sum(0), (J1 * J1).sum(0), (J0 * J1).sum(0)
    det = a * c - b * b
    inv = np.array([[c / det, -b / det], [-b / det, a / det]])
    dXdx = np.stack([inv[i, 0] * J0 + inv[i, 1] * J1 for i in range(2)])  # [2][3][n]
    np.testing.assert_allclose(ref[4:], dXdx.reshape(6, n), rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("hllc", [False, True])
def test_face_diagonal_is_the_oracle_jacobian_diagonal(hllc):
    """freestream_diagonal equals e_i^T J e_i of the oracle's face Jacobian (itself pinned to the reference's
    Freestream_Jacobian above), on a small box with every side a free-stream face."""
    import importlib
    prob = importlib.import_module("honee-4aiad_b200.problem")
    U, Y, cv, cp = _ext()
    mesh = prob.box_mesh((2, 1, 1), 3)
    basis = prob.tensor_basis(3, 3)
    gas = prob.GasProperties(cv=cv, cp=cp)
    q = prob.gaussian_pulse_state(mesh, basis, gas, seed=2)
    off, xn, _ = prob.box_faces(mesh, basis)
    qd = FO.face_qdata(basis.interp1d, basis.grad1d, basis.qweight1d, 3, 3, xn)
    B = np.asarray(basis.interp1d).reshape(3, 3)
    Bq = np.einsum("jb,ia->jiba", B, B).reshape(9, 9)
    jac = np.stack([(Bq @ q.reshape(-1, 5)[off[f] // 5]).T for f in range(off.shape[0])])
    d = FO.freestream_diagonal(off, basis.interp1d, 3, 3, qd, jac, U, Y, cv, cp, hllc=hllc, l_size=mesh.l_size)
    rng = np.random.default_rng(1)
    for i in rng.choice(np.unique(off.reshape(-1)), 12, replace=False) + rng.integers(0, 5, 12):
        e = np.zeros(mesh.l_size)
        e[i] = 1.0
        col = FO.freestream_apply(off, basis.interp1d, 3, 3, qd, q, U, Y, cv, cp, hllc=hllc, dq=e, jac=jac)
        assert abs(col[i] - d[i]) <= 1e-12 * np.abs(d).max()


@pytest.mark.parametrize("sv,flux", [(1, "HLLC"), (2, "HLL")])
def test_state_variables_match_reference(sv, flux):
    """The oracle's free-stream flux and tangent in primitive (Freestream_Prim_HLLC) and entropy (Freestream_Entropy_HLL)
    variables against the reference's QFunctions compiled in oracle/_ref, on the fixture's points converted to those
    variables (the stored face state is the state in its own variables)."""
    import importlib
    import oracle as O
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    prob = importlib.import_module("honee-4aiad_b200.problem")
    U, Y, cv, cp = _ext()
    name = ("Conserv", "Prim", "Entropy")[sv]
    qd = np.ascontiguousarray(G["qdata"])
    n = qd.shape[1]
    newt = prob.newtonian_context(2, cv=cv, cp=cp)
    newt.state_var = sv
    ctx = prob.freestream_context(newt, float(G["P_inf"]), np.asarray(G["u_inf"]), float(G["T_inf"]))
    qv = np.ascontiguousarray(prob.state_to_q(newt.gas, G["q"].T.reshape(-1), sv).reshape(-1, 5).T)
    v, jac = np.zeros((5, n)), np.zeros((5, n))
    grad, x = np.zeros((10, n)), np.zeros((3, n))
    assert O.call_qf(getattr(O.ref(), f"ref_Freestream_{name}_{flux}"), ctx, n, [qv, grad, qd, x], [v, jac]) == 0
    np.testing.assert_array_equal(jac, qv)
    s = FO.state_from_q(qv, sv, cv, cp)
    F = FO.riemann(s, FO.exterior(U, Y, n), qd[1:4], cv, cp, hllc=flux == "HLLC")
    np.testing.assert_allclose(qd[0] * F, v, rtol=1e-11, atol=1e-11 * np.abs(v).max())
    dq = qv * 1e-3 * np.random.default_rng(sv).normal(size=qv.shape)
    dv = np.zeros((5, n))
    assert O.call_qf(getattr(O.ref(), f"ref_Freestream_Jacobian_{name}_{flux}"), ctx, n, [dq, grad, qd, x, jac], [dv]) == 0
    ds = FO.state_from_q_fwd(s, dq, sv, cv, cp)
    zero = FO.St(np.zeros(n), np.zeros((3, n)), np.zeros(n), np.zeros(n), np.zeros((3, n)), np.zeros(n))
    dF = FO.riemann(s, FO.exterior(U, Y, n), qd[1:4], cv, cp, hllc=flux == "HLLC", dL=ds, dR=zero)
    np.testing.assert_allclose(qd[0] * dF, dv, rtol=1e-9, atol=1e-9 * np.abs(dv).max())
