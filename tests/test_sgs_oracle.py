"""CPU checks of the SGS-closure oracle (oracle/sgs_oracle.py) against the reference's own QFunctions: the committed
golden fixture (tests/golden/sgs_points.npz, made by make_sgs_golden.py from oracle/_ref) and, where it is built, the
reference library itself.  Also pins the oracle's back-propagation against finite differences."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import sgs_oracle as SO  # noqa: E402

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "sgs_points.npz"))


def test_eigensolver_matches_reference():
    for i in range(GOLD["mats"].shape[0]):
        ev, E = SO.eig3(GOLD["mats"][i], 5)
        np.testing.assert_allclose(ev, GOLD["evals"][i], rtol=1e-13, atol=1e-14)
        np.testing.assert_allclose(E, GOLD["evecs"][i], rtol=1e-12, atol=1e-13)


def test_anisotropy_and_inputs_match_reference():
    n = GOLD["G"].shape[0]
    for i in range(n):
        kmA, delta = SO.anisotropy(GOLD["dXdx"][i])
        np.testing.assert_allclose(kmA, GOLD["Aij_delta"][:6, i], rtol=1e-12, atol=1e-14)
        assert delta == pytest.approx(GOLD["Aij_delta"][6, i], rel=1e-13)
        x, E, g = SO.inputs(GOLD["G"][i], GOLD["Aij_delta"][:6, i], GOLD["Aij_delta"][6, i], GOLD["nu"][i])
        np.testing.assert_allclose(x, GOLD["inputs"][i], rtol=1e-11, atol=1e-13)
        np.testing.assert_allclose(E, GOLD["E"][i], rtol=1e-11, atol=1e-12)
        assert g == pytest.approx(GOLD["gmag"][i], rel=1e-13)


def test_stress_pipeline_with_reference_weights_matches_reference():
    w = GOLD["weights"].astype(np.float64)
    n = GOLD["G"].shape[0]
    for i in range(n):
        x, E, g = SO.inputs(GOLD["G"][i], GOLD["Aij_delta"][:6, i], GOLD["Aij_delta"][6, i], GOLD["nu"][i])
        y, _, _ = SO.forward(w, 20, 0, x[None, :])
        tau = SO.outputs_to_stress(y[0], GOLD["Aij_delta"][6, i], E, GOLD["bounds"], g)
        ref = GOLD["km_sgs"][:, i]
        np.testing.assert_allclose(tau, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_training_pairs_match_reference():
    q, u = GOLD["q"], GOLD["q"][1:4] / GOLD["q"][0]
    n = q.shape[1]
    for i in range(n):
        x, _, _ = SO.inputs(GOLD["G"][i], GOLD["Aij_delta"][:6, i], GOLD["Aij_delta"][6, i], GOLD["nu"][i])
        np.testing.assert_allclose(x, GOLD["train"][:6, i], rtol=1e-11, atol=1e-13)
    vp = GOLD["velo_prod"]
    tau = vp - np.stack([u[0] * u[0], u[1] * u[1], u[2] * u[2], u[1] * u[2], u[0] * u[2], u[0] * u[1]])
    np.testing.assert_allclose(tau, GOLD["train"][6:], rtol=1e-12, atol=1e-9)


def test_sframe_target_inverts_the_output_map():
    rng = np.random.default_rng(3)
    for i in range(16):
        x, E, g = SO.inputs(GOLD["G"][i], GOLD["Aij_delta"][:6, i], GOLD["Aij_delta"][6, i], GOLD["nu"][i])
        out_n = rng.uniform(0, 1, 6)
        km = SO.outputs_to_stress(out_n, GOLD["Aij_delta"][6, i], E, GOLD["bounds"], g)
        tau = SO.km_unpack(km)
        tau6 = np.array([tau[0, 0], tau[1, 1], tau[2, 2], tau[1, 2], tau[0, 2], tau[0, 1]])
        o = SO.stress_to_sframe(tau6, GOLD["Aij_delta"][6, i], E, g)
        b = GOLD["bounds"].reshape(6, 2)
        np.testing.assert_allclose((o - b[:, 0]) / (b[:, 1] - b[:, 0]), out_n, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("h2,alpha", [(20, 0.0), (0, 0.0), (20, 0.1)])
def test_backprop_matches_finite_differences(h2, alpha):
    rng = np.random.default_rng(5)
    nparam = len(np.concatenate([np.zeros(a * b + b) for a, b in SO.shapes(20, h2)]))
    p = rng.normal(0, 0.4, nparam)
    X, Y = rng.normal(0, 1, (40, 6)), rng.normal(0, 1, (40, 6))
    loss, g = SO.loss_and_grad(p, 20, h2, X, Y, alpha)
    for k in rng.choice(nparam, 25, replace=False):
        e = np.zeros(nparam)
        e[k] = 1e-6
        fd = (SO.loss_and_grad(p + e, 20, h2, X, Y, alpha)[0] - SO.loss_and_grad(p - e, 20, h2, X, Y, alpha)[0]) / 2e-6
        assert g[k] == pytest.approx(fd, rel=1e-5, abs=1e-9)


def test_reference_weight_files_load_into_the_fixture_layout():
    sgs = importlib.import_module("honee-4aiad_b200.sgs")
    from helpers import reference_dir
    ref = reference_dir()
    if ref is None:
        pytest.skip("reference tree not present (set HONEE_REFERENCE_DIR)")
    dd = os.path.join(ref, "examples", "dd_sgs_data")
    d, flat = sgs.load_reference_model(dd)
    np.testing.assert_array_equal(flat, GOLD["weights"])
    assert (d.hidden1, d.hidden2) == (20, 0)
    np.testing.assert_allclose(np.array(d.out_bounds[:]), GOLD["bounds"], rtol=1e-7)


def test_oracle_equals_reference_library_on_fresh_points():
    import oracle as O
    R = O.ref()
    if R is None:
        pytest.skip("oracle/_ref not built")
    import ctypes as C
    rng = np.random.default_rng(77)
    dp = C.POINTER(C.c_double)
    for _ in range(50):
        M = rng.normal(0, 3, (3, 3))
        M = np.ascontiguousarray(M + M.T)
        ev = np.zeros(3)
        Ev = np.zeros((3, 3))
        e2, E2 = SO.eig3(M, 5)
        Mc = M.copy()  # Diagonalize3 works in place
        R.ref_Diagonalize3(Mc.ctypes.data_as(dp), ev.ctypes.data_as(dp), Ev.ctypes.data_as(dp), 5)
        np.testing.assert_array_equal(e2, ev)
        np.testing.assert_array_equal(E2, Ev)


def _filter_ctx(R, newt: bytes, grid_based, ws, ks):
    import ctypes as C
    lay = (C.c_size_t * 4)()
    R.ref_diff_filter_ctx_layout(lay)
    size, o_newt, o_ks, o_damp = lay[:]
    buf = bytearray(size)
    buf[0] = 1 if grid_based else 0
    np.frombuffer(buf, dtype=np.float64, count=3, offset=8)[:] = ws           # width_scaling follows the bool
    np.frombuffer(buf, dtype=np.float64, count=1, offset=o_ks)[:] = ks
    np.frombuffer(buf, dtype=np.int32, count=1, offset=o_damp)[:] = 0         # DIFF_FILTER_DAMP_NONE
    buf[o_newt:o_newt + len(newt)] = newt
    return bytes(buf)


@pytest.mark.parametrize("grid_based", [False, True])
def test_filter_pointwise_forms_match_reference(grid_based):
    import oracle as O
    import filter_oracle as FO
    R = O.ref()
    if R is None:
        pytest.skip("oracle/_ref not built")
    prob = importlib.import_module("honee-4aiad_b200.problem")
    rng = np.random.default_rng(31)
    n, N = 64, 11
    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)
    ws, ks = np.array([1.5, 0.7, 2.0]), 0.1
    cb = _filter_ctx(R, prob.context_bytes(ctx), grid_based, ws, ks)
    q = rng.normal(0, 1, (N, n))
    gq = rng.normal(0, 1, (3 * N, n))
    dXdx = np.stack([np.diag(rng.uniform(5, 50, 3)) + rng.normal(0, 2, (3, 3)) for _ in range(n)])
    qdata = np.zeros((10, n))
    qdata[0] = rng.uniform(0.5, 2, n)
    qdata[1:] = dXdx.reshape(n, 9).T
    Aij = np.zeros((7, n))
    O.call_qf(R.ref_AnisotropyTensorCollocate, None, n, [np.ascontiguousarray(qdata)], [Aij])
    v = np.zeros((N, n))
    gv = np.zeros((3 * N, n))
    O.call_qf(R.ref_DifferentialFilter_LHS_11, cb, n, [q, gq, Aij, np.zeros((3, n)), np.ascontiguousarray(qdata)], [v, gv])
    for i in range(n):
        al = FO.alpha_at(dXdx[i], grid_based, ws, ks)
        vv, gg = FO.lhs_point(q[:, i], gq[:, i].reshape(3, N), dXdx[i], qdata[0, i], al)
        np.testing.assert_allclose(vv, v[:, i], rtol=1e-14)
        np.testing.assert_allclose(gg, gv[:, i].reshape(3, N), rtol=1e-11, atol=1e-12 * np.abs(gg).max())
    # right-hand side integrand: wdetJ * (P, u, T, u_i u_j)
    P = 101325 * (1 + 0.01 * rng.uniform(-1, 1, n))
    T = 288 * (1 + 0.01 * rng.uniform(-1, 1, n))
    u = rng.uniform(-20, 20, (3, n))
    qc = prob.conservative_from_primitive(ctx.gas, P, u, T)
    v0, v1 = np.zeros((5, n)), np.zeros((6, n))
    O.call_qf(R.ref_DifferentialFilter_RHS_Conserv, cb, n, [np.ascontiguousarray(qc), np.ascontiguousarray(qdata)], [v0, v1])
    w = qdata[0]
    np.testing.assert_allclose(v0, w * np.stack([P, u[0], u[1], u[2], T]), rtol=1e-12)
    np.testing.assert_allclose(v1, w * np.stack([u[0] ** 2, u[1] ** 2, u[2] ** 2, u[1] * u[2], u[0] * u[2], u[0] * u[1]]), rtol=1e-11)


@pytest.mark.parametrize("sv", [1, 2])
def test_filter_rhs_in_other_state_variables_matches_reference(sv):
    """DifferentialFilter_RHS_Prim / _Entropy (qfunctions/differential_filter.h:62-68): the same integrand w (P, u, T, u_i u_j)
    from the state given in primitive or entropy variables."""
    import oracle as O
    prob = importlib.import_module("honee-4aiad_b200.problem")
    R = O.ref()
    if R is None:
        pytest.skip("oracle/_ref not built")
    ctx = prob.newtonian_context(2)
    ctx.state_var = sv
    cb = _filter_ctx(R, prob.context_bytes(ctx), False, (1.0, 1.0, 1.0), 0.1)
    rng = np.random.default_rng(8)
    n = 64
    qdata = np.zeros((10, n))
    qdata[0] = rng.uniform(1e-4, 1e-2, n)
    P = 101325 * (1 + 0.01 * rng.uniform(-1, 1, n))
    T = 288 * (1 + 0.01 * rng.uniform(-1, 1, n))
    u = rng.uniform(-20, 20, (3, n))
    qc = prob.conservative_from_primitive(ctx.gas, P, u, T)
    qv = np.ascontiguousarray(prob.state_to_q(ctx.gas, qc.T.reshape(-1), sv).reshape(-1, 5).T)
    v0, v1 = np.zeros((5, n)), np.zeros((6, n))
    name = ("Conserv", "Prim", "Entropy")[sv]
    O.call_qf(getattr(R, f"ref_DifferentialFilter_RHS_{name}"), cb, n, [qv, np.ascontiguousarray(qdata)], [v0, v1])
    w = qdata[0]
    np.testing.assert_allclose(v0, w * np.stack([P, u[0], u[1], u[2], T]), rtol=1e-11)
    np.testing.assert_allclose(v1, w * np.stack([u[0] ** 2, u[1] ** 2, u[2] ** 2, u[1] * u[2], u[0] * u[2], u[0] * u[1]]), rtol=1e-10)
