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
    dd = "/root/reference/examples/dd_sgs_data"
    if not os.path.isdir(dd):
        pytest.skip("reference tree not present")
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
