"""The oracle's point-wise restatement against the reference's own QFunctions and known-answer tests (CPU only).

Pins: qfunctions/newtonian.h:205-315 (IFunction/IJacobian, all three state variables, none/SU/SUPG, IDL, gravity)
through the golden vectors in tests/golden/pointwise_newtonian.npz (generated by tests/golden/make_golden.py from the
reference compiled unchanged), and problems/newtonian.c:947-987 (UnitTests_Newtonian state round trips at 20 eps and
forward-mode tangents against finite differences at 5e-6).
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
QF = {"Conserv": "conserv", "Prim": "prim", "Entropy": "entropy"}


def _golden():
    z = np.load(os.path.join(GOLD, "pointwise_newtonian.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    return z, meta, int(z["Q"])


@pytest.mark.parametrize("ci", range(11))
def test_pointwise_matches_reference_golden(oracle, ci):
    z, meta, Q = _golden()
    cs = meta[ci]
    k = lambda n: np.ascontiguousarray(z[f"c{ci}_{n}"])  # noqa: E731
    ctx = bytes(k("ctx"))
    v = np.zeros((5, Q)); gv = np.zeros((3, 5, Q)); jd = np.zeros((cs["njd"], Q))
    fn = getattr(oracle.lib(), f"oracle_qf_ifunction_{QF[cs['qf']]}")
    assert oracle.call_qf(fn, ctx, Q, [k("q"), k("grad_q"), k("q_dot"), k("qdata"), k("x")], [v, gv, jd]) == 0
    # bit-exact: same operations in the same order under -ffp-contract=off
    np.testing.assert_array_equal(v, k("v"))
    np.testing.assert_array_equal(gv, k("grad_v"))
    np.testing.assert_array_equal(jd, k("jac_data"))
    jv = np.zeros((5, Q)); jgv = np.zeros((3, 5, Q))
    fn = getattr(oracle.lib(), f"oracle_qf_ijacobian_{QF[cs['qf']]}")
    assert oracle.call_qf(fn, ctx, Q, [k("dq"), k("grad_dq"), k("qdata"), k("jac_data")], [jv, jgv]) == 0
    np.testing.assert_array_equal(jv, k("jv"))
    np.testing.assert_array_equal(jgv, k("jgrad_v"))


def test_pointwise_matches_reference_build_directly(oracle, prob):
    """Fresh random points through both builds (needs oracle/_ref, i.e. the reference sources at build time)."""
    R = oracle.ref()
    if R is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    rng = np.random.default_rng(7)
    Q = 40
    for stab in (0, 1, 2):
        ctx = prob.newtonian_context(4, stab=stab, dt=3e-4, ijacobian_time_shift=5e3, g=(1., 2., -3.))
        cb = prob.context_bytes(ctx)
        P = 1e5 * (1 + 0.05 * rng.uniform(-1, 1, Q)); T = 300 * (1 + 0.05 * rng.uniform(-1, 1, Q)); u = rng.uniform(-50, 50, (3, Q))
        q = prob.conservative_from_primitive(ctx.gas, P, u, T)
        ins = [np.ascontiguousarray(a) for a in (q, rng.normal(size=(3, 5, Q)) * q[None], rng.normal(size=(5, Q)) * q,
                                                 np.concatenate([np.ones((1, Q)), rng.normal(size=(9, Q))]), rng.uniform(size=(3, Q)))]
        outs = {}
        for tag, fn in (("o", oracle.lib().oracle_qf_ifunction_conserv), ("r", R.ref_IFunction_Newtonian_Conserv)):
            o = [np.zeros((5, Q)), np.zeros((3, 5, Q)), np.zeros((14, Q))]
            oracle.call_qf(fn, cb, Q, ins, o)
            outs[tag] = o
        for a, b in zip(outs["o"], outs["r"]):
            np.testing.assert_array_equal(a, b)


def _check_q(q_a, q_b, q_s, rtol0, rtolu, rtol4):
    """CheckQWithTolerance (problems/newtonian.c:860-889): component-wise relative error with the velocity norm scale."""
    thr = 10 * np.finfo(float).eps
    err0 = (q_a[0] - q_b[0]) / (q_s[0] if abs(q_s[0]) > thr else 1)
    err4 = (q_a[4] - q_b[4]) / (q_s[4] if abs(q_s[4]) > thr else 1)
    um = np.sqrt(q_s[1] ** 2 + q_s[2] ** 2 + q_s[3] ** 2)
    erru = [(q_a[i] - q_b[i]) / (um if um > thr else 1) for i in (1, 2, 3)]
    assert abs(err0) < rtol0 and abs(err4) < rtol4 and all(abs(e) < rtolu for e in erru), (err0, erru, err4)


def test_unit_tests_newtonian_roundtrip(oracle, prob):
    """TestState: A -> B -> A round trips at 20 eps for every pair (problems/newtonian.c:966-972)."""
    g = json.load(open(os.path.join(GOLD, "unit_state.json")))
    gas = prob.newtonian_context(2).gas
    eps = np.finfo(float).eps
    A = {0: np.array(g["U0"]), 1: np.array(g["Y0"]), 2: np.array(g["V0"])}
    for a, b in ((1, 0), (1, 2), (0, 1), (0, 2), (2, 0), (2, 1)):
        s = oracle.lib().oracle_state_from_q
        s.restype = None
        st = _state_from_q(oracle, gas, A[a], a)
        qb = _state_to_q(oracle, gas, st, b)
        np.testing.assert_array_equal(qb, np.array(g["state_to_q"][f"{a}->{b}"]))  # same bits as the reference
        back = _state_to_q(oracle, gas, _state_from_q(oracle, gas, qb, b), a)
        _check_q(back, A[a], A[a], 20 * eps, 20 * eps, 20 * eps)


def test_unit_tests_newtonian_fwd_vs_fd(oracle, prob):
    """TestState_fwd: StateFromQ_fwd/StateToQ_fwd against finite differences (problems/newtonian.c:974-986)."""
    g = json.load(open(os.path.join(GOLD, "unit_state.json")))
    gas = prob.newtonian_context(2).gas
    A = {0: np.array(g["U0"]), 1: np.array(g["Y0"]), 2: np.array(g["V0"])}
    rtol, eps = 5e-6, 4e-7
    tol = {(1, 0): (1, 1, 1), (1, 2): (1, 1, 1), (0, 1): (1, 1, 1), (0, 2): (10, 1, 1), (2, 0): (5, 1, 1), (2, 1): (5, 5, 5)}
    for (a, b), (f0, fu, f4) in tol.items():
        A0 = A[a]
        s0 = _state_from_q(oracle, gas, A0, a)
        for i in range(5):
            dA = np.zeros(5); dA[i] = A0[i]
            ds = _state_from_q_fwd(oracle, gas, s0, dA, a)
            dB = _state_to_q_fwd(oracle, gas, s0, ds, b)
            A1 = A0 * (1 + eps * (np.arange(5) == i))
            dB_fd = (_state_to_q(oracle, gas, _state_from_q(oracle, gas, A1, a), b) - _state_to_q(oracle, gas, s0, b)) / eps
            _check_q(dB_fd, dB, dB_fd, f0 * rtol, fu * rtol, f4 * rtol)


# ---- ctypes plumbing for OracleState
class _St(C.Structure):
    _fields_ = [("U", C.c_double * 5), ("Y", C.c_double * 5)]


def _fn(oracle, name, restype):
    f = getattr(oracle.lib(), name)
    f.restype = restype
    return f


def _state_from_q(oracle, gas, q, var):
    return _fn(oracle, "oracle_state_from_q", _St)(C.byref(gas), (C.c_double * 5)(*q), var)


def _state_from_q_fwd(oracle, gas, s, dq, var):
    return _fn(oracle, "oracle_state_from_q_fwd", _St)(C.byref(gas), C.byref(s), (C.c_double * 5)(*dq), var)


def _state_to_q(oracle, gas, s, var):
    out = (C.c_double * 5)()
    _fn(oracle, "oracle_state_to_q", None)(C.byref(gas), C.byref(s), out, var)
    return np.array(out[:])


def _state_to_q_fwd(oracle, gas, s, ds, var):
    out = (C.c_double * 5)()
    _fn(oracle, "oracle_state_to_q_fwd", None)(C.byref(gas), C.byref(s), C.byref(ds), out, var)
    return np.array(out[:])
