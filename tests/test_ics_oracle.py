"""The initial-condition and CFL oracle (oracle/ics_oracle.py) against the reference's own QFunctions compiled unchanged
(oracle/_ref): ICsNewtonianIG_*, ICsTaylorGreen, ICsChannel, IC_GaussianWave_* at random points in every state
variable, and MonitorCFL_3D_* per point.  CPU only; skipped where the reference build is absent.  Tolerance 1e-13
relative: the restatement evaluates the same expressions in the same order, numpy's cos / sin / exp / log may differ from
the C library's by an ulp."""
import importlib

import numpy as np
import pytest

import ics_oracle as IO
from helpers import O

prob = importlib.import_module("honee-4aiad_b200.problem")
R = O.ref()
pytestmark = pytest.mark.skipif(R is None, reason="reference QFunctions not built (oracle/_ref)")
SV_NAME = {0: "Conserv", 1: "Prim", 2: "Entropy"}


def _ref_ic(name, ctx, X):
    n = X.shape[1]
    q0 = np.zeros((5, n))
    dx = np.zeros((9, n))
    assert O.call_qf(getattr(R, name), bytes(ctx), n, [np.ascontiguousarray(X), dx], [q0]) == 0
    return q0


def _pts(seed, lo=0.0, hi=1.0, n=64):
    return np.random.default_rng(seed).uniform(lo, hi, (3, n))


def _newt(sv):
    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)
    ctx.state_var = sv
    return ctx


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_newtonian_ic(sv):
    ctx = prob.setup_context(_newt(sv), 101325.0, (10.0, -2.0, 1.0), 288.0)
    X = _pts(1)
    np.testing.assert_allclose(IO.ics_newtonian(ctx, X, sv), _ref_ic(f"ref_ICsNewtonianIG_{SV_NAME[sv]}", ctx, X), rtol=1e-13)


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_taylor_green_ic(sv):
    tg = prob.taylor_green_context(3)
    tg.newt_ctx.state_var = sv
    tg.u[:] = [0.3, -0.1, 0.05]
    X = _pts(2, 0, 2 * np.pi)
    np.testing.assert_allclose(IO.ics_taylor_green(tg, X), _ref_ic("ref_ICsTaylorGreen", tg, X), rtol=1e-13)


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_channel_ic(sv):
    newt = _newt(sv)
    ch = prob.channel_context(newt, (0, -1, 0), (1, 1, 1), umax=12.0, theta0=300.0, P0=1.0e5)
    X = _pts(3, -1, 1)
    np.testing.assert_allclose(IO.ics_channel(ch, X), _ref_ic("ref_ICsChannel", ch, X), rtol=1e-13)


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_gaussian_wave_ic(sv):
    gw = prob.gaussian_wave_context(_newt(sv), 101325.0, (20.0, 5.0, 0.0), 288.0, epicenter=(0.4, 0.6, 0.0), width=0.1, amplitude=0.05)
    X = _pts(4)
    np.testing.assert_allclose(IO.ics_gaussian_wave(gw, X, sv), _ref_ic(f"ref_IC_GaussianWave_{SV_NAME[sv]}", gw, X), rtol=1e-13)


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_cfl_points(sv):
    rng = np.random.default_rng(5)
    n = 40
    newt = _newt(sv)
    X = _pts(6)
    q = IO.ics_gaussian_wave(prob.gaussian_wave_context(_newt(sv), 101325.0, (30.0, -5.0, 2.0), 288.0, width=0.2, amplitude=0.1), X[:, :n], sv)
    dXdx = rng.normal(size=(3, 3, n)) * 4
    qdata = np.zeros((10, n))
    qdata[0] = 1.0
    qdata[1:] = dXdx.reshape(9, n)
    v = np.zeros((1, n))
    assert O.call_qf(getattr(R, f"ref_MonitorCFL_3D_{SV_NAME[sv]}"), bytes(newt), n, [np.ascontiguousarray(q), qdata], [v]) == 0
    np.testing.assert_allclose(IO.cfl_points(newt.gas, q, dXdx, sv), v[0], rtol=1e-13)
