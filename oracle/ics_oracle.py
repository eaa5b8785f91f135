"""CPU restatement of HONEE's initial-condition QFunctions and of the per-point CFL monitor (TEST INFRASTRUCTURE ONLY).

Checker for the B200 initial-condition and monitor operators reached through the libCEED API.  Only ``tests/`` import
this module.  Each function follows the reference QFunction it names, evaluated at given points (numpy arrays
[3][n] of coordinates), and returns the state in the requested state variable, [5][n]:

  ics_newtonian     ICsNewtonianIG_{Conserv,Prim,Entropy}    qfunctions/newtonian.h:17-42
  ics_taylor_green  ICsTaylorGreen                           qfunctions/taylorgreen.h:23-51 (cos(2 z + 2) kept)
  ics_channel       ICsChannel / Exact_Channel               qfunctions/channel.h:24-73 (Pr = mu / (cp k) as written)
  ics_gaussian_wave IC_GaussianWave_{Conserv,Prim,Entropy}   qfunctions/gaussianwave.h:20-71
  state_to_q        StateToQ (StateToU / StateToY / StateToV) qfunctions/newtonian_state.h:91-103, 282-304
  cfl_points        MonitorCFL_3D_*                          qfunctions/monitor_cfl.h:9-58 (per point, before x dt)

The restatement is pinned to the reference's own QFunctions compiled unchanged (oracle/_ref) by
tests/test_ics_oracle.py.
"""
from __future__ import annotations

import math

import numpy as np

CONSERVATIVE, PRIMITIVE, ENTROPY = 0, 1, 2


def _gas(gas):
    return gas.cv, gas.cp, gas.cp - gas.cv, gas.cp / gas.cv


def state_from_Y(gas, Y):
    """StateConservativeFromPrimitive (newtonian_state.h:159-168): U from (P, u, T); returns (U, Y)."""
    cv, cp, R, gamma = _gas(gas)
    P, u, T = Y[0], Y[1:4], Y[4]
    rho = P / (R * T)
    e_internal = cv * T
    e_kinetic = .5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
    U = np.stack([rho, rho * u[0], rho * u[1], rho * u[2], rho * (e_internal + e_kinetic)])
    return U, np.asarray(Y, dtype=np.float64)


def state_from_U(gas, U):
    """StatePrimitiveFromConservative (newtonian_state.h:64-73)."""
    cv, cp, R, gamma = _gas(gas)
    u = U[1:4] / U[0]
    e_kinetic = .5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
    e_internal = U[4] / U[0] - e_kinetic
    T = e_internal / cv
    P = (gamma - 1) * U[0] * e_internal
    return np.asarray(U, dtype=np.float64), np.stack([P, u[0], u[1], u[2], T])


def state_to_q(gas, U, Y, state_var):
    """StateToQ (newtonian_state.h:282-304); entropy variables by StateEntropyFromPrimitive (:91-103)."""
    if state_var == PRIMITIVE:
        return np.array(Y)
    if state_var == ENTROPY:
        cv, cp, R, gamma = _gas(gas)
        P, u, T = Y[0], Y[1:4], Y[4]
        rho = P / (R * T)
        entropy = np.log(P) - gamma * np.log(rho)
        rho_div_p = rho / P
        e_kinetic = 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
        return np.stack([(gamma - entropy) / (gamma - 1) - rho_div_p * e_kinetic, rho_div_p * u[0], rho_div_p * u[1], rho_div_p * u[2],
                         -rho_div_p])
    return np.array(U)


def ics_newtonian(setup_ctx, X, state_var):
    """ICsNewtonianIG (newtonian.h:17-30): the context's reference state at every point."""
    ref, gas = setup_ctx.reference, setup_ctx.newt_ctx.gas
    n = X.shape[1]
    Y = np.array([[ref.pressure], [ref.velocity[0]], [ref.velocity[1]], [ref.velocity[2]], [ref.temperature]]) * np.ones(n)
    return state_to_q(gas, *state_from_Y(gas, Y), state_var)


def ics_taylor_green(tg, X):
    """ICsTaylorGreen (taylorgreen.h:23-51), state variable from the context."""
    gas, ref = tg.newt_ctx.gas, tg.reference
    R = gas.cp - gas.cv
    V0 = math.sqrt(ref.velocity[0] ** 2 + ref.velocity[1] ** 2 + ref.velocity[2] ** 2)
    density0 = ref.pressure / (ref.temperature * R)
    x = X * (2 * math.pi / tg.lx)
    Y = np.stack([ref.pressure + (density0 * V0 * V0 / 16) * (np.cos(2 * x[0]) + np.cos(2 * x[1])) * (np.cos(2 * x[2] + 2)),
                  tg.u[0] + V0 * np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2]), tg.u[1] - V0 * np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2]),
                  tg.u[2] + 0 * x[0], ref.temperature + 0 * x[0]])
    return state_to_q(gas, *state_from_Y(gas, Y), tg.newt_ctx.state_var)


def ics_channel(ch, X):
    """ICsChannel (channel.h:58-73) with Exact_Channel (:24-53) at time 0, state variable from the context."""
    gas = ch.newt_ctx.gas
    Pr = gas.mu / (gas.cp * gas.k)
    Ec = (ch.umax * ch.umax) / (gas.cp * ch.theta0)
    eta = (X[1] - ch.center) / ch.H
    theta = ch.theta0 * (1 + (Pr * Ec / 3) * (1 - (eta * eta) ** 2))
    Y = np.stack([ch.P0 + 0 * eta, ch.umax * (1 - eta * eta), 0 * eta, 0 * eta, theta])
    return state_to_q(gas, *state_from_Y(gas, Y), ch.newt_ctx.state_var)


def ics_gaussian_wave(gw, X, state_var):
    """IC_GaussianWave (gaussianwave.h:20-58)."""
    gas = gw.newt_ctx.gas
    gamma = gas.cp / gas.cv
    rho, P, u = gw.S_infty.U[0], gw.S_infty.Y[0], np.array(gw.S_infty.Y[1:4])
    x0, y0 = X[0] - gw.epicenter[0], X[1] - gw.epicenter[1]
    e_kinetic = 0.5 * rho * (u @ u)
    pert = 1 + gw.amplitude * np.exp(-(x0 * x0 + y0 * y0) / (2 * (gw.width * gw.width)))
    U0 = rho * pert
    U = np.stack([U0, u[0] * U0, u[1] * U0, u[2] * U0, P / (gamma - 1) * pert + e_kinetic])
    return state_to_q(gas, *state_from_U(gas, U), state_var)


def cfl_points(gas, q_pts, X_pts, state_var):
    """MonitorCFL_3D (monitor_cfl.h:9-58) at points: sqrt(u . g u), g = 0.25 dXdx^T dXdx.  q_pts [5][n] in the state variable,
    X_pts [3][3][n] the inverse mapping Jacobian dX/dx."""
    if state_var == CONSERVATIVE:
        u = q_pts[1:4] / q_pts[0]
    elif state_var == PRIMITIVE:
        u = q_pts[1:4]
    else:
        u = -q_pts[1:4] / q_pts[4]
    g = 0.25 * np.einsum("kin,kjn->ijn", X_pts, X_pts)
    return np.sqrt(np.einsum("in,ijn,jn->n", u, g, u))
