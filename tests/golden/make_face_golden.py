"""Generate tests/golden/face_points.npz from the reference itself (run in a container that has the reference).

  python tests/golden/make_face_golden.py

Seeded face-point data run through the reference's own free-stream boundary QFunctions, compiled unchanged into
oracle/_ref/libhonee_ref.so (oracle/Makefile): Freestream_Conserv_HLL / _HLLC and Freestream_Jacobian_Conserv_HLL / _HLLC
(qfunctions/bc_freestream.h:14-138, qfunctions/riemann_solver.h) and SetupBoundary (qfunctions/setupgeo.h:100-117).
Interior normal velocities span supersonic outflow to supersonic inflow so every Riemann branch is exercised.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    import oracle as O
    O.build()
    R = O.ref()
    assert R is not None, "oracle/_ref not built (needs the reference tree)"
    prob = importlib.import_module("honee-4aiad_b200.problem")
    rng = np.random.default_rng(77)
    n = 400
    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, implicit=True)
    gas = ctx.gas
    P_inf, u_inf, T_inf = 101325.0, np.array([40.0, 5.0, -3.0]), 288.0
    cb = prob.freestream_context(ctx, P_inf, u_inf, T_inf)
    normal = rng.normal(0, 1, (3, n))
    normal /= np.linalg.norm(normal, axis=0)
    c = np.sqrt(gas.cp / gas.cv * (gas.cp - gas.cv) * 288.0)
    un = rng.uniform(-3.5, 3.5, n) * c                       # interior normal velocity: supersonic in .. supersonic out
    ut = rng.normal(0, 30, (3, n))
    ut -= (ut * normal).sum(0) * normal
    u = un * normal + ut
    P = P_inf * (1 + 0.2 * rng.uniform(-1, 1, n))
    T = T_inf * (1 + 0.2 * rng.uniform(-1, 1, n))
    q = prob.conservative_from_primitive(gas, P, u, T)
    qdata = np.zeros((10, n))
    qdata[0] = rng.uniform(0.5, 2.0, n)
    qdata[1:4] = normal
    out = {}
    for name in ("HLL", "HLLC"):
        v = np.zeros((5, n))
        jac = np.zeros((5, n))
        O.call_qf(getattr(R, f"ref_Freestream_Conserv_{name}"), cb, n, [np.ascontiguousarray(q), np.zeros((15, n)), qdata], [v, jac])
        dq = q * 1e-3 * rng.uniform(-1, 1, q.shape)
        dv = np.zeros((5, n))
        O.call_qf(getattr(R, f"ref_Freestream_Jacobian_Conserv_{name}"), cb, n, [np.ascontiguousarray(dq), np.zeros((15, n)), qdata, np.zeros((3, n)), jac],
                  [dv])
        out[f"v_{name}"], out[f"jac_{name}"], out[f"dq_{name}"], out[f"dv_{name}"] = v, jac, dq, dv
    # face geometric factors
    J = rng.normal(0, 1, (2, 3, n))
    w = rng.uniform(0.1, 1.0, n)
    qs = np.zeros((10, n))
    O.call_qf(R.ref_SetupBoundary, None, n, [np.ascontiguousarray(J), w], [qs])
    np.savez_compressed(os.path.join(HERE, "face_points.npz"), q=q, qdata=qdata, P_inf=P_inf, u_inf=u_inf, T_inf=T_inf, cv=gas.cv, cp=gas.cp,
                        J=J, w=w, qdata_sur=qs, **out)
    print("wrote", os.path.join(HERE, "face_points.npz"))


if __name__ == "__main__":
    main()
