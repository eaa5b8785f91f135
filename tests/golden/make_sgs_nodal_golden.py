"""Generate tests/golden/sgs_nodal_points.npz from the reference itself (run in a container that has the reference).

  python tests/golden/make_sgs_nodal_golden.py

Seeded point data run through the reference's own QFunctions of the nodal data-driven SGS pipeline, compiled unchanged
into oracle/_ref/libhonee_ref.so (oracle/Makefile), for each state variable (conservative, primitive, entropy):
  VelocityGradientProjectionRHS_*   (qfunctions/velocity_gradient_projection.h:9-49)
  ComputeSgsDDNodal_*               (qfunctions/sgs_dd_model.h:69-108) with the reference's published 6-20-6 weights and
                                    a random inverse multiplicity
  IFunction_NodalSgs_*              (qfunctions/sgs_dd_model.h:219-255)
and once: AnisotropyTensorProjection (qfunctions/grid_anisotropy_tensor.h:35-55), InverseMultiplicity
(qfunctions/inverse_multiplicity.h) and Mass_9 (qfunctions/mass.h).  The weights are those of sgs_points.npz.
"""
from __future__ import annotations

import ctypes as C
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)


def state_in(R, gas, q_cons, sv):
    """conservative states [5][n] -> the same states in the state variable sv (StateToQ, newtonian_state.h:292-306)"""
    if sv == 0:
        return q_cons.copy()
    out = np.zeros_like(q_cons)
    for i in range(q_cons.shape[1]):
        qa = np.ascontiguousarray(q_cons[:, i])
        qb = np.zeros(5)
        R.ref_StateToQ(C.byref(gas), qa.ctypes.data_as(C.POINTER(C.c_double)), 0, sv, qb.ctypes.data_as(C.POINTER(C.c_double)))
        out[:, i] = qb
    return out


def main():
    import oracle as O
    from make_sgs_golden import sgs_ctx_bytes
    O.build()
    R = O.ref()
    assert R is not None, "oracle/_ref not built (needs the reference tree)"
    prob = importlib.import_module("honee-4aiad_b200.problem")
    gold = np.load(os.path.join(HERE, "sgs_points.npz"))
    flat, bounds = gold["weights"], gold["bounds"]
    W1, b1, W2, b2 = flat[:120].reshape(20, 6), flat[120:140], flat[140:260].reshape(6, 20), flat[260:266]
    blob = np.concatenate([b1, np.pad(b2, (0, 14)), W1.reshape(-1), W2.reshape(-1), bounds])

    rng = np.random.default_rng(77)
    n = 128
    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)
    gas = ctx.gas
    P = 101325 * (1 + 0.01 * rng.uniform(-1, 1, n))
    T = 288 * (1 + 0.01 * rng.uniform(-1, 1, n))
    u = rng.uniform(-20, 20, (3, n))
    q_cons = prob.conservative_from_primitive(gas, P, u, T)
    h = rng.uniform(0.01, 0.1, (n, 3))
    dXdx = np.stack([np.diag(2 / h[i]) + rng.normal(0, 2, (3, 3)) for i in range(n)])
    qdata = np.zeros((10, n))
    qdata[0] = rng.uniform(0.5, 2.0, n) * 1e-6
    qdata[1:] = dXdx.reshape(n, 9).T
    x = rng.uniform(0, 1, (3, n))
    G = rng.normal(0, 50, (n, 3, 3))
    grad_velo = np.ascontiguousarray(G.transpose(1, 2, 0))
    km = rng.normal(0, 1.0, (6, n))
    inv_mult = 1.0 / rng.integers(1, 9, n).astype(np.float64)
    mult = np.stack([1.0 / inv_mult] * 6)
    u9 = rng.normal(0, 1, (9, n))

    aniso = np.zeros((7, n))
    O.call_qf(R.ref_AnisotropyTensorProjection, None, n, [qdata], [aniso])
    Aij_delta = np.zeros((7, n))
    O.call_qf(R.ref_AnisotropyTensorCollocate, None, n, [qdata], [Aij_delta])
    inv_out = np.zeros(n)
    O.call_qf(R.ref_InverseMultiplicity, None, n, [np.ascontiguousarray(mult)], [inv_out])
    mass9 = np.zeros((9, n))
    O.call_qf(R.ref_Mass_9, None, n, [u9, qdata], [mass9])

    res = dict(q_cons=q_cons, qdata=qdata, x=x, G=G, km=km, inv_mult=inv_mult, mult=mult, u9=u9, aniso=aniso, Aij_delta=Aij_delta,
               inv_out=inv_out, mass9=mass9, mu=gas.mu, cv=gas.cv, cp=gas.cp)
    for sv, name in enumerate(("Conserv", "Prim", "Entropy")):
        ctx.state_var = sv
        newt = prob.context_bytes(ctx)
        q = state_in(R, gas, q_cons, sv)
        grad_q = rng.normal(0, 1, (3, 5, n)) * np.abs(q)[None] * 5.0
        vg = np.zeros((9, n))
        O.call_qf(getattr(R, f"ref_VelocityGradientProjectionRHS_{name}"), newt, n, [q, np.ascontiguousarray(grad_q), qdata, x], [vg])
        kms = np.zeros((6, n))
        O.call_qf(getattr(R, f"ref_ComputeSgsDDNodal_{name}"), sgs_ctx_bytes(R, newt, blob), n,
                  [q, x, grad_velo, Aij_delta, inv_mult], [kms])
        gv = np.zeros((3, 5, n))
        O.call_qf(getattr(R, f"ref_IFunction_NodalSgs_{name}"), newt, n, [q, qdata, km], [gv])
        res.update({f"q_{name}": q, f"grad_q_{name}": grad_q, f"velgrad_{name}": vg, f"km_sgs_{name}": kms, f"grad_v_{name}": gv})
    np.savez_compressed(os.path.join(HERE, "sgs_nodal_points.npz"), **res)
    print("wrote", os.path.join(HERE, "sgs_nodal_points.npz"))


if __name__ == "__main__":
    main()
