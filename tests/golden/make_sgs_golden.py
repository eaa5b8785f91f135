"""Generate tests/golden/sgs_points.npz from the reference itself (run in a container that has the reference).

  python tests/golden/make_sgs_golden.py [--ref REFERENCE_TREE]

Seeded quadrature-point data run through the reference's own data-driven SGS QFunctions, compiled unchanged into
oracle/_ref/libhonee_ref.so (oracle/Makefile):
  AnisotropyTensorCollocate              (qfunctions/grid_anisotropy_tensor.h:55-78)  -> A_ij (KM) and delta
  ComputeSgsDDInputs                     (qfunctions/sgs_dd_utils.h:58-96)            -> model inputs, eigenframe, |G A|
  ComputeSgsDDNodal_Conserv              (qfunctions/sgs_dd_model.h:65-98)            -> SGS stress (KM) with the
                                         reference's published 6-20-6 weights (examples/dd_sgs_data/*.dat)
  ComputeSGS_DDAnisotropicTrainingData   (qfunctions/sgs_dd_training.h:22-56)          -> training pairs
  Diagonalize3                           (qfunctions/utils_eigensolver_jacobi.h:172)   -> eigenpairs of random matrices
The weights and the OutScaling bounds are stored in the fixture (in the flat layout of the CUDA kernels) so the GPU
tests need no reference tree.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def sgs_ctx_bytes(R, newt_ctx: bytes, flat_ref_layout: np.ndarray) -> bytes:
    """struct SgsDDContext_ (qfunctions/sgs_dd_model.h:16-31) with its trailing data blob, laid out by the compiler."""
    lay = (C.c_size_t * 4)()
    R.ref_sgs_dd_ctx_layout(lay)
    size, o_newt, o_off, o_data = lay[:]
    nI, nO, nN = 6, 6, 20
    off = {"bias1": 0, "bias2": nN, "weight1": 2 * nN, "weight2": 2 * nN + nN * nI, "out_scaling": 2 * nN + nN * nI + nI * nN}
    total = o_data + 8 * (off["out_scaling"] + 2 * nO)
    buf = bytearray(max(total, size))
    np.frombuffer(buf, dtype=np.int32, count=4, offset=0)[:] = [nI, nO, 2, nN]
    np.frombuffer(buf, dtype=np.float64, count=1, offset=16)[:] = 0.0  # alpha (after the 4 ints)
    buf[o_newt:o_newt + len(newt_ctx)] = newt_ctx
    np.frombuffer(buf, dtype=np.uint64, count=6, offset=o_off)[:] = [off["bias1"], off["bias2"], off["weight1"], off["weight2"],
                                                                    off["out_scaling"], total]
    np.frombuffer(buf, dtype=np.float64, count=flat_ref_layout.size, offset=o_data)[:] = flat_ref_layout
    return bytes(buf)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HONEE_REFERENCE_DIR"),
                    help="the reference tree (default: HONEE_REFERENCE_DIR, else the tree oracle/_ref was built from)")
    args = ap.parse_args()
    import oracle as O
    O.build()
    R = O.ref()
    assert R is not None, "oracle/_ref not built (needs the reference tree)"
    prob = importlib.import_module("honee-4aiad_b200.problem")
    sgs = importlib.import_module("honee-4aiad_b200.sgs")
    rng = np.random.default_rng(2024)
    n = 256

    # weights: the reference's files, in its data-blob layout (b1 | b2 (20 slots) | W1 [20][6] | W2 [6][20] | bounds)
    if not args.ref:
        args.ref = open(os.path.join(os.path.dirname(O.__file__), "_ref", "reference_dir.txt")).read().strip()
    dd = os.path.join(args.ref, "examples", "dd_sgs_data")
    b1, b2 = sgs.read_dat(os.path.join(dd, "b1.dat")), sgs.read_dat(os.path.join(dd, "b2.dat"))
    w1, w2 = sgs.read_dat(os.path.join(dd, "w1.dat")), sgs.read_dat(os.path.join(dd, "w2.dat"))
    bounds = sgs.read_dat(os.path.join(dd, "OutScaling.dat"))
    W1 = w1.reshape(6, 20).T
    W2 = w2.reshape(20, 6).T
    blob = np.concatenate([b1[:20], np.pad(b2[:6], (0, 14)), W1.reshape(-1), W2.reshape(-1), bounds])
    _, flat = sgs.load_reference_model(dd)

    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)
    newt = prob.context_bytes(ctx)
    gas = ctx.gas

    # points: states, velocity gradients of LES size, stretched and sheared element maps
    P = 101325 * (1 + 0.01 * rng.uniform(-1, 1, n))
    T = 288 * (1 + 0.01 * rng.uniform(-1, 1, n))
    u = rng.uniform(-20, 20, (3, n))
    q = prob.conservative_from_primitive(gas, P, u, T)                 # [5][n]
    G = rng.normal(0, 50, (n, 3, 3))
    h = rng.uniform(0.01, 0.1, (n, 3))
    dXdx = np.stack([np.diag(2 / h[i]) + rng.normal(0, 2, (3, 3)) for i in range(n)])
    qdata = np.zeros((10, n))
    qdata[0] = 1.0
    qdata[1:] = dXdx.reshape(n, 9).T

    Aij_delta = np.zeros((7, n))
    O.call_qf(R.ref_AnisotropyTensorCollocate, None, n, [np.ascontiguousarray(qdata)], [Aij_delta])

    nu = gas.mu / q[0]
    inp = np.zeros((n, 6))
    E = np.zeros((n, 3, 3))
    gmag = np.zeros(n)
    dp = C.POINTER(C.c_double)
    for i in range(n):
        Gi = np.ascontiguousarray(G[i])
        Ai = np.ascontiguousarray(Aij_delta[:6, i])
        Ei = np.zeros((3, 3))
        xi = np.zeros(6)
        g = C.c_double()
        R.ref_ComputeSgsDDInputs(Gi.ctypes.data_as(dp), Ai.ctypes.data_as(dp), C.c_double(Aij_delta[6, i]), C.c_double(nu[i]),
                                 Ei.ctypes.data_as(dp), xi.ctypes.data_as(dp), C.byref(g))
        inp[i], E[i], gmag[i] = xi, Ei, g.value

    grad_velo = np.ascontiguousarray(G.transpose(1, 2, 0))            # [3][3][n]
    inv_mult = np.ones(n)
    km_sgs = np.zeros((6, n))
    cbytes = sgs_ctx_bytes(R, newt, blob)
    O.call_qf(R.ref_ComputeSgsDDNodal_Conserv, cbytes, n, [np.ascontiguousarray(q), np.zeros((3, n)), grad_velo, Aij_delta, inv_mult],
              [km_sgs])

    velo_prod = np.stack([u[0] * u[0], u[1] * u[1], u[2] * u[2], u[1] * u[2], u[0] * u[2], u[0] * u[1]]) * (1 + 0.05 * rng.uniform(-1, 1, (6, n)))
    train = np.zeros((12, n))
    O.call_qf(R.ref_ComputeSGS_DDAnisotropicTrainingDataNodal_Conserv, newt, n,
              [np.ascontiguousarray(q), np.ascontiguousarray(velo_prod), grad_velo, Aij_delta, inv_mult], [train])

    mats = rng.normal(0, 1, (64, 3, 3))
    mats = mats + mats.transpose(0, 2, 1)
    evals = np.zeros((64, 3))
    evecs = np.zeros((64, 3, 3))
    for i in range(64):
        A = mats[i].copy()  # Diagonalize3 works in place
        ev = np.zeros(3)
        Ev = np.zeros((3, 3))
        R.ref_Diagonalize3(A.ctypes.data_as(dp), ev.ctypes.data_as(dp), Ev.ctypes.data_as(dp), 5)
        evals[i], evecs[i] = ev, Ev

    np.savez_compressed(os.path.join(HERE, "sgs_points.npz"), q=q, G=G, dXdx=dXdx, Aij_delta=Aij_delta, nu=nu, inputs=inp, E=E, gmag=gmag,
                        km_sgs=km_sgs, velo_prod=velo_prod, train=train, weights=flat, bounds=bounds, mats=mats,
                        evals=evals, evecs=evecs, mu=gas.mu, cv=gas.cv, cp=gas.cp)
    print("wrote", os.path.join(HERE, "sgs_points.npz"))


if __name__ == "__main__":
    main()
