"""Test helpers: oracle meshes built from the same caller-side inputs the backend gets, and error norms."""
import importlib
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

prob = importlib.import_module("honee-4aiad_b200.problem")


def reference_dir():
    """The reference source tree, or None: HONEE_REFERENCE_DIR when set, else the tree oracle/Makefile built oracle/_ref
    from (recorded in oracle/_ref/reference_dir.txt).  Tests that read reference sources skip when it is None."""
    d = os.environ.get("HONEE_REFERENCE_DIR")
    if not d:
        rec = os.path.join(ROOT, "oracle", "_ref", "reference_dir.txt")
        d = open(rec).read().strip() if os.path.exists(rec) else None
    return d if d and os.path.isdir(os.path.join(d, "qfunctions")) else None


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def oracle_mesh(mesh, basis, threads=0):
    return O.Mesh(mesh.num_elem, basis.P, basis.Q, mesh.offsets, basis.interp1d, basis.grad1d, basis.qweight1d, colors=mesh.colors,
                  num_threads=threads)


def case(n=(4, 4, 4), P=3, Q=3, periodic=(0, 0, 0), stab=prob.STAB_SUPG, seed=0, dt=1e-5, shift=None, idl=None, state="pulse", g=(0, 0, 0)):
    """A box, basis, context and state in the form of the benchmark workloads (3D Gaussian pulse or multi-mode)."""
    mesh = prob.box_mesh(n, P, periodic=periodic)
    basis = prob.tensor_basis(P, Q)
    ctx = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=stab, dt=dt,
                                 ijacobian_time_shift=(1.5 / dt if shift is None else shift), idl=idl, g=g)
    if state == "pulse":
        q = prob.gaussian_pulse_state(mesh, basis, ctx.gas, seed=seed)
    else:
        q = prob.multimode_state(mesh, basis, ctx.gas, seed=seed)
    rng = np.random.default_rng(seed + 1)
    q_dot = q * 1e-3 * rng.uniform(-1, 1, q.shape)
    return mesh, basis, ctx, q, q_dot


def oracle_ifunction(mesh, basis, ctx, q, q_dot, use_ref=False):
    m = oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    njd = 15 if ctx.idl_enable else 14
    jd = np.zeros(mesh.num_elem * njd * basis.Q ** 3)
    xq = O.coords_at_qpts(mesh.num_elem, basis.Q, mesh.x_elem)
    v = O.apply_ifunction(m, prob.context_bytes(ctx), q, q_dot, qdata, jd, num_jd=njd, x_q=xq, use_ref=use_ref)
    return v, jd, qdata, m
