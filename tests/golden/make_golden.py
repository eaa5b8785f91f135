"""Generate the golden fixtures in tests/golden/ from the reference itself (run in a container that has the reference).

  python tests/golden/make_golden.py [--ref REFERENCE_TREE]

Outputs (committed, so the tests need no reference tree):
  pointwise_newtonian.npz   seeded quadrature-point inputs and the outputs of the reference's own
                            IFunction_Newtonian_* / IJacobian_Newtonian_* QFunctions (qfunctions/newtonian.h:205-315),
                            compiled unchanged into oracle/_ref/libhonee_ref.so by oracle/Makefile
  taylorgreen_ke_step0.json the step-0 row of tests/output/taylorgreen_totalke.csv with the configuration that produced
                            it (examples/navierstokes.c:222, examples/taylor_green_vortex.yaml)
  unit_state.json           the UnitTests_Newtonian inputs and tolerances (problems/newtonian.c:947-987) with the
                            reference's StateToQ outputs for every (A, B) pair
  channel_prim_be5.npz      the same for "Channel, Primitive" (examples/navierstokes.c:253, -state_var primitive),
                            tests/output/channel-prim.bin
  channel_be5.npz           the free DOFs of the final state of the "Channel" run (examples/navierstokes.c:252:
                            examples/channel.yaml, 5 x 5 x 1 faces, 5 backward-Euler steps), tests/output/channel.bin
  gaussianwave_explicit.npz the free DOFs of the final state of "Gaussian Wave, explicit, supg, IDL" (examples/navierstokes.c:233),
                            tests/output/gaussianwave-explicit.bin (a 64-bit-index HONEE file)
  ref_*.bin                 copies of tests/output/{channel,channel-prim,taylor-green,gaussianwave-explicit}.bin, the reference's own
                            solution files, for the checks of the file-format reader (honee-4aiad_b200/honee_file.py)
  taylorgreen_rk4.npz       every row of tests/output/taylorgreen_totalke.csv (steps 0, 2, 3 of the explicit RK4 run of
                            examples/navierstokes.c:222) and the final state of that run, tests/output/taylor-green.bin
                            (HONEE binary format, src/honee-file.c:194-217: int32 token, int32 step, float64 time, then a
                            PETSc Vec: int32 class id, int32 length, big-endian float64 values in DMPlex order)
"""
from __future__ import annotations

import argparse
import csv
import ctypes as C
import importlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def seeded_points(rng, gas, Q, state_var):
    """Perturbed states around an atmospheric background, with reference gradients and an affine-ish dXdx."""
    prob = importlib.import_module("honee-4aiad_b200.problem")
    P = 101325 * (1 + 0.01 * rng.uniform(-1, 1, Q))
    T = 288 * (1 + 0.01 * rng.uniform(-1, 1, Q))
    u = rng.uniform(-30, 30, (3, Q))
    U = prob.conservative_from_primitive(gas, P, u, T)
    Y = np.stack([P, u[0], u[1], u[2], T])
    if state_var == 0:
        q = U
    elif state_var == 1:
        q = Y
    else:
        import oracle as O
        q = np.zeros((5, Q))
        for i in range(Q):
            out = (C.c_double * 5)()
            O.ref().ref_StateToQ(C.byref(gas), (C.c_double * 5)(*Y[:, i]), 1, 2, out)
            q[:, i] = out[:]
    scale = np.abs(q) + 1e-3
    grad_q = rng.normal(size=(3, 5, Q)) * scale[None] * 0.05
    q_dot = rng.normal(size=(5, Q)) * scale * 3.0
    h = 1 / 16.
    dXdx = np.eye(3)[:, :, None] * (2 / h) + rng.normal(size=(3, 3, Q)) * 1.5
    qdata = np.concatenate([rng.uniform(0.5, 1, (1, Q)) * (h / 2) ** 3, dXdx.reshape(9, Q)])
    x = rng.uniform(0, 1, (3, Q))
    dq = rng.normal(size=(5, Q)) * scale * 1e-3
    grad_dq = rng.normal(size=(3, 5, Q)) * scale[None] * 1e-2
    return q, grad_q, q_dot, qdata, x, dq, grad_dq


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HONEE_REFERENCE_DIR"),
                    help="the reference tree (default: HONEE_REFERENCE_DIR, else the tree oracle/_ref was built from)")
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")] + ([f"REF={args.ref}"] if args.ref else []), check=True)
    if not args.ref:
        args.ref = open(os.path.join(ROOT, "oracle", "_ref", "reference_dir.txt")).read().strip()
    import oracle as O
    R = O.ref()
    assert R is not None, "reference QFunctions were not built"
    prob = importlib.import_module("honee-4aiad_b200.problem")

    # ---- point-wise golden vectors
    rng = np.random.default_rng(20240611)
    Q = 24
    cases = []
    names = {0: "Conserv", 1: "Prim", 2: "Entropy"}
    for state_var in (0, 1, 2):
        for stab in (0, 1, 2):
            cases.append(dict(state_var=state_var, stab=stab, idl=False))
    cases.append(dict(state_var=0, stab=2, idl=True))
    cases.append(dict(state_var=0, stab=2, idl=False, gravity=True))
    arrays = {}
    meta = []
    for ci, cs in enumerate(cases):
        ctx = prob.newtonian_context(3, stab=cs["stab"], state_var=cs["state_var"], dt=1e-5, ijacobian_time_shift=1.5e5,
                                     g=(0.3, -9.81, 0.1) if cs.get("gravity") else (0., 0., 0.),
                                     idl=(2e-3, 0.2, 0.5, 101000.) if cs["idl"] else None)
        cb = prob.context_bytes(ctx)
        njd = 15 if cs["idl"] else 14
        q, gq, qd, qdata, x, dq, gdq = seeded_points(rng, ctx.gas, Q, cs["state_var"])
        ins = [np.ascontiguousarray(a) for a in (q, gq, qd, qdata, x)]
        v = np.zeros((5, Q)); gv = np.zeros((3, 5, Q)); jd = np.zeros((njd, Q))
        assert O.call_qf(getattr(R, f"ref_IFunction_Newtonian_{names[cs['state_var']]}"), cb, Q, ins, [v, gv, jd]) == 0
        jv = np.zeros((5, Q)); jgv = np.zeros((3, 5, Q))
        jins = [np.ascontiguousarray(a) for a in (dq, gdq, qdata, jd)]
        assert O.call_qf(getattr(R, f"ref_IJacobian_Newtonian_{names[cs['state_var']]}"), cb, Q, jins, [jv, jgv]) == 0
        for k, a in dict(ctx=np.frombuffer(cb, dtype=np.uint8), q=q, grad_q=gq, q_dot=qd, qdata=qdata, x=x, v=v, grad_v=gv, jac_data=jd, dq=dq,
                         grad_dq=gdq, jv=jv, jgrad_v=jgv).items():
            arrays[f"c{ci}_{k}"] = a
        meta.append(dict(cs, njd=njd, qf=names[cs["state_var"]]))
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    arrays["Q"] = np.array(Q)
    np.savez_compressed(os.path.join(HERE, "pointwise_newtonian.npz"), **arrays)

    # ---- Taylor-Green KE step 0 (tests/output/taylorgreen_totalke.csv)
    rows = [r for r in csv.reader(open(os.path.join(args.ref, "tests/output/taylorgreen_totalke.csv"))) if r and not r[0].startswith("#")]
    header, first = rows[0], rows[1]
    ke = {h: float(v) for h, v in zip(header, first)}
    ke.update(dict(source="tests/output/taylorgreen_totalke.csv (step 0)", faces=[2, 2, 2], degree=2, P=3, Q=3, box=[0, 6.283185307179586],
                   periodic=True, reference_velocity=[1, 0, 0], reference_temperature=0.2490535963, reference_pressure=71.42857143,
                   mu=0.000625, k=0.8836267606, cv=717, cp=1003.8, csv_rtol=1e-9, csv_ztol=3e-10))
    json.dump(ke, open(os.path.join(HERE, "taylorgreen_ke_step0.json"), "w"), indent=1)

    # ---- Taylor-Green explicit RK4 run: every KE row and the final state (tests/output/taylor-green.bin)
    names = header[2:]
    table = np.array([[float(v) for v in r] for r in rows[1:]])
    raw = open(os.path.join(args.ref, "tests/output/taylor-green.bin"), "rb").read()
    token, step = np.frombuffer(raw[:8], dtype=">i4")
    t_final = np.frombuffer(raw[8:16], dtype=">f8")[0]
    classid, length = np.frombuffer(raw[16:24], dtype=">i4")
    state = np.frombuffer(raw[24:24 + 8 * int(length)], dtype=">f8").astype(np.float64)
    assert len(raw) == 24 + 8 * int(length) and int(token) == 0x0CEEDF32 and int(classid) == 1211214
    np.savez_compressed(os.path.join(HERE, "taylorgreen_rk4.npz"), ke_steps=table[:, 0].astype(np.int64), ke_times=table[:, 1],
                        ke=table[:, 2:], ke_names=np.array(names), final_step=np.int64(step), final_time=np.float64(t_final),
                        final_state=state, dt=np.float64(2e-3), tableau=np.array("4"), mass_ksp=np.array("gmres"),
                        mass_pc_jacobi=np.array("diagonal"), source=np.array("tests/output/taylorgreen_totalke.csv, tests/output/taylor-green.bin"))

    # ---- Channel run (examples/navierstokes.c:252): free DOFs of the final state
    raw = open(os.path.join(args.ref, "tests/output/channel.bin"), "rb").read()
    token, step = np.frombuffer(raw[:8], dtype=">i4")
    t_final = np.frombuffer(raw[8:16], dtype=">f8")[0]
    classid, length = np.frombuffer(raw[16:24], dtype=">i4")
    assert len(raw) == 24 + 8 * int(length) and int(classid) == 1211214
    np.savez_compressed(os.path.join(HERE, "channel_be5.npz"), final_step=np.int64(step), final_time=np.float64(t_final),
                        free_state=np.frombuffer(raw[24:], dtype=">f8").astype(np.float64), faces=np.array([5, 5, 1]), degree=np.int64(1),
                        q_extra=np.int64(2), box_hi=np.array([0.01, 0.01, 0.001]), mu=np.float64(0.01), umax=np.float64(40.0),
                        dt=np.float64(5e-6), steps=np.int64(5), essential=np.array("y-:1,2,3 y+:1,2,3 z-:3 z+:3"), compare_atol=np.float64(2e-11),
                        source=np.array("tests/output/channel.bin (examples/navierstokes.c:252, examples/channel.yaml)"))

    # ---- "Channel, Primitive" (examples/navierstokes.c:253): the same run with -state_var primitive
    raw = open(os.path.join(args.ref, "tests/output/channel-prim.bin"), "rb").read()
    token, step = np.frombuffer(raw[:8], dtype=">i4")
    t_final = np.frombuffer(raw[8:16], dtype=">f8")[0]
    classid, length = np.frombuffer(raw[16:24], dtype=">i4")
    assert len(raw) == 24 + 8 * int(length) and int(classid) == 1211214
    np.savez_compressed(os.path.join(HERE, "channel_prim_be5.npz"), final_step=np.int64(step), final_time=np.float64(t_final),
                        free_state=np.frombuffer(raw[24:], dtype=">f8").astype(np.float64), faces=np.array([5, 5, 1]), degree=np.int64(1),
                        q_extra=np.int64(2), box_hi=np.array([0.01, 0.01, 0.001]), mu=np.float64(0.01), umax=np.float64(40.0),
                        dt=np.float64(5e-6), steps=np.int64(5), essential=np.array("y-:1,2,3 y+:1,2,3 z-:3 z+:3"), compare_atol=np.float64(2e-11),
                        state_var=np.int64(1),
                        source=np.array("tests/output/channel-prim.bin (examples/navierstokes.c:253, examples/channel.yaml, -state_var primitive)"))

    # ---- Gaussian wave, explicit, SUPG, IDL (examples/navierstokes.c:233): free DOFs of the final state, a 64-bit-index file
    #      (token 0x0CEEDF64: int64 step, float64 time, int64 class id, int64 length, values)
    raw = open(os.path.join(args.ref, "tests/output/gaussianwave-explicit.bin"), "rb").read()
    assert int(np.frombuffer(raw[:4], dtype=">i4")[0]) == 0x0CEEDF64
    step = np.frombuffer(raw[4:12], dtype=">i8")[0]
    t_final = np.frombuffer(raw[12:20], dtype=">f8")[0]
    classid, length = np.frombuffer(raw[20:36], dtype=">i8")
    assert int(classid) == 1211214 and len(raw) == 36 + 8 * int(length)
    np.savez_compressed(os.path.join(HERE, "gaussianwave_explicit.npz"), final_step=np.int64(step), final_time=np.float64(t_final),
                        free_state=np.frombuffer(raw[36:], dtype=">f8").astype(np.float64), faces=np.array([2, 2, 1]), degree=np.int64(3),
                        box_hi=np.array([1.0, 1.0, 0.025]), reference_PuT=np.array([71.75, 2.0, 2.0, 0.0, 0.25]),
                        epicenter=np.array([0.33, 0.75, 0.0]), amplitude=np.float64(2.0), width=np.float64(0.05), mu=np.float64(0.0),
                        dt=np.float64(2e-3), steps=np.int64(5), rk_type=np.array("5f"), mass_ksp=np.array("gmres"),
                        mass_pc_jacobi=np.array("diagonal"), idl=np.array([2e-3, 0.0, 0.25, 70.0]), compare_atol=np.float64(1e-8),
                        source=np.array("tests/output/gaussianwave-explicit.bin (examples/navierstokes.c:233, examples/gaussianwave.yaml)"))

    # ---- raw solution files of the reference's runs (32- and 64-bit-index HONEE files) for the file-format reader
    import shutil
    for name in ("channel.bin", "channel-prim.bin", "taylor-green.bin", "gaussianwave-explicit.bin"):
        shutil.copyfile(os.path.join(args.ref, "tests/output", name), os.path.join(HERE, "ref_" + name))

    # ---- UnitTests_Newtonian inputs (problems/newtonian.c:947-987) and reference StateToQ outputs
    ctx = prob.newtonian_context(2)
    gas = ctx.gas
    T, rho, ub = 200., 1.2, 40.
    gamma = gas.cp / gas.cv
    Pp = (gamma - 1) * rho * gas.cv * T
    u = [ub, ub * 1.1, ub * 1.2]
    ek = 0.5 * sum(a * a for a in u)
    ei = gas.cv * T
    ent = np.log(Pp) - gamma * np.log(rho)
    rp = rho / Pp
    Y0 = [Pp, *u, T]
    U0 = [rho, rho * u[0], rho * u[1], rho * u[2], rho * (ek + ei)]
    V0 = [(gamma - ent) / (gamma - 1) - rp * ek, rp * u[0], rp * u[1], rp * u[2], -rp]
    conv = {}
    for a, A0 in ((0, U0), (1, Y0), (2, V0)):
        for b in (0, 1, 2):
            out = (C.c_double * 5)()
            R.ref_StateToQ(C.byref(gas), (C.c_double * 5)(*A0), a, b, out)
            conv[f"{a}->{b}"] = list(out)
    json.dump(dict(Y0=Y0, U0=U0, V0=V0, rtol_roundtrip="20*DBL_EPSILON", rtol_fwd=5e-6, fd_eps=4e-7, state_to_q=conv,
                   source="problems/newtonian.c:947-987"), open(os.path.join(HERE, "unit_state.json"), "w"), indent=1)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
