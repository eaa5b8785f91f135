"""Implicit time-stepping driver on one GPU: the part of HONEE's `navierstokes` executable (examples/navierstokes.c) that
this backend covers.  It builds a periodic box problem, the geometric factors, the fused Newtonian operators and the BDF
time loop (hb_ts_*), runs it and reports the total-kinetic-energy and CFL monitors (src/monitor_totalkineticenergy.c,
src/monitor_cfl.c) with the solver's iteration counts and step times.

    python -m honee-4aiad_b200.navierstokes --problem taylor_green --faces 32 --degree 4 --steps 200 --cfl 1 [--mixed|--both]

`--cfl` is the acoustic CFL number on the node spacing, dt = cfl * h_node / (|u|max + c).

Problems: `taylor_green` (examples/taylor_green_vortex.yaml parameters, Re 1600, Ma 0.1, box [0, 2 pi]^3) and
`gaussian_pulse` (the acoustic pulse of the small configuration, on a periodic unit box).  Device buffers are torch
tensors; every operator, Krylov step and monitor is a kernel of this package.
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import sys
from dataclasses import dataclass, field

import numpy as np

from . import kernels as K
from . import problem as prob
from . import solver as S


@dataclass
class Run:
    rows: list = field(default_factory=list)      # monitor rows: step, time, KE, dissipations, min/max CFL
    stats: list = field(default_factory=list)     # solver statistics per step
    dofs: int = 0
    dt: float = 0.0

    def steps_per_second(self, skip=1):
        s = [st.seconds for st in self.stats[skip:]] or [st.seconds for st in self.stats]
        return 1.0 / (sum(s) / len(s))


def build_problem(name, faces, degree, q_extra=1, stab=prob.STAB_SUPG):
    P, Q = degree + 1, degree + 1 + q_extra
    if name == "taylor_green":
        L = 2 * math.pi
        mesh = prob.box_mesh((faces,) * 3, P, periodic=(1, 1, 1), hi=(L, L, L))
        basis = prob.tensor_basis(P, Q)
        tg = prob.taylor_green_context(degree, stab=stab)
        q0 = prob.taylor_green_state(mesh, basis, tg)
        ctx = tg.newt_ctx
        gas = ctx.gas
        V0 = math.sqrt(sum(tg.reference.velocity[i] ** 2 for i in range(3)))
        c0 = math.sqrt(gas.cp / gas.cv * (gas.cp - gas.cv) * tg.reference.temperature)
        vmax, volume = V0 + c0, L ** 3
    elif name == "gaussian_pulse":
        mesh = prob.box_mesh((faces,) * 3, P, periodic=(1, 1, 1))
        basis = prob.tensor_basis(P, Q)
        ctx = prob.newtonian_context(degree, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=stab)
        q0 = prob.gaussian_pulse_state(mesh, basis, ctx.gas)
        gas = ctx.gas
        vmax, volume = 10.0 + math.sqrt(gas.cp / gas.cv * (gas.cp - gas.cv) * 288.0), 1.0
    else:
        raise ValueError(f"unknown problem {name!r}")
    return mesh, basis, ctx, q0, vmax, volume


def run(name="taylor_green", faces=32, degree=4, q_extra=1, steps=10, dt=None, cfl=1.0, mixed=False, monitor_every=1,
        options=None, device="cuda:0", log=None):
    """Run `steps` BDF2 steps; dt defaults to the acoustic CFL number `cfl` on the node spacing,
    dt = cfl * h_node / (|u|max + c) with the initial state's velocity scale and sound speed."""
    import torch
    dev = torch.device(device)
    mesh, basis, ctx, q0, vmax, volume = build_problem(name, faces, degree, q_extra)
    h_node = (mesh.xs[-1] - mesh.xs[0]) / (faces * (basis.P - 1))
    dt = dt if dt is not None else cfl * h_node / vmax
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(dev)
    qdata = torch.empty(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=dev)
    op.setup_qdata(x, qdata)
    opts = S.default_options(dt=dt, bdf_order=2, jacobian_fp32=int(mixed), **(options or {}))
    cb = prob.context_bytes(ctx)
    ts = S.TimeStepper(op, cb, qdata, opts)
    q = torch.from_numpy(q0).to(dev)
    ts.set_state(q, 0.0)
    scratch = torch.empty(5 * mesh.num_elem, dtype=torch.float64, device=dev)
    out = Run(dofs=mesh.l_size, dt=dt)

    def monitor(step, t):
        ts.get_state(q)
        ke = S.monitor_ke(op, cb, q, qdata, scratch) / volume
        cmin, cmax = S.monitor_cfl(op, cb, q, qdata, dt, scratch)
        row = {"step": step, "time": t, "TotalKineticEnergy": ke[0], "StrainDissipation": ke[1], "DivergenceDissipation": ke[2],
               "VolumeExpansion": ke[3], "MuVorticity2": ke[4], "mincfl": cmin, "maxcfl": cmax}
        out.rows.append(row)
        return row

    monitor(0, 0.0)
    t = 0.0
    for step in range(1, steps + 1):
        st = ts.step()
        t += dt
        out.stats.append(st)
        if st.converged_reason != 1:
            raise RuntimeError(f"step {step}: Newton did not converge ({st})")
        if step % monitor_every == 0 or step == steps:
            row = monitor(step, t)
            if log:
                print(json.dumps({**row, "newton_its": st.newton_its, "ksp_its": st.ksp_its, "step_s": st.seconds}), file=log, flush=True)
    return out


def compare(a: Run, b: Run):
    """Largest relative difference of the kinetic energy and the strain dissipation between two runs (b against a), over
    the monitored steps they share."""
    keys = ["TotalKineticEnergy", "StrainDissipation"]
    res = {}
    for k in keys:
        ra = np.array([r[k] for r in a.rows])
        rb = np.array([r[k] for r in b.rows])
        n = min(len(ra), len(rb))
        res[k] = float(np.max(np.abs(rb[:n] - ra[:n])) / max(np.max(np.abs(ra[:n])), 1e-300))
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--problem", default="taylor_green", choices=["taylor_green", "gaussian_pulse"])
    ap.add_argument("--faces", type=int, default=32)
    ap.add_argument("--degree", type=int, default=4)
    ap.add_argument("--q-extra", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--dt", type=float, default=None)
    ap.add_argument("--cfl", type=float, default=1.0)
    ap.add_argument("--mixed", action="store_true", help="FP32 Krylov basis, Jacobian action and diagonal")
    ap.add_argument("--both", action="store_true", help="run FP64 and mixed and compare the monitors")
    ap.add_argument("--monitor-every", type=int, default=10)
    ap.add_argument("--csv", default=None, help="write the monitor rows of each run here (suffix _fp64 / _mixed)")
    ap.add_argument("--pc-type", default="jacobi", choices=["none", "jacobi", "vpbjacobi"], help="-pc_type of the Newton-Krylov solve")
    args = ap.parse_args(argv)
    pc = {"none": 0, "jacobi": 1, "vpbjacobi": 2}[args.pc_type]
    variants = [False, True] if args.both else [args.mixed]
    runs = {}
    for mixed in variants:
        r = run(args.problem, args.faces, args.degree, args.q_extra, args.steps, args.dt, args.cfl, mixed, args.monitor_every,
                options={"pc_jacobi": pc}, log=sys.stderr)
        runs[mixed] = r
        tag = "mixed" if mixed else "fp64"
        if args.csv:
            with open(args.csv.replace(".csv", f"_{tag}.csv"), "w", newline="") as f:
                w = csv.DictWriter(f, fieldnames=list(r.rows[0].keys()))
                w.writeheader()
                w.writerows(r.rows)
        newton = [s.newton_its for s in r.stats]
        ksp = [s.ksp_its for s in r.stats]
        print(json.dumps({"run": tag, "problem": args.problem, "faces": args.faces, "degree": args.degree, "dofs": r.dofs, "dt": r.dt,
                          "steps": len(r.stats), "steps_per_s": r.steps_per_second(), "newton_its_mean": float(np.mean(newton)),
                          "ksp_its_mean": float(np.mean(ksp)), "final": r.rows[-1]}), flush=True)
    if args.both:
        print(json.dumps({"mixed_vs_fp64": compare(runs[False], runs[True]),
                          "speedup_steps_per_s": runs[True].steps_per_second() / runs[False].steps_per_second()}), flush=True)


if __name__ == "__main__":
    main()
