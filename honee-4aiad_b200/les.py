"""Learned-closure coarse LES of the decaying Taylor-Green vortex, end to end on one GPU.

  1. fine run: the plain method (no closure) on `fine_faces`^3 elements, snapshots of the state every `snap_every`
     coarse steps' worth of time
  2. each snapshot through the differential filter (filter width = the coarse element size: grid-based width, width
     scaling = fine/coarse element ratio, kernel scaling 0.1 as src/differential_filter.c defaults) and into training
     pairs at the fine quadrature points (model inputs of the filtered velocity gradient, the filtered stress
     u_i u_j - u_i u_j in the model's output frame)
  3. min-max normalisation of the targets (their bounds become the model's de-normalisation bounds, OutScaling), the
     network (6-20-20-6, ReLU, Xavier init from a seed) trained with Adam on the GPU by this package's kernels
  4. two coarse runs on `coarse_faces`^3 elements from the filtered initial state (the coarse nodes are a subset of the
     fine ones for these nested meshes, so the filtered fine field is injected): without the closure, and with the
     trained network in the residual (hb_ts_set_sgs), implicit with matrix-free Krylov products by default
  5. both compared with the filtered fine solution through the kinetic-energy monitor (total KE and the resolved strain
     dissipation), with the GPU time of each run

    python -m honee-4aiad_b200.les [--fine-faces 96 --coarse-faces 24 --degree 2 --t-end 2.0 ...]

Everything on the device is a kernel of this package (operators, Krylov, filter, training, inference); torch tensors are
the buffers.  Time steps are the BDF2 time loop of hb_solver.c at acoustic CFL `cfl` on each mesh's node spacing, the
fine step a divisor of the coarse step so the snapshots fall on coarse step boundaries.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import filter as FL
from . import kernels as K
from . import problem as prob
from . import sgs as SG
from . import solver as S


class TGMesh:
    """Periodic Taylor-Green box with its element operator, geometric factors and monitors."""

    def __init__(self, faces, degree, q_extra=1, device="cuda:0"):
        import torch
        self.torch = torch
        L = 2 * math.pi
        self.faces, self.P, self.Q = faces, degree + 1, degree + 1 + q_extra
        self.mesh = prob.box_mesh((faces,) * 3, self.P, periodic=(1, 1, 1), hi=(L, L, L))
        self.basis = prob.tensor_basis(self.P, self.Q)
        self.tg = prob.taylor_green_context(degree)
        self.ctx = self.tg.newt_ctx
        self.cb = prob.context_bytes(self.ctx)
        self.op = K.ElemOp(self.mesh, self.basis)
        dev = torch.device(device)
        self.dev = dev
        x = torch.from_numpy(np.ascontiguousarray(self.mesh.x_elem)).to(dev)
        self.qdata = torch.empty(self.mesh.num_elem * 10 * self.Q ** 3, dtype=torch.float64, device=dev)
        self.op.setup_qdata(x, self.qdata)
        self.scratch = torch.empty(5 * self.mesh.num_elem, dtype=torch.float64, device=dev)
        self.volume = L ** 3
        gas = self.ctx.gas
        self.wave_speed = 1.0 + math.sqrt(gas.cp / gas.cv * (gas.cp - gas.cv) * self.tg.reference.temperature)
        self.h_node = L / (faces * (self.P - 1))

    def initial_state(self):
        return self.torch.from_numpy(prob.taylor_green_state(self.mesh, self.basis, self.tg)).to(self.dev)

    def ke(self, q):
        s = S.monitor_ke(self.op, self.cb, q, self.qdata, self.scratch) / self.volume
        return {"TotalKineticEnergy": float(s[0]), "StrainDissipation": float(s[1]), "MuVorticity2": float(s[4])}


def run_steps(m: TGMesh, dt, n_steps, every, mixed=True, sgs=None, on_snapshot=None, q0=None, **opts):
    """BDF2 steps from q0 (default: the Taylor-Green initial condition); calls on_snapshot(k, q) every `every` steps
    (and at step 0).  Returns the monitor rows and the summed step time (CUDA events inside hb_ts_step)."""
    ts = S.TimeStepper(m.op, m.cb, m.qdata, dt=dt, bdf_order=2, jacobian_fp32=int(mixed), **opts)
    if sgs is not None:
        ts.set_sgs(*sgs)
    q = m.initial_state() if q0 is None else q0.clone()
    ts.set_state(q, 0.0)
    rows, seconds = [], 0.0
    rows.append({"time": 0.0, **m.ke(q)})
    if on_snapshot:
        on_snapshot(0, q)
    for k in range(1, n_steps + 1):
        st = ts.step()
        if st.converged_reason != 1:
            raise RuntimeError(f"step {k}: Newton did not converge ({st})")
        seconds += st.seconds
        if k % every == 0:
            ts.get_state(q)
            rows.append({"time": k * dt, **m.ke(q)})
            if on_snapshot:
                on_snapshot(k // every, q)
    return rows, seconds


def _max_rel_err(rows, ref, key, scale, from_start=False, upto=None):
    """max over the monitored times after t = 0 (up to row `upto`) of |a - b| / scale; from_start compares the changes
    since t = 0."""
    n = min(len(rows), len(ref), (upto + 1) if upto else 1 << 30)
    a0, b0 = (rows[0][key], ref[0][key]) if from_start else (0.0, 0.0)
    return max(abs((rows[k][key] - a0) - (ref[k][key] - b0)) for k in range(1, n)) / scale


def study(fine_faces=96, coarse_faces=24, degree=2, t_end=2.0, snaps=4, cfl=1.0, train_steps=4000, batch=65536, lr=1e-3, seed=0,
          clip=1e-3, implicit_closure=False, coarse_substeps=1, cache=None, clamp_outputs=False, no_backscatter=True, log=None, scales=None):
    """implicit_closure: the closure inside Newton with matrix-free Krylov products (FP64); by default it is evaluated once
    per step at the previous state (explicit, mixed-precision Krylov).  coarse_substeps divides the coarse step of both
    coarse runs.  cache: a directory where the fine-run products (filtered monitors, injected initial state, trained
    model) are stored after stages 1-3 and reused by later calls with the same fine configuration.  clamp_outputs and
    no_backscatter select the inference limiters of the fused closure (HbMlpDesc; both off = the reference's evaluation).
    Backscatter limiting is on by default: without it the trained closure fed energy into the resolved scales of the 24^3
    Taylor-Green run and the run diverged near t = 1.5 at every time step tried.

    scales: candidate stress scales gamma (each multiplies the de-normalisation bounds, so the modelled stress scales by
    gamma).  With candidates, every scale runs the coarse closure and the one whose worst error ratio to the plain coarse
    run is smallest on the first half of the snapshots (validation) is kept; the reported errors cover all snapshots.
    Without, the trained model is used as it is (gamma = 1)."""
    import os
    import torch

    def say(**kw):
        if log:
            print(json.dumps(kw), file=log, flush=True)

    if fine_faces % coarse_faces:
        raise ValueError("the fine element count must be a multiple of the coarse one")
    ratio = fine_faces // coarse_faces
    coarse = TGMesh(coarse_faces, degree)
    dt_c = cfl * coarse.h_node / coarse.wave_speed
    every_c = max(1, int(round(t_end / dt_c / snaps)))
    n_c = every_c * snaps
    dt_f, n_f, every_f = dt_c / ratio, n_c * ratio, every_c * ratio
    out = {"fine_faces": fine_faces, "coarse_faces": coarse_faces, "degree": degree, "dt_fine": dt_f, "dt_coarse": dt_c, "steps_fine": n_f,
           "steps_coarse": n_c, "t_end": n_c * dt_c, "snapshots": snaps}

    key = f"tg_f{fine_faces}_c{coarse_faces}_d{degree}_t{t_end}_s{snaps}_cfl{cfl}_n{train_steps}_b{batch}_seed{seed}"
    cpath = os.path.join(cache, key + ".npz") if cache else None
    if cpath and os.path.exists(cpath):
        z = np.load(cpath, allow_pickle=False)
        saved = json.loads(str(z["meta"]))
        out.update(saved)
        ref_rows, weights, bounds = saved["filtered_fine"], z["weights"], z["bounds"]
        q_inject = [torch.from_numpy(z["q_inject"]).to(coarse.dev)]
        sec_f = saved["fine"]["gpu_seconds"]
        say(stage="loaded fine run and model", path=cpath)
    else:
        ref_rows, weights, bounds, q_inject, sec_f, d = _fine_and_train(out, coarse, fine_faces, degree, ratio, dt_f, n_f, every_f, clip, seed, batch,
                                                                      lr, train_steps, say)
        if cpath:
            os.makedirs(cache, exist_ok=True)
            meta = {k: out[k] for k in ("fine", "filtered_fine", "filter_seconds", "training", "dofs_fine", "dofs_coarse")}
            np.savez(cpath, meta=json.dumps(meta), weights=weights, bounds=bounds, q_inject=q_inject[0].cpu().numpy())
    out["weights"] = np.asarray(weights).tolist()

    out["limiters"] = {"clamp_outputs": bool(clamp_outputs), "no_backscatter": bool(no_backscatter)}

    # 4. coarse runs without and with the closure (same step, from the same filtered initial state)
    dt_cs, n_cs, every_cs = dt_c / coarse_substeps, n_c * coarse_substeps, every_c * coarse_substeps
    out["coarse_dt"], out["coarse_steps"] = dt_cs, n_cs
    rows_c0, sec_c0 = run_steps(coarse, dt_cs, n_cs, every_cs, mixed=True, q0=q_inject[0])
    out["coarse_plain"] = {"gpu_seconds": sec_c0, "rows": rows_c0}

    def closure_run(gamma):
        d = SG.desc(20, 20, 0.0, np.asarray(bounds) * gamma, clamp_outputs=clamp_outputs, no_backscatter=no_backscatter)
        try:
            rows, sec = run_steps(coarse, dt_cs, n_cs, every_cs, mixed=not implicit_closure, sgs=(d, np.asarray(weights, dtype=np.float32)),
                                  q0=q_inject[0], jfnk=int(implicit_closure))
            return rows, sec, None
        except RuntimeError as e:
            return [], float("nan"), str(e)

    half = max(1, snaps // 2)
    if scales:
        cands = []
        for g in scales:
            rows, sec, div = closure_run(float(g))
            score = None
            if div is None:
                ev = _errors(ref_rows, rows, upto=half)
                e0 = _errors(ref_rows, rows_c0, upto=half)
                score = max(ev[k] / e0[k] for k in ev)
            cands.append({"gamma": float(g), "diverged": div, "validation_worst_error_ratio": score, "rows": rows, "gpu_seconds": sec})
            say(stage="closure scale", gamma=g, diverged=div, score=score)
        ok = [c for c in cands if c["diverged"] is None]
        best = min(ok, key=lambda c: c["validation_worst_error_ratio"]) if ok else cands[-1]
        out["scale_selection"] = {"validation_snapshots": half, "candidates": [{k: v for k, v in c.items() if k != "rows"} for c in cands],
                                  "chosen_gamma": best["gamma"]}
        rows_c1, sec_c1, diverged = best["rows"], best["gpu_seconds"], best["diverged"]
    else:
        rows_c1, sec_c1, diverged = closure_run(1.0)
    out["coarse_closure"] = {"gpu_seconds": sec_c1, "rows": rows_c1, "diverged": diverged, "implicit": bool(implicit_closure)}
    return _compare(out, ref_rows, rows_c0, rows_c1, sec_f, sec_c1)


def _errors(ref_rows, rows, upto=None):
    """KE, KE-decay and resolved-dissipation errors of a coarse run against the filtered fine rows."""
    ke0 = ref_rows[0]["TotalKineticEnergy"]
    eps_scale = max(abs(r["StrainDissipation"]) for r in ref_rows)
    return {"ke_err": _max_rel_err(rows, ref_rows, "TotalKineticEnergy", ke0, upto=upto),
            "ke_decay_err": _max_rel_err(rows, ref_rows, "TotalKineticEnergy", max(ke0 - r["TotalKineticEnergy"] for r in ref_rows),
                                         from_start=True, upto=upto),
            "dissipation_err": _max_rel_err(rows, ref_rows, "StrainDissipation", eps_scale, upto=upto)}


def _fine_and_train(out, coarse, fine_faces, degree, ratio, dt_f, n_f, every_f, clip, seed, batch, lr, train_steps, say):
    import torch
    # 1-2. fine run, filtered snapshots, training pairs
    fine = TGMesh(fine_faces, degree)
    out["dofs_fine"], out["dofs_coarse"] = fine.mesh.l_size, coarse.mesh.l_size
    filt = FL.DifferentialFilter(fine.op, fine.qdata, fine.cb, grid_based_width=True, width_scaling=(float(ratio),) * 3, kernel_scaling=0.1)
    nq = fine.mesh.num_elem * fine.Q ** 3
    Xs, Ys, ref_rows = [], [], []
    t_filter = [0.0]
    q_inject = [None]

    def on_snap(k, q):
        t0 = time.perf_counter()
        fbar, its, rel = filt.filter_state(q)
        qf = torch.empty(fine.mesh.l_size, dtype=torch.float64, device=fine.dev)
        filt.conservative(fbar, qf)
        ref_rows.append({"time": k * every_f * dt_f, **fine.ke(qf), "filter_cg_its": its})
        if k == 0:  # the coarse runs start from the filtered initial state, injected at the shared nodes
            Nf = fine.mesh.node_dims[0]
            q_inject[0] = qf.view(Nf, Nf, Nf, 5)[::ratio, ::ratio, ::ratio, :].contiguous().view(-1)
        if k > 0:
            X = torch.empty(nq, 6, dtype=torch.float32, device=fine.dev)
            Y = torch.empty_like(X)
            filt.training_pairs(fbar, float(ratio), X, Y)
            Xs.append(X)
            Ys.append(Y)
        torch.cuda.synchronize()
        t_filter[0] += time.perf_counter() - t0
        say(stage="fine snapshot", k=k, **ref_rows[-1])

    rows_f, sec_f = run_steps(fine, dt_f, n_f, every_f, mixed=True, on_snapshot=on_snap)
    out["fine"] = {"gpu_seconds": sec_f, "rows": rows_f}
    out["filtered_fine"] = ref_rows
    out["filter_seconds"] = t_filter[0]
    del fine, filt
    torch.cuda.empty_cache()

    # 3. targets: drop non-finite rows, clip to the [clip, 1 - clip] quantiles per column, min-max normalise; train
    X = torch.cat(Xs)
    Y = torch.cat(Ys)
    del Xs, Ys
    keep = torch.isfinite(X).all(1) & torch.isfinite(Y).all(1)
    X, Y = X[keep].contiguous(), Y[keep].contiguous()
    g = torch.Generator(device=X.device).manual_seed(seed)
    sub = Y[torch.randint(0, Y.shape[0], (min(Y.shape[0], 1_000_000),), device=Y.device, generator=g)]
    lo = torch.quantile(sub, clip, dim=0)
    hi = torch.quantile(sub, 1 - clip, dim=0)
    Y = torch.maximum(torch.minimum(Y, hi), lo).contiguous()
    bounds = np.stack([lo.cpu().numpy(), hi.cpu().numpy()], 1).reshape(12).astype(np.float64)
    SG.normalize_targets(Y, bounds)
    d = SG.desc(20, 20, 0.0, bounds)
    tr = SG.Trainer(d, SG.xavier_init(d, seed), batch=batch, lr=lr, seed=seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = tr.train(X, Y, train_steps, log_every=max(1, train_steps // 10))
    torch.cuda.synchronize()
    out["training"] = {"samples": int(X.shape[0]), "steps": train_steps, "batch": batch, "lr": lr, "seconds": time.perf_counter() - t0,
                       "loss": hist, "bounds": bounds.tolist()}
    say(stage="trained", **{k: v for k, v in out["training"].items() if k != "bounds"})
    weights = tr.params()
    del X, Y, tr
    torch.cuda.empty_cache()
    return ref_rows, weights, bounds, q_inject, sec_f, d


def _compare(out, ref_rows, rows_c0, rows_c1, sec_f, sec_c1):
    """errors of both coarse runs against the filtered fine solution at the snapshot times"""
    res = {}
    for name, rows in (("plain", rows_c0), ("closure", rows_c1)):
        if len(rows) < 2:
            continue
        res[name] = _errors(ref_rows, rows)
    out["errors_vs_filtered_fine"] = res
    out["cost_ratio_fine_over_closure"] = sec_f / sec_c1 if sec_c1 == sec_c1 and sec_c1 > 0 else None
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="learned-closure coarse LES of the Taylor-Green vortex")
    ap.add_argument("--fine-faces", type=int, default=96)
    ap.add_argument("--coarse-faces", type=int, default=24)
    ap.add_argument("--degree", type=int, default=2)
    ap.add_argument("--t-end", type=float, default=2.0)
    ap.add_argument("--snaps", type=int, default=4)
    ap.add_argument("--cfl", type=float, default=1.0)
    ap.add_argument("--train-steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--coarse-substeps", type=int, default=1, help="divide the coarse time step of both coarse runs")
    ap.add_argument("--implicit-closure", action="store_true", help="closure inside Newton with matrix-free Krylov products")
    ap.add_argument("--cache", default=None, help="directory to keep / reuse the fine run and the trained model")
    ap.add_argument("--clamp-outputs", action="store_true", help="limit the network outputs to the training range")
    ap.add_argument("--backscatter", action="store_true", help="keep the model's stress where tau : S > 0 (the reference's evaluation)")
    ap.add_argument("--out", default=None, help="write the full result (monitor rows, loss history, weights) as JSON here")
    ap.add_argument("--scales", default=None, help="comma-separated candidate stress scales, chosen on the first half of the snapshots")
    a = ap.parse_args(argv)
    res = study(a.fine_faces, a.coarse_faces, a.degree, a.t_end, a.snaps, a.cfl, a.train_steps, a.batch, a.lr, a.seed,
                implicit_closure=a.implicit_closure, coarse_substeps=a.coarse_substeps, cache=a.cache, clamp_outputs=a.clamp_outputs,
                no_backscatter=not a.backscatter, log=sys.stderr, scales=[float(v) for v in a.scales.split(",")] if a.scales else None)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
    summary = {k: v for k, v in res.items() if k not in ("weights", "fine", "coarse_plain", "coarse_closure", "filtered_fine", "training")}
    summary["cost_ratio_fine_over_plain"] = res["fine"]["gpu_seconds"] / res["coarse_plain"]["gpu_seconds"]
    summary["fine_gpu_seconds"] = res["fine"]["gpu_seconds"]
    summary["coarse_plain_gpu_seconds"] = res["coarse_plain"]["gpu_seconds"]
    summary["coarse_closure_gpu_seconds"] = res["coarse_closure"]["gpu_seconds"]
    summary["final_loss"] = res["training"]["loss"][-1]
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
