"""Benchmark: GDoF/s of the Newtonian residual + Jacobian apply on B200, FP64 and FP32-mixed.

Workload (the at-scale operator configuration): unit cube, 64^3 hex elements, degree 3 (P=4 nodes, Q=5 Gauss points per
direction), 5 conservative fields, ideal gas (cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257), SUPG, dt=1e-5, BDF2 shift
3/(2 dt); state = background (P=101325, T=288, u=(10,0,0)) plus 8 seeded sinusoidal modes (|k| <= 8, 1e-3 relative).
L-vector 7,189,057 nodes x 5 = 35,945,285 DOF; 32,768,000 quadrature points.

One step = one IFunction apply (writes the residual and the stored Jacobian data) + one IJacobian action, the unit of
work of a Newton-Krylov iteration.  value = DOF / step time (GDoF/s), whole job over N GPUs (replicas, weak scaling).
Inputs are larger than L2 (qdata alone is 2.6 GB), so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--size 64]
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
METRIC = "GDoF/s residual+Jacobian apply, FP64 vs FP32-mixed, at stated FP64-oracle error"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def workload(n, P=4, Q=5):
    prob = importlib.import_module("honee-4aiad_b200.problem")
    mesh = prob.box_mesh((n, n, n), P)
    basis = prob.tensor_basis(P, Q)
    ctx = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=prob.STAB_SUPG, dt=1e-5, ijacobian_time_shift=1.5e5)
    q = prob.multimode_state(mesh, basis, ctx.gas, seed=0)
    rng = np.random.default_rng(1)
    q_dot = q * 1e-3 * rng.uniform(-1, 1, q.shape)
    dq = q * 1e-4 * rng.uniform(-1, 1, q.shape)
    return prob, mesh, basis, ctx, q, q_dot, dq


def algorithmic_bytes(N_L, N_q, E, P, f32=False):
    """Per-apply algorithmic bytes: unique L-vector traffic, qdata (10 doubles) and jac_data (14 values) per point, int32
    offsets.  IFunction reads q, q_dot, writes v; IJacobian reads dq, writes v."""
    b_if = 8 * 3 * N_L + 8 * N_q * 10 + (4 if f32 else 8) * N_q * 14 + 4 * E * P ** 3
    b_ij = (4 if f32 else 8) * 2 * N_L + 8 * N_q * 10 + (4 if f32 else 8) * N_q * 14 + 4 * E * P ** 3
    return b_if, b_ij


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.count(",") >= 8]
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------------------------------------------------------------
# CPU legs (oracle = the checker / baseline; never the measured product)

def cpu_leg(n_sample, use_ref, reps=3, warmup=1):
    """Time the reference CPU path (reference QFunctions under the libCEED-semantics oracle driver, OpenMP over element
    colours, all host threads) on `n_sample`^3 elements of the same workload: `warmup` untimed steps, then the median of
    `reps` timed steps, each one IFunction apply + one IJacobian action."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    if use_ref and O.ref() is None:
        use_ref = False
    prob, mesh, basis, ctx, q, q_dot, dq = workload(n_sample)
    threads = os.cpu_count() or 1
    m = O.Mesh(mesh.num_elem, basis.P, basis.Q, mesh.offsets, basis.interp1d, basis.grad1d, basis.qweight1d, colors=mesh.colors,
               num_threads=threads)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    jd = np.zeros(mesh.num_elem * 14 * basis.Q ** 3)
    cb = prob.context_bytes(ctx)
    for _ in range(warmup):
        O.apply_ifunction(m, cb, q, q_dot, qdata, jd, use_ref=use_ref)
        O.apply_ijacobian(m, cb, dq, qdata, jd, use_ref=use_ref)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        O.apply_ifunction(m, cb, q, q_dot, qdata, jd, use_ref=use_ref)
        O.apply_ijacobian(m, cb, dq, qdata, jd, use_ref=use_ref)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return {"value": mesh.l_size / t / 1e9, "unit": "GDoF/s", "cores": threads, "kind": "reference" if use_ref else "port",
            "sample": f"{n_sample}^3 elements P=4 Q=5 ({mesh.l_size} DOF), IFunction+IJacobian, {warmup} untimed + median of {reps} timed steps",
            "seconds_per_step": t, "reps": reps, "warmup": warmup, "dofs": mesh.l_size, "elements": mesh.num_elem}


def run_reference(args, rank):
    """The reference's own CPU implementation of the path (its QFunctions compiled unchanged, driven by the oracle's
    libCEED-semantics operator, OpenMP over element colours on every host thread): W untimed and K timed steps of the
    benchmark workload, each step one IFunction apply + one IJacobian action on the full mesh.  When K + W is large enough
    that full-size steps would take more than a few minutes, each step is a 32^3 sample of the same operator instead
    (stated in `config`)."""
    if rank != 0:
        return
    n_sample = args.size if args.steps + args.warmup <= 40 else min(args.size, 32)
    res = cpu_leg(n_sample, use_ref=True, reps=args.steps, warmup=args.warmup)
    full = n_sample == args.size
    line = {"metric": METRIC, "value": res["value"], "unit": "GDoF/s", "n_gpus": args.gpus, "steps": res["reps"], "warmup": res["warmup"],
            "ms_per_step": res["seconds_per_step"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: background + 8 seeded sinusoidal modes (|k|<=8, 1e-3 relative)", "impl": "reference",
            "config": {"workload": f"{args.size}^3 hex elements, P=4 Q=5, Newtonian IFunction + IJacobian (SUPG, conservative, FP64)"
                                   + ("" if full else f" -- bounded CPU sample of {n_sample}^3 elements per step"),
                       "dofs": res["dofs"], "elements": res["elements"], "parallelism": f"CPU, {res['cores']} OpenMP threads"},
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": res["value"], "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------------------------------------
# GPU arm

def max_over_ranks(ms, world, device):
    """The job's time for one step: the slowest rank's (replicas run the same work; the job ends with the last one)."""
    if world > 1:
        import torch
        t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return t.item()
    return ms


def job_gdofs(world, dofs_per_rank, ms):
    """Whole-job throughput of `world` replicas, each doing dofs_per_rank per step, in GDoF/s."""
    return world * dofs_per_rank / (ms * 1e-3) / 1e9


def run_gpu(args, rank, world):
    import torch
    hb = importlib.import_module("honee-4aiad_b200")
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    ce = importlib.import_module("honee-4aiad_b200.ceed")
    hon = importlib.import_module("honee-4aiad_b200.honee")
    hb.lib()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    prob, mesh, basis, ctx, q, q_dot, dq = workload(args.size)
    P, Q, E = basis.P, basis.Q, mesh.num_elem
    N_L, N_q = mesh.l_size, E * Q ** 3
    cb = prob.context_bytes(ctx)

    op = kern.ElemOp(mesh, basis)
    f64 = dict(dtype=torch.float64, device=dev)
    t_q = torch.from_numpy(q).to(dev)
    t_qd = torch.from_numpy(q_dot).to(dev)
    t_dq = torch.from_numpy(dq).to(dev)
    t_v = torch.empty(N_L, **f64)
    t_jv = torch.empty(N_L, **f64)
    t_x = torch.from_numpy(mesh.x_elem).to(dev)
    t_qdata = torch.empty(E * 10 * Q ** 3, **f64)
    t_jd = torch.empty(E * 14 * Q ** 3, **f64)
    op.setup_qdata(t_x, t_qdata)
    del t_x
    t_jd32 = torch.empty(E * 14 * Q ** 3, dtype=torch.float32, device=dev)
    t_dq32 = t_dq.float()
    t_jv32 = torch.empty(N_L, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def step64():
        op.ifunction(cb, t_q, t_qd, t_qdata, t_v, jac_data=t_jd)
        op.ijacobian(cb, t_qdata, t_jd, t_dq, t_jv)

    def step32():
        op.ifunction(cb, t_q, t_qd, t_qdata, t_v, jac_data_f32=t_jd32)
        op.ijacobian(cb, t_qdata, t_jd32, t_dq32, t_jv32, fp32=True)

    def timed(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(k):
            fn()
        b.record()
        torch.cuda.synchronize()
        return max_over_ranks(a.elapsed_time(b) / k, world, dev)

    if args.profile_apply:  # one apply of every operator kernel after one warm-up apply: the launches ncu captures
        t_diag, t_diag32 = torch.empty(N_L, **f64), torch.empty(N_L, dtype=torch.float32, device=dev)
        for _ in range(2):  # per round: IFunction (FP64 jac_data), IJacobian FP64, IFunction (FP32 jac_data), IJacobian FP32,
            op.ifunction(cb, t_q, t_qd, t_qdata, t_v, jac_data=t_jd)  # diagonal FP64, diagonal FP32: 6 x colours launches
            op.ijacobian(cb, t_qdata, t_jd, t_dq, t_jv)
            op.ifunction(cb, t_q, t_qd, t_qdata, t_v, jac_data_f32=t_jd32)
            op.ijacobian(cb, t_qdata, t_jd32, t_dq32, t_jv32, fp32=True)
            op.diagonal(cb, t_qdata, t_jd, t_diag)
            op.diagonal(cb, t_qdata, t_jd32, t_diag32, fp32=True)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile_apply": args.size, "elements": E, "colours": op.num_colors, "rounds": 2}), flush=True)
        return
    with ClockSampler(dev.index) as clk:
        ms64 = timed(step64, args.steps)
    clocks = clk.summary()
    ms32 = timed(step32, args.steps)
    if args.only_kernels:
        if rank == 0:
            print(json.dumps({"ms_per_step_f64": ms64, "ms_per_step_f32": ms32, "gdofs_f64": N_L / ms64 / 1e6, "clocks": clocks}), flush=True)
        return
    ms_if = timed(lambda: op.ifunction(cb, t_q, t_qd, t_qdata, t_v, jac_data=t_jd), args.steps)
    ms_ij = timed(lambda: op.ijacobian(cb, t_qdata, t_jd, t_dq, t_jv), args.steps)
    ms_if32 = timed(lambda: op.ifunction(cb, t_q, t_qd, t_qdata, t_v, jac_data_f32=t_jd32), args.steps)
    ms_ij32 = timed(lambda: op.ijacobian(cb, t_qdata, t_jd32, t_dq32, t_jv32, fp32=True), args.steps)
    t_diag = torch.empty(N_L, **f64)
    ms_diag = timed(lambda: op.diagonal(cb, t_qdata, t_jd, t_diag), max(1, min(args.steps, 3)))

    # FP32 Jacobian error against the FP64 kernel on the full workload; these outputs are also checked against the oracle
    step64()
    jv64 = t_jv.clone()
    step32()
    torch.cuda.synchronize()
    err32 = (torch.linalg.vector_norm(t_jv32.double() - jv64) / torch.linalg.vector_norm(jv64)).item()
    gpu_out = {"v": t_v.cpu().numpy(), "jac_data": t_jd.cpu().numpy(), "jv": jv64.cpu().numpy(), "jv32": t_jv32.double().cpu().numpy()}
    del jv64, t_jd32, t_dq32, t_jv32

    # e2e through the libCEED API with host (pinned) buffers: H2D of q, q_dot, dq and D2H of both results every step.
    # Two steps in flight: the results of step k are read back (CeedVectorSyncArray) after step k+1 is enqueued, into a
    # second pair of output vectors, so step k's read-back (device->host) shares the bus with step k+1's upload
    # (host->device); the serial variant reads each step back before enqueuing the next.
    ceed = ce.Ceed("/gpu/b200")
    ops = hon.NewtonianOperators(ceed, mesh, basis, ctx)
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    h_q, h_qd, h_dq = pin(q), pin(q_dot), pin(dq)
    h_g, h_j = [pin(np.zeros(N_L)) for _ in range(2)], [pin(np.zeros(N_L)) for _ in range(2)]
    qv, dv = ce.Vector(ceed, N_L), ce.Vector(ceed, N_L)
    gv, jvv = [ce.Vector(ceed, N_L) for _ in range(2)], [ce.Vector(ceed, N_L) for _ in range(2)]

    def e2e_enqueue(s):
        qv.set_array_host(h_q, copy=False)
        ops.q_dot.set_array_host(h_qd, copy=False)
        dv.set_array_host(h_dq, copy=False)
        gv[s].set_array_host(h_g[s], copy=False)
        jvv[s].set_array_host(h_j[s], copy=False)
        ops.op_ifunction.apply(qv, gv[s])
        ops.op_ijacobian.apply(dv, jvv[s])

    def e2e_read(s):
        ce.L().CeedVectorSyncArray(gv[s].ptr, ce.CEED_MEM_HOST)
        ce.L().CeedVectorSyncArray(jvv[s].ptr, ce.CEED_MEM_HOST)

    def e2e_steps(k, in_flight):
        for i in range(k):
            e2e_enqueue(i % 2)
            if in_flight == 1:
                e2e_read(i % 2)
            elif i:
                e2e_read((i - 1) % 2)
        if in_flight == 2:
            e2e_read((k - 1) % 2)

    k_e2e = max(2, min(args.steps, 10))
    ms_e2e_serial = timed(lambda: e2e_steps(1, 1), k_e2e)
    ms_e2e = timed(lambda: e2e_steps(k_e2e, 2), 1) / k_e2e
    err_e2e = max(float(np.linalg.norm(h_j[s] - gpu_out["jv"]) / np.linalg.norm(gpu_out["jv"])) for s in range(2))

    # parity against the CPU oracle: the benchmarked outputs themselves (full size), and a small case of the same operator
    acc, cpu_full = parity_full(prob, mesh, basis, ctx, q, q_dot, dq, gpu_out, args.size) if rank == 0 and not args.no_cpu else ({}, None)
    del gpu_out
    acc["small_case"] = parity_sample(prob, kern, torch, dev)

    pk, pk_kind = peaks()
    b_if, b_ij = algorithmic_bytes(N_L, N_q, E, P)
    _, b_ij32 = algorithmic_bytes(N_L, N_q, E, P, f32=True)
    b_diag = 8 * N_L + 8 * N_q * 24 + 4 * E * P ** 3
    achieved_if = b_if / (ms_if * 1e-3) / 1e9
    fma64, fma32 = kern.fma_peak(True), kern.fma_peak(False)
    sides = two_sided_roofline({"ifunction": ms_if, "ijacobian": ms_ij, "ijacobian_f32": ms_ij32, "diagonal_f64": ms_diag},
                               {"ifunction": b_if, "ijacobian": b_ij, "ijacobian_f32": b_ij32, "diagonal_f64": b_diag}, E, pk, fma64, fma32)
    launches = 2 * op.num_colors * args.steps
    line = {
        "metric": METRIC, "value": job_gdofs(world, N_L, ms64), "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: background + 8 seeded sinusoidal modes (|k|<=8, 1e-3 relative)",
        "config": {"workload": f"{args.size}^3 hex elements, P=4 Q=5, Newtonian IFunction + IJacobian (SUPG, conservative, FP64)",
                   "dofs": N_L, "elements": E, "qpts": N_q, "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (qdata 2.6 GB, jac_data 3.7 GB per GPU); no flush"},
        "fp32_mixed": {"value": job_gdofs(world, N_L, ms32), "unit": "GDoF/s", "ms_per_step": ms32,
                       "jacobian_rel_l2_vs_fp64": err32, "residual": "FP64", "jacobian": "FP32 (FP32 jac_data, FP64 qdata)"},
        "breakdown_ms": {"ifunction": ms_if, "ijacobian": ms_ij, "ifunction_f32_jacdata": ms_if32, "ijacobian_f32": ms_ij32,
                         "diagonal_f64": ms_diag},
        "accuracy": acc,
        "roofline": {"bound": "hbm", "kernel": "k_ifunction (fused IFunction, one launch per colour)", "achieved": achieved_if,
                     "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved_if / pk["hbm_gbs"], "peak_source": pk_kind,
                     "algorithmic_bytes_per_apply": b_if, "algorithmic_bytes_per_launch": b_if / op.num_colors,
                     "traffic": KERNEL_COUNTERS["ifunction"]["dram_per_elem"] * E / op.num_colors,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, mean of the 8 colour launches of one 64^3 apply "
                                       "(--cache-control none, steady state), per launch",
                     "ijacobian": {"achieved": b_ij / (ms_ij * 1e-3) / 1e9, "frac": b_ij / (ms_ij * 1e-3) / 1e9 / pk["hbm_gbs"]},
                     "pipe_peaks": {"fp64_fma_per_s": fma64, "fp32_fma_per_s": fma32, "fp64_tflops": 2 * fma64 / 1e12,
                                    "fp32_tflops": 2 * fma32 / 1e12,
                                    "source": "hb_fma_peak_probe (independent FMA chains, 8 CTAs/SM), best of 5 launches, CUDA events, this run"},
                     "two_sided": sides},
        "e2e": {"value": job_gdofs(world, N_L, ms_e2e), "unit": "GDoF/s", "h2d_bytes_per_step": 3 * 8 * N_L, "d2h_bytes_per_step": 2 * 8 * N_L,
                "api": "CeedVectorSetArray(HOST, USE_POINTER) + CeedOperatorApply x2 + CeedVectorSyncArray(HOST)", "steps_in_flight": 2,
                "steps": k_e2e, "serial_value": job_gdofs(world, N_L, ms_e2e_serial), "jacobian_rel_l2_vs_kernel": err_e2e},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if not args.no_timeloop:
        line["timeloop"] = timeloop_leg(args.timeloop_steps)
    if cpu_full is not None:
        line["cpu_baseline"] = cpu_full
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_gpu_partitioned(args, rank, world):
    """N > 1: the operator partitioned into z-slabs (weak scaling: rank r holds a size^3 slab of a size x size x (N size) box),
    each step one ghost-plane exchange of q and q_dot, the IFunction, the ghost contributions summed into their owners, the
    same for the Jacobian action on dq -- the exchanges of HONEE's DMGlobalToLocal / DMLocalToGlobal around every apply,
    over NCCL point-to-point between neighbouring ranks.  value = DOF of the whole box / the slowest rank's step time."""
    import torch
    import torch.distributed as dist
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    prob = importlib.import_module("honee-4aiad_b200.problem")
    part = importlib.import_module("honee-4aiad_b200.partition")
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    n = args.size
    slab = part.partition_box((n, n, n * world), 4, rank, world)
    mesh, basis = slab.local, prob.tensor_basis(4, 5)
    ctx = prob.newtonian_context(3, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=prob.STAB_SUPG, dt=1e-5, ijacobian_time_shift=1.5e5)
    q = prob.multimode_state(mesh, basis, ctx.gas, seed=0)
    rng = np.random.default_rng(1 + rank)
    q_dot, dq = q * 1e-3 * rng.uniform(-1, 1, q.shape), q * 1e-4 * rng.uniform(-1, 1, q.shape)
    E, Q, NL, no = mesh.num_elem, basis.Q, mesh.l_size, slab.owned_size
    cb = prob.context_bytes(ctx)
    op = kern.ElemOp(mesh, basis)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    t_q, t_qd, t_dq = T(q), T(q_dot), T(dq)
    t_v, t_jv = torch.empty_like(t_q), torch.empty_like(t_q)
    t_qdata = torch.empty(E * 10 * Q ** 3, dtype=torch.float64, device=dev)
    op.setup_qdata(T(mesh.x_elem), t_qdata)
    t_jd = torch.empty(E * 14 * Q ** 3, dtype=torch.float64, device=dev)
    ex = part.HaloExchange(slab, dist)
    own_v, own_jv = torch.empty(no, dtype=torch.float64, device=dev), torch.empty(no, dtype=torch.float64, device=dev)

    def step():
        ex.global_to_local(t_q[:no], t_q)
        ex.global_to_local(t_qd[:no], t_qd)
        op.ifunction(cb, t_q, t_qd, t_qdata, t_v, jac_data=t_jd)
        ex.local_to_global(t_v, own_v)
        ex.global_to_local(t_dq[:no], t_dq)
        op.ijacobian(cb, t_qdata, t_jd, t_dq, t_jv)
        ex.local_to_global(t_jv, own_jv)

    def timed(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(k):
            fn()
        b.record()
        torch.cuda.synchronize()
        return max_over_ranks(a.elapsed_time(b) / k, world, dev)

    with ClockSampler(dev.index) as clk:
        ms = timed(step, args.steps)
    clocks = clk.summary()
    # end to end: this rank's owned state from pinned host memory, the exchanged step, both owned results back to the host
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a[:no])).pin_memory()  # noqa: E731
    h_q, h_qd, h_dq = pin(q), pin(q_dot), pin(dq)
    h_v, h_j = torch.empty(no, dtype=torch.float64).pin_memory(), torch.empty(no, dtype=torch.float64).pin_memory()

    def e2e():
        t_q[:no].copy_(h_q, non_blocking=True)
        t_qd[:no].copy_(h_qd, non_blocking=True)
        t_dq[:no].copy_(h_dq, non_blocking=True)
        step()
        h_v.copy_(own_v, non_blocking=True)
        h_j.copy_(own_jv, non_blocking=True)

    ms_e2e = timed(e2e, max(1, min(args.steps, 5)))
    dofs = torch.tensor([float(no)], dtype=torch.float64, device=dev)
    dist.all_reduce(dofs)
    total = dofs.item()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": total / (ms * 1e-3) / 1e9, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: background + 8 seeded sinusoidal modes (|k|<=8, 1e-3 relative)",
            "config": {"workload": f"{n}x{n}x{n * world} hex box in {world} z-slabs of {n}^3 elements, P=4 Q=5, Newtonian IFunction + IJacobian "
                                   "(SUPG, conservative, FP64) with the ghost-plane exchanges of every apply", "dofs": total,
                       "parallelism": f"z-slab element partition over {world} GPUs (NCCL point-to-point halo planes)",
                       "l2": "inputs larger than L2 per GPU; no flush"},
            "e2e": {"value": total / (ms_e2e * 1e-3) / 1e9, "unit": "GDoF/s", "h2d_bytes_per_step": 3 * 8 * no * world,
                    "d2h_bytes_per_step": 2 * 8 * no * world, "api": "pinned host owned vectors -> exchange + ElemOp applies -> host"},
            "gpu_launches": 2 * op.num_colors * args.steps, "clocks": clocks}), flush=True)


def timeloop_leg(steps):
    """Implicit BDF2 steps of the mixed-precision configuration (Taylor-Green, periodic [0, 2 pi]^3, 32^3 elements, P=5 Q=6,
    10,485,760 DOF, acoustic CFL 1) in FP64 and in mixed precision: time-steps per second after the first (BDF1) step, with
    the Newton/GMRES iteration counts and the largest relative difference of the monitors between the two runs."""
    NS = importlib.import_module("honee-4aiad_b200.navierstokes")
    out = {"workload": "Taylor-Green 32^3 hex, P=5 Q=6, periodic, Re 1600, Ma 0.1, acoustic CFL 1, BDF2 + Newton + GMRES(30) + Jacobi",
           "steps": steps}
    runs = {}
    for tag, mixed in (("fp64", False), ("mixed", True)):
        r = NS.run("taylor_green", faces=32, degree=4, steps=steps, cfl=1.0, mixed=mixed, monitor_every=steps)
        runs[tag] = r
        out[tag] = {"steps_per_s": r.steps_per_second(), "newton_its": [s.newton_its for s in r.stats],
                    "ksp_its": [s.ksp_its for s in r.stats], "final_rel_residual": max(s.res_final / s.res0 for s in r.stats)}
    out["dofs"] = runs["fp64"].dofs
    out["dt"] = runs["fp64"].dt
    out["mixed_speedup"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    out["mixed_vs_fp64_monitor_rel_diff"] = NS.compare(runs["fp64"], runs["mixed"])
    return out


# Per-element counters of the fused kernels at P=4, Q=5 (profiles/roofline_counters_64cube_P4Q5.md has the commands):
#   pipe ops: FP64 (DFMA + DADD + DMUL) or FP32 (FFMA + FADD + FMUL) thread instructions, ncu
#             smsp__sass_thread_inst_executed_op_{d,f}{fma,add,mul}_pred_on.sum over one apply at 32^3 / elements;
#   dram:     dram__bytes_read.sum + dram__bytes_write.sum per element over the 8 colour launches of one apply at 64^3
#             with --cache-control none (steady state: each launch pays for the dirty lines the previous one left).
# The FP32 element-pair kernel's packed f32x2 instructions are not among those metrics: its ops are the single-element
# FP32 kernel's count, the arithmetic both lanes do per element.
KERNEL_COUNTERS = {
    "ifunction": {"pipe": "fp64", "ops_per_elem": 99010, "dram_per_elem": 39257},
    "ijacobian": {"pipe": "fp64", "ops_per_elem": 90250, "dram_per_elem": 35426},
    "ijacobian_f32": {"pipe": "fp32", "ops_per_elem": 88695, "dram_per_elem": 23289},
    "diagonal_f64": {"pipe": "fp64", "ops_per_elem": 204800, "dram_per_elem": 31384},
}


def two_sided_roofline(ms, bytes_alg, E, pk, fma64, fma32):
    """Per kernel: the HBM floor (algorithmic bytes / measured copy bandwidth), the arithmetic-pipe floor (thread
    instructions / measured FMA-pipe rate; DFMA, DADD and DMUL each take one pipe slot), the binding (larger) floor and
    the measured time's fraction of it.  fma64 / fma32: measured pipe rates in thread instructions per second."""
    out = {}
    for name, t_ms in ms.items():
        k = KERNEL_COUNTERS[name]
        t = t_ms * 1e-3
        t_hbm = bytes_alg[name] / (pk["hbm_gbs"] * 1e9)
        rate = fma64 if k["pipe"] == "fp64" else fma32
        t_pipe = k["ops_per_elem"] * E / rate
        out[name] = {"ms": t_ms, "algorithmic_bytes": bytes_alg[name], "hbm_floor_ms": t_hbm * 1e3, "hbm_frac": t_hbm / t,
                     f"{k['pipe']}_pipe_floor_ms": t_pipe * 1e3, "pipe_frac": t_pipe / t, "pipe_ops_per_elem": k["ops_per_elem"],
                     "binding": "hbm" if t_hbm >= t_pipe else f"{k['pipe']} pipe", "binding_floor_ms": max(t_hbm, t_pipe) * 1e3,
                     "frac_of_binding": max(t_hbm, t_pipe) / t, "dram_traffic_per_elem": k["dram_per_elem"],
                     "dram_traffic_over_algorithmic": k["dram_per_elem"] * E / bytes_alg[name]}
    return out


def parity_full(prob, mesh, basis, ctx, q, q_dot, dq, gpu, n):
    """The benchmarked GPU outputs against the CPU oracle on the same full-size inputs: relative L2 of the residual, the
    stored Jacobian data, and the FP64 and FP32 Jacobian actions (the oracle restates the reference QFunctions and is
    pinned to them bit for bit; it computes its own qdata and Jacobian data from the same mesh and state).  The oracle's
    step (IFunction + IJacobian on every host thread) is timed as the CPU baseline."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    m = O.Mesh(mesh.num_elem, basis.P, basis.Q, mesh.offsets, basis.interp1d, basis.grad1d, basis.qweight1d, colors=mesh.colors,
               num_threads=threads)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    jd = np.zeros(mesh.num_elem * 14 * basis.Q ** 3)
    cb = prob.context_bytes(ctx)
    t0 = time.perf_counter()
    v_ref = O.apply_ifunction(m, cb, q, q_dot, qdata, jd)
    j_ref = O.apply_ijacobian(m, cb, dq, qdata, jd)
    t = time.perf_counter() - t0
    r = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    acc = {"case": f"{n}^3 P=4 Q=5: the benchmarked outputs vs the CPU oracle on the same inputs",
           "ifunction_rel_l2": r(gpu["v"], v_ref), "jac_data_rel_l2": r(gpu["jac_data"], jd), "ijacobian_rel_l2": r(gpu["jv"], j_ref),
           "ijacobian_f32_rel_l2": r(gpu["jv32"], j_ref), "bar": "FP64 <= 1e-12; FP32 Jacobian within FP32 rounding (~1e-7)"}
    cpu = {"value": mesh.l_size / t / 1e9, "unit": "GDoF/s", "cores": threads, "kind": "port",
           "sample": f"{n}^3 elements P=4 Q=5 ({mesh.l_size} DOF): one IFunction + IJacobian step of the oracle, the run that checks the "
                     f"benchmarked outputs ({t:.2f} s)"}
    return acc, cpu


def parity_sample(prob, kern, torch, dev):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    mesh = prob.box_mesh((6, 6, 6), 4)
    basis = prob.tensor_basis(4, 5)
    ctx = prob.newtonian_context(3, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=prob.STAB_SUPG, dt=1e-5, ijacobian_time_shift=1.5e5)
    q = prob.multimode_state(mesh, basis, ctx.gas, seed=3)
    qd = q * 1e-3
    dq = q * 1e-4 * np.random.default_rng(2).uniform(-1, 1, q.shape)
    cb = prob.context_bytes(ctx)
    m = O.Mesh(mesh.num_elem, 4, 5, mesh.offsets, basis.interp1d, basis.grad1d, basis.qweight1d, colors=mesh.colors)
    qdata = O.setup_qdata(mesh.num_elem, 5, mesh.x_elem)
    jd = np.zeros(mesh.num_elem * 14 * 125)
    v_ref = O.apply_ifunction(m, cb, q, qd, qdata, jd)
    j_ref = O.apply_ijacobian(m, cb, dq, qdata, jd)
    op = kern.ElemOp(mesh, basis)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    tq, tqd, tdq, tqdata = T(q), T(qd), T(dq), T(qdata)
    tv, tj = torch.empty_like(tq), torch.empty_like(tq)
    tjd = torch.empty(mesh.num_elem * 14 * 125, dtype=torch.float64, device=dev)
    tjd32 = torch.empty(mesh.num_elem * 14 * 125, dtype=torch.float32, device=dev)
    op.ifunction(cb, tq, tqd, tqdata, tv, jac_data=tjd, jac_data_f32=tjd32)
    op.ijacobian(cb, tqdata, tjd, tdq, tj)
    tj32 = torch.empty(mesh.l_size, dtype=torch.float32, device=dev)
    op.ijacobian(cb, tqdata, tjd32, tdq.float(), tj32, fp32=True)
    torch.cuda.synchronize()
    r = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    return {"case": "6^3 P=4 Q=5 same operator", "ifunction_rel_l2": r(tv.cpu().numpy(), v_ref), "ijacobian_rel_l2": r(tj.cpu().numpy(), j_ref),
            "ijacobian_f32_rel_l2": r(tj32.double().cpu().numpy(), j_ref)}


def run_contraction_ab(args):
    """A/B of the basis-contraction mechanism on one GPU (hb_contraction_probe): 32 rounds of the in-plane collocated
    derivatives of five FP64 components at Q = 5 on 65,536 elements (328 MB in, 328 MB out), by shared-memory fibre passes
    (the operator kernels' mechanism) and by warp shuffles, each at its own occupancy limit and at the operator kernels'
    three CTAs per SM; best of 5 CUDA-event-timed launches.  Prints one JSON line; no part of the benchmark step."""
    import torch
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    prob = importlib.import_module("honee-4aiad_b200.problem")
    qx, _ = prob.gauss_legendre(5)
    _, D = prob.lagrange_tabulate(qx, qx)
    D = D / np.abs(D).sum(1).max()
    E, reps = 65536, 32
    u = torch.from_numpy(np.random.default_rng(0).normal(size=(E, 5, 125))).cuda()
    fma64 = kern.fma_peak(True)
    res, outs = {}, {}
    for variant, name in ((0, "shared_fibre_passes"), (1, "warp_shuffles")):
        for ctas in (0, 3):
            ms, fmas, out = kern.contraction_probe(variant, D, u, reps, ctas_per_sm=ctas)
            res[f"{name}_{'max_occupancy' if ctas == 0 else '3_ctas_per_sm'}"] = {
                "ms": ms, "ns_per_element_round": ms * 1e6 / (E * reps), "fp64_pipe_fraction": fmas / (ms * 1e-3) / fma64}
            outs[(variant, ctas)] = out
        del out
    same = all(torch.equal(o, outs[(0, 0)]) for o in outs.values())
    print(json.dumps({"contraction_ab": "in-plane collocated derivatives, 5 FP64 components, Q=5", "elements": E, "rounds": reps,
                      "fma_per_element_round": 6250, "fp64_fma_peak_per_s": fma64, "bit_identical": same, "variants": res}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--only-kernels", action="store_true", help="time the fused kernels only (profiling runs)")
    ap.add_argument("--profile-apply", action="store_true",
                    help="run two applies of every operator kernel (IFunction, IJacobian FP64/FP32, diagonal FP64/FP32) and exit: "
                         "the launches an ncu capture selects with -k/-s/-c")
    ap.add_argument("--contraction-ab", action="store_true",
                    help="time the basis-contraction A/B probe (shared-memory fibre passes against warp shuffles) and exit")
    ap.add_argument("--no-timeloop", action="store_true", help="skip the implicit time-loop leg")
    ap.add_argument("--timeloop-steps", type=int, default=5)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        # the reference arm is CPU work on rank 0 alone (minutes at full size) while the other ranks wait at the final
        # barrier: a CPU process group with a long timeout; the GPU arm's ranks exchange over NCCL with a short one
        if args.impl == "reference":
            torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=3600))
        else:
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank)
        elif args.contraction_ab:
            run_contraction_ab(args)
        elif world > 1:
            run_gpu_partitioned(args, rank, world)
        else:
            run_gpu(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
