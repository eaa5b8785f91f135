"""The z-slab element partition (honee-4aiad_b200/partition.py) on CPU ranks: two gloo processes each apply the operator
to their slab (the CPU oracle stands in for the device kernels), exchange one node plane per apply (global-to-local
before, local-to-global with ADD after) and reduce their Krylov inner products.  The two-rank IFunction, IJacobian,
Jacobi diagonal and one Jacobi-preconditioned GMRES solve must equal the single-rank results on the whole box: the
operator outputs to 1e-13 relative L2 (only the summation order at the slab boundary differs), the GMRES solution to
1e-8 (both solves stop at relative residual 1e-10).  Also checked: one rank with z periodic, whose ghost plane is its
own first plane."""
import importlib
import multiprocessing as mp
import os
import socket
import sys
import traceback

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem(n, P, Q, periodic):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    prob = importlib.import_module("honee-4aiad_b200.problem")
    mesh = prob.box_mesh(n, P, periodic=periodic)
    basis = prob.tensor_basis(P, Q)
    ctx = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=prob.STAB_SUPG, dt=1e-5, ijacobian_time_shift=1.5e5)
    q = prob.multimode_state(mesh, basis, ctx.gas, seed=11)
    rng = np.random.default_rng(12)
    q_dot = q * 1e-3 * rng.uniform(-1, 1, q.shape)
    dq = q * 1e-4 * rng.normal(size=q.shape)
    return prob, mesh, basis, ctx, q, q_dot, dq


class _Ops:
    """IFunction / IJacobian / diagonal of one mesh through the oracle."""

    def __init__(self, O, prob, mesh, basis, ctx):
        self.O, self.mesh = O, mesh
        self.m = O.Mesh(mesh.num_elem, basis.P, basis.Q, mesh.offsets, basis.interp1d, basis.grad1d, basis.qweight1d, colors=mesh.colors)
        self.qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
        self.jd = np.zeros(mesh.num_elem * 14 * basis.Q ** 3)
        self.cb = prob.context_bytes(ctx)

    def ifunction(self, q, q_dot):
        return self.O.apply_ifunction(self.m, self.cb, q, q_dot, self.qdata, self.jd)

    def ijacobian(self, dq):
        return self.O.apply_ijacobian(self.m, self.cb, dq, self.qdata, self.jd)

    def diagonal(self):
        return self.O.assemble_diagonal(self.m, self.cb, self.qdata, self.jd, self.mesh.l_size)


def _rank_main(rank, world, port, n, P, Q, periodic, out):
    try:
        import torch
        import torch.distributed as dist
        os.environ.setdefault("OMP_NUM_THREADS", "1")
        if world > 1:
            import datetime
            dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                    timeout=datetime.timedelta(seconds=60))
        import oracle as O
        part = importlib.import_module("honee-4aiad_b200.partition")
        prob, mesh, basis, ctx, q, q_dot, dq = _problem(n, P, Q, periodic)
        s = part.partition_box(n, P, rank, world, periodic=periodic)
        ex = part.HaloExchange(s, dist if world > 1 else None)
        g0, no = s.global_node0 * 5, s.owned_size
        own = lambda v: np.ascontiguousarray(v[g0:g0 + no])  # noqa: E731
        loc = _Ops(O, prob, s.local, basis, ctx)
        ql = ex.global_to_local(own(q), np.zeros(s.local_size))
        qdl = ex.global_to_local(own(q_dot), np.zeros(s.local_size))
        v = ex.local_to_global(loc.ifunction(ql, qdl), np.zeros(no))
        dql = ex.global_to_local(own(dq), np.zeros(s.local_size))
        jv = ex.local_to_global(loc.ijacobian(dql), np.zeros(no))
        diag = ex.local_to_global(loc.diagonal(), np.zeros(no))

        def apply(x):
            return ex.local_to_global(loc.ijacobian(ex.global_to_local(x, np.zeros(s.local_size))), np.zeros(no))

        b = own(q) * 1e-3
        x, its, res = part.gmres(apply, b, ex, precond=lambda r: r / diag, rtol=1e-10)
        # the single-rank reference on the whole box
        ref = _Ops(O, prob, mesh, basis, ctx)
        v_ref = ref.ifunction(q, q_dot)
        jv_ref = ref.ijacobian(dq)
        d_ref = ref.diagonal()
        ex1 = part.HaloExchange(part.partition_box(n, P, 0, 1, periodic=periodic))
        x_ref, its_ref, _ = part.gmres(ref.ijacobian, q * 1e-3, _Whole(ex1), precond=lambda r: r / d_ref, rtol=1e-10)
        r = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
        out.put((rank, {"v": r(v, own(v_ref)), "jv": r(jv, own(jv_ref)), "diag": r(diag, own(d_ref)), "x": r(x, own(x_ref)), "its": its, "its_ref": its_ref,
                        "res": res}))
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
    except Exception:
        out.put((rank, traceback.format_exc()))


class _Whole:
    """Inner products of whole vectors on one process (the single-rank reference solve)."""

    def __init__(self, ex):
        self.s = ex.s

    def dot(self, a, b):
        return float((a * b).sum())


def _run(world, n, P, Q, periodic):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n, P, Q, periodic, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, val = out.get(timeout=240)
        res[rank] = val
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0, f"rank process exited with {p.exitcode}"
    for rank, val in res.items():
        assert not isinstance(val, str), f"rank {rank} failed:\n{val}"
    return res


@pytest.mark.parametrize("periodic", [(False, False, False), (True, True, True)])
def test_two_rank_slabs_equal_the_single_rank_operator_and_solve(periodic):
    res = _run(2, (3, 2, 4), 3, 3, periodic)
    for rank, d in res.items():
        assert d["v"] < 1e-13 and d["jv"] < 1e-13 and d["diag"] < 1e-13, (rank, d)
        assert d["res"] <= 1e-10 and d["x"] < 1e-8, (rank, d)
    assert res[0]["its"] == res[1]["its"]


def test_one_rank_periodic_ghost_is_its_own_first_plane():
    res = _run(1, (2, 2, 3), 3, 3, (False, False, True))
    d = res[0]
    assert d["v"] < 1e-13 and d["jv"] < 1e-13 and d["diag"] < 1e-13 and d["x"] < 1e-8, d


def test_slab_bounds_and_ownership():
    part = importlib.import_module("honee-4aiad_b200.partition")
    assert part.slab_bounds(10, 3) == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError):
        part.slab_bounds(2, 3)
    P, n = 4, (2, 3, 5)
    sizes = []
    for periodic in (False, True):
        owned = [part.partition_box(n, P, r, 2, periodic=(False, False, periodic)) for r in range(2)]
        total_planes = n[2] * (P - 1) + (0 if periodic else 1)
        assert sum(s.owned_planes for s in owned) == total_planes
        assert owned[0].global_node0 == 0 and owned[1].global_node0 == owned[0].owned_planes * owned[0].plane_nodes
        assert owned[0].has_ghost and owned[1].has_ghost == periodic
        sizes.append(owned[0].local_size)
    assert sizes[0] == sizes[1]
