"""The z-slab partition of `bench.py --gpus N` on one GPU: the operator applied slab by slab with the device kernels, the
ghost planes moved by device copies in one process (the NCCL point-to-point exchange of a multi-GPU run carries the same
planes), equals the whole-box operator: IFunction and IJacobian within 1e-13 relative L2 (only the summation order at the
slab boundaries differs).  Nothing waits on another slab, so the slabs run one after another on one GPU."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

prob = importlib.import_module("honee-4aiad_b200.problem")
part = importlib.import_module("honee-4aiad_b200.partition")
kern = importlib.import_module("honee-4aiad_b200.kernels")


def _apply(mesh, basis, ctx, q, q_dot, dq, dev):
    import torch
    op = kern.ElemOp(mesh, basis)
    T = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev).contiguous()  # noqa: E731
    E, Q = mesh.num_elem, basis.Q
    qdata = torch.empty(E * 10 * Q ** 3, dtype=torch.float64, device=dev)
    op.setup_qdata(T(mesh.x_elem), qdata)
    jd = torch.empty(E * 14 * Q ** 3, dtype=torch.float64, device=dev)
    v, jv = torch.zeros_like(T(q)), torch.zeros_like(T(q))
    cb = prob.context_bytes(ctx)
    op.ifunction(cb, T(q), T(q_dot), qdata, v, jac_data=jd)
    op.ijacobian(cb, qdata, jd, T(dq), jv)
    torch.cuda.synchronize()
    return v, jv


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("periodic", [(False, False, False), (True, True, True)])
def test_slab_by_slab_operator_equals_the_whole_box(world, periodic):
    import torch
    dev = torch.device("cuda:0")
    n, P, Q = (3, 3, 6), 4, 5
    mesh, basis = prob.box_mesh(n, P, periodic=periodic), prob.tensor_basis(P, Q)
    ctx = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, stab=prob.STAB_SUPG, dt=1e-5, ijacobian_time_shift=1.5e5)
    q = prob.multimode_state(mesh, basis, ctx.gas, seed=3)
    rng = np.random.default_rng(4)
    q_dot, dq = q * 1e-3 * rng.uniform(-1, 1, q.shape), q * 1e-4 * rng.normal(size=q.shape)
    v_ref, jv_ref = _apply(mesh, basis, ctx, q, q_dot, dq, dev)
    slabs = [part.partition_box(n, P, r, world, periodic=periodic) for r in range(world)]
    g = [torch.as_tensor(a, device=dev) for a in (q, q_dot, dq)]
    v, jv = torch.zeros_like(v_ref), torch.zeros_like(jv_ref)
    for s in slabs:
        g0, no, ps = s.global_node0 * 5, s.owned_size, s.plane_size
        gn = slabs[s.next_rank].global_node0 * 5
        # global-to-local: the owned planes, then the owner's first plane as the ghost
        loc = [torch.cat([a[g0:g0 + no], a[gn:gn + ps]]) if s.has_ghost else a[g0:g0 + no].clone() for a in g]
        assert loc[0].numel() == s.local_size
        lv, ljv = _apply(s.local, basis, ctx, *(x.cpu().numpy() for x in loc), dev)
        # local-to-global (ADD): owned entries, and the ghost contributions into the owner's first plane
        for out, lo in ((v, lv), (jv, ljv)):
            out[g0:g0 + no] += lo[:no]
            if s.has_ghost:
                out[gn:gn + ps] += lo[no:no + ps]
    r = lambda a, b: float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))  # noqa: E731
    assert r(v, v_ref) < 1e-13, r(v, v_ref)
    assert r(jv, jv_ref) < 1e-13, r(jv, jv_ref)
