"""GPU parity: the fused sm_100a operators, reached through the libCEED C API, against the CPU oracle.

Tolerances: restriction maps bit-exact; FP64 residual, Jacobian action and diagonal within
1e-12 relative L2 of the oracle; geometric factors within 1e-14; the FP32 (mixed-precision) Jacobian action and
diagonal within 2e-6 relative L2 (single-precision arithmetic on FP64 geometry).
"""
import importlib

import numpy as np
import pytest

from helpers import O, case, oracle_ifunction, oracle_mesh, prob, rel_l2

pytestmark = pytest.mark.gpu

ce = importlib.import_module("honee-4aiad_b200.ceed")
hon = importlib.import_module("honee-4aiad_b200.honee")

TOL64 = 1e-12
TOL32 = 2e-6

CASES = {
    # config-1 shape: 3D Gaussian pulse, degree 2 (P=3, Q=3), SUPG
    "cfg1_P3Q3": dict(n=(8, 8, 8), P=3, Q=3),
    # config-2 shape at reduced size: degree 3 with q_extra 1 (P=4, Q=5), multi-mode state
    "cfg2_P4Q5": dict(n=(6, 5, 4), P=4, Q=5, state="modes"),
    # config-3 shape: periodic, degree 4 with q_extra 1 (P=5, Q=6)
    "cfg3_P5Q6_periodic": dict(n=(4, 4, 4), P=5, Q=6, periodic=(1, 1, 1), state="modes"),
    "su_gravity_P4Q4": dict(n=(3, 3, 3), P=4, Q=4, stab=prob.STAB_SU, g=(0.5, -9.81, 0.2)),
    "nostab_P3Q4": dict(n=(3, 4, 2), P=3, Q=4, stab=prob.STAB_NONE),
    "idl_P3Q3": dict(n=(6, 3, 3), P=3, Q=3, idl=(2e-3, 0.2, 0.5, 101000.0)),
    # edge sizes: one element (one colour, the other launches empty), the smallest and the largest compiled bases
    "single_elem_P4Q5": dict(n=(1, 1, 1), P=4, Q=5, state="modes"),
    "min_basis_P2Q2": dict(n=(5, 3, 4), P=2, Q=2),
    "max_basis_P6Q7": dict(n=(2, 2, 1), P=6, Q=7, state="modes"),
}


def _setup(name, resource="/gpu/b200"):
    kw = dict(CASES[name])
    mesh, basis, ctx, q, qd = case(**kw)
    ceed = ce.Ceed(resource)
    ops = hon.NewtonianOperators(ceed, mesh, basis, ctx)
    qv = ce.Vector(ceed, mesh.l_size)
    qv.set_array_host(q)
    ops.q_dot.set_array_host(qd)
    g = ce.Vector(ceed, mesh.l_size)
    return mesh, basis, ctx, q, qd, ceed, ops, qv, g


@pytest.mark.parametrize("name", list(CASES))
def test_ifunction_ijacobian_diagonal_fp64(name):
    mesh, basis, ctx, q, qd, ceed, ops, qv, g = _setup(name)
    v_ref, jd_ref, qdata_ref, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    # geometric factors (Setup QFunction)
    assert rel_l2(ops.q_data.to_numpy(), qdata_ref) < 1e-14
    # residual
    ops.ifunction(qv, ops.q_dot, g)
    v = g.to_numpy()
    assert rel_l2(v, v_ref) < TOL64, rel_l2(v, v_ref)
    assert rel_l2(ops.jac_data.to_numpy(), jd_ref) < TOL64
    # Jacobian action
    cb = prob.context_bytes(ctx)
    dq = np.random.default_rng(3).normal(size=q.shape) * np.abs(q) * 1e-4
    dv = ce.Vector(ceed, mesh.l_size)
    dv.set_array_host(dq)
    jv = ce.Vector(ceed, mesh.l_size)
    ops.ijacobian(dv, jv)
    j_ref = O.apply_ijacobian(m, cb, dq, qdata_ref, jd_ref, num_jd=ops.num_jd)
    assert rel_l2(jv.to_numpy(), j_ref) < TOL64, rel_l2(jv.to_numpy(), j_ref)
    # ApplyAdd accumulates
    ops.ijacobian(dv, jv, add=True)
    assert rel_l2(jv.to_numpy(), 2 * j_ref) < TOL64
    # diagonal
    if mesh.num_elem <= 216:
        d = ce.Vector(ceed, mesh.l_size)
        ops.diagonal(d)
        d_ref = O.assemble_diagonal(m, cb, qdata_ref, jd_ref, mesh.l_size, num_jd=ops.num_jd)
        assert rel_l2(d.to_numpy(), d_ref) < TOL64, rel_l2(d.to_numpy(), d_ref)


@pytest.mark.parametrize("name", ["cfg1_P3Q3", "cfg2_P4Q5", "cfg3_P5Q6_periodic", "single_elem_P4Q5", "max_basis_P6Q7"])
def test_mixed_precision_jacobian(name):
    mesh, basis, ctx, q, qd, ceed, ops, qv, g = _setup(name, "/gpu/b200/mixed")
    v_ref, jd_ref, qdata_ref, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    ops.ifunction(qv, ops.q_dot, g)
    assert rel_l2(g.to_numpy(), v_ref) < TOL64  # the residual stays FP64
    # the stored Jacobian data is written in FP32 only; reading it on the host widens it on the compute stream first, and
    # the read-back must wait for that conversion, not only for the operator that wrote the FP32 copy
    assert rel_l2(ops.jac_data.to_numpy(), jd_ref) < 1e-7
    cb = prob.context_bytes(ctx)
    dq = np.random.default_rng(4).normal(size=q.shape) * np.abs(q) * 1e-4
    dv = ce.Vector(ceed, mesh.l_size)
    dv.set_array_host(dq)
    jv = ce.Vector(ceed, mesh.l_size)
    ops.ijacobian(dv, jv)
    j_ref = O.apply_ijacobian(m, cb, dq, qdata_ref, jd_ref)
    err = rel_l2(jv.to_numpy(), j_ref)
    assert err < TOL32, err
    d = ce.Vector(ceed, mesh.l_size)
    ops.diagonal(d)
    d_ref = O.assemble_diagonal(m, cb, qdata_ref, jd_ref, mesh.l_size)
    assert rel_l2(d.to_numpy(), d_ref) < TOL32


def test_context_labels_update_the_kernels():
    """FormIJacobian_NS sets "ijacobian time shift" by label before the Krylov solve (src/setupts.c:141)."""
    mesh, basis, ctx, q, qd, ceed, ops, qv, g = _setup("cfg1_P3Q3")
    ops.ifunction(qv, ops.q_dot, g)
    dq = np.random.default_rng(5).normal(size=q.shape) * np.abs(q) * 1e-4
    dv = ce.Vector(ceed, mesh.l_size)
    dv.set_array_host(dq)
    jv = ce.Vector(ceed, mesh.l_size)
    ops.set_ijacobian_shift(12345.0)
    assert ops.op_ijacobian.get_context_double("ijacobian time shift") == [12345.0]
    ops.ijacobian(dv, jv)
    ctx2 = prob.newtonian_context(2)
    import ctypes as C
    C.memmove(C.addressof(ctx2), C.addressof(ctx), C.sizeof(ctx))
    _, jd_ref, qdata_ref, m = oracle_ifunction(mesh, basis, ctx2, q, qd)
    ctx2.ijacobian_time_shift = 12345.0
    j_ref = O.apply_ijacobian(m, prob.context_bytes(ctx2), dq, qdata_ref, jd_ref)
    assert rel_l2(jv.to_numpy(), j_ref) < TOL64


def test_restriction_maps_bit_exact():
    mesh = prob.box_mesh((3, 2, 2), 4, periodic=(1, 0, 1))
    ceed = ce.Ceed("/gpu/b200")
    r = ce.ElemRestriction(ceed, mesh.num_elem, 64, 5, 1, mesh.l_size, offsets=mesh.offsets)
    lv, ev = r.create_vectors()
    rng = np.random.default_rng(8)
    l = rng.normal(size=mesh.l_size)
    lv.set_array_host(l)
    r.apply(False, lv, ev)
    e = ev.to_numpy()
    e_ref = np.zeros_like(e)
    O.lib().oracle_restrict(mesh.num_elem, 64, 5, 1, O.ptr(mesh.offsets), O.ptr(l), O.ptr(e_ref))
    np.testing.assert_array_equal(e, e_ref)
    lv.set_value(0.0)
    r.apply(True, ev, lv)
    lt_ref = np.zeros(mesh.l_size)
    O.lib().oracle_restrict_t(mesh.num_elem, 64, 5, 1, O.ptr(mesh.offsets), O.ptr(e_ref), O.ptr(lt_ref))
    np.testing.assert_array_equal(lv.to_numpy(), lt_ref)


def test_colouring_is_conflict_free():
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    mesh = prob.box_mesh((6, 4, 4), 4, periodic=(1, 0, 1))
    basis = prob.tensor_basis(4, 5)
    op = kern.ElemOp(mesh, basis)
    assert op.num_colors == 8 and sum(op.color_sizes()) == mesh.num_elem


def test_unsupported_qfunction_fails_loudly():
    ceed = ce.Ceed("/gpu/b200")
    mesh = prob.box_mesh((1, 1, 1), 3)
    basis = prob.tensor_basis(3, 3)
    b = ce.Basis(ceed, 3, 5, 3, 3, basis.interp1d, basis.grad1d, basis.qref1d, basis.qweight1d)
    r = ce.ElemRestriction(ceed, 1, 27, 5, 1, mesh.l_size, offsets=mesh.offsets)
    qf = ce.QFunction(ceed, "advection.h:RHSFunction_Advection")
    qf.add_input("q", 5, ce.CEED_EVAL_INTERP)
    qf.add_output("v", 5, ce.CEED_EVAL_INTERP)
    op = ce.Operator(ceed, qf)
    op.set_field("q", r, b, ceed.active)
    op.set_field("v", r, b, ceed.active)
    x = ce.Vector(ceed, mesh.l_size)
    x.set_value(1.0)
    y = ce.Vector(ceed, mesh.l_size)
    with pytest.raises(ce.CeedError) as ei:
        op.apply(x, y)
    assert ei.value.code == ce.CEED_ERROR_UNSUPPORTED and "no CPU fallback" in str(ei.value)


def test_direct_kernel_abi_matches_ceed_path():
    """The kernel ABI on caller-managed device buffers (torch tensors) equals the libCEED path."""
    import torch
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    mesh, basis, ctx, q, qd, ceed, ops, qv, g = _setup("cfg2_P4Q5")
    ops.ifunction(qv, ops.q_dot, g)
    v_ceed = g.to_numpy()
    op = kern.ElemOp(mesh, basis)
    dev = torch.device("cuda:0")
    tq = torch.from_numpy(q).to(dev)
    tqd = torch.from_numpy(qd).to(dev)
    tqdata = torch.from_numpy(ops.q_data.to_numpy()).to(dev)
    tv = torch.zeros_like(tq)
    tjd = torch.zeros(mesh.num_elem * 14 * basis.Q ** 3, dtype=torch.float64, device=dev)
    op.ifunction(prob.context_bytes(ctx), tq, tqd, tqdata, tv, jac_data=tjd)
    torch.cuda.synchronize()
    assert rel_l2(tv.cpu().numpy(), v_ceed) < 1e-15


def test_host_backed_vectors_across_steps_match_the_device_path():
    """Inputs handed over as host arrays (CEED_USE_POINTER, pinned), rewritten between steps, and outputs read back: the
    copies run on their own streams ordered by events (an input copy overlaps the kernels enqueued before it, an output
    read-back the kernels enqueued after its producer).  Every step must equal the kernel ABI on device buffers, bit for
    bit, with the host arrays reused as a time loop reuses them."""
    import torch
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    mesh, basis, ctx, q, qd, ceed, ops, qv, g = _setup("cfg2_P4Q5")
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_q, h_qd, h_dq, h_g, h_j = pin(q), pin(qd), pin(q * 0), pin(q * 0), pin(q * 0)
    dv, jv = ce.Vector(ceed, mesh.l_size), ce.Vector(ceed, mesh.l_size)
    op = kern.ElemOp(mesh, basis)
    dev = torch.device("cuda:0")
    tqdata = torch.from_numpy(ops.q_data.to_numpy()).to(dev)
    cb = prob.context_bytes(ctx)
    rng = np.random.default_rng(4)
    for step in range(3):
        h_q[:] = q * (1 + 1e-3 * rng.uniform(-1, 1, q.shape))
        h_qd[:] = qd * (1 + 0.1 * rng.uniform(-1, 1, q.shape))
        h_dq[:] = q * 1e-4 * rng.normal(size=q.shape)
        qv.set_array_host(h_q, copy=False)
        ops.q_dot.set_array_host(h_qd, copy=False)
        dv.set_array_host(h_dq, copy=False)
        g.set_array_host(h_g, copy=False)
        jv.set_array_host(h_j, copy=False)
        ops.op_ifunction.apply(qv, g)
        ops.op_ijacobian.apply(dv, jv)
        ce.L().CeedVectorSyncArray(g.ptr, ce.CEED_MEM_HOST)
        ce.L().CeedVectorSyncArray(jv.ptr, ce.CEED_MEM_HOST)
        tq, tqd, tdq = (torch.from_numpy(a.copy()).to(dev) for a in (h_q, h_qd, h_dq))
        tv, tj = torch.zeros_like(tq), torch.zeros_like(tq)
        tjd = torch.zeros(mesh.num_elem * 14 * basis.Q ** 3, dtype=torch.float64, device=dev)
        op.ifunction(cb, tq, tqd, tqdata, tv, jac_data=tjd)
        op.ijacobian(cb, tqdata, tjd, tdq, tj)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(h_g, tv.cpu().numpy(), err_msg=f"step {step}")
        np.testing.assert_array_equal(h_j, tj.cpu().numpy(), err_msg=f"step {step}")
    # An operator marks g's device array used; a device-to-device copy into it (SetArray DEVICE, COPY_VALUES) is enqueued
    # on the compute stream after that.  The read-back must wait for the copy, not only for the operator's event.
    ops.op_ifunction.apply(qv, g)
    src = torch.from_numpy(q * 3.0 + 1.0).to(dev)
    torch.cuda.synchronize()
    g.set_array_device(src.data_ptr(), copy=True)
    ce.L().CeedVectorSyncArray(g.ptr, ce.CEED_MEM_HOST)
    np.testing.assert_array_equal(h_g, src.cpu().numpy())


def test_host_backed_vectors_with_two_steps_in_flight():
    """Two steps in flight through the libCEED API, as a pipelined host loop runs them: step k+1's host inputs are handed
    over (CEED_USE_POINTER) and its operators enqueued before step k's outputs are read back, into a second pair of output
    vectors.  The input vectors are shared by both steps, so step k+1's upload may start only after step k's operator has
    read the device array (its last-use event), and each step's inputs differ: any overlap of the two would change step k's
    results.  Every step equals the kernel ABI on device buffers, bit for bit."""
    import torch
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    mesh, basis, ctx, q, qd, ceed, ops, qv, _ = _setup("cfg2_P4Q5")
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    rng = np.random.default_rng(6)
    K = 5
    h_q = [pin(q * (1 + 1e-3 * rng.uniform(-1, 1, q.shape))) for _ in range(K)]
    h_qd = [pin(qd * (1 + 0.1 * rng.uniform(-1, 1, q.shape))) for _ in range(K)]
    h_dq = [pin(q * 1e-4 * rng.normal(size=q.shape)) for _ in range(K)]
    h_g, h_j = [pin(q * 0) for _ in range(2)], [pin(q * 0) for _ in range(2)]
    dv = ce.Vector(ceed, mesh.l_size)
    gv, jv = [ce.Vector(ceed, mesh.l_size) for _ in range(2)], [ce.Vector(ceed, mesh.l_size) for _ in range(2)]
    op = kern.ElemOp(mesh, basis)
    dev = torch.device("cuda:0")
    tqdata = torch.from_numpy(ops.q_data.to_numpy()).to(dev)
    cb = prob.context_bytes(ctx)

    def expected(k):
        tq, tqd, tdq = (torch.from_numpy(a[k].copy()).to(dev) for a in (h_q, h_qd, h_dq))
        tv, tj = torch.zeros_like(tq), torch.zeros_like(tq)
        tjd = torch.zeros(mesh.num_elem * 14 * basis.Q ** 3, dtype=torch.float64, device=dev)
        op.ifunction(cb, tq, tqd, tqdata, tv, jac_data=tjd)
        op.ijacobian(cb, tqdata, tjd, tdq, tj)
        torch.cuda.synchronize()
        return tv.cpu().numpy(), tj.cpu().numpy()

    def read_and_check(k):
        s = k % 2
        ce.L().CeedVectorSyncArray(gv[s].ptr, ce.CEED_MEM_HOST)
        ce.L().CeedVectorSyncArray(jv[s].ptr, ce.CEED_MEM_HOST)
        v_exp, j_exp = expected(k)
        np.testing.assert_array_equal(h_g[s], v_exp, err_msg=f"residual of step {k}")
        np.testing.assert_array_equal(h_j[s], j_exp, err_msg=f"Jacobian action of step {k}")

    for k in range(K):
        s = k % 2
        qv.set_array_host(h_q[k], copy=False)
        ops.q_dot.set_array_host(h_qd[k], copy=False)
        dv.set_array_host(h_dq[k], copy=False)
        gv[s].set_array_host(h_g[s], copy=False)
        jv[s].set_array_host(h_j[s], copy=False)
        ops.op_ifunction.apply(qv, gv[s])
        ops.op_ijacobian.apply(dv, jv[s])
        if k:
            read_and_check(k - 1)
    read_and_check(K - 1)


def test_operator_over_zero_elements_contributes_nothing():
    """A partition may own no elements: libCEED accepts restrictions with num_elem 0 and an operator over them adds zero.
    HONEE's operators built over zero elements (same L-vector) give a zero residual with Apply, leave the output of
    ApplyAdd unchanged, assemble zero (point-block) diagonals, and change nothing, bit for bit, as sub-operators of the
    real composites."""
    from types import SimpleNamespace
    mesh, basis, ctx, q, qd, ceed, ops, qv, g = _setup("cfg2_P4Q5")
    empty = SimpleNamespace(num_elem=0, l_size=mesh.l_size, offsets=np.zeros(0, np.int32), x_elem=np.zeros((0, 3, 8)))
    eops = hon.NewtonianOperators(ceed, empty, basis, ctx)
    assert eops.q_data.to_numpy().size == 0
    rng = np.random.default_rng(5)
    dq = q * 1e-4 * rng.normal(size=q.shape)
    dv = ce.Vector(ceed, mesh.l_size)
    dv.set_array_host(dq)
    out = ce.Vector(ceed, mesh.l_size)
    out.set_array_host(np.full(mesh.l_size, 7.0))
    eops.op_ifunction.apply(qv, out)
    np.testing.assert_array_equal(out.to_numpy(), 0.0)
    out.set_array_host(np.full(mesh.l_size, 7.0))
    eops.op_ijacobian.apply(dv, out, add=True)
    np.testing.assert_array_equal(out.to_numpy(), 7.0)
    eops.op_ijacobian.assemble_diagonal(out)
    np.testing.assert_array_equal(out.to_numpy(), 0.0)
    pb = ce.Vector(ceed, 5 * mesh.l_size)
    eops.op_ijacobian.assemble_point_block_diagonal(pb)
    np.testing.assert_array_equal(pb.to_numpy(), 0.0)
    # reference results of the real composites, then the same composites with an empty sub-operator joined
    ops.ifunction(qv, ops.q_dot, g)
    v_ref = g.to_numpy()
    jv = ce.Vector(ceed, mesh.l_size)
    ops.ijacobian(dv, jv)
    j_ref = jv.to_numpy()
    d = ce.Vector(ceed, mesh.l_size)
    ops.diagonal(d)
    d_ref = d.to_numpy()
    ops.op_ifunction.add_sub(eops.op_ifunction_volume)
    ops.op_ijacobian.add_sub(eops.op_ijacobian_volume)
    ops.ifunction(qv, ops.q_dot, g)
    ops.ijacobian(dv, jv)
    ops.diagonal(d)
    np.testing.assert_array_equal(g.to_numpy(), v_ref)
    np.testing.assert_array_equal(jv.to_numpy(), j_ref)
    np.testing.assert_array_equal(d.to_numpy(), d_ref)

