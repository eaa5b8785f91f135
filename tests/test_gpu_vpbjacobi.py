"""GPU tests of point-block Jacobi (HONEE's -pc_type vpbjacobi) in the implicit time loop: the 5 x 5 block inversion and
application kernels against numpy, a singular block reported instead of used, and BDF steps preconditioned by the point
blocks that solve the same equations as the Jacobi-preconditioned ones (the oracle evaluates the BDF1 residual), in FP64
and mixed precision, with free-stream faces included."""
import ctypes as C
import importlib

import numpy as np
import pytest

from helpers import O, case, prob, rel_l2
from test_gpu_solver import _oracle_bdf1_residual, _problem, _run

pytestmark = pytest.mark.gpu

K = importlib.import_module("honee-4aiad_b200.kernels")
S = importlib.import_module("honee-4aiad_b200.solver")
hb = importlib.import_module("honee-4aiad_b200")


def _dev():
    import torch
    return torch.device("cuda:0")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_block_inversion_and_apply_match_numpy():
    import torch
    L = hb.lib()
    rng = np.random.default_rng(0)
    nodes = 1000
    B = rng.normal(size=(nodes, 5, 5)) + 6 * np.eye(5)[None] * rng.uniform(0.5, 2, (nodes, 1, 1))
    B[7] = 0.0                      # no pivot at all
    B[11, :, 2] = 0.0               # a zero column
    tb = torch.from_numpy(B.reshape(-1).copy()).to(_dev())
    inv = torch.empty_like(tb)
    d_sing = torch.zeros(1, dtype=torch.int32, device=_dev())
    h_sing = C.c_int(-1)
    assert L.hb_pb_invert_f64(_ptr(tb), _ptr(inv), C.c_int64(nodes), _ptr(d_sing), C.byref(h_sing), None) == 0
    assert h_sing.value == 2
    got = inv.cpu().numpy().reshape(nodes, 5, 5)
    ok = np.ones(nodes, dtype=bool)
    ok[[7, 11]] = False
    np.testing.assert_allclose(got[ok], np.linalg.inv(B[ok]), rtol=1e-12, atol=1e-14)
    np.testing.assert_array_equal(got[7], np.eye(5))
    # in place, and the FP32 form
    assert L.hb_pb_invert_f64(_ptr(tb), _ptr(tb), C.c_int64(nodes), _ptr(d_sing), None, None) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(tb.cpu().numpy(), inv.cpu().numpy())
    tb = torch.from_numpy(B.reshape(-1).copy()).to(_dev())
    inv32 = torch.empty(25 * nodes, dtype=torch.float32, device=_dev())
    assert L.hb_pb_invert_f64_to_f32(_ptr(tb), _ptr(inv32), C.c_int64(nodes), _ptr(d_sing), C.byref(h_sing), None) == 0
    assert h_sing.value == 2
    np.testing.assert_allclose(inv32.cpu().numpy().reshape(nodes, 5, 5)[ok], np.linalg.inv(B[ok]), rtol=1e-6, atol=1e-7)
    x = rng.normal(size=5 * nodes)
    tx = torch.from_numpy(x).to(_dev())
    y = torch.empty_like(tx)
    assert L.hb_pb_apply_f64(_ptr(inv), _ptr(tx), _ptr(y), C.c_int64(nodes), None) == 0
    np.testing.assert_allclose(y.cpu().numpy().reshape(nodes, 5), np.einsum("nij,nj->ni", got, x.reshape(nodes, 5)), rtol=1e-13, atol=1e-13)
    y32 = torch.empty(5 * nodes, dtype=torch.float32, device=_dev())
    assert L.hb_pb_apply_f32(_ptr(inv32), _ptr(tx.float()), _ptr(y32), C.c_int64(nodes), None) == 0
    assert rel_l2(y32.double().cpu().numpy(), y.cpu().numpy()) < 1e-6
    assert L.hb_pb_apply_f64(_ptr(inv), _ptr(tx), _ptr(tx), C.c_int64(nodes), None) != 0  # x and y must differ


@pytest.mark.parametrize("name,kw", [("pulse_P3Q3", dict()), ("modes_P4Q5", dict(n=(3, 3, 3), P=4, Q=5, state="modes"))])
def test_bdf1_step_with_point_block_jacobi(name, kw):
    mesh, basis, ctx, q0, op, qdata = _problem(**kw)
    dt = ctx.dt
    rtol = 1e-9
    for fp32 in (0, 1):
        out = {}
        for pc in (1, 2):
            q1, t, (st,), _ = _run(op, ctx, qdata, q0, 1, dt=dt, bdf_order=1, newton_rtol=rtol, jacobian_fp32=fp32, pc_jacobi=pc)
            assert st.converged_reason == 1, (pc, fp32, st)
            r = _oracle_bdf1_residual(mesh, basis, ctx, q1, q0, dt)
            assert np.linalg.norm(r) <= 2 * rtol * st.res0, (pc, fp32, np.linalg.norm(r) / st.res0)
            out[pc] = (q1, st)
        (qj, sj), (qb, sb) = out[1], out[2]
        assert rel_l2(qb - q0, qj - q0) < 1e-6
        # the time-derivative shift dominates these blocks, so the coupling they add saves few iterations: in FP64 they cost
        # none; built from FP32 Jacobian data their off-diagonal entries carry ~1e-4 relative error and cost up to ~15% more
        assert sb.ksp_its <= (1.3 if fp32 else 1.1) * sj.ksp_its + 2, (fp32, sb.ksp_its, sj.ksp_its)


def test_bdf2_with_freestream_faces_and_point_block_jacobi():
    """The small configuration's boundary (free-stream faces on every side) with vpbjacobi: the face blocks join the volume
    ones, and every step converges in FP64 and mixed precision to states that agree."""
    import torch
    mesh, basis, ctx, q, _ = case(n=(4, 4, 4), P=3, Q=3, dt=1e-5)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    off, xn, _ = prob.box_faces(mesh, basis)
    fop = K.FaceOp(off, mesh.l_size, basis, xn)
    cb = prob.freestream_context(ctx, 101325.0, np.array([10.0, 0.0, 0.0]), 288.0)
    res = {}
    for fp32 in (0, 1):
        ts = S.TimeStepper(op, prob.context_bytes(ctx), qdata, dt=1e-5, bdf_order=2, newton_rtol=1e-9, jacobian_fp32=fp32, pc_jacobi=2)
        ts.set_freestream(fop, cb, flux_type=1)
        tq = torch.from_numpy(q).to(_dev())
        ts.set_state(tq, 0.0)
        stats = [ts.step() for _ in range(4)]
        assert all(s.converged_reason == 1 for s in stats), stats
        out = torch.empty_like(tq)
        ts.get_state(out)
        res[fp32] = out.cpu().numpy()
    assert rel_l2(res[1] - q, res[0] - q) < 1e-6
