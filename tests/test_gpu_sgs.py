"""GPU tests of the learned-closure kernels against the reference QFunctions (golden fixture) and the CPU oracle:
point-wise maps (FP64, 1e-10), FP32 network inference with the reference's weights (1e-5), the training kernels'
gradient (against float64 back-propagation, 1e-4 relative) and Adam step, and a training run that fits a teacher network."""
import importlib
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import sgs_oracle as SO  # noqa: E402

S = importlib.import_module("honee-4aiad_b200.sgs")
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "sgs_points.npz"))


def _t(a, dtype=None):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).to("cuda:0")


def test_point_maps_and_reference_model_match_reference_qfunctions():
    import torch
    n = GOLD["G"].shape[0]
    dXdx = _t(GOLD["dXdx"].reshape(n, 9))
    kmA = torch.empty(n, 6, dtype=torch.float64, device="cuda:0")
    delta = torch.empty(n, dtype=torch.float64, device="cuda:0")
    S.point_anisotropy(dXdx, kmA, delta)
    torch.cuda.synchronize()
    np.testing.assert_allclose(kmA.cpu().numpy(), GOLD["Aij_delta"][:6].T, rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(delta.cpu().numpy(), GOLD["Aij_delta"][6], rtol=1e-12)
    inp = torch.empty(n, 6, dtype=torch.float64, device="cuda:0")
    E = torch.empty(n, 9, dtype=torch.float64, device="cuda:0")
    gmag = torch.empty(n, dtype=torch.float64, device="cuda:0")
    S.point_inputs(_t(GOLD["G"].reshape(n, 9)), _t(GOLD["Aij_delta"][:6].T), _t(GOLD["Aij_delta"][6]), _t(GOLD["nu"]), inp, E, gmag)
    torch.cuda.synchronize()
    np.testing.assert_allclose(inp.cpu().numpy(), GOLD["inputs"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(E.cpu().numpy().reshape(n, 3, 3), GOLD["E"], rtol=1e-10, atol=1e-11)
    np.testing.assert_allclose(gmag.cpu().numpy(), GOLD["gmag"], rtol=1e-12)
    # the reference's 6-20-6 network in FP32, then the de-normalisation and rotation in FP64
    d = S.desc(20, 0, 0.0, GOLD["bounds"])
    w = _t(GOLD["weights"], torch.float32)
    x32 = inp.float().contiguous()
    y32 = torch.empty_like(x32)
    S.forward(d, w, x32, y32)
    tau = torch.empty(n, 6, dtype=torch.float64, device="cuda:0")
    S.point_stress(y32.double().contiguous(), _t(GOLD["Aij_delta"][6]), E, gmag, GOLD["bounds"], tau)
    torch.cuda.synchronize()
    ref = GOLD["km_sgs"].T
    err = np.linalg.norm(tau.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < 1e-5, err  # FP32 weights and arithmetic in the network


@pytest.mark.parametrize("h2", [20, 0])
def test_training_gradient_matches_float64_backprop(h2):
    import torch
    rng = np.random.default_rng(11)
    d = S.desc(20, h2, 0.0)
    p = S.xavier_init(d, seed=3)
    n = 5000
    X = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
    Y = rng.uniform(0, 1, (n, 6)).astype(np.float32)
    idx = rng.integers(0, n, 1000).astype(np.int32)
    tr = S.Trainer(d, p, batch=1000)
    g = torch.empty(S.num_params(d), dtype=torch.float32, device="cuda:0")
    tr.step(_t(X), _t(Y), idx=_t(idx), lr=0.0, grad=g)
    torch.cuda.synchronize()
    loss_ref, g_ref = SO.loss_and_grad(p.astype(np.float64), 20, h2, X[idx].astype(np.float64), Y[idx].astype(np.float64))
    assert tr.loss.item() == pytest.approx(loss_ref, rel=1e-5)
    gg = g.cpu().numpy()
    assert np.linalg.norm(gg - g_ref) / np.linalg.norm(g_ref) < 1e-4
    np.testing.assert_array_equal(tr.params(), p)  # lr 0: gradient only


def test_adam_step_matches_oracle():
    import torch
    rng = np.random.default_rng(12)
    d = S.desc(20, 20, 0.0)
    p = S.xavier_init(d, seed=4)
    n = 3000
    X = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
    Y = rng.uniform(0, 1, (n, 6)).astype(np.float32)
    idx = np.arange(512, dtype=np.int32)
    tr = S.Trainer(d, p, batch=512, lr=1e-3)
    g = torch.empty(S.num_params(d), dtype=torch.float32, device="cuda:0")
    pp, m, v = p.astype(np.float64), np.zeros(p.size), np.zeros(p.size)
    for t in range(1, 4):
        tr.step(_t(X), _t(Y), idx=_t(idx), grad=g)
        torch.cuda.synchronize()
        gg = g.cpu().numpy().astype(np.float64)
        pp, m, v = SO.adam_step(pp, m, v, gg, t, 1e-3)
        np.testing.assert_allclose(tr.params(), pp, rtol=1e-5, atol=1e-7)
        pp = tr.params().astype(np.float64)


def test_training_fits_a_teacher_network():
    import torch
    rng = np.random.default_rng(13)
    teacher = S.desc(20, 20, 0.0)
    pt = S.xavier_init(teacher, seed=99) * 1.5
    n = 200_000
    X = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
    Yt, _, _ = SO.forward(pt.astype(np.float64), 20, 20, X.astype(np.float64))
    d = S.desc(20, 20, 0.0)
    tr = S.Trainer(d, S.xavier_init(d, seed=1), batch=8192, lr=3e-3, seed=7)
    tx, ty = _t(X), _t(Yt.astype(np.float32))
    hist = tr.train(tx, ty, 1500, log_every=500)
    assert hist[-1][1] < 0.1 * hist[0][1], hist
    # the device inference agrees with the oracle forward pass of the trained weights
    yd = torch.empty_like(tx)
    S.forward(d, tr.w, tx, yd)
    yo, _, _ = SO.forward(tr.params().astype(np.float64), 20, 20, X[:1000].astype(np.float64))
    np.testing.assert_allclose(yd[:1000].cpu().numpy(), yo, rtol=1e-4, atol=1e-5)


def test_target_bounds_and_normalisation():
    import torch
    rng = np.random.default_rng(14)
    Y = rng.normal(0, 3, (100_003, 6)).astype(np.float32)
    ty = _t(Y)
    work = torch.empty(4096, dtype=torch.float32, device="cuda:0")
    b = S.target_bounds(ty, work).reshape(6, 2)
    np.testing.assert_array_equal(b[:, 0], Y.min(0))
    np.testing.assert_array_equal(b[:, 1], Y.max(0))
    S.normalize_targets(ty, b)
    torch.cuda.synchronize()
    yn = ty.cpu().numpy()
    assert yn.min() >= 0 and yn.max() <= 1.0000001
    np.testing.assert_allclose(yn, (Y - b[:, 0]) / (b[:, 1] - b[:, 0]), rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("model", ["reference_6_20_6", "xavier_6_20_20_6"])
def test_residual_with_fused_closure_matches_oracle(model):
    """IFunction with the closure minus IFunction without it equals the closure's flux contribution computed by the
    oracle (FP32 network, FP64 elsewhere: 1e-5 relative)."""
    import torch
    from helpers import prob, rel_l2
    import filter_oracle  # noqa: F401  (used by the oracle contribution)
    K = importlib.import_module("honee-4aiad_b200.kernels")
    L = 2 * np.pi
    mesh = prob.box_mesh((3, 3, 3), 3, periodic=(1, 1, 1), hi=(L, L, L))
    basis = prob.tensor_basis(3, 4)
    tg = prob.taylor_green_context(2)
    tg.u[0], tg.u[1], tg.u[2] = 0.2, 0.1, 0.3
    q = prob.taylor_green_state(mesh, basis, tg)
    ctx = tg.newt_ctx
    ctx.dt, ctx.ijacobian_time_shift = 0.01, 150.0
    cb = prob.context_bytes(ctx)
    if model == "reference_6_20_6":
        d, w = S.desc(20, 0, 0.0, GOLD["bounds"]), GOLD["weights"].astype(np.float32)
    else:
        d = S.desc(20, 20, 0.0, np.array([-1, 1] * 6, dtype=np.float64) * 0.5)
        w = S.xavier_init(d, seed=8)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to("cuda:0")
    qdata = torch.zeros(mesh.num_elem * 10 * basis.Q ** 3, dtype=torch.float64, device="cuda:0")
    op.setup_qdata(x, qdata)
    tq = torch.from_numpy(q).to("cuda:0")
    tqd = torch.zeros_like(tq)
    v0, v1 = torch.empty_like(tq), torch.empty_like(tq)
    op.ifunction(cb, tq, tqd, qdata, v0)
    op.ifunction_sgs(cb, tq, tqd, qdata, v1, d, w)
    torch.cuda.synchronize()
    got = (v1 - v0).cpu().numpy()
    ref = SO.residual_contribution(mesh, basis, qdata.cpu().numpy(), q, ctx.gas, w, d.hidden1, d.hidden2, np.array(d.out_bounds[:]))
    assert np.linalg.norm(ref) > 0
    assert rel_l2(got, ref) < 1e-5, rel_l2(got, ref)
