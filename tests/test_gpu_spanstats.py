"""GPU parity of the spanwise turbulence statistics (k_stats.cu, hb_stats.c) against the oracle (oracle/spanstats_oracle.py,
which follows the reference's child collection, coordinate star forest and projection and is pinned to the reference's
ChildStatsCollection_Conserv).

Tolerances: the parent-point sums 1e-13 relative L2 (FP64 sums in a different order: over the span per step, then over
time, where the reference sums over time per child point first); the parent mass operator 1e-14; the processed
statistics 1e-12 as a whole and 1e-9 per component with the CG driven to rtol 1e-14 (the oracle solves directly; one CG
over all 22 components converges in one norm, dominated by the largest fields), and the reference's own stopping rule
(rtol 1e-10 in the natural norm) leaves them within 1e-8."""
import ctypes as C
import importlib

import numpy as np
import pytest

from helpers import O, prob, rel_l2

import spanstats_oracle as SO  # noqa: E402

pytestmark = pytest.mark.gpu

K = importlib.import_module("honee-4aiad_b200.kernels")
SP = importlib.import_module("honee-4aiad_b200.spanstats")
hb = importlib.import_module("honee-4aiad_b200")


def _dev():
    import torch
    return torch.device("cuda:0")


def channel_case(n=(3, 4, 3), P=3, Q=4, beta=1.8, seed=0):
    planes = [np.linspace(0, 4 * np.pi / 3, n[0] + 1), prob.tanh_planes(n[1], -1.0, 1.0, beta), np.linspace(0, 2 * np.pi / 9, n[2] + 1)]
    mesh = prob.box_mesh(n, P, periodic=(1, 0, 1), planes=planes)
    basis = prob.tensor_basis(P, Q)
    newt = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)
    ch = prob.channel_context(newt, (0, -1, 0), (1, 1, 1), umax=20.0)
    q = prob.perturbed_channel_state(mesh, basis, ch, amplitude=0.05, seed=seed)
    return mesh, basis, ch, q


def _oracle(mesh, basis, ctx, qdata, states, times, lay):
    xy_p, wdetJ_p = SO.parent_points(lay.parent_x, basis.Q, basis.qref1d, basis.qweight1d)
    match = SO.star_forest(SO.child_points_xy(mesh, basis.Q), xy_p)
    child = None
    for k, qk in enumerate(states):
        child = SO.collect_child(mesh, basis, qdata, qk, ctx.gas.cv, ctx.gas.cp, times[k + 1] - times[k], child)
    parent = SO.reduce_to_parent(child, match, xy_p.shape[0] * xy_p.shape[1])
    stats = SO.process(parent, times[-1] - times[0], lay.span_width, lay.parent_offsets, lay.num_parent_nodes, basis.interp1d, basis.P,
                       basis.Q, wdetJ_p)
    return parent, stats, wdetJ_p


@pytest.mark.parametrize("n,P,Q", [((3, 4, 3), 3, 4), ((2, 3, 2), 4, 5), ((3, 2, 2), 2, 2), ((2, 2, 3), 6, 7)])
def test_collection_and_processing_match_oracle(n, P, Q):
    import torch
    mesh, basis, ch, q0 = channel_case(n, P, Q)
    ctx = ch.newt_ctx
    cb = prob.context_bytes(ctx)
    op = K.ElemOp(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, Q, mesh.x_elem)
    tqd = torch.from_numpy(qdata).to(_dev())
    lay = SP.box_span_layout(mesh)
    rng = np.random.default_rng(5)
    states = [q0 * (1 + 0.01 * rng.uniform(-1, 1, q0.shape)) for _ in range(3)]
    times = [0.5, 0.5 + 1e-3, 0.5 + 2.5e-3, 0.5 + 3e-3]
    st = SP.SpanStats(op, lay, initial_time=times[0])
    for k, qk in enumerate(states):
        st.collect(cb, torch.from_numpy(qk).to(_dev()), tqd, times[k + 1])
    parent_ref, stats_ref, wdetJ_ref = _oracle(mesh, basis, ctx, qdata, states, times, lay)
    assert rel_l2(st.sums().reshape(-1, 22), parent_ref) < 1e-13
    stats, its, rel = st.process(times[-1], rtol=1e-14)
    got = stats.cpu().numpy()
    assert rel <= 1e-14 and its > 0
    assert rel_l2(got, stats_ref) < 1e-12
    for c in range(22):  # one CG for all components converges in one norm: the small fields carry the large ones' error
        assert rel_l2(got[:, c], stats_ref[:, c]) < 1e-9, (c, SP.COMPONENTS[c])
    stats, its10, rel10 = st.process(times[-1])  # the reference's rtol 1e-10
    assert rel10 <= 1e-10 and its10 <= its
    assert rel_l2(stats.cpu().numpy(), stats_ref) < 1e-8


def test_parent_mass_operator_matches_oracle():
    import torch
    mesh, basis, ch, q0 = channel_case((3, 4, 2), 4, 5)
    op = K.ElemOp(mesh, basis)
    lay = SP.box_span_layout(mesh)
    st = SP.SpanStats(op, lay)
    _, wdetJ_ref = SO.parent_points(lay.parent_x, basis.Q, basis.qref1d, basis.qweight1d)
    _, M = SO.plane_operators(lay.parent_offsets, lay.num_parent_nodes, basis.interp1d, basis.P, basis.Q, wdetJ_ref)
    u = np.random.default_rng(2).normal(size=(lay.num_parent_nodes, 22))
    tu = torch.from_numpy(u.reshape(-1).copy()).to(_dev())
    tv = torch.empty_like(tu)
    L = hb.lib()
    pl = st.plane()
    assert L.hb_plane_mass_apply(pl, C.c_void_p(tu.data_ptr()), C.c_void_p(tv.data_ptr()), 0, None) == 0
    assert rel_l2(tv.cpu().numpy().reshape(-1, 22), M @ u) < 1e-14
    d = torch.empty(lay.num_parent_nodes, dtype=torch.float64, device=_dev())
    assert L.hb_plane_mass_diagonal(pl, C.c_void_p(d.data_ptr()), 0, None) == 0
    assert rel_l2(d.cpu().numpy(), M.diagonal()) < 1e-14
    # the parent geometric factors integrate the plane's area
    assert float(wdetJ_ref.sum()) == pytest.approx(4 * np.pi / 3 * 2.0, rel=1e-14)


def test_steady_polynomial_field_is_reproduced_at_full_channel_width():
    """48 x 32 parent elements of degree 3 on the tanh-graded plane (the parent of the 48 x 32 x 24 channel), 4 spanwise
    elements: a steady state whose velocity is quadratic in y averages to itself at every parent node."""
    import torch
    n, P, Q = (48, 32, 4), 4, 5
    planes = [np.linspace(0, 4 * np.pi, n[0] + 1), prob.tanh_planes(n[1], -1.0, 1.0, 1.8), np.linspace(0, 2 * np.pi / 3, n[2] + 1)]
    mesh = prob.box_mesh(n, P, periodic=(1, 0, 1), planes=planes)
    basis = prob.tensor_basis(P, Q)
    gas = prob.newtonian_context(P - 1, cv=717.5, cp=1004.5).gas
    X = prob.node_coordinates(mesh, basis)
    rho0 = 1.16
    u = np.stack([20 * (1 - X[1] ** 2), 0.0 * X[1], 0.0 * X[1]])
    q = np.vstack([rho0 + 0 * X[1], rho0 * u, rho0 * (gas.cv * 300.0 + 0.5 * (u * u).sum(0))]).T.reshape(-1)
    op = K.ElemOp(mesh, basis)
    x = torch.from_numpy(np.ascontiguousarray(mesh.x_elem)).to(_dev())
    qdata = torch.zeros(mesh.num_elem * 10 * Q ** 3, dtype=torch.float64, device=_dev())
    op.setup_qdata(x, qdata)
    lay = SP.box_span_layout(mesh)
    st = SP.SpanStats(op, lay)
    tq = torch.from_numpy(q).to(_dev())
    cb = prob.context_bytes(prob.newtonian_context(P - 1, cv=717.5, cp=1004.5))
    for t in (1e-3, 3e-3, 4e-3):
        st.collect(cb, tq, qdata, t)
    stats, its, rel = st.process(4e-3, rtol=1e-13)
    got = stats.cpu().numpy()
    Nx, Ny = lay.parent_dims
    yn = X[1].reshape(-1)[: Nx * Ny]
    np.testing.assert_allclose(got[:, 0], rho0, rtol=1e-12)
    np.testing.assert_allclose(got[:, 19], 20 * (1 - yn ** 2), rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(got[:, 10], rho0 * 20 * (1 - yn ** 2), rtol=1e-11, atol=1e-11)
    assert np.abs(got[:, 20:22]).max() < 1e-11


def test_errors_are_reported():
    import torch
    mesh, basis, ch, q0 = channel_case((2, 2, 2), 3, 4)
    op = K.ElemOp(mesh, basis)
    lay = SP.box_span_layout(mesh)
    st = SP.SpanStats(op, lay, initial_time=1.0)
    with pytest.raises(K.HbError):
        st.process(1.0)  # no time has elapsed
    bad = SP.SpanLayout(lay.column_elems + mesh.num_elem, lay.parent_offsets, lay.num_parent_nodes, lay.parent_x, lay.span_width,
                        lay.parent_dims)
    with pytest.raises(K.HbError):
        SP.SpanStats(op, bad)
    ctx = prob.newtonian_context(2)
    ctx.state_var = 7  # not a state variable
    qdata = torch.zeros(mesh.num_elem * 10 * 64, dtype=torch.float64, device=_dev())
    with pytest.raises(K.HbError):
        st.collect(prob.context_bytes(ctx), torch.from_numpy(q0).to(_dev()), qdata, 1.5)


@pytest.mark.parametrize("sv", [prob.STATEVAR_PRIMITIVE, prob.STATEVAR_ENTROPY])
def test_collection_in_other_state_variables_matches_oracle(sv):
    """ChildStatsCollection_Prim / _Entropy: the state handed over in primitive or entropy variables (interpolated in
    those variables, then converted at each point)."""
    import torch
    mesh, basis, ch, q0 = channel_case((3, 3, 2), 3, 4)
    ctx = ch.newt_ctx
    ctx.state_var = sv
    cb = prob.context_bytes(ctx)
    op = K.ElemOp(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, 4, mesh.x_elem)
    tqd = torch.from_numpy(qdata).to(_dev())
    lay = SP.box_span_layout(mesh)
    rng = np.random.default_rng(6)
    states = [prob.state_to_q(ctx.gas, q0 * (1 + 0.01 * rng.uniform(-1, 1, q0.shape)), sv) for _ in range(2)]
    times = [0.0, 2e-3, 3e-3]
    st = SP.SpanStats(op, lay, initial_time=times[0])
    for k, qk in enumerate(states):
        st.collect(cb, torch.from_numpy(qk).to(_dev()), tqd, times[k + 1])
    xy_p, wdetJ_p = SO.parent_points(lay.parent_x, basis.Q, basis.qref1d, basis.qweight1d)
    match = SO.star_forest(SO.child_points_xy(mesh, basis.Q), xy_p)
    child = None
    for k, qk in enumerate(states):
        child = SO.collect_child(mesh, basis, qdata, qk, ctx.gas.cv, ctx.gas.cp, times[k + 1] - times[k], child, sv=sv)
    parent = SO.reduce_to_parent(child, match, xy_p.shape[0] * xy_p.shape[1])
    got = st.sums().reshape(-1, 22)
    for c in range(22):
        assert rel_l2(got[:, c], parent[:, c]) < 1e-12, (c, SP.COMPONENTS[c])
