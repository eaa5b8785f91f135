"""CPU checks of the spanwise-statistics oracle (oracle/spanstats_oracle.py) and of the box layout the GPU monitor uses.

* the statistics of every point equal the reference's ChildStatsCollection_Conserv (qfunctions/spanstats/turbulence.h,
  compiled unchanged in oracle/_ref) bit for bit, including the w detJ * (t - t_prev) weighting and its context layout
* the star forest built from coordinates, as the reference builds it (src/spanstats/spanstats.c:253-289), sends child
  point (qi, qj, qk) of element (ex, ey, ez) to parent point qi + Q qj of parent element ex + nx ey: the column structure
  spanstats.box_span_layout hands the GPU, on uniform, tanh-graded and periodic boxes
* averaging a time-invariant state whose density is constant and whose velocity is a polynomial of the parent space
  returns that velocity at the parent nodes (the L2 projection reproduces its own space) and the density exactly
"""
import ctypes as C
import importlib

import numpy as np
import pytest

from helpers import O, prob

import spanstats_oracle as SO  # noqa: E402

SP = importlib.import_module("honee-4aiad_b200.spanstats")


def _ctx():
    return prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)


def test_statistics_match_reference_qfunction_bit_for_bit():
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    ctx = _ctx()
    cb = prob.context_bytes(ctx)
    assert O.ref().ref_turb_spanstats_ctx_size() == 16 + len(cb)
    rng = np.random.default_rng(3)
    n = 257
    rho = rng.uniform(0.8, 1.4, n)
    u = rng.normal(0, 30, (3, n))
    T = rng.uniform(250, 350, n)
    U = np.vstack([rho, rho * u, rho * (ctx.gas.cv * T + 0.5 * (u * u).sum(0))])
    qdata = np.zeros((10, n))
    qdata[0] = rng.uniform(1e-6, 1e-3, n)
    x = np.zeros((3, n))
    t_prev, t_now = 0.37, 0.37 + 2.5e-3
    ctx_stats = np.array([t_now, t_prev]).tobytes() + cb
    v = np.zeros((22, n))
    assert O.call_qf(O.ref().ref_ChildStatsCollection_Conserv, ctx_stats, n, [U, qdata, x], [v]) == 0
    mine = SO.stats_weighted(U, qdata[0] * (t_now - t_prev), ctx.gas.cv, ctx.gas.cp)
    np.testing.assert_array_equal(mine, v)
    assert len(SP.COMPONENTS) == 22 == SO.NS


@pytest.mark.parametrize("n,P,periodic,beta", [((3, 2, 2), 2, (0, 0, 1), 0.0), ((3, 4, 3), 3, (1, 0, 1), 1.8), ((2, 3, 2), 4, (1, 0, 0), 1.2)])
def test_star_forest_is_the_column_layout(n, P, periodic, beta):
    Q = P + 1
    planes = [np.linspace(0, 4.0, n[0] + 1), prob.tanh_planes(n[1], -1.0, 1.0, beta), np.linspace(0, 2.0, n[2] + 1)]
    mesh = prob.box_mesh(n, P, periodic=periodic, planes=planes)
    basis = prob.tensor_basis(P, Q)
    lay = SP.box_span_layout(mesh)
    xy_p, _ = SO.parent_points(lay.parent_x, Q, basis.qref1d, basis.qweight1d)
    match = SO.star_forest(SO.child_points_xy(mesh, Q), xy_p)
    expect = np.zeros((mesh.num_elem, Q ** 3), dtype=np.int64)
    qxy = np.arange(Q ** 3) % (Q * Q)
    for col in range(lay.column_elems.shape[0]):
        for e in lay.column_elems[col]:
            expect[e] = col * Q * Q + qxy
    np.testing.assert_array_equal(match, expect.reshape(-1))
    assert lay.span_width == pytest.approx(2.0)
    # every child element lies in exactly one column
    assert np.array_equal(np.sort(lay.column_elems.reshape(-1)), np.arange(mesh.num_elem))


def test_tanh_planes_cluster_at_the_walls():
    y = prob.tanh_planes(32, -1.0, 1.0, 1.8)
    dy = np.diff(y)
    assert y[0] == -1.0 and y[-1] == 1.0 and np.all(dy > 0)
    assert dy[0] < dy[16] / 4 and np.allclose(dy, dy[::-1])
    np.testing.assert_allclose(prob.tanh_planes(4, 0, 1, 0.0), np.linspace(0, 1, 5))


def test_average_of_steady_polynomial_field_is_exact():
    n, P, Q = (3, 3, 2), 3, 4
    planes = [np.linspace(0, 3.0, n[0] + 1), prob.tanh_planes(n[1], -1.0, 1.0, 1.5), np.linspace(0, 1.0, n[2] + 1)]
    mesh = prob.box_mesh(n, P, periodic=(1, 0, 1), planes=planes)
    basis = prob.tensor_basis(P, Q)
    ctx = _ctx()
    X = prob.node_coordinates(mesh, basis)
    rho0 = 1.2
    u = np.stack([3 + 2 * X[1] - X[1] ** 2, 0.5 * X[1], 0 * X[1] + 0.25])  # quadratic in y: inside the parent space
    T = 300.0 + 0 * X[1]
    q = np.vstack([rho0 + 0 * T, rho0 * u, rho0 * (ctx.gas.cv * T + 0.5 * (u * u).sum(0))]).T.reshape(-1)
    qdata = O.setup_qdata(mesh.num_elem, Q, mesh.x_elem)
    lay = SP.box_span_layout(mesh)
    xy_p, wdetJ_p = SO.parent_points(lay.parent_x, Q, basis.qref1d, basis.qweight1d)
    match = SO.star_forest(SO.child_points_xy(mesh, Q), xy_p)
    child = None
    times = [0.0, 0.1, 0.25, 0.32]
    for t0, t1 in zip(times[:-1], times[1:]):
        child = SO.collect_child(mesh, basis, qdata, q, ctx.gas.cv, ctx.gas.cp, t1 - t0, child)
    parent = SO.reduce_to_parent(child, match, xy_p.shape[0] * xy_p.shape[1])
    stats = SO.process(parent, times[-1] - times[0], lay.span_width, lay.parent_offsets, lay.num_parent_nodes, basis.interp1d, P, Q, wdetJ_p)
    Nx, Ny = lay.parent_dims
    yn = X[1].reshape(-1)[: Nx * Ny]  # the k = 0 plane of the node grid (node i + Nx (j + Ny k))
    np.testing.assert_allclose(stats[:, 0], rho0, rtol=1e-13)
    np.testing.assert_allclose(stats[:, 19], 3 + 2 * yn - yn ** 2, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(stats[:, 20], 0.5 * yn, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(stats[:, 12], rho0 * 0.25, rtol=1e-12)


@pytest.mark.parametrize("sv", [1, 2])
def test_statistics_in_other_state_variables_match_reference(sv):
    """ChildStatsCollection_Prim / _Entropy (compiled in oracle/_ref) against the oracle's StateFromQ + statistics."""
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    ctx = _ctx()
    ctx.state_var = sv
    cb = prob.context_bytes(ctx)
    rng = np.random.default_rng(5)
    n = 129
    rho = rng.uniform(0.8, 1.4, n)
    u = rng.normal(0, 30, (3, n))
    T = rng.uniform(250, 350, n)
    U = np.vstack([rho, rho * u, rho * (ctx.gas.cv * T + 0.5 * (u * u).sum(0))])
    qv = np.ascontiguousarray(prob.state_to_q(ctx.gas, U.T.reshape(-1), sv).reshape(-1, 5).T)
    qdata = np.zeros((10, n))
    qdata[0] = rng.uniform(1e-6, 1e-3, n)
    v = np.zeros((22, n))
    name = ("Conserv", "Prim", "Entropy")[sv]
    ctx_stats = np.array([0.5 + 1e-3, 0.5]).tobytes() + cb
    assert O.call_qf(getattr(O.ref(), f"ref_ChildStatsCollection_{name}"), ctx_stats, n, [qv, qdata, np.zeros((3, n))], [v]) == 0
    import face_oracle as FaceO
    mine = SO.stats_state(FaceO.state_from_q(qv, sv, ctx.gas.cv, ctx.gas.cp), qdata[0] * 1e-3)
    for c in range(22):
        np.testing.assert_allclose(mine[c], v[c], rtol=1e-12, atol=1e-14 * np.abs(v[c]).max(), err_msg=SP.COMPONENTS[c])
