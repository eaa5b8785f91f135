"""CPU checks of the nodal SGS-pipeline oracle (oracle/sgs_nodal_oracle.py) against the reference's own QFunctions: the
committed fixture tests/golden/sgs_nodal_points.npz (made by make_sgs_nodal_golden.py from oracle/_ref) holds
VelocityGradientProjectionRHS_*, ComputeSgsDDNodal_* and IFunction_NodalSgs_* for the three state variables, and
AnisotropyTensorProjection, InverseMultiplicity and Mass_9, on seeded points.  Also checks the oracle's operators on a
small mesh: the mass diagonal against the assembled matrix, the projections' solvers, and the multiplicity weights."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
import sgs_nodal_oracle as SN  # noqa: E402

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "sgs_nodal_points.npz"))
SGS = np.load(os.path.join(ROOT, "tests", "golden", "sgs_points.npz"))
NAMES = ("Conserv", "Prim", "Entropy")


def _X(qdata):
    return qdata[1:].reshape(3, 3, -1)


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_velocity_gradient_points_match_reference(sv):
    name = NAMES[sv]
    v = SN.velgrad_points(GOLD[f"q_{name}"], GOLD[f"grad_q_{name}"], GOLD["qdata"][0], _X(GOLD["qdata"]), sv, float(GOLD["cv"]), float(GOLD["cp"]))
    ref = GOLD[f"velgrad_{name}"]
    np.testing.assert_allclose(v, ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())


def test_anisotropy_projection_points_match_reference():
    a = SN.aniso_points(GOLD["qdata"][0], _X(GOLD["qdata"]))
    np.testing.assert_allclose(a, GOLD["aniso"], rtol=1e-12, atol=1e-14 * np.abs(GOLD["aniso"]).max())


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_nodal_closure_matches_reference(sv):
    name = NAMES[sv]
    net = SN.Net(SGS["weights"], SGS["bounds"])
    q, G, A, im = GOLD[f"q_{name}"], GOLD["G"], GOLD["Aij_delta"], GOLD["inv_mult"]
    ref = GOLD[f"km_sgs_{name}"]
    for i in range(q.shape[1]):
        tau = im[i] * SN.closure_point(net, q[:, i], G[i], A[:, i], sv, float(GOLD["mu"]), float(GOLD["cv"]), float(GOLD["cp"]))
        np.testing.assert_allclose(tau, ref[:, i], rtol=1e-10, atol=1e-10 * np.abs(ref[:, i]).max())


@pytest.mark.parametrize("sv", [0, 1, 2])
def test_sgs_flux_points_match_reference(sv):
    name = NAMES[sv]
    gv = SN.sgs_flux_points(GOLD[f"q_{name}"], GOLD["km"], GOLD["qdata"][0], _X(GOLD["qdata"]), sv, float(GOLD["cv"]), float(GOLD["cp"]))
    ref = GOLD[f"grad_v_{name}"]
    np.testing.assert_allclose(gv, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def test_inverse_multiplicity_and_mass_points_match_reference():
    np.testing.assert_array_equal(1.0 / GOLD["mult"][0], GOLD["inv_out"])
    np.testing.assert_allclose(GOLD["qdata"][0] * GOLD["u9"], GOLD["mass9"], rtol=0, atol=0)


def _small():
    prob = importlib.import_module("honee-4aiad_b200.problem")
    import oracle as O
    mesh = prob.box_mesh((2, 1, 2), 3, periodic=(True, False, False))
    basis = prob.tensor_basis(3, 4)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    return prob, mesh, basis, qdata


def test_mass_diagonal_and_projection_solvers():
    prob, mesh, basis, qdata = _small()
    nc = 7
    n = mesh.num_nodes * nc
    M = np.stack([SN.mass_apply(mesh, basis, qdata, np.eye(1, n, k).ravel(), nc) for k in range(n)], axis=1)
    np.testing.assert_allclose(SN.mass_diagonal(mesh, basis, qdata, nc), np.diag(M), rtol=1e-13)
    rng = np.random.default_rng(5)
    b = rng.normal(size=n)
    x = SN.project_cg(mesh, basis, qdata, b, nc, rtol=1e-12)
    np.testing.assert_allclose(M @ x, b, rtol=1e-9, atol=1e-10 * np.abs(b).max())
    np.testing.assert_allclose(SN.project_rowsum(mesh, basis, qdata, b, nc), b / M.sum(1), rtol=1e-13)


def test_inverse_multiplicity_sums_to_one_per_node():
    _, mesh, _, _ = _small()
    im = SN.inverse_multiplicity(mesh)
    nodes = (mesh.offsets.reshape(mesh.num_elem, -1) // 5)
    w = np.bincount(nodes.ravel(), weights=im.ravel(), minlength=mesh.num_nodes)
    np.testing.assert_allclose(w, 1.0, rtol=1e-15)


def test_sgs_dd_context_blob_runs_the_reference_closure():
    """sgs.sgs_dd_context lays the blob out as the reference compiler does, and the reference's ComputeSgsDDNodal_Conserv
    run on it gives the golden stresses (skipped without oracle/_ref)."""
    import oracle as O
    R = O.ref()
    if R is None:
        pytest.skip("oracle/_ref not built")
    import ctypes as C
    prob = importlib.import_module("honee-4aiad_b200.problem")
    sgs = importlib.import_module("honee-4aiad_b200.sgs")
    lay = (C.c_size_t * 4)()
    R.ref_sgs_dd_ctx_layout(lay)
    assert list(lay) == [264, 24, 208, 256]
    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257)
    blob = bytes(sgs.sgs_dd_context(prob.context_bytes(ctx), SGS["weights"], SGS["bounds"]))
    n = GOLD["q_Conserv"].shape[1]
    out = np.zeros((6, n))
    O.call_qf(R.ref_ComputeSgsDDNodal_Conserv, blob, n, [GOLD["q_Conserv"], GOLD["x"], np.ascontiguousarray(GOLD["G"].transpose(1, 2, 0)),
                                                         GOLD["Aij_delta"], GOLD["inv_mult"]], [out])
    np.testing.assert_array_equal(out, GOLD["km_sgs_Conserv"])


def test_nodal_pipeline_closure_matches_reference_on_a_mesh():
    """SN.sgs_nodal on a small mesh with a generic state (all velocity components perturbed) equals the reference's
    ComputeSgsDDNodal_Prim at every node (skipped without oracle/_ref).  At degenerate states (v = w = 0: repeated
    strain-rate eigenvalues, an eigenframe orthogonal to the vorticity) the reference's own result depends on rounding."""
    import oracle as O
    R = O.ref()
    if R is None:
        pytest.skip("oracle/_ref not built")
    prob = importlib.import_module("honee-4aiad_b200.problem")
    sgs = importlib.import_module("honee-4aiad_b200.sgs")
    mesh = prob.box_mesh((2, 2, 1), 3, periodic=(True, False, False))
    basis = prob.tensor_basis(3, 4)
    ctx = prob.newtonian_context(2, cv=717.5, cp=1004.5, mu=1.8e-5, k=0.0257, state_var=1)
    gas = ctx.gas
    q = prob.multimode_state(mesh, basis, gas, seed=4).reshape(-1, 5).copy()
    rng = np.random.default_rng(8)
    q[:, 2:4] += q[:, 0:1] * rng.normal(0, 2.0, (q.shape[0], 2))
    q = prob.state_to_q(gas, q.reshape(-1), 1)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    A7 = SN.project_cg(mesh, basis, qdata, SN.aniso_rhs(mesh, basis, qdata), 7, rtol=1e-12)
    G9 = SN.project_rowsum(mesh, basis, qdata, SN.velgrad_rhs(mesh, basis, qdata, q, 1, gas.cv, gas.cp), 9)
    km = SN.sgs_nodal(mesh, SN.Net(SGS["weights"], SGS["bounds"]), q, G9, A7, SN.inverse_multiplicity(mesh), 1, gas.mu, gas.cv, gas.cp)
    N = mesh.num_nodes
    blob = bytes(sgs.sgs_dd_context(prob.context_bytes(ctx), SGS["weights"], SGS["bounds"]))
    out = np.zeros((6, N))
    O.call_qf(R.ref_ComputeSgsDDNodal_Prim, blob, N, [np.ascontiguousarray(q.reshape(N, 5).T), np.zeros((3, N)),
                                                      np.ascontiguousarray(G9.reshape(N, 3, 3).transpose(1, 2, 0)),
                                                      np.ascontiguousarray(A7.reshape(N, 7).T), np.ones(N)], [out])
    ref = out.T.reshape(-1)
    assert np.linalg.norm(km - ref) / np.linalg.norm(ref) < 1e-13
