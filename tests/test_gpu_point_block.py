"""GPU parity of the point-block diagonal (hb_point_block_diagonal_*, hb_freestream_point_block_diagonal,
hb_mass_point_block_diagonal, and CeedOperatorLinearAssemblePointBlockDiagonal[Symbolic] as MatCEED calls them for
-pc_type vpbjacobi) against the CPU oracle (oracle_assemble_point_block, face_oracle.freestream_point_block, both checked
block by block against the oracle's Jacobian action on CPU).

Tolerances: FP64 1e-12 relative L2.  FP32 (the mixed-precision resource: Jacobian data stored in FP32): the diagonal
entries 2e-6; the whole blocks within 10x the error that rounding the stored Jacobian data to FP32 already causes (the oracle
evaluated on that rounded data): the off-diagonal entries are differences of larger terms, so FP32 inputs alone move them
by up to ~5e-5 relative.
"""
import importlib

import numpy as np
import pytest

from helpers import O, case, oracle_ifunction, oracle_mesh, prob, rel_l2

import explicit_oracle as X  # noqa: E402
import face_oracle as FO  # noqa: E402

pytestmark = pytest.mark.gpu

K = importlib.import_module("honee-4aiad_b200.kernels")

CASES = {
    "P3Q3": dict(n=(3, 2, 2), P=3, Q=3),
    "P4Q5_modes": dict(n=(2, 3, 2), P=4, Q=5, state="modes"),
    "P5Q6_periodic": dict(n=(2, 2, 2), P=5, Q=6, periodic=(1, 1, 1), state="modes"),
    "P6Q7": dict(n=(2, 1, 1), P=6, Q=7),
    "P3Q4_idl_su": dict(n=(3, 2, 1), P=3, Q=4, stab=prob.STAB_SU, idl=(2e-3, 0.2, 0.5, 101000.0)),
}


def _dev():
    import torch
    return torch.device("cuda:0")


def check_fp32_blocks(pb32, pb_ref, pb_ref_rounded_inputs):
    eye = np.eye(5, dtype=bool)
    got, ref = pb32.reshape(-1, 5, 5), pb_ref.reshape(-1, 5, 5)
    assert rel_l2(got[:, eye], ref[:, eye]) < 2e-6
    floor = max(rel_l2(pb_ref_rounded_inputs, pb_ref), 1e-6)
    assert rel_l2(pb32, pb_ref) < 10 * floor, (rel_l2(pb32, pb_ref), floor)


@pytest.mark.parametrize("name", list(CASES))
def test_point_block_matches_oracle(name):
    import torch
    mesh, basis, ctx, q, qd = case(**CASES[name])
    v, jd, qdata, m = oracle_ifunction(mesh, basis, ctx, q, qd)
    njd = 15 if ctx.idl_enable else 14
    cb = prob.context_bytes(ctx)
    pb_ref = O.assemble_point_block(m, cb, qdata, jd, mesh.l_size, num_jd=njd)
    d_ref = O.assemble_diagonal(m, cb, qdata, jd, mesh.l_size, num_jd=njd)
    op = K.ElemOp(mesh, basis)
    if ctx.idl_enable:
        op.set_vertex_coords(np.ascontiguousarray(mesh.x_elem))
    tqd = torch.from_numpy(qdata).to(_dev())
    tjd = torch.from_numpy(jd).to(_dev())
    pb = torch.zeros(5 * mesh.l_size, dtype=torch.float64, device=_dev())
    op.point_block_diagonal(cb, tqd, tjd, pb)
    assert rel_l2(pb.cpu().numpy(), pb_ref) < 1e-12
    np.testing.assert_allclose(pb.cpu().numpy().reshape(-1, 5, 5)[:, np.arange(5), np.arange(5)].reshape(-1), d_ref, rtol=1e-11,
                               atol=1e-13 * np.abs(d_ref).max())
    # add mode accumulates onto what is there
    op.point_block_diagonal(cb, tqd, tjd, pb, add=True)
    assert rel_l2(pb.cpu().numpy(), 2 * pb_ref) < 1e-12
    # FP32 Jacobian data
    tjd32 = tjd.float()
    pb32 = torch.zeros(5 * mesh.l_size, dtype=torch.float32, device=_dev())
    op.point_block_diagonal(cb, tqd, tjd32, pb32, fp32=True)
    pb_rounded = O.assemble_point_block(m, cb, qdata, jd.astype(np.float32).astype(np.float64), mesh.l_size, num_jd=njd)
    check_fp32_blocks(pb32.double().cpu().numpy(), pb_ref, pb_rounded)


def test_face_and_mass_point_blocks_match_oracle():
    import torch
    mesh, basis, ctx, q, _ = case(n=(2, 3, 2), P=3, Q=4, state="pulse")
    off, xn, names = prob.box_faces(mesh, basis)
    fop = K.FaceOp(off, mesh.l_size, basis, xn)
    u_inf = np.array([60.0, -25.0, 10.0])
    gas = ctx.gas
    cb = prob.freestream_context(ctx, 101325.0 * 1.02, u_inf, 290.0)
    rho = 101325.0 * 1.02 / ((gas.cp - gas.cv) * 290.0)
    U = np.array([rho, *(rho * u_inf), rho * (gas.cv * 290.0 + 0.5 * u_inf @ u_inf)])
    Y = np.array([101325.0 * 1.02, *u_inf, 290.0])
    tq = torch.from_numpy(q).to(_dev())
    fop.freestream(cb, tq, torch.zeros_like(tq), flux_type=1)
    out = torch.zeros(5 * mesh.l_size, dtype=torch.float64, device=_dev())
    fop.freestream_point_block(cb, out, flux_type=1)
    qd_ref = FO.face_qdata(basis.interp1d, basis.grad1d, basis.qweight1d, basis.P, basis.Q, xn)
    jac = fop.jac.cpu().numpy().reshape(len(names), 5, basis.Q ** 2)
    ref = FO.freestream_point_block(off, basis.interp1d, basis.P, basis.Q, qd_ref, jac, U, Y, gas.cv, gas.cp, hllc=True, l_size=mesh.l_size)
    assert rel_l2(out.cpu().numpy(), ref) < 1e-12
    # mass: its diagonal on each block's diagonal
    op = K.ElemOp(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    mb = torch.zeros(5 * mesh.l_size, dtype=torch.float64, device=_dev())
    op.mass_point_block_diagonal(torch.from_numpy(qdata).to(_dev()), mb)
    md = X.mass_diagonal(oracle_mesh(mesh, basis), basis.P, basis.Q, qdata, mesh.l_size)
    expect = np.zeros((mesh.l_size // 5, 5, 5))
    expect[:, np.arange(5), np.arange(5)] = md.reshape(-1, 5)
    assert rel_l2(mb.cpu().numpy(), expect.reshape(-1)) < 1e-14


@pytest.mark.parametrize("resource", ["/gpu/b200", "/gpu/b200/mixed"])
def test_point_blocks_through_the_ceed_api(resource):
    """The IJacobian composite with free-stream faces: the COO triplets MatCEED would hand PETSc (symbolic rows/cols plus
    values) assemble to the sum of the volume and face blocks of the oracle."""
    ce = importlib.import_module("honee-4aiad_b200.ceed")
    hon = importlib.import_module("honee-4aiad_b200.honee")
    mesh, basis, ctx, q, qdv = case(n=(3, 2, 2), P=3, Q=3)
    ceed = ce.Ceed(resource)
    ops = hon.NewtonianOperators(ceed, mesh, basis, ctx)
    bc = ops.add_freestream(101325.0 * 1.02, np.array([60.0, -25.0, 10.0]), 290.0, riemann="hllc")
    qv = ce.Vector(ceed, mesh.l_size)
    qv.set_array_host(q)
    ops.q_dot.set_array_host(qdv)
    ops.ifunction(qv, ops.q_dot, ce.Vector(ceed, mesh.l_size))
    rows, cols = ops.op_ijacobian.point_block_symbolic()
    assert rows.size == 5 * mesh.l_size == cols.size
    vals = ce.Vector(ceed, 5 * mesh.l_size)
    ops.op_ijacobian.assemble_point_block_diagonal(vals)
    dense = np.zeros((mesh.l_size, 5))  # row, column within the row's node block
    np.add.at(dense, (rows, cols % 5), vals.to_numpy())
    assert np.all(rows // 5 == cols // 5)
    # oracle: volume blocks + face blocks
    v, jd, qdata, m = oracle_ifunction(mesh, basis, ctx, q, qdv)
    pb_vol = O.assemble_point_block(m, prob.context_bytes(ctx), qdata, jd, mesh.l_size)
    pb_vol_rounded = O.assemble_point_block(m, prob.context_bytes(ctx), qdata, jd.astype(np.float32).astype(np.float64), mesh.l_size)
    gas = ctx.gas
    u_inf = np.array([60.0, -25.0, 10.0])
    rho = 101325.0 * 1.02 / ((gas.cp - gas.cv) * 290.0)
    U = np.array([rho, *(rho * u_inf), rho * (gas.cv * 290.0 + 0.5 * u_inf @ u_inf)])
    Y = np.array([101325.0 * 1.02, *u_inf, 290.0])
    P, Q = basis.P, basis.Q
    F = bc["offsets"].shape[0]
    qd_sur = bc["q_data"].to_numpy().reshape(F, 10, Q * Q)
    jac = bc["jac_data"].to_numpy().reshape(F, 5, Q * Q)
    pb_face = FO.freestream_point_block(bc["offsets"], basis.interp1d, P, Q, qd_sur, jac, U, Y, gas.cv, gas.cp, hllc=True, l_size=mesh.l_size)
    got = dense.reshape(-1)
    if resource == "/gpu/b200":
        assert rel_l2(got, pb_vol + pb_face) < 1e-12
    else:  # FP32 volume blocks, FP64 faces
        check_fp32_blocks(got, pb_vol + pb_face, pb_vol_rounded + pb_face)
    # and the diagonal of those blocks is the assembled diagonal
    d = ce.Vector(ceed, mesh.l_size)
    ops.diagonal(d)
    assert rel_l2(got.reshape(-1, 5, 5)[:, np.arange(5), np.arange(5)].reshape(-1), d.to_numpy()) < (1e-12 if resource == "/gpu/b200" else 2e-6)
