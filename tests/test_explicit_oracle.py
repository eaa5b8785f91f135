"""CPU checks of the explicit-path oracle (oracle/explicit_oracle.py, the RHS and mass operators of oracle/honee_oracle.c):

* the restated RHSFunction_Newtonian (the IFunction integrand at q_dot = 0, negated) equals the reference's own
  RHSFunction_Newtonian (qfunctions/newtonian.h:133-202) and the restated Mass_5 the reference's (qfunctions/mass.h), when
  oracle/_ref is built;
* the mass diagonal equals e_i^T M e_i;
* the restated loop (TSRK4 + KSPGMRES/PCJacobi-diagonal mass solves) reproduces the reference's own explicit run of
  examples/navierstokes.c:222: the kinetic-energy rows of tests/output/taylorgreen_totalke.csv at steps 0, 2, 3 and the
  final state tests/output/taylor-green.bin (carried in tests/golden/taylorgreen_rk4.npz), the state compared the way the
  reference's regression test does (src/misc.c:111-118: max |Q - Q_ref| / max |Q_ref| <= 1e-10), as sorted component
  columns because DMPlex numbers the nodes differently from the box mesh here.
"""
import json
import os

import numpy as np
import pytest

from helpers import O, case, oracle_mesh, prob, rel_l2

import explicit_oracle as X  # noqa: E402  (oracle/ is on sys.path through helpers)

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def taylor_green_rk4_case():
    """The configuration of examples/navierstokes.c:222 (examples/taylor_green_vortex.yaml, 2^3 faces, degree 2)."""
    import ctypes as C
    g = json.load(open(os.path.join(GOLD, "taylorgreen_ke_step0.json")))
    L = g["box"][1]
    mesh = prob.box_mesh(g["faces"], g["P"], periodic=(1, 1, 1), hi=(L, L, L))
    basis = prob.tensor_basis(g["P"], g["Q"])
    tg = prob.TaylorGreenContext()
    tg.reference = prob.StatePrimitive(g["reference_pressure"], (C.c_double * 3)(*g["reference_velocity"]), g["reference_temperature"])
    tg.newt_ctx = prob.newtonian_context(g["degree"], cv=g["cv"], cp=g["cp"], mu=g["mu"], k=g["k"], stab=prob.STAB_SUPG, Ctau_t=1.0,
                                         Ctau_v=60, Ctau_C=0.5, Ctau_M=0.5, Ctau_E=0.5, implicit=False)
    tg.lx = tg.ly = tg.lz = L
    X_ = prob.node_coordinates(mesh, basis)
    q = np.zeros((5, X_.shape[1]))
    O.call_qf(O.lib().oracle_qf_ics_taylorgreen, bytes(memoryview(tg)), X_.shape[1], [np.ascontiguousarray(X_)], [q])
    return mesh, basis, tg, np.ascontiguousarray(q.T.reshape(-1)), L


def ke_rows_match(rows, G, rtol=1e-11, ztol=3e-10):
    """Relative tolerance on the physical columns; the columns that are round-off in the reference (|ref| < 1e-12:
    divergence dissipation and volume expansion of an incompressible initial field) against an absolute one."""
    for i, st in enumerate(G["ke_steps"]):
        for j, name in enumerate(G["ke_names"]):
            ref, got = G["ke"][i, j], rows[int(st)][j]
            tol = rtol * abs(ref) if abs(ref) >= 1e-12 else ztol
            assert abs(got - ref) <= tol, (int(st), str(name), got, ref)


def state_matches(q, G, tol=1e-10):
    ref = G["final_state"].reshape(-1, 5)
    ours = np.asarray(q).reshape(-1, 5)
    assert ref.shape == ours.shape
    err = max(np.abs(np.sort(ref[:, c]) - np.sort(ours[:, c])).max() for c in range(5)) / np.abs(ref).max()
    assert err <= tol, err
    return err


@pytest.mark.parametrize("P,Q,periodic,idl", [(3, 3, (0, 0, 0), None), (4, 5, (1, 0, 0), (2e-3, 0.2, 0.5, 101000.0))])
def test_rhs_and_mass_restatements_equal_reference(P, Q, periodic, idl):
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    mesh, basis, ctx, q, _ = case((2, 2, 2), P, Q, periodic=periodic, idl=idl, g=(0.3, -9.81, 0.1))
    m = oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    xq = O.coords_at_qpts(mesh.num_elem, basis.Q, mesh.x_elem)
    cb = prob.context_bytes(ctx)
    r_o = O.apply_rhs(m, cb, q, qdata, xq)
    r_r = O.apply_rhs(m, cb, q, qdata, xq, use_ref=True)
    assert rel_l2(r_o, r_r) < 1e-14
    # and it is the negated IFunction at zero rate
    njd = 15 if ctx.idl_enable else 14
    v = O.apply_ifunction(m, cb, q, np.zeros_like(q), qdata, np.zeros(mesh.num_elem * njd * Q ** 3), num_jd=njd, x_q=xq)
    assert rel_l2(-v, r_r) < 1e-14
    u = np.random.default_rng(0).normal(size=q.shape)
    np.testing.assert_array_equal(O.apply_mass(m, u, qdata), O.apply_mass(m, u, qdata, use_ref=True))


def test_mass_diagonal_is_the_operator_diagonal():
    mesh, basis, ctx, q, _ = case((2, 1, 2), 3, 4, periodic=(1, 0, 0))
    m = oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    d = X.mass_diagonal(m, basis.P, basis.Q, qdata, mesh.l_size)
    for i in np.random.default_rng(3).choice(mesh.l_size, 25, replace=False):
        e = np.zeros(mesh.l_size)
        e[i] = 1.0
        assert abs(O.apply_mass(m, e, qdata)[i] - d[i]) <= 1e-15 * np.abs(d).max()


def run_oracle_tg(mass_ksp, pc_jacobi, steps=3):
    mesh, basis, tg, q, L = taylor_green_rk4_case()
    m = oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    cb = bytes(memoryview(tg.newt_ctx))
    ex = X.Explicit(m, basis.P, basis.Q, cb, qdata, mesh.l_size, dt=2e-3, tableau="4", mass_ksp=mass_ksp, pc_jacobi=pc_jacobi)
    rows, t = {}, 0.0
    for step in range(steps + 1):
        rows[step] = O.monitor_ke(m, cb, q, qdata) / L ** 3
        if step < steps:
            q = ex.step(q, t)
            t += 2e-3
    return rows, q, ex


def test_explicit_rk4_reproduces_reference_run():
    G = np.load(os.path.join(GOLD, "taylorgreen_rk4.npz"))
    rows, q, ex = run_oracle_tg("gmres", "diagonal")
    ke_rows_match(rows, G)
    assert state_matches(q, G) < 1e-10
    assert len(ex.mass_its) == 12 and all(0 < i < 30 for i in ex.mass_its)


def test_lumped_mass_is_distinguishable_from_the_reference_run():
    """The comparison above is sharp: HONEE's default lumped mass (not what the reference run used) misses it by ~1e-6."""
    G = np.load(os.path.join(GOLD, "taylorgreen_rk4.npz"))
    rows, q, _ = run_oracle_tg("preonly", "rowsum")
    ke3 = rows[3][0]
    assert abs(ke3 - G["ke"][2, 0]) > 1e-8 * abs(G["ke"][2, 0])


@pytest.mark.parametrize("stab", [prob.STAB_SUPG, prob.STAB_SU, prob.STAB_NONE])
def test_stabilized_mass_restatement_equals_reference(stab):
    """MassFunction_Newtonian (qfunctions/newtonian.h:44-86), the mass operator HONEE uses for explicit SUPG runs."""
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    mesh, basis, ctx, q, qd = case((2, 2, 1), 4, 4, stab=stab)
    m = oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    cb = prob.context_bytes(ctx)
    np.testing.assert_array_equal(O.apply_mass_stab(m, cb, qd, q, qdata), O.apply_mass_stab(m, cb, qd, q, qdata, use_ref=True))


def test_stabilized_mass_diagonal_is_the_operator_diagonal():
    mesh, basis, ctx, q, _ = case((2, 1, 1), 3, 4, periodic=(1, 0, 0))
    m = oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, basis.Q, mesh.x_elem)
    cb = prob.context_bytes(ctx)
    d = O.mass_stab_diagonal(m, cb, q, qdata, mesh.l_size)
    for i in np.random.default_rng(4).choice(mesh.l_size, 25, replace=False):
        e = np.zeros(mesh.l_size)
        e[i] = 1.0
        assert abs(O.apply_mass_stab(m, cb, e, q, qdata)[i] - d[i]) <= 1e-13 * np.abs(d).max()


def gaussian_wave_explicit_case():
    """"Gaussian Wave, explicit, supg, IDL" (examples/navierstokes.c:233, examples/gaussianwave.yaml): degree 3 on 2 x 2 x 1 faces
    of [0,1]^2 x [0,0.025], free-stream faces (HLLC) on the x and y sides, symmetry planes (z momentum) on the z sides, SUPG,
    the internal damping layer, TSRK5F with dt 2e-3, GMRES + Jacobi-diagonal solves of the stabilized mass."""
    import face_oracle as FO
    G = np.load(os.path.join(GOLD, "gaussianwave_explicit.npz"))
    hi = tuple(float(v) for v in G["box_hi"])
    deg = int(G["degree"])
    P = Q = deg + 1
    mesh = prob.box_mesh(tuple(int(v) for v in G["faces"]), P, hi=hi)
    basis = prob.tensor_basis(P, Q)
    Pr, ux, uy, uz, T = (float(v) for v in G["reference_PuT"])
    decay, start, length, p_idl = (float(v) for v in G["idl"])
    newt = prob.newtonian_context(deg, mu=float(G["mu"]), stab=prob.STAB_SUPG, implicit=False, idl=(decay, start, length, p_idl), dt=float(G["dt"]))
    gw = prob.gaussian_wave_context(newt, Pr, (ux, uy, uz), T, epicenter=tuple(float(v) for v in G["epicenter"]), width=float(G["width"]),
                                    amplitude=float(G["amplitude"]))
    q = prob.gaussian_wave_state(mesh, basis, gw)
    ess = prob.box_essential(mesh, {"z-": (3,), "z+": (3,)})
    q[ess] = 0.0
    off, xn, _ = prob.box_faces(mesh, basis, sides=["x-", "x+", "y-", "y+"])
    fs = prob.freestream_context(newt, Pr, (ux, uy, uz), T)
    U, Y = prob.state_from_primitive(newt.gas, Pr, (ux, uy, uz), T)
    return G, mesh, basis, newt, gw, q, ess, off, xn, fs, U, Y, FO


def test_gaussian_wave_initial_state_equals_reference():
    if O.ref() is None:
        pytest.skip("oracle/_ref not built")
    G, mesh, basis, newt, gw, q, ess, off, xn, fs, U, Y, FO = gaussian_wave_explicit_case()
    import ctypes as C
    assert O.ref().ref_gaussianwave_ctx_size() == C.sizeof(gw)
    X_ = prob.node_coordinates(mesh, basis)
    qr = np.zeros((5, X_.shape[1]))
    O.call_qf(O.ref().ref_IC_GaussianWave_Conserv, bytes(memoryview(gw)), X_.shape[1], [np.ascontiguousarray(X_)], [qr])
    qr = qr.T.reshape(-1)
    qr[ess] = 0.0  # the reference's IC has zero z momentum there too
    np.testing.assert_array_equal(q, qr)


def test_oracle_reproduces_reference_gaussian_wave_explicit_run():
    G, mesh, basis, newt, gw, q, ess, off, xn, fs, U, Y, FO = gaussian_wave_explicit_case()
    P, Q = basis.P, basis.Q
    m = oracle_mesh(mesh, basis)
    qdata = O.setup_qdata(mesh.num_elem, Q, mesh.x_elem)
    xq = O.coords_at_qpts(mesh.num_elem, Q, mesh.x_elem)
    qd_sur = FO.face_qdata(basis.interp1d, basis.grad1d, basis.qweight1d, P, Q, xn)
    gas = newt.gas
    faces = lambda qq: FO.freestream_apply(off, basis.interp1d, P, Q, qd_sur, qq, U, Y, gas.cv, gas.cp, hllc=True, l_size=mesh.l_size)  # noqa
    ex = X.Explicit(m, P, Q, prob.context_bytes(newt), qdata, mesh.l_size, dt=float(G["dt"]), tableau=str(G["rk_type"]),
                    mass_ksp=str(G["mass_ksp"]), pc_jacobi=str(G["mass_pc_jacobi"]), x_q=xq, essential=ess, faces=faces)
    assert ex.stab_mass
    t = 0.0
    for _ in range(int(G["steps"])):
        q = ex.step(q, t)
        t += float(G["dt"])
    free = np.setdiff1d(np.arange(mesh.l_size), ess)
    ref = G["free_state"]
    err = np.abs(np.sort(q[free]) - np.sort(ref)).max() / np.abs(ref).max()
    assert err <= float(G["compare_atol"]), err
