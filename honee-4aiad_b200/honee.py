"""HONEE's operator set-up for the Newtonian volume operator, written against the libCEED binding.

Mirrors, call for call, what the reference does before time stepping:
  * QDataGet (src/qdata.c:133-190): the ``Setup`` QFunction on the coordinate field -> qdata [elem][10][Q^3]
  * SetupLibceed (src/setuplibceed.c:97-340): bases, restrictions, jac_data, the IFunction and IJacobian volume
    operators with the field names of src/setuplibceed.c:216-266, wrapped in composite operators (:295-306)
  * NS_NEWTONIAN_IG context registration (problems/newtonian.c:744-753): "timestep size", "ijacobian time shift",
    "solution time" labels
and exposes the calls the reference makes in its hot loop:
  * IFunction_NS (src/setupts.c:78-125)      -> :meth:`NewtonianOperators.ifunction`
  * FormIJacobian_NS (src/setupts.c:131-157) -> :meth:`NewtonianOperators.set_ijacobian_shift`
  * MatMult_Ceed (src/mat-ceed.c:1643-1700)  -> :meth:`NewtonianOperators.ijacobian`
  * MatGetDiagonal_Ceed (src/mat-ceed.c:1603-1634) -> :meth:`NewtonianOperators.diagonal`
and, for the free-stream boundary (problems/bc_freestream.c:112-190), the face sub-operators the reference adds to both
composites: QDataBoundaryGet (src/qdata.c:228-270, ``SetupBoundary``), HoneeBCAddIFunctionOp / HoneeBCAddIJacobianOp
(src/boundary_condition.c:371-470) with the QFunctions of HoneeBCCreateIFunctionQF / HoneeBCCreateIJacobianQF
(:276-364) -> :meth:`NewtonianOperators.add_freestream`.
The structured box mesh stands in for DMPlex; all arithmetic happens in libceed_b200.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import ceed as ce
from .problem import CONTEXT_LABELS, BoxMesh, TensorBasis, box_faces, context_bytes, freestream_context


def linear_coordinate_basis(Q: int, qref1d, qweight1d):
    """P=2 Lagrange basis of the trilinear coordinate field at the solution's quadrature points."""
    x = np.asarray(qref1d)
    B = np.stack([0.5 * (1 - x), 0.5 * (1 + x)], axis=1)
    G = np.tile(np.array([[-0.5, 0.5]]), (Q, 1))
    return B, G


class NewtonianOperators:
    def __init__(self, ceed: ce.Ceed, mesh: BoxMesh, basis: TensorBasis, ctx, *, num_comps_jac_data=None):
        self.ceed, self.mesh, self.basis, self.ctx = ceed, mesh, basis, ctx
        P, Q, E = basis.P, basis.Q, mesh.num_elem
        Q3 = Q ** 3
        njd = num_comps_jac_data or (15 if ctx.idl_enable else 14)
        self.num_jd = njd
        # -- bases (src/dm-utils.c:766-879)
        self.basis_q = ce.Basis(ceed, 3, 5, P, Q, basis.interp1d, basis.grad1d, basis.qref1d, basis.qweight1d)
        Bx, Gx = linear_coordinate_basis(Q, basis.qref1d, basis.qweight1d)
        self.basis_x = ce.Basis(ceed, 3, 3, 2, Q, Bx, Gx, basis.qref1d, basis.qweight1d)
        # -- restrictions (src/dm-utils.c:83-137, :235)
        self.rstr_q = ce.ElemRestriction(ceed, E, P ** 3, 5, 1, mesh.l_size, offsets=mesh.offsets)
        off_x = (np.arange(E * 8, dtype=np.int64) * 3).astype(np.int32)  # element-local (periodic-safe) coordinates
        self.rstr_x = ce.ElemRestriction(ceed, E, 8, 3, 1, E * 24, offsets=off_x)
        self.rstr_qd = ce.ElemRestriction(ceed, E, Q3, 10, 0, E * Q3 * 10)
        self.rstr_jd = ce.ElemRestriction(ceed, E, Q3, njd, 0, E * Q3 * njd)
        # -- coordinates as an interleaved L-vector [elem][vertex][3]
        x_elem = mesh.x_elem.reshape(E, 3, 8)
        self.x_coord = ce.Vector(ceed, E * 24)
        self.x_coord.set_array_host(np.ascontiguousarray(x_elem.transpose(0, 2, 1)).reshape(-1))
        # -- qdata (QDataGet, src/qdata.c:153-178)
        self.q_data = ce.Vector(ceed, E * Q3 * 10)
        qf_setup = ce.QFunction(ceed, "setupgeo.h:Setup")
        qf_setup.add_input("dx", 9, ce.CEED_EVAL_GRAD)
        qf_setup.add_input("weight", 1, ce.CEED_EVAL_WEIGHT)
        qf_setup.add_output("surface qdata", 10, ce.CEED_EVAL_NONE)
        op_setup = ce.Operator(ceed, qf_setup)
        op_setup.set_field("dx", self.rstr_x, self.basis_x, ceed.active)
        op_setup.set_field("weight", ceed.rstr_none, self.basis_x, ceed.vector_none)
        op_setup.set_field("surface qdata", self.rstr_qd, ceed.basis_none, ceed.active)
        op_setup.apply(self.x_coord, self.q_data)
        self.op_setup = op_setup
        # -- context (problems/newtonian.c:744-753)
        self.qfctx = ce.QFunctionContext(ceed, ctx)
        for name, off in CONTEXT_LABELS.items():
            self.qfctx.register_double(name, off, 1)
        # -- vectors (src/setuplibceed.c:125-131)
        self.jac_data = ce.Vector(ceed, E * Q3 * njd)
        self.q_dot = ce.Vector(ceed, mesh.l_size)
        # -- IFunction volume operator (src/setuplibceed.c:209-243)
        sv_name = ("Conserv", "Prim", "Entropy")[ctx.state_var]  # problems/newtonian.c:771-787: the QFunctions of the state variable
        qf_if = ce.QFunction(ceed, f"newtonian.h:IFunction_Newtonian_{sv_name}")
        for name, size, mode in (("q", 5, ce.CEED_EVAL_INTERP), ("Grad_q", 15, ce.CEED_EVAL_GRAD), ("q dot", 5, ce.CEED_EVAL_INTERP),
                                 ("qdata", 10, ce.CEED_EVAL_NONE), ("x", 3, ce.CEED_EVAL_INTERP)):
            qf_if.add_input(name, size, mode)
        qf_if.add_output("v", 5, ce.CEED_EVAL_INTERP)
        qf_if.add_output("Grad_v", 15, ce.CEED_EVAL_GRAD)
        qf_if.add_output("jac_data", njd, ce.CEED_EVAL_NONE)
        qf_if.set_context(self.qfctx)
        op_if = ce.Operator(ceed, qf_if)
        op_if.set_name("IFunction Domain Operator")
        op_if.set_field("q", self.rstr_q, self.basis_q, ceed.active)
        op_if.set_field("Grad_q", self.rstr_q, self.basis_q, ceed.active)
        op_if.set_field("q dot", self.rstr_q, self.basis_q, self.q_dot)
        op_if.set_field("qdata", self.rstr_qd, ceed.basis_none, self.q_data)
        op_if.set_field("x", self.rstr_x, self.basis_x, self.x_coord)
        op_if.set_field("v", self.rstr_q, self.basis_q, ceed.active)
        op_if.set_field("Grad_v", self.rstr_q, self.basis_q, ceed.active)
        op_if.set_field("jac_data", self.rstr_jd, ceed.basis_none, self.jac_data)
        # -- IJacobian volume operator (src/setuplibceed.c:245-269)
        qf_ij = ce.QFunction(ceed, f"newtonian.h:IJacobian_Newtonian_{sv_name}")
        for name, size, mode in (("dq", 5, ce.CEED_EVAL_INTERP), ("Grad_dq", 15, ce.CEED_EVAL_GRAD), ("qdata", 10, ce.CEED_EVAL_NONE),
                                 ("jac_data", njd, ce.CEED_EVAL_NONE)):
            qf_ij.add_input(name, size, mode)
        qf_ij.add_output("v", 5, ce.CEED_EVAL_INTERP)
        qf_ij.add_output("Grad_v", 15, ce.CEED_EVAL_GRAD)
        qf_ij.set_context(self.qfctx)
        op_ij = ce.Operator(ceed, qf_ij)
        op_ij.set_name("IJacobian Domain Operator")
        op_ij.set_field("dq", self.rstr_q, self.basis_q, ceed.active)
        op_ij.set_field("Grad_dq", self.rstr_q, self.basis_q, ceed.active)
        op_ij.set_field("qdata", self.rstr_qd, ceed.basis_none, self.q_data)
        op_ij.set_field("jac_data", self.rstr_jd, ceed.basis_none, self.jac_data)
        op_ij.set_field("v", self.rstr_q, self.basis_q, ceed.active)
        op_ij.set_field("Grad_v", self.rstr_q, self.basis_q, ceed.active)
        # -- composites (src/setuplibceed.c:295-306)
        self.op_ifunction = ce.Operator(ceed)
        self.op_ifunction.set_name("IFunction Composite Operator")
        self.op_ifunction.add_sub(op_if)
        self.op_ijacobian = ce.Operator(ceed)
        self.op_ijacobian.set_name("IJacobian Composite Operator")
        self.op_ijacobian.add_sub(op_ij)
        self._vol = (op_if, op_ij, qf_if, qf_ij, qf_setup)
        self.op_ifunction_volume, self.op_ijacobian_volume = op_if, op_ij
        self.boundaries = []

    # ---- explicit path (src/setuplibceed.c:179-205 for the RHS operator, :15-53 for the mass operator of CreateKSPMass)
    def add_explicit(self):
        """The RHSFunction_Newtonian volume operator (fields q, Grad_q, qdata, x -> v, Grad_v) in an "RHS" composite and the
        Mass_5 operator on the state fields, as SetupLibceed builds them for -ts_type rk."""
        ceed = self.ceed
        qf_rhs = ce.QFunction(ceed, "newtonian.h:RHSFunction_Newtonian")
        for name, size, mode in (("q", 5, ce.CEED_EVAL_INTERP), ("Grad_q", 15, ce.CEED_EVAL_GRAD), ("qdata", 10, ce.CEED_EVAL_NONE),
                                 ("x", 3, ce.CEED_EVAL_INTERP)):
            qf_rhs.add_input(name, size, mode)
        qf_rhs.add_output("v", 5, ce.CEED_EVAL_INTERP)
        qf_rhs.add_output("Grad_v", 15, ce.CEED_EVAL_GRAD)
        qf_rhs.set_context(self.qfctx)
        op_rhs_vol = ce.Operator(ceed, qf_rhs)
        op_rhs_vol.set_field("q", self.rstr_q, self.basis_q, ceed.active)
        op_rhs_vol.set_field("Grad_q", self.rstr_q, self.basis_q, ceed.active)
        op_rhs_vol.set_field("qdata", self.rstr_qd, ceed.basis_none, self.q_data)
        op_rhs_vol.set_field("x", self.rstr_x, self.basis_x, self.x_coord)
        op_rhs_vol.set_field("v", self.rstr_q, self.basis_q, ceed.active)
        op_rhs_vol.set_field("Grad_v", self.rstr_q, self.basis_q, ceed.active)
        self.op_rhs = ce.Operator(ceed)
        self.op_rhs.set_name("RHS Composite Operator")
        self.op_rhs.add_sub(op_rhs_vol)
        if self.ctx.stabilization == 2:  # SUPG: CreateKSPMassOperator_NewtonianStabilized (problems/newtonian.c:212-265, 795)
            self.q_state = ce.Vector(ceed, self.mesh.l_size)  # the state RHS_NS last evaluated at (honee->q_ceed)
            qf_mass = ce.QFunction(ceed, "newtonian.h:MassFunction_Newtonian_Conserv")
            qf_mass.add_input("q_dot", 5, ce.CEED_EVAL_INTERP)
            qf_mass.add_input("q", 5, ce.CEED_EVAL_INTERP)
            qf_mass.add_input("qdata", 10, ce.CEED_EVAL_NONE)
            qf_mass.add_output("v", 5, ce.CEED_EVAL_INTERP)
            qf_mass.add_output("Grad_v", 15, ce.CEED_EVAL_GRAD)
            qf_mass.set_context(self.qfctx)
            self.op_mass = ce.Operator(ceed, qf_mass)
            self.op_mass.set_name("RHS Mass Operator, Newtonian Stabilized")
            self.op_mass.set_field("q_dot", self.rstr_q, self.basis_q, ceed.active)
            self.op_mass.set_field("q", self.rstr_q, self.basis_q, self.q_state)
            self.op_mass.set_field("qdata", self.rstr_qd, ceed.basis_none, self.q_data)
            self.op_mass.set_field("v", self.rstr_q, self.basis_q, ceed.active)
            self.op_mass.set_field("Grad_v", self.rstr_q, self.basis_q, ceed.active)
        else:  # CreateKSPMassOperator_Unstabilized (src/setuplibceed.c:15-53)
            self.q_state = None
            qf_mass = ce.QFunction(ceed, "mass.h:Mass_5")
            qf_mass.add_input("u", 5, ce.CEED_EVAL_INTERP)
            qf_mass.add_input("qdata", 10, ce.CEED_EVAL_NONE)
            qf_mass.add_output("v", 5, ce.CEED_EVAL_INTERP)
            self.op_mass = ce.Operator(ceed, qf_mass)
            self.op_mass.set_name("RHS Mass Operator")
            self.op_mass.set_field("u", self.rstr_q, self.basis_q, ceed.active)
            self.op_mass.set_field("qdata", self.rstr_qd, ceed.basis_none, self.q_data)
            self.op_mass.set_field("v", self.rstr_q, self.basis_q, ceed.active)
        self._explicit = (op_rhs_vol, qf_rhs, qf_mass)

    def rhs(self, q: ce.Vector, g: ce.Vector):
        """R = RHS(q) before the mass solve (ApplyCeedOperatorLocalToGlobal in RHS_NS, src/setupts.c:50); the stabilized mass
        operator then sees the same state (the reference points honee->q_ceed at it, src/setupts.c:54)."""
        self.op_rhs.apply(q, g)
        if self.q_state is not None:
            q.copy_to(self.q_state)

    # ---- boundary faces
    def add_freestream(self, P_inf, u_inf, T_inf, *, riemann="hllc", sides=None, implicit=True):
        """Free-stream condition on the non-periodic box sides: face restriction and 2D basis of the state, the bilinear
        face coordinate field, surface qdata from ``SetupBoundary``, and the ``Freestream_[Jacobian_]{Conserv,Prim,Entropy}_HLL[C]`` sub-
        operators joined to the IFunction and IJacobian composites (num_comps_jac_data 5 for implicit runs,
        problems/bc_freestream.c:175)."""
        ceed, mesh, basis = self.ceed, self.mesh, self.basis
        P, Q = basis.P, basis.Q
        off, xn, names = box_faces(mesh, basis, sides)
        F = off.shape[0]
        Q2 = Q * Q
        flux = {"hll": "HLL", "hllc": "HLLC"}[riemann]
        sv_name = ("Conserv", "Prim", "Entropy")[self.ctx.state_var]  # the QFunctions of the state variable
        # -- face restriction and basis of the state (DMPlexCeedElemRestrictionCreate / DMPlexCeedBasisCreate at the face height)
        rstr_q = ce.ElemRestriction(ceed, F, P * P, 5, 1, mesh.l_size, offsets=off)
        basis_q = ce.Basis(ceed, 2, 5, P, Q, basis.interp1d, basis.grad1d, basis.qref1d, basis.qweight1d)
        # -- bilinear face coordinates (DMPlexCeedCoordinateCreateField at the face height): the face's corner nodes
        corners = [0, P - 1, P * (P - 1), P * P - 1]
        x_face = np.ascontiguousarray(xn[:, :, corners].transpose(0, 2, 1)).reshape(-1)      # [F][vertex][3]
        x_coord = ce.Vector(ceed, F * 12)
        x_coord.set_array_host(x_face)
        rstr_x = ce.ElemRestriction(ceed, F, 4, 3, 1, F * 12, offsets=(np.arange(F * 4, dtype=np.int64) * 3).astype(np.int32))
        Bx, Gx = linear_coordinate_basis(Q, basis.qref1d, basis.qweight1d)
        basis_x = ce.Basis(ceed, 2, 3, 2, Q, Bx, Gx, basis.qref1d, basis.qweight1d)
        # -- surface qdata (QDataBoundaryGet)
        rstr_qd = ce.ElemRestriction(ceed, F, Q2, 10, 0, F * Q2 * 10)
        q_data = ce.Vector(ceed, F * Q2 * 10)
        qf_setup = ce.QFunction(ceed, "setupgeo.h:SetupBoundary")
        qf_setup.add_input("dx", 6, ce.CEED_EVAL_GRAD)
        qf_setup.add_input("weight", 1, ce.CEED_EVAL_WEIGHT)
        qf_setup.add_output("surface qdata", 10, ce.CEED_EVAL_NONE)
        op_setup = ce.Operator(ceed, qf_setup)
        op_setup.set_field("dx", rstr_x, basis_x, ceed.active)
        op_setup.set_field("weight", ceed.rstr_none, basis_x, ceed.vector_none)
        op_setup.set_field("surface qdata", rstr_qd, ceed.basis_none, ceed.active)
        op_setup.apply(x_coord, q_data)
        # -- context: FreestreamContext_ (the Newtonian context and the exterior State)
        fs_bytes = freestream_context(self.ctx, P_inf, u_inf, T_inf)
        fs_ctx = ce.QFunctionContext(ceed, (ctypes.c_char * len(fs_bytes)).from_buffer_copy(fs_bytes))
        njd = 5 if implicit else 0
        rstr_jd = ce.ElemRestriction(ceed, F, Q2, 5, 0, F * Q2 * 5) if njd else None
        jac_data = ce.Vector(ceed, F * Q2 * 5) if njd else None
        # -- IFunction face sub-operator
        qf_if = ce.QFunction(ceed, f"bc_freestream.h:Freestream_{sv_name}_{flux}")
        for name, size, mode in (("q", 5, ce.CEED_EVAL_INTERP), ("Grad_q", 10, ce.CEED_EVAL_GRAD), ("surface qdata", 10, ce.CEED_EVAL_NONE),
                                 ("x", 3, ce.CEED_EVAL_INTERP)):
            qf_if.add_input(name, size, mode)
        qf_if.add_output("v", 5, ce.CEED_EVAL_INTERP)
        if njd:
            qf_if.add_output("surface jacobian data", njd, ce.CEED_EVAL_NONE)
        qf_if.set_context(fs_ctx)
        op_if = ce.Operator(ceed, qf_if)
        op_if.set_name("Freestream IFunction")
        op_if.set_field("q", rstr_q, basis_q, ceed.active)
        op_if.set_field("Grad_q", rstr_q, basis_q, ceed.active)
        op_if.set_field("surface qdata", rstr_qd, ceed.basis_none, q_data)
        op_if.set_field("x", rstr_x, basis_x, x_coord)
        op_if.set_field("v", rstr_q, basis_q, ceed.active)
        if njd:
            op_if.set_field("surface jacobian data", rstr_jd, ceed.basis_none, jac_data)
        self.op_ifunction.add_sub(op_if)
        op_ij = None
        if njd:
            qf_ij = ce.QFunction(ceed, f"bc_freestream.h:Freestream_Jacobian_{sv_name}_{flux}")
            for name, size, mode in (("dq", 5, ce.CEED_EVAL_INTERP), ("Grad_dq", 10, ce.CEED_EVAL_GRAD),
                                     ("surface qdata", 10, ce.CEED_EVAL_NONE), ("x", 3, ce.CEED_EVAL_INTERP),
                                     ("surface jacobian data", njd, ce.CEED_EVAL_NONE)):
                qf_ij.add_input(name, size, mode)
            qf_ij.add_output("v", 5, ce.CEED_EVAL_INTERP)
            qf_ij.set_context(fs_ctx)
            op_ij = ce.Operator(ceed, qf_ij)
            op_ij.set_name("Freestream IJacobian")
            op_ij.set_field("dq", rstr_q, basis_q, ceed.active)
            op_ij.set_field("Grad_dq", rstr_q, basis_q, ceed.active)
            op_ij.set_field("surface qdata", rstr_qd, ceed.basis_none, q_data)
            op_ij.set_field("x", rstr_x, basis_x, x_coord)
            op_ij.set_field("surface jacobian data", rstr_jd, ceed.basis_none, jac_data)
            op_ij.set_field("v", rstr_q, basis_q, ceed.active)
            self.op_ijacobian.add_sub(op_ij)
        bc = dict(offsets=off, x_nodes=xn, sides=names, q_data=q_data, jac_data=jac_data, ctx_bytes=fs_bytes, op_ifunction=op_if,
                  op_ijacobian=op_ij, hllc=flux == "HLLC",
                  _keep=(rstr_q, basis_q, x_coord, rstr_x, basis_x, rstr_qd, qf_setup, op_setup, fs_ctx, rstr_jd, qf_if))
        self.boundaries.append(bc)
        return bc

    # ---- data-driven SGS model, fused nodal implementation (problems/sgs_dd_model.c:645-737)
    def add_sgs_dd(self, flat_params, bounds, alpha=0.0, aniso_rtol=1e-10):
        """SgsDDSetup for a box mesh: the velocity-gradient projection (src/velocity_gradient_projection.c:44-140: right-hand
        side ``VelocityGradientProjectionRHS_*`` and ``Mass_9``, solved by one row-sum Jacobi step), the anisotropy tensor
        projected once (src/grid_anisotropy_tensor.c:10-118: ``AnisotropyTensorProjection``, ``Mass_7``, CG with Jacobi to
        ``aniso_rtol`` in the natural norm), the local inverse multiplicity (src/inverse_multiplicity.c:24-80), the nodal
        closure ``ComputeSgsDDNodal_*`` with the network's ``SgsDDContext_`` (flat_params and bounds in the layout of
        sgs.load_reference_model) and the residual term ``IFunction_NodalSgs_*``.  Afterwards :meth:`ifunction` adds the SGS
        term as IFunction_NS does through SgsDDApplyIFunction (problems/sgs_dd_model.c:559-587)."""
        from .sgs import sgs_dd_context
        ceed, mesh, basis = self.ceed, self.mesh, self.basis
        P, Q, E, N = basis.P, basis.Q, mesh.num_elem, mesh.num_nodes
        a, none_b = ceed.active, ceed.basis_none
        sv_name = ("Conserv", "Prim", "Entropy")[self.ctx.state_var]
        keep = []

        def rstr(nc):  # DMPlexCeedElemRestrictionCreate on the nc-field clone of the solution DM
            return ce.ElemRestriction(ceed, E, P ** 3, nc, 1, N * nc, offsets=(mesh.offsets // 5) * nc)

        def bas(nc):
            return ce.Basis(ceed, 3, nc, P, Q, basis.interp1d, basis.grad1d, basis.qref1d, basis.qweight1d)

        def qfunction(name, ins, outs, ctx=None):
            q = ce.QFunction(ceed, name)
            for nm, size, mode in ins:
                q.add_input(nm, size, mode)
            for nm, size, mode in outs:
                q.add_output(nm, size, mode)
            if ctx is not None:
                q.set_context(ctx)
            keep.append(q)
            return q

        def operator(qf, fields, name):
            op = ce.Operator(ceed, qf)
            op.set_name(name)
            for nm, r, b, v in fields:
                op.set_field(nm, r, b, v)
            keep.append(op)
            return op

        def mass(nc, r, b):
            qf = qfunction(f"mass.h:Mass_{nc}", [("u", nc, ce.CEED_EVAL_INTERP), ("qdata", 10, ce.CEED_EVAL_NONE)], [("v", nc, ce.CEED_EVAL_INTERP)])
            return operator(qf, [("u", r, b, a), ("qdata", self.rstr_qd, none_b, self.q_data), ("v", r, b, a)], f"Mass_{nc}")

        r9, r7, r6, b9, b7, b6 = rstr(9), rstr(7), rstr(6), bas(9), bas(7), bas(6)
        keep += [r9, r7, r6, b9, b7, b6]
        # -- velocity-gradient projection
        qf = qfunction(f"velocity_gradient_projection.h:VelocityGradientProjectionRHS_{sv_name}",
                       [("q", 5, ce.CEED_EVAL_INTERP), ("Grad_q", 15, ce.CEED_EVAL_GRAD), ("qdata", 10, ce.CEED_EVAL_NONE), ("x", 3, ce.CEED_EVAL_INTERP)],
                       [("velocity gradient", 9, ce.CEED_EVAL_INTERP)], self.qfctx)
        self.op_sgs_velgrad = operator(qf, [("q", self.rstr_q, self.basis_q, a), ("Grad_q", self.rstr_q, self.basis_q, a),
                                            ("qdata", self.rstr_qd, none_b, self.q_data), ("x", self.rstr_x, self.basis_x, self.x_coord),
                                            ("velocity gradient", r9, b9, a)], "velocity gradient projection RHS")
        op_m9 = mass(9, r9, b9)
        ones, self.sgs_rowsum_inv = ce.Vector(ceed, N * 9), ce.Vector(ceed, N * 9)
        ones.set_value(1.0)
        op_m9.apply(ones, self.sgs_rowsum_inv)  # PC_JACOBI_ROWSUM: MatGetRowSum = M 1
        self.sgs_rowsum_inv.reciprocal()
        # -- anisotropy tensor, projected once
        qf = qfunction("grid_anisotropy_tensor.h:AnisotropyTensorProjection", [("qdata", 10, ce.CEED_EVAL_NONE)], [("v", 7, ce.CEED_EVAL_INTERP)])
        op_a = operator(qf, [("qdata", self.rstr_qd, none_b, self.q_data), ("v", r7, b7, a)], "anisotropy tensor projection RHS")
        op_m7 = mass(7, r7, b7)
        rhs, diag, tmp = ce.Vector(ceed, N * 7), ce.Vector(ceed, N * 7), ce.Vector(ceed, N * 7)
        op_a.apply(None, rhs)
        op_m7.assemble_diagonal(diag)
        b_h, dinv = rhs.to_numpy(), 1.0 / diag.to_numpy()

        def m7(x):
            tmp.set_array_host(x)
            out = ce.Vector(ceed, N * 7)
            op_m7.apply(tmp, out)
            return out.to_numpy()

        x = np.zeros_like(b_h)
        r = b_h.copy()
        z = dinv * r
        p = z.copy()
        rz = rz0 = float(r @ z)
        for _ in range(1000):  # KSPCG, KSP_NORM_NATURAL, PCJACOBI diagonal (src/grid_anisotropy_tensor.c:84-95)
            if rz <= aniso_rtol * aniso_rtol * rz0:
                break
            Ap = m7(p)
            al = rz / float(p @ Ap)
            x += al * p
            r -= al * Ap
            z = dinv * r
            rz_new = float(r @ z)
            p = z + (rz_new / rz) * p
            rz = rz_new
        self.sgs_aniso = ce.Vector(ceed, N * 7)
        self.sgs_aniso.set_array_host(x)
        # -- inverse multiplicity (local)
        r_inv = ce.ElemRestriction(ceed, E, P ** 3, 1, None, E * P ** 3)
        mult = ce.Vector(ceed, N * 6)
        mult.set_value(0.0)
        r6.multiplicity(mult)
        qf = qfunction("inverse_multiplicity.h:InverseMultiplicity", [("multiplicity", 6, ce.CEED_EVAL_NONE)], [("inverse multiplicity", 1, ce.CEED_EVAL_NONE)])
        op_im = operator(qf, [("multiplicity", r6, none_b, a), ("inverse multiplicity", r_inv, none_b, a)], "InverseMultiplicity")
        self.sgs_inv_mult = ce.Vector(ceed, E * P ** 3)
        op_im.apply(mult, self.sgs_inv_mult)
        keep += [r_inv, mult]
        # -- nodal closure
        self.sgs_ctx_blob = sgs_dd_context(context_bytes(self.ctx), flat_params, bounds, alpha)
        self.sgs_qfctx = ce.QFunctionContext(ceed, self.sgs_ctx_blob)
        basis_x_to_q = ce.Basis.projection(self.basis_x, self.basis_q)
        keep.append(basis_x_to_q)
        self.sgs_q, self.sgs_grad_velo, self.sgs_km = ce.Vector(ceed, mesh.l_size), ce.Vector(ceed, N * 9), ce.Vector(ceed, N * 6)
        qf = qfunction(f"sgs_dd_model.h:ComputeSgsDDNodal_{sv_name}",
                       [("q", 5, ce.CEED_EVAL_NONE), ("x", 3, ce.CEED_EVAL_INTERP), ("gradient velocity", 9, ce.CEED_EVAL_NONE),
                        ("anisotropy tensor", 7, ce.CEED_EVAL_NONE), ("inverse multiplicity", 1, ce.CEED_EVAL_NONE)],
                       [("km_sgs", 6, ce.CEED_EVAL_NONE)], self.sgs_qfctx)
        self.op_sgs_nodal = operator(qf, [("q", self.rstr_q, none_b, self.sgs_q), ("x", self.rstr_x, basis_x_to_q, self.x_coord),
                                          ("gradient velocity", r9, none_b, a), ("anisotropy tensor", r7, none_b, self.sgs_aniso),
                                          ("inverse multiplicity", r_inv, none_b, self.sgs_inv_mult), ("km_sgs", r6, none_b, a)],
                                     "nodal data-driven SGS")
        # -- SGS residual term
        qf = qfunction(f"sgs_dd_model.h:IFunction_NodalSgs_{sv_name}",
                       [("q", 5, ce.CEED_EVAL_INTERP), ("qdata", 10, ce.CEED_EVAL_NONE), ("km_sgs", 6, ce.CEED_EVAL_INTERP)],
                       [("Grad_v", 15, ce.CEED_EVAL_GRAD)], self.qfctx)
        self.op_sgs_apply = operator(qf, [("q", self.rstr_q, self.basis_q, a), ("qdata", self.rstr_qd, none_b, self.q_data),
                                          ("km_sgs", r6, b6, self.sgs_km), ("Grad_v", self.rstr_q, self.basis_q, a)], "SGS residual")
        self._sgs_keep = keep

    def sgs_stress(self, q: ce.Vector) -> ce.Vector:
        """The nodal SGS stress (KM, [node][6]) of the state q: VelocityGradientProjectionApply, then the nodal closure."""
        self.op_sgs_velgrad.apply(q, self.sgs_grad_velo)
        self.sgs_grad_velo.pointwise_mult(self.sgs_grad_velo, self.sgs_rowsum_inv)
        q.copy_to(self.sgs_q)  # q_ceed is the closure's implicit input (problems/sgs_dd_model.c:105)
        self.op_sgs_nodal.apply(self.sgs_grad_velo, self.sgs_km)
        return self.sgs_km

    # ---- context updates (src/setupts.c:91-93, :141)
    def set_time(self, t):
        self.op_ifunction.set_context_double("solution time", [t])

    def set_timestep(self, dt):
        self.op_ifunction.set_context_double("timestep size", [dt])

    def set_ijacobian_shift(self, shift):
        self.op_ijacobian.set_context_double("ijacobian time shift", [shift])

    # ---- hot-path calls
    def ifunction(self, q: ce.Vector, q_dot: ce.Vector, g: ce.Vector):
        """G = F(q, q_dot): HONEE points its q_dot CeedVector at the PETSc array, then applies (src/setupts.c:102-109)."""
        q_dot.copy_to(self.q_dot) if q_dot is not self.q_dot else None
        self.op_ifunction.apply(q, g)
        if getattr(self, "op_sgs_apply", None) is not None:  # SgsDDApplyIFunction (src/setupts.c:118-120)
            self.sgs_stress(q)
            self.op_sgs_apply.apply(q, g, add=True)

    def ijacobian(self, dq: ce.Vector, out: ce.Vector, add=False):
        self.op_ijacobian.apply(dq, out, add=add)

    def diagonal(self, out: ce.Vector):
        self.op_ijacobian.assemble_diagonal(out)

    def host_inputs(self):
        """qdata as a numpy array (for checks against the oracle)."""
        return self.q_data.to_numpy()

    def context_bytes(self):
        return context_bytes(self.ctx)
