"""The C-ABI library loads and exports every symbol the public headers declare; struct layouts match the reference.
CPU only: no call here touches a device."""
import ctypes as C
import importlib
import os
import re

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEADERS = [os.path.join(ROOT, "include", "honee_b200.h"), os.path.join(ROOT, "include", "ceed", "ceed.h")]


def _declared():
    funcs, data = [], []
    for h in HEADERS:
        src = "\n".join(l for l in open(h).read().splitlines() if not l.lstrip().startswith("#"))
        funcs += re.findall(r"(?:CEED_EXTERN|HB_EXPORT)\s+(?:const\s+)?\w+\s*\**\s*(\w+)\s*\(", src)
        data += re.findall(r"CEED_EXTERN\s+(?:const\s+)?\w+\s*\*?\s*(?:const\s+)?(CEED_\w+)\s*(?:\[\d+\])?;", src)
    return sorted(set(funcs)), sorted(set(data))


def _lib(hb):
    if not os.path.exists(hb.LIB_PATH):
        hb.build()
    return hb.lib()


def test_library_exports_every_declared_symbol(hb):
    L = _lib(hb)
    funcs, data = _declared()
    assert len(funcs) > 100 and len(data) >= 8
    missing = [f for f in funcs + data if not hasattr(L, f)]
    assert not missing, missing


def test_kernel_abi_entry_points_present(hb):
    L = _lib(hb)
    for name in ("hb_ifunction_apply", "hb_ijacobian_apply_f64", "hb_ijacobian_apply_f32", "hb_diagonal_assemble_f64",
                 "hb_diagonal_assemble_f32", "hb_setup_qdata", "hb_elemop_create", "hb_elemop_destroy"):
        assert hasattr(L, name)
    assert hb.version().startswith("honee-b200")


def test_context_layout_matches_reference(prob, oracle):
    assert C.sizeof(prob.NewtonianContext) == 184
    assert prob.NewtonianContext.time.offset == 64
    assert prob.NewtonianContext.ijacobian_time_shift.offset == 72
    assert prob.NewtonianContext.dt.offset == 168
    R = oracle.ref()
    if R is not None:
        assert R.ref_context_size() == 184 and R.ref_setup_context_size() == 304


def test_ceed_init_rejects_unknown_resource(hb):
    L = _lib(hb)
    c = C.c_void_p()
    assert L.CeedInit(b"/cpu/self", C.byref(c)) == -3  # CEED_ERROR_UNSUPPORTED: no CPU backend here
    msg = C.c_char_p()
    L.CeedGetErrorMessage(None, C.byref(msg))
    assert b"/gpu/b200" in msg.value


def test_elemop_rejects_out_of_range_offsets(hb, prob):
    """Host-side validation refuses offsets outside the L-vector before anything is uploaded."""
    L = _lib(hb)
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    mesh = prob.box_mesh((1, 1, 1), 2)
    basis = prob.tensor_basis(2, 2)
    bad = mesh.offsets.copy()
    bad[3] = mesh.l_size  # one past the end
    p = C.POINTER(kern.HbElemOp)()
    import numpy as np
    code = L.hb_elemop_create(1, 2, 2, bad.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int64(mesh.l_size), kern._dp(basis.interp1d),
                              kern._dp(basis.grad1d), kern._dp(basis.qref1d), kern._dp(basis.qweight1d), C.byref(p))
    assert code == -4 and not p  # HB_ERROR_INVALID, nothing allocated


def test_solver_options_defaults_and_validation_on_host():
    """Defaults mirror the PETSc settings HONEE's BDF runs use; invalid options are refused before any device work."""
    import ctypes as C
    S = importlib.import_module("honee-4aiad_b200.solver")
    K = importlib.import_module("honee-4aiad_b200.kernels")
    o = S.default_options()
    assert o.bdf_order == 2 and o.ksp_rtol == 1e-5 and o.gmres_restart == 30 and o.pc_jacobi == 1 and o.jacobian_fp32 == 0
    L = importlib.import_module("honee-4aiad_b200").lib()
    fake = K.HbElemOp()
    ctx = C.create_string_buffer(184)
    ts = C.c_void_p()
    for bad in (dict(gmres_restart=0), dict(gmres_restart=32), dict(bdf_order=3), dict(dt=0.0)):
        ob = S.default_options(**bad)
        assert L.hb_ts_create(C.byref(fake), ctx, C.c_void_p(16), C.byref(ob), None, C.byref(ts)) == -4, bad
        assert not ts.value
