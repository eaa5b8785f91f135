"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (the C restatement in ``honee_oracle.c``) and, when present,
``oracle/_ref/libhonee_ref.so`` (the reference's own QFunction headers compiled unchanged by
``oracle/Makefile``).  Only ``tests/``, the smoke check in ``__graft_entry__.py`` and the CPU legs of
``bench.py`` import this module: it is the checker and the CPU baseline, never the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhonee_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
QF_TYPE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(_dp), C.POINTER(_dp))


def build(force: bool = False) -> None:
    """Compile the oracle (and the reference QFunctions when the reference sources exist)."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(path):
    return C.CDLL(path)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = _load(ORACLE_SO)
        _declare(_lib)
    return _lib


def ref():
    """The reference's QFunctions compiled unchanged, or None when they were not built here."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = _load(REF_SO)
    return _ref


def _declare(L):
    for name in ("oracle_qf_ifunction_conserv", "oracle_qf_ifunction_prim", "oracle_qf_ifunction_entropy",
                 "oracle_qf_ijacobian_conserv", "oracle_qf_ijacobian_prim", "oracle_qf_ijacobian_entropy",
                 "oracle_qf_setup", "oracle_qf_monitor_ke_conserv", "oracle_qf_ics_taylorgreen"):
        getattr(L, name).restype = C.c_int
    L.oracle_apply_ifunction.restype = C.c_int
    L.oracle_apply_rhs.restype = C.c_int
    L.oracle_apply_mass.restype = C.c_int
    L.oracle_qf_rhs_conserv.restype = C.c_int
    L.oracle_qf_mass.restype = C.c_int
    L.oracle_qf_mass_stab_conserv.restype = C.c_int
    L.oracle_apply_ijacobian.restype = C.c_int
    L.oracle_assemble_diagonal.restype = C.c_int
    L.oracle_assemble_point_block.restype = C.c_int
    L.oracle_box_num_nodes.restype = C.c_int64


def ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags.c_contiguous
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_ip)
    raise TypeError(a.dtype)


def _arr_of_ptrs(arrs):
    return (_dp * len(arrs))(*[ptr(a) if a is not None else None for a in arrs])


def call_qf(fn, ctx_bytes: bytes | np.ndarray | None, Q: int, ins, outs) -> int:
    """Call a libCEED-style QFunction ``fn`` (a ctypes function) on numpy arrays."""
    cbuf = None
    if ctx_bytes is not None:
        raw = bytes(ctx_bytes) if not isinstance(ctx_bytes, np.ndarray) else ctx_bytes.tobytes()
        cbuf = C.create_string_buffer(raw, len(raw))
    return fn(cbuf, C.c_int(Q), _arr_of_ptrs(ins), _arr_of_ptrs(outs))


# ----------------------------------------------------------------------------------------------------------------------
# operator-level helpers


class OracleMesh(C.Structure):
    _fields_ = [("num_elem", C.c_int), ("P", C.c_int), ("Q", C.c_int), ("offsets", _ip), ("interp1d", _dp), ("grad1d", _dp),
                ("qweight1d", _dp), ("num_threads", C.c_int), ("color_ptr", _ip), ("color_elem", _ip), ("num_colors", C.c_int)]


class Mesh:
    """Keeps numpy arrays alive for an OracleMesh."""

    def __init__(self, num_elem, P, Q, offsets, interp1d, grad1d, qweight1d, colors=None, num_threads=0):
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        self.interp1d = np.ascontiguousarray(interp1d, dtype=np.float64)
        self.grad1d = np.ascontiguousarray(grad1d, dtype=np.float64)
        self.qweight1d = np.ascontiguousarray(qweight1d, dtype=np.float64)
        self.c = OracleMesh(num_elem, P, Q, ptr(self.offsets), ptr(self.interp1d), ptr(self.grad1d), ptr(self.qweight1d),
                            num_threads, None, None, 0)
        if colors is not None:
            self.color_ptr = np.ascontiguousarray(colors[0], dtype=np.int32)
            self.color_elem = np.ascontiguousarray(colors[1], dtype=np.int32)
            self.c.color_ptr = ptr(self.color_ptr)
            self.c.color_elem = ptr(self.color_elem)
            self.c.num_colors = len(self.color_ptr) - 1


def qf(name: str, use_ref: bool = False):
    """A QFunction pointer from the oracle (default) or the reference build."""
    L = ref() if use_ref else lib()
    if L is None:
        raise RuntimeError("reference QFunctions not built")
    return C.cast(getattr(L, name), C.c_void_p)


def apply_ifunction(mesh: Mesh, ctx: bytes, q, q_dot, qdata, jac_data, num_jd=14, x_q=None, qf_name=None, use_ref=False):
    L = lib()
    fn = qf(qf_name or ("ref_IFunction_Newtonian_Conserv" if use_ref else "oracle_qf_ifunction_conserv"), use_ref)
    v = np.zeros_like(q)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    err = L.oracle_apply_ifunction(C.byref(mesh.c), fn, cbuf, ptr(q), ptr(q_dot), ptr(qdata), ptr(x_q), ptr(jac_data),
                                   C.c_int(num_jd), ptr(v), C.c_int64(v.size))
    if err:
        raise RuntimeError("oracle IFunction failed")
    return v


def apply_ijacobian(mesh: Mesh, ctx: bytes, dq, qdata, jac_data, num_jd=14, qf_name=None, use_ref=False):
    L = lib()
    fn = qf(qf_name or ("ref_IJacobian_Newtonian_Conserv" if use_ref else "oracle_qf_ijacobian_conserv"), use_ref)
    v = np.zeros_like(dq)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    err = L.oracle_apply_ijacobian(C.byref(mesh.c), fn, cbuf, ptr(dq), ptr(qdata), ptr(jac_data), C.c_int(num_jd), ptr(v),
                                   C.c_int64(v.size))
    if err:
        raise RuntimeError("oracle IJacobian failed")
    return v


def assemble_diagonal(mesh: Mesh, ctx: bytes, qdata, jac_data, l_size, num_jd=14, qf_name=None, use_ref=False):
    L = lib()
    fn = qf(qf_name or ("ref_IJacobian_Newtonian_Conserv" if use_ref else "oracle_qf_ijacobian_conserv"), use_ref)
    d = np.zeros(l_size)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    err = L.oracle_assemble_diagonal(C.byref(mesh.c), fn, cbuf, ptr(qdata), ptr(jac_data), C.c_int(num_jd), ptr(d), C.c_int64(l_size))
    if err:
        raise RuntimeError("oracle diagonal failed")
    return d


def apply_rhs(mesh: Mesh, ctx: bytes, q, qdata, x_q=None, use_ref=False):
    """RHSFunction_Newtonian as an operator (restatement, or the reference QFunction with use_ref)."""
    L = lib()
    fn = qf("ref_RHSFunction_Newtonian" if use_ref else "oracle_qf_rhs_conserv", use_ref)
    v = np.zeros_like(q)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    if L.oracle_apply_rhs(C.byref(mesh.c), fn, cbuf, ptr(q), ptr(qdata), ptr(x_q), ptr(v), C.c_int64(v.size)):
        raise RuntimeError("oracle RHS failed")
    return v


def apply_mass(mesh: Mesh, u, qdata, use_ref=False):
    """v = M u with the Mass_5 QFunction (restatement, or the reference's with use_ref)."""
    L = lib()
    fn = qf("ref_Mass_5" if use_ref else "oracle_qf_mass", use_ref)
    v = np.zeros_like(u)
    if L.oracle_apply_mass(C.byref(mesh.c), fn, ptr(u), ptr(qdata), ptr(v), C.c_int64(v.size)):
        raise RuntimeError("oracle mass failed")
    return v


def assemble_point_block(mesh: Mesh, ctx: bytes, qdata, jac_data, l_size, num_jd=14, qf_name=None, use_ref=False):
    """Row-major 5 x 5 blocks per node, [(node * 5 + i) * 5 + j], of the IJacobian operator."""
    L = lib()
    fn = qf(qf_name or ("ref_IJacobian_Newtonian_Conserv" if use_ref else "oracle_qf_ijacobian_conserv"), use_ref)
    out = np.zeros(5 * l_size)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    if L.oracle_assemble_point_block(C.byref(mesh.c), fn, cbuf, ptr(qdata), ptr(jac_data), C.c_int(num_jd), ptr(out), C.c_int64(l_size)):
        raise RuntimeError("oracle point-block assembly failed")
    return out


def apply_mass_stab(mesh: Mesh, ctx: bytes, q_dot, q, qdata, use_ref=False):
    """The SUPG-stabilized mass applied to q_dot at state q (MassFunction_Newtonian: the restatement, or the reference's)."""
    L = lib()
    fn = qf("ref_MassFunction_Newtonian_Conserv" if use_ref else "oracle_qf_mass_stab_conserv", use_ref)
    v = np.zeros_like(q_dot)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    L.oracle_apply_mass_stab.restype = C.c_int
    if L.oracle_apply_mass_stab(C.byref(mesh.c), fn, cbuf, ptr(np.ascontiguousarray(q_dot)), ptr(np.ascontiguousarray(q)), ptr(qdata), ptr(v),
                                C.c_int64(v.size)):
        raise RuntimeError("oracle stabilized mass failed")
    return v


def mass_stab_diagonal(mesh: Mesh, ctx: bytes, q, qdata, l_size, use_ref=False):
    """Diagonal of the stabilized mass at the state q."""
    L = lib()
    fn = qf("ref_MassFunction_Newtonian_Conserv" if use_ref else "oracle_qf_mass_stab_conserv", use_ref)
    d = np.zeros(l_size)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    L.oracle_assemble_mass_stab_diagonal.restype = C.c_int
    if L.oracle_assemble_mass_stab_diagonal(C.byref(mesh.c), fn, cbuf, ptr(np.ascontiguousarray(q)), ptr(qdata), ptr(d), C.c_int64(l_size)):
        raise RuntimeError("oracle stabilized-mass diagonal failed")
    return d


def setup_qdata(num_elem, Q, x_elem):
    qdata = np.zeros(num_elem * 10 * Q ** 3)
    lib().oracle_setup_qdata(C.c_int(num_elem), C.c_int(Q), ptr(np.ascontiguousarray(x_elem)), ptr(qdata))
    return qdata


def coords_at_qpts(num_elem, Q, x_elem):
    xq = np.zeros(num_elem * 3 * Q ** 3)
    lib().oracle_coords_at_qpts(C.c_int(num_elem), C.c_int(Q), ptr(np.ascontiguousarray(x_elem)), ptr(xq))
    return xq


def monitor_ke(mesh: Mesh, ctx: bytes, q, qdata):
    sums = np.zeros(5)
    cbuf = C.create_string_buffer(bytes(ctx), len(ctx))
    lib().oracle_monitor_ke(C.byref(mesh.c), cbuf, ptr(q), ptr(qdata), ptr(sums))
    return sums


def gauss_legendre(Q):
    x = np.zeros(Q)
    w = np.zeros(Q)
    lib().oracle_gauss_legendre(C.c_int(Q), ptr(x), ptr(w))
    return x, w


def gauss_lobatto(P):
    x = np.zeros(P)
    lib().oracle_gauss_lobatto(C.c_int(P), ptr(x))
    return x


def lagrange_tabulate(nodes, pts):
    P, Q = len(nodes), len(pts)
    B = np.zeros((Q, P))
    G = np.zeros((Q, P))
    lib().oracle_lagrange_tabulate(C.c_int(P), ptr(np.ascontiguousarray(nodes, dtype=np.float64)), C.c_int(Q),
                                   ptr(np.ascontiguousarray(pts, dtype=np.float64)), ptr(B), ptr(G))
    return B, G


def box_offsets(n, P, periodic=(0, 0, 0), ncomp=5):
    n_arr = (C.c_int * 3)(*n)
    p_arr = (C.c_int * 3)(*periodic)
    ne = n[0] * n[1] * n[2]
    off = np.zeros(ne * P ** 3, dtype=np.int32)
    lib().oracle_box_offsets(n_arr, C.c_int(P), p_arr, C.c_int(ncomp), ptr(off))
    nn = lib().oracle_box_num_nodes(n_arr, C.c_int(P), p_arr)
    return off, int(nn)


def box_elem_coords(n, xs, ys, zs):
    ne = n[0] * n[1] * n[2]
    x = np.zeros(ne * 24)
    lib().oracle_box_elem_coords((C.c_int * 3)(*n), ptr(np.ascontiguousarray(xs, dtype=np.float64)),
                                 ptr(np.ascontiguousarray(ys, dtype=np.float64)), ptr(np.ascontiguousarray(zs, dtype=np.float64)), ptr(x))
    return x
