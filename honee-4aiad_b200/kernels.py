"""ctypes binding of the kernel-level C ABI (include/honee_b200.h) on device pointers.

Used by callers that manage device memory themselves -- the Newton-Krylov driver, the benchmark and the parity tests --
with torch tensors serving only as device buffers and streams.  Every call is asynchronous on the stream it is given.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as _load

HB_MAX_P = 8


class HbElemOp(C.Structure):
    _fields_ = [("num_elem", C.c_int), ("P", C.c_int), ("Q", C.c_int), ("l_size", C.c_int64), ("d_offsets", C.c_void_p),
                ("num_colors", C.c_int), ("h_color_ptr", C.POINTER(C.c_int32)), ("d_color_elem", C.c_void_p),
                ("interp1d", C.c_double * 64), ("grad1d", C.c_double * 64), ("colo_grad1d", C.c_double * 64),
                ("qref1d", C.c_double * 8), ("qweight1d", C.c_double * 8), ("d_x_elem", C.c_void_p), ("num_sms", C.c_int),
                ("device", C.c_int), ("d_status", C.c_void_p)]


class HbIFunctionIO(C.Structure):
    _fields_ = [("q", C.c_void_p), ("q_dot", C.c_void_p), ("qdata", C.c_void_p), ("jac_data", C.c_void_p), ("jac_data_f32", C.c_void_p),
                ("v", C.c_void_p), ("add", C.c_int)]


def _dp(a: np.ndarray):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _addr(t):
    if t is None:
        return None
    return C.c_void_p(t.data_ptr() if hasattr(t, "data_ptr") else int(t))


def _stream(s):
    if s is None:
        return None
    return C.c_void_p(s.cuda_stream if hasattr(s, "cuda_stream") else int(s))


class HbError(RuntimeError):
    pass


def _chk(code, what):
    if code != 0:
        raise HbError(f"{what} failed with status {code}")


class ElemOp:
    """Device description of the hex element operator (restriction + colouring + tensor basis)."""

    def __init__(self, mesh, basis):
        L = _load()
        self.ptr = C.POINTER(HbElemOp)()
        off = np.ascontiguousarray(mesh.offsets, dtype=np.int32)
        _chk(L.hb_elemop_create(mesh.num_elem, basis.P, basis.Q, off.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int64(mesh.l_size),
                                _dp(basis.interp1d), _dp(basis.grad1d), _dp(basis.qref1d), _dp(basis.qweight1d), C.byref(self.ptr)),
             "hb_elemop_create")
        self.num_elem, self.P, self.Q, self.l_size = mesh.num_elem, basis.P, basis.Q, mesh.l_size
        self.qref1d = np.ascontiguousarray(basis.qref1d)
        self.qweight1d = np.ascontiguousarray(basis.qweight1d)

    @property
    def num_colors(self):
        return self.ptr.contents.num_colors

    def color_sizes(self):
        c = self.ptr.contents
        return [c.h_color_ptr[i + 1] - c.h_color_ptr[i] for i in range(c.num_colors)]

    def set_vertex_coords(self, x_elem):
        _chk(_load().hb_elemop_set_vertex_coords(self.ptr, _dp(x_elem)), "hb_elemop_set_vertex_coords")

    def __del__(self):
        try:
            if self.ptr:
                _load().hb_elemop_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    # ---- operators
    def setup_qdata(self, x_elem_dev, qdata_dev, stream=None):
        _chk(_load().hb_setup_qdata(self.num_elem, self.Q, _dp(self.qref1d), _dp(self.qweight1d), _addr(x_elem_dev), _addr(qdata_dev),
                                    _stream(stream)), "hb_setup_qdata")

    def ifunction(self, ctx_bytes: bytes, q, q_dot, qdata, v, jac_data=None, jac_data_f32=None, add=False, stream=None):
        io = HbIFunctionIO(_addr(q), _addr(q_dot), _addr(qdata), _addr(jac_data), _addr(jac_data_f32), _addr(v), int(add))
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        _chk(_load().hb_ifunction_apply(self.ptr, cb, C.byref(io), _stream(stream)), "hb_ifunction_apply")

    def ifunction_sgs(self, ctx_bytes: bytes, q, q_dot, qdata, v, desc, weights, jac_data=None, jac_data_f32=None, add=False, stream=None):
        """IFunction with the learned closure fused in (desc: sgs.HbMlpDesc, weights: float32 host array)."""
        io = HbIFunctionIO(_addr(q), _addr(q_dot), _addr(qdata), _addr(jac_data), _addr(jac_data_f32), _addr(v), int(add))
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        w = np.ascontiguousarray(weights, dtype=np.float32)
        _chk(_load().hb_ifunction_apply_sgs(self.ptr, cb, C.byref(io), C.byref(desc), w.ctypes.data_as(C.POINTER(C.c_float)), _stream(stream)),
             "hb_ifunction_apply_sgs")

    def ijacobian(self, ctx_bytes: bytes, qdata, jac_data, dq, v, add=False, fp32=False, stream=None):
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        fn = _load().hb_ijacobian_apply_f32 if fp32 else _load().hb_ijacobian_apply_f64
        _chk(fn(self.ptr, cb, _addr(qdata), _addr(jac_data), _addr(dq), _addr(v), int(add), _stream(stream)), "hb_ijacobian_apply")

    def diagonal(self, ctx_bytes: bytes, qdata, jac_data, diag, add=False, fp32=False, stream=None):
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        fn = _load().hb_diagonal_assemble_f32 if fp32 else _load().hb_diagonal_assemble_f64
        _chk(fn(self.ptr, cb, _addr(qdata), _addr(jac_data), _addr(diag), int(add), _stream(stream)), "hb_diagonal_assemble")

    def point_block_diagonal(self, ctx_bytes: bytes, qdata, jac_data, out, add=False, fp32=False, stream=None):
        """out[(node * 5 + i) * 5 + j] (+)= the node's 5 x 5 block of the IJacobian (5 * l_size values)."""
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        fn = _load().hb_point_block_diagonal_f32 if fp32 else _load().hb_point_block_diagonal_f64
        _chk(fn(self.ptr, cb, _addr(qdata), _addr(jac_data), _addr(out), int(add), _stream(stream)), "hb_point_block_diagonal")

    def mass(self, qdata, u, v, add=False, stream=None):
        """v (+)= M u, the Mass_5 operator of the explicit path."""
        _chk(_load().hb_mass_apply(self.ptr, _addr(qdata), _addr(u), _addr(v), int(add), _stream(stream)), "hb_mass_apply")

    def mass_diagonal(self, qdata, diag, add=False, stream=None):
        _chk(_load().hb_mass_diagonal(self.ptr, _addr(qdata), _addr(diag), int(add), _stream(stream)), "hb_mass_diagonal")

    def mass_stab(self, ctx_bytes: bytes, qdata, q_state, u, v, add=False, stream=None):
        """v (+)= M_stab(q_state) u, the SUPG-stabilized mass of explicit SUPG runs (MassFunction_Newtonian)."""
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        _chk(_load().hb_mass_stab_apply(self.ptr, cb, _addr(qdata), _addr(q_state), _addr(u), _addr(v), int(add), _stream(stream)),
             "hb_mass_stab_apply")

    def mass_stab_diagonal(self, ctx_bytes: bytes, qdata, q_state, diag, add=False, stream=None):
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        _chk(_load().hb_mass_stab_diagonal(self.ptr, cb, _addr(qdata), _addr(q_state), _addr(diag), int(add), _stream(stream)),
             "hb_mass_stab_diagonal")

    def mass_point_block_diagonal(self, qdata, out, add=False, stream=None):
        _chk(_load().hb_mass_point_block_diagonal(self.ptr, _addr(qdata), _addr(out), int(add), _stream(stream)), "hb_mass_point_block_diagonal")


class HbFaceOp(C.Structure):
    _fields_ = [("num_faces", C.c_int), ("P", C.c_int), ("Q", C.c_int), ("l_size", C.c_int64), ("d_offsets", C.c_void_p), ("num_colors", C.c_int),
                ("h_color_ptr", C.POINTER(C.c_int32)), ("d_color_elem", C.c_void_p), ("interp1d", C.c_double * 64), ("grad1d", C.c_double * 64),
                ("qweight1d", C.c_double * 8), ("device", C.c_int)]


class FaceOp:
    """Boundary faces of a volume mesh (problem.box_faces) with the free-stream boundary condition."""

    HLL, HLLC = 0, 1

    def __init__(self, offsets, l_size, basis, x_nodes):
        import torch
        L = _load()
        self.ptr = C.POINTER(HbFaceOp)()
        off = np.ascontiguousarray(offsets, dtype=np.int32)
        self.num_faces, self.P2 = off.shape
        _chk(L.hb_faceop_create(self.num_faces, basis.P, basis.Q, off.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int64(l_size), _dp(basis.interp1d),
                                _dp(basis.grad1d), _dp(basis.qweight1d), C.byref(self.ptr)), "hb_faceop_create")
        self.Q = basis.Q
        dev = torch.device("cuda:0")
        xn = torch.from_numpy(np.ascontiguousarray(x_nodes, dtype=np.float64)).to(dev)
        self.qdata = torch.empty(self.num_faces * 10 * self.Q ** 2, dtype=torch.float64, device=dev)
        _chk(L.hb_face_setup_qdata(self.ptr, _addr(xn), _addr(self.qdata), None), "hb_face_setup_qdata")
        self.jac = torch.empty(self.num_faces * 5 * self.Q ** 2, dtype=torch.float64, device=dev)

    def __del__(self):
        try:
            if self.ptr:
                _load().hb_faceop_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def freestream(self, ctx264: bytes, q, v, flux_type=1, stream=None):
        cb = C.create_string_buffer(bytes(ctx264), len(ctx264))
        _chk(_load().hb_freestream_apply(self.ptr, cb, C.c_int(flux_type), _addr(self.qdata), _addr(q), _addr(self.jac), _addr(v), _stream(stream)),
             "hb_freestream_apply")

    def freestream_point_block(self, ctx264: bytes, out, flux_type=1, stream=None):
        """out[(node * 5 + i) * 5 + j] += the face Jacobian's 5 x 5 node blocks (after freestream() stored the face state)."""
        cb = C.create_string_buffer(bytes(ctx264), len(ctx264))
        _chk(_load().hb_freestream_point_block_diagonal(self.ptr, cb, C.c_int(flux_type), _addr(self.qdata), _addr(self.jac), _addr(out),
                                                        _stream(stream)), "hb_freestream_point_block_diagonal")

    def freestream_jacobian(self, ctx264: bytes, dq, v, flux_type=1, stream=None):
        cb = C.create_string_buffer(bytes(ctx264), len(ctx264))
        _chk(_load().hb_freestream_jacobian_apply(self.ptr, cb, C.c_int(flux_type), _addr(self.qdata), _addr(self.jac), _addr(dq), _addr(v),
                                                  _stream(stream)), "hb_freestream_jacobian_apply")


def contraction_probe(variant, D, u, reps, ctas_per_sm=0, launches=5):
    """Run the library's contraction A/B probe (hb_contraction_probe) on u, a CUDA float64 tensor [E][5][125]: returns
    (best CUDA-event milliseconds of `launches` timed launches after one warm-up, FMA count per launch, output tensor).
    variant 0 = shared-memory fibre passes, 1 = warp shuffles."""
    import torch
    assert u.is_cuda and u.dtype == torch.float64 and u.is_contiguous() and u.numel() % 625 == 0
    E = u.numel() // 625
    out = torch.empty_like(u)
    Dh = np.ascontiguousarray(np.asarray(D, dtype=np.float64).reshape(5, 5))
    s = torch.cuda.current_stream(u.device)
    cnt = C.c_int64()
    fn = _load().hb_contraction_probe
    args = lambda: (int(variant), Dh.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),  # noqa: E731
                    int(E), int(reps), int(ctas_per_sm), C.byref(cnt), _stream(s))
    _chk(fn(*args()), "hb_contraction_probe")
    best = None
    for _ in range(launches):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        _chk(fn(*args()), "hb_contraction_probe")
        b.record(s)
        b.synchronize()
        t = a.elapsed_time(b)
        best = t if best is None else min(best, t)
    return best, cnt.value, out


def fma_peak(fp64=True, iters=4096, reps=5, device=None):
    """Measured FMA throughput of the FP64 (or FP32) pipe in FMA/s: the best of `reps` launches of the library's probe
    (independent FMA chains over 8 CTAs per SM), timed with CUDA events on torch's current stream after one warm-up."""
    import torch
    dev = device or torch.device("cuda", torch.cuda.current_device())
    n = 2048 * torch.cuda.get_device_properties(dev).multi_processor_count
    sink = torch.empty(n, dtype=torch.float64 if fp64 else torch.float32, device=dev)
    s = torch.cuda.current_stream(dev)
    cnt = C.c_int64()
    fn = _load().hb_fma_peak_probe
    _chk(fn(int(fp64), iters, _addr(sink), C.c_int64(n), C.byref(cnt), _stream(s)), "hb_fma_peak_probe")
    best = None
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        _chk(fn(int(fp64), iters, _addr(sink), C.c_int64(n), C.byref(cnt), _stream(s)), "hb_fma_peak_probe")
        b.record(s)
        b.synchronize()
        t = a.elapsed_time(b) * 1e-3
        best = t if best is None else min(best, t)
    return cnt.value / best
