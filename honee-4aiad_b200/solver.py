"""ctypes binding of the implicit time loop (hb_ts_* in include/honee_b200.h) and the device monitors.

The loop restates what HONEE asks of PETSc for the Newtonian problem (TSBDF, SNES Newton, KSP GMRES, PC Jacobi:
src/setupts.c:333-480) on device buffers: every residual is the fused IFunction, every Krylov product the fused IJacobian,
the preconditioner the fused diagonal.  `jacobian_fp32=True` selects the mixed-precision solve (FP32 Krylov basis,
Jacobian data and diagonal; FP64 residual, update and inner-product accumulation).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import lib as _load
from .kernels import _addr, _chk, _stream


class HbSolverOptions(C.Structure):
    _fields_ = [("dt", C.c_double), ("bdf_order", C.c_int), ("newton_rtol", C.c_double), ("newton_atol", C.c_double),
                ("newton_max_it", C.c_int), ("ksp_rtol", C.c_double), ("ksp_max_it", C.c_int), ("gmres_restart", C.c_int),
                ("pc_jacobi", C.c_int), ("pc_every_newton", C.c_int), ("jacobian_fp32", C.c_int), ("cgs_refine", C.c_int),
                ("sgs_lagged", C.c_int), ("jfnk", C.c_int)]


class HbStepStats(C.Structure):
    _fields_ = [("newton_its", C.c_int), ("ksp_its", C.c_int), ("converged_reason", C.c_int), ("res0", C.c_double),
                ("res_final", C.c_double), ("seconds", C.c_double)]


@dataclass
class StepStats:
    newton_its: int
    ksp_its: int
    converged_reason: int
    res0: float
    res_final: float
    seconds: float


def default_options(**kw) -> HbSolverOptions:
    o = HbSolverOptions()
    _load().hb_solver_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class TimeStepper:
    """BDF time stepper over one ElemOp (kernels.ElemOp); device state is a torch tensor or a raw device address."""

    def __init__(self, elemop, ctx_bytes: bytes, qdata, options: HbSolverOptions | None = None, stream=None, **kw):
        L = _load()
        self.options = options if options is not None else default_options(**kw)
        self._ctx = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        self._op = elemop  # keeps the element operator alive
        self._stream = _stream(stream)
        self.ptr = C.c_void_p()
        _chk(L.hb_ts_create(elemop.ptr, self._ctx, _addr(qdata), C.byref(self.options), self._stream, C.byref(self.ptr)), "hb_ts_create")

    def set_state(self, q, t=0.0):
        _chk(_load().hb_ts_set_state(self.ptr, _addr(q), C.c_double(t)), "hb_ts_set_state")

    def get_state(self, q) -> float:
        t = C.c_double()
        _chk(_load().hb_ts_get_state(self.ptr, _addr(q), C.byref(t)), "hb_ts_get_state")
        return t.value

    def step(self) -> StepStats:
        s = HbStepStats()
        _chk(_load().hb_ts_step(self.ptr, C.byref(s)), "hb_ts_step")
        return StepStats(s.newton_its, s.ksp_its, s.converged_reason, s.res0, s.res_final, s.seconds)

    def set_freestream(self, faceop=None, ctx264: bytes = b"", flux_type=1):
        """Add the free-stream boundary (kernels.FaceOp, FreestreamContext bytes, 0 HLL / 1 HLLC), or remove it."""
        if faceop is None:
            _chk(_load().hb_ts_set_freestream(self.ptr, None, None, 0, None), "hb_ts_set_freestream")
            return
        self._bc = (faceop, C.create_string_buffer(bytes(ctx264), len(ctx264)))
        _chk(_load().hb_ts_set_freestream(self.ptr, faceop.ptr, self._bc[1], C.c_int(flux_type), _addr(faceop.qdata)), "hb_ts_set_freestream")

    def set_essential(self, idx=None, values=None):
        """Strong Dirichlet DOFs (L-vector indices node * 5 + component, values default 0), or none (no arguments)."""
        L = _load()
        if idx is None or len(idx) == 0:
            _chk(L.hb_ts_set_essential(self.ptr, None, None, C.c_int64(0)), "hb_ts_set_essential")
            return
        i = np.ascontiguousarray(idx, dtype=np.int32)
        v = None if values is None else np.ascontiguousarray(values, dtype=np.float64)
        _chk(L.hb_ts_set_essential(self.ptr, i.ctypes.data_as(C.POINTER(C.c_int32)), None if v is None else v.ctypes.data_as(C.POINTER(C.c_double)),
                                   C.c_int64(i.size)), "hb_ts_set_essential")

    def set_sgs(self, desc=None, weights=None):
        """Fuse the learned closure (sgs.HbMlpDesc, float32 weights) into the residual, or remove it (no arguments)."""
        if desc is None:
            _chk(_load().hb_ts_set_sgs(self.ptr, None, None), "hb_ts_set_sgs")
            return
        self._sgs_w = np.ascontiguousarray(weights, dtype=np.float32)
        self._sgs_desc = desc
        _chk(_load().hb_ts_set_sgs(self.ptr, C.byref(desc), self._sgs_w.ctypes.data_as(C.POINTER(C.c_float))), "hb_ts_set_sgs")

    def context_bytes(self) -> bytes:
        L = _load()
        L.hb_ts_context.restype = C.c_void_p
        return C.string_at(L.hb_ts_context(self.ptr), len(self._ctx))

    def __del__(self):
        try:
            if self.ptr:
                _load().hb_ts_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


# ---- explicit time loop (hb_explicit_*): HONEE's -ts_type rk path, RHS_NS with the mass KSP (src/setupts.c:31-75)
RK_MAX_STAGES = 6

# PETSc TSRK tableaux by -ts_rk_type name: (A, b, c), published Butcher tables
RK_TABLEAUX = {
    "1fe": ([[0.0]], [1.0], [0.0]),
    "2a": ([[0, 0], [1.0, 0]], [0.5, 0.5], [0, 1.0]),
    "3": ([[0, 0, 0], [0.5, 0, 0], [-1.0, 2.0, 0]], [1 / 6, 2 / 3, 1 / 6], [0, 0.5, 1.0]),
    "3bs": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.75, 0, 0], [2 / 9, 1 / 3, 4 / 9, 0]], [2 / 9, 1 / 3, 4 / 9, 0], [0, 0.5, 0.75, 1.0]),
    "4": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.5, 0, 0], [0, 0, 1.0, 0]], [1 / 6, 1 / 3, 1 / 3, 1 / 6], [0, 0.5, 0.5, 1.0]),
    # Fehlberg's six-stage pair, advanced with its fifth-order weights (TSRK5F, HONEE's explicit default, src/setupts.c:355)
    "5f": ([[0, 0, 0, 0, 0, 0], [1 / 4, 0, 0, 0, 0, 0], [3 / 32, 9 / 32, 0, 0, 0, 0], [1932 / 2197, -7200 / 2197, 7296 / 2197, 0, 0, 0],
            [439 / 216, -8, 3680 / 513, -845 / 4104, 0, 0], [-8 / 27, 2, -3544 / 2565, 1859 / 4104, -11 / 40, 0]],
           [16 / 135, 0, 6656 / 12825, 28561 / 56430, -9 / 50, 2 / 55], [0, 1 / 4, 3 / 8, 12 / 13, 1, 1 / 2]),
}


class HbExplicitOptions(C.Structure):
    _fields_ = [("dt", C.c_double), ("rk_stages", C.c_int), ("rk_a", C.c_double * (RK_MAX_STAGES * RK_MAX_STAGES)),
                ("rk_b", C.c_double * RK_MAX_STAGES), ("rk_c", C.c_double * RK_MAX_STAGES), ("mass_ksp", C.c_int),
                ("mass_pc_rowsum", C.c_int), ("mass_rtol", C.c_double), ("mass_atol", C.c_double), ("mass_max_it", C.c_int),
                ("mass_restart", C.c_int), ("mass_type", C.c_int)]


class HbExplicitStats(C.Structure):
    _fields_ = [("mass_its", C.c_int), ("converged_reason", C.c_int), ("seconds", C.c_double)]


def explicit_options(*, dt, rk_type="4", mass_ksp="preonly", pc_jacobi="rowsum", rtol=1e-5, atol=1e-50, max_it=10000,
                     restart=30, mass="auto") -> HbExplicitOptions:
    """Options in HONEE's vocabulary: -ts_rk_type, -mass_ksp_type preonly|gmres, -mass_pc_jacobi_type rowsum|diagonal."""
    o = HbExplicitOptions()
    _load().hb_explicit_default_options(C.byref(o))
    A, b, c = RK_TABLEAUX[rk_type]
    o.dt = dt
    o.rk_stages = len(b)
    for i in range(RK_MAX_STAGES * RK_MAX_STAGES):
        o.rk_a[i] = 0.0
    for i, row in enumerate(A):
        for j, a in enumerate(row):
            o.rk_a[i * RK_MAX_STAGES + j] = a
    for i in range(RK_MAX_STAGES):
        o.rk_b[i] = b[i] if i < len(b) else 0.0
        o.rk_c[i] = c[i] if i < len(c) else 0.0
    o.mass_ksp = {"preonly": 0, "gmres": 1}[mass_ksp]
    o.mass_pc_rowsum = {"rowsum": 1, "diagonal": 0}[pc_jacobi]
    o.mass_rtol, o.mass_atol, o.mass_max_it, o.mass_restart = rtol, atol, max_it, restart
    o.mass_type = {"auto": 0, "plain": 1}[mass]  # auto: the SUPG-stabilized mass when stab = supg, as HONEE chooses
    return o


@dataclass
class ExplicitStats:
    mass_its: int
    converged_reason: int
    seconds: float


class ExplicitStepper:
    """Explicit RK time stepper over one ElemOp: q_{n+1} from the tableau with G = M^-1 RHS(q) (RHS_NS)."""

    def __init__(self, elemop, ctx_bytes: bytes, qdata, options: HbExplicitOptions | None = None, stream=None, **kw):
        L = _load()
        self.options = options if options is not None else explicit_options(**kw)
        self._ctx = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        self._op = elemop
        self._stream = _stream(stream)
        self.ptr = C.c_void_p()
        _chk(L.hb_explicit_create(elemop.ptr, self._ctx, _addr(qdata), C.byref(self.options), self._stream, C.byref(self.ptr)),
             "hb_explicit_create")

    def set_state(self, q, t=0.0):
        _chk(_load().hb_explicit_set_state(self.ptr, _addr(q), C.c_double(t)), "hb_explicit_set_state")

    def get_state(self, q) -> float:
        t = C.c_double()
        _chk(_load().hb_explicit_get_state(self.ptr, _addr(q), C.byref(t)), "hb_explicit_get_state")
        return t.value

    def rhs(self, q, g, t=0.0) -> tuple[int, int]:
        """g = M^-1 RHS(q) at time t; returns (mass-solve iterations, converged reason)."""
        its, reason = C.c_int(), C.c_int()
        _chk(_load().hb_explicit_rhs(self.ptr, _addr(q), C.c_double(t), _addr(g), C.byref(its), C.byref(reason)), "hb_explicit_rhs")
        return its.value, reason.value

    def set_essential(self, idx=None, values=None):
        """Strong Dirichlet DOFs (L-vector indices node * 5 + component, values default 0), or none."""
        L = _load()
        if idx is None or len(idx) == 0:
            _chk(L.hb_explicit_set_essential(self.ptr, None, None, C.c_int64(0)), "hb_explicit_set_essential")
            return
        i = np.ascontiguousarray(idx, dtype=np.int32)
        v = None if values is None else np.ascontiguousarray(values, dtype=np.float64)
        _chk(L.hb_explicit_set_essential(self.ptr, i.ctypes.data_as(C.POINTER(C.c_int32)), None if v is None else v.ctypes.data_as(C.POINTER(C.c_double)),
                                         C.c_int64(i.size)), "hb_explicit_set_essential")

    def set_freestream(self, faceop=None, ctx264: bytes = b"", flux_type=1):
        if faceop is None:
            _chk(_load().hb_explicit_set_freestream(self.ptr, None, None, 0, None), "hb_explicit_set_freestream")
            return
        self._bc = (faceop, C.create_string_buffer(bytes(ctx264), len(ctx264)))
        _chk(_load().hb_explicit_set_freestream(self.ptr, faceop.ptr, self._bc[1], C.c_int(flux_type), _addr(faceop.qdata)),
             "hb_explicit_set_freestream")

    def step(self) -> ExplicitStats:
        s = HbExplicitStats()
        _chk(_load().hb_explicit_step(self.ptr, C.byref(s)), "hb_explicit_step")
        return ExplicitStats(s.mass_its, s.converged_reason, s.seconds)

    def __del__(self):
        try:
            if self.ptr:
                _load().hb_explicit_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


def monitor_ke(elemop, ctx_bytes: bytes, q, qdata, scratch, stream=None) -> np.ndarray:
    """Kinetic-energy integrand sums (TotalKineticEnergy, StrainDissipation, DivergenceDissipation, VolumeExpansion,
    MuVorticity2), not yet divided by the domain volume.  scratch: >= 5 * num_elem doubles on the device."""
    sums = np.zeros(5)
    cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
    _chk(_load().hb_monitor_ke(elemop.ptr, cb, _addr(q), _addr(qdata), _addr(scratch), sums.ctypes.data_as(C.POINTER(C.c_double)),
                               _stream(stream)), "hb_monitor_ke")
    return sums


def monitor_cfl(elemop, ctx_bytes: bytes, q, qdata, dt, scratch, stream=None) -> tuple[float, float]:
    """(min, max) over quadrature points of dt * sqrt(u . g u), g = 0.25 dXdx^T dXdx.  scratch: >= 2 * num_elem doubles."""
    mm = np.zeros(2)
    cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
    _chk(_load().hb_monitor_cfl(elemop.ptr, cb, _addr(q), _addr(qdata), C.c_double(dt), _addr(scratch),
                                mm.ctypes.data_as(C.POINTER(C.c_double)), _stream(stream)), "hb_monitor_cfl")
    return float(mm[0]), float(mm[1])
