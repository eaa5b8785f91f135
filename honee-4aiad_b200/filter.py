"""Differential filter on the GPU (ctypes over include/honee_b200.h): HONEE's src/differential_filter.c with the fused
operator of k_filter.cu and the CG + Jacobi solve of hb_filter.c.  Filters the resolved state into the 11 fields the
SGS training needs (P, u, T and the velocity products) and turns them into training pairs at the quadrature points."""
from __future__ import annotations

import ctypes as C

from . import lib as _load
from .kernels import _addr, _chk, _stream


class HbFilterOptions(C.Structure):
    _fields_ = [("grid_based_width", C.c_int), ("width_scaling", C.c_double * 3), ("kernel_scaling", C.c_double)]


class FilterError(RuntimeError):
    pass


class DifferentialFilter:
    """(M + K_alpha) u_bar = int phi f on the mesh of `elemop` (kernels.ElemOp), qdata its geometric factors."""

    def __init__(self, elemop, qdata, ctx_bytes: bytes, grid_based_width=True, width_scaling=(1.0, 1.0, 1.0), kernel_scaling=0.1, stream=None):
        import torch
        self.op, self.qdata, self.stream = elemop, qdata, stream
        self.ctx = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        self.opts = HbFilterOptions(int(grid_based_width), (C.c_double * 3)(*width_scaling), kernel_scaling)
        self.nodes = elemop.l_size // 5
        self.device = qdata.device
        self._work = {}
        self.torch = torch

    def _work_for(self, nc):
        if nc not in self._work:
            L = _load()
            L.hb_filter_work_doubles.restype = C.c_size_t
            n = L.hb_filter_work_doubles(self.op.ptr, C.c_int(nc))
            self._work[nc] = self.torch.empty(n, dtype=self.torch.float64, device=self.device)
        return self._work[nc]

    def apply(self, x, y, nc):
        _chk(_load().hb_filter_apply(self.op.ptr, C.c_int(nc), C.byref(self.opts), _addr(self.qdata), _addr(x), _addr(y), _stream(self.stream)),
             "hb_filter_apply")

    def diagonal(self, diag):
        _chk(_load().hb_filter_diagonal(self.op.ptr, C.byref(self.opts), _addr(self.qdata), _addr(diag), _stream(self.stream)), "hb_filter_diagonal")

    def rhs(self, q, out):
        _chk(_load().hb_filter_rhs(self.op.ptr, self.ctx, _addr(self.qdata), _addr(q), _addr(out), _stream(self.stream)), "hb_filter_rhs")

    def solve(self, b, x, nc, rtol=1e-10, max_it=500):
        its, rel = C.c_int(), C.c_double()
        code = _load().hb_filter_solve(self.op.ptr, C.c_int(nc), C.byref(self.opts), _addr(self.qdata), _addr(b), _addr(x), C.c_double(rtol),
                                       C.c_int(max_it), _addr(self._work_for(nc)), C.byref(its), C.byref(rel), _stream(self.stream))
        if code == 3:
            raise FilterError(f"filter CG did not reach rtol {rtol} in {max_it} iterations (relative norm {rel.value:.3e})")
        _chk(code, "hb_filter_solve")
        return its.value, rel.value

    def filter_state(self, q, rtol=1e-10, max_it=500):
        """Filtered (P, u, T, u_i u_j) [node][11] of the state q (in the context's state variable), with the CG statistics."""
        b = self.torch.empty(self.nodes * 11, dtype=self.torch.float64, device=self.device)
        x = self.torch.empty_like(b)
        self.rhs(q, b)
        its, rel = self.solve(b, x, 11, rtol, max_it)
        return x, its, rel

    def conservative(self, filtered, q):
        """State [node][5] of filtered fields in the context's state variable (to run the monitors on the filtered solution)."""
        _chk(_load().hb_filtered_state(_addr(filtered), C.c_int64(self.nodes), self.ctx, _addr(q), _stream(self.stream)), "hb_filtered_state")

    def training_pairs(self, filtered, width_scale, X, Y):
        _chk(_load().hb_sgs_training_pairs(self.op.ptr, self.ctx, _addr(self.qdata), _addr(filtered), C.c_double(width_scale), _addr(X), _addr(Y),
                                           _stream(self.stream)), "hb_sgs_training_pairs")
