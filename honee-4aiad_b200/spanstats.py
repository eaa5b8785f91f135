"""Spanwise turbulence statistics on the GPU (hb_spanstats_* of include/honee_b200.h): HONEE's
-ts_monitor_spanstats_turbulence (src/spanstats/turbulence.c:152-278, src/spanstats/spanstats.c).

The spanwise direction is z.  For a box mesh the parent plane is the z- face (spanstats.c:55-95 filters the periodic
face, or face set 1 = z- without periodicity), a 2D mesh of nx * ny elements whose nodes are those of the box's
(x, y) node grid; the elements of column ex + nx * ey are (ex, ey, ez) for ez = 0 .. nz - 1, and their quadrature points
share the (x, y) of the parent element's points (the star forest of spanstats.c:253-289).

Collection follows the reference's monitor (turbulence.c:223-278): nothing is collected on the initial condition; each
later step adds its statistics weighted by the time since the previous collection; processing averages over the time
since the start of collection (spanstats.c:445-448) and the span width.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import lib as _load
from .kernels import HB_MAX_P, _addr, _chk, _stream

NUM_COMPONENTS = 22
# component names in the reference's order (turbulence.c:172-193)
COMPONENTS = ("MeanDensity", "MeanPressure", "MeanPressureSquared", "MeanPressureVelocityX", "MeanPressureVelocityY",
              "MeanPressureVelocityZ", "MeanDensityTemperature", "MeanDensityTemperatureFluxX", "MeanDensityTemperatureFluxY",
              "MeanDensityTemperatureFluxZ", "MeanMomentumX", "MeanMomentumY", "MeanMomentumZ", "MeanMomentumFluxXX",
              "MeanMomentumFluxYY", "MeanMomentumFluxZZ", "MeanMomentumFluxYZ", "MeanMomentumFluxXZ", "MeanMomentumFluxXY",
              "MeanVelocityX", "MeanVelocityY", "MeanVelocityZ")


class HbPlaneOp(C.Structure):
    _fields_ = [("num_elem", C.c_int), ("P", C.c_int), ("Q", C.c_int), ("num_nodes", C.c_int64), ("d_offsets", C.c_void_p),
                ("num_colors", C.c_int), ("h_color_ptr", C.POINTER(C.c_int32)), ("d_color_elem", C.c_void_p),
                ("interp1d", C.c_double * (HB_MAX_P * HB_MAX_P)), ("qref1d", C.c_double * HB_MAX_P), ("qweight1d", C.c_double * HB_MAX_P),
                ("d_wdetJ", C.c_void_p)]


@dataclass
class SpanLayout:
    column_elems: np.ndarray    # int32 [num_columns][nz]
    parent_offsets: np.ndarray  # int32 [num_columns][P^2] parent node index
    num_parent_nodes: int
    parent_x: np.ndarray        # [num_columns][3][4] vertex coordinates (vertex a + 2b)
    span_width: float
    parent_dims: tuple          # (Nx, Ny) parent node grid, node i + Nx * j


def box_span_layout(mesh) -> SpanLayout:
    """Columns, parent plane and span width of a problem.BoxMesh (elements numbered ex + nx (ey + ny ez))."""
    nx, ny, nz = mesh.n
    P = mesh.P
    Nx, Ny = mesh.node_dims[0], mesh.node_dims[1]
    ex, ey = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")  # column index ex + nx * ey, ex fastest
    ex, ey = ex.reshape(-1), ey.reshape(-1)
    cols = (ex + nx * ey).astype(np.int64)
    column_elems = (cols[:, None] + nx * ny * np.arange(nz)[None, :]).astype(np.int32)
    a = np.arange(P)
    A, Bb = np.meshgrid(a, a, indexing="xy")  # local node a + P b, a fastest
    A, Bb = A.reshape(-1), Bb.reshape(-1)
    i = (ex[:, None] * (P - 1) + A[None, :]) % Nx
    j = (ey[:, None] * (P - 1) + Bb[None, :]) % Ny
    parent_offsets = (i + Nx * j).astype(np.int32)
    px = np.zeros((nx * ny, 3, 4))
    for v in range(4):
        va, vb = v & 1, v >> 1
        px[:, 0, v] = mesh.xs[ex + va]
        px[:, 1, v] = mesh.ys[ey + vb]
        px[:, 2, v] = mesh.zs[0]
    return SpanLayout(column_elems, parent_offsets, Nx * Ny, px, float(mesh.zs[-1] - mesh.zs[0]), (Nx, Ny))


class SpanStats:
    """The statistics monitor on device buffers: collect(q, t) after every step, process(t) for the averaged fields
    [parent node][22] (a torch tensor on cuda:0)."""

    def __init__(self, op, layout: SpanLayout, initial_time=0.0):
        import torch
        L = _load()
        self.ptr = C.c_void_p()
        self.layout = layout
        ce = np.ascontiguousarray(layout.column_elems, dtype=np.int32)
        po = np.ascontiguousarray(layout.parent_offsets, dtype=np.int32)
        px = np.ascontiguousarray(layout.parent_x, dtype=np.float64)
        _chk(L.hb_spanstats_create(op.ptr, C.c_int(ce.shape[0]), C.c_int(ce.shape[1]), ce.ctypes.data_as(C.POINTER(C.c_int32)),
                                   po.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int64(layout.num_parent_nodes),
                                   px.ctypes.data_as(C.POINTER(C.c_double)), C.c_double(layout.span_width), C.byref(self.ptr)),
             "hb_spanstats_create")
        self.num_nodes = layout.num_parent_nodes
        self.Q = op.Q
        self.num_columns = ce.shape[0]
        self.stats = torch.zeros(self.num_nodes * NUM_COMPONENTS, dtype=torch.float64, device="cuda:0")
        self.reset(initial_time)

    def __del__(self):
        try:
            if self.ptr:
                _load().hb_spanstats_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def reset(self, initial_time=0.0, stream=None):
        self.initial_time = float(initial_time)
        _chk(_load().hb_spanstats_reset(self.ptr, C.c_double(initial_time), _stream(stream)), "hb_spanstats_reset")

    def collect(self, ctx_bytes: bytes, q, qdata, solution_time, stream=None):
        cb = C.create_string_buffer(bytes(ctx_bytes), len(ctx_bytes))
        _chk(_load().hb_spanstats_collect(self.ptr, cb, _addr(q), _addr(qdata), C.c_double(solution_time), _stream(stream)),
             "hb_spanstats_collect")

    def sums(self):
        """Host copy of the parent-point sums [num_columns][Q^2][22]."""
        out = np.empty(self.num_columns * self.Q ** 2 * NUM_COMPONENTS)
        _chk(_load().hb_spanstats_copy_sums(self.ptr, out.ctypes.data_as(C.POINTER(C.c_double))), "hb_spanstats_copy_sums")
        return out.reshape(self.num_columns, self.Q ** 2, NUM_COMPONENTS)

    def plane(self):
        """The parent plane's HbPlaneOp (for the plane operators of the kernel ABI)."""
        pl = C.POINTER(HbPlaneOp)()
        _chk(_load().hb_spanstats_view(self.ptr, None, C.byref(pl)), "hb_spanstats_view")
        return pl

    def process(self, solution_time, rtol=1e-10, max_it=10000, stream=None):
        """Averaged statistics [parent node][22] on the device, plus (iterations, final relative natural residual)."""
        its, rel = C.c_int(0), C.c_double(0)
        _chk(_load().hb_spanstats_process(self.ptr, C.c_double(solution_time), C.c_double(rtol), C.c_int(max_it), _addr(self.stats),
                                          C.byref(its), C.byref(rel), _stream(stream)), "hb_spanstats_process")
        return self.stats.view(self.num_nodes, NUM_COMPONENTS), its.value, rel.value

