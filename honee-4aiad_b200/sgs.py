"""The learned subgrid-stress closure: model description, weights, GPU training and inference (ctypes over
include/honee_b200.h).

Model: the data-driven SGS model of HONEE (qfunctions/sgs_dd_model.h), inputs = rotation-invariant features of the
velocity gradient in the grid-anisotropy frame, outputs = the SGS stress in the strain-rate eigenframe, min-max
normalised.  `load_reference_model` reads the reference's published 6-20-6 weights (examples/dd_sgs_data/*.dat,
PHASTA ASCII format, problems/sgs_dd_model.c:600-646); `Trainer` trains a 6-20-20-6 (or 6-20-6) network on the GPU
with this package's forward / backward / Adam kernels.  Device buffers are torch tensors (plumbing).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import lib as _load
from .kernels import _addr, _chk, _stream


class HbMlpDesc(C.Structure):
    _fields_ = [("hidden1", C.c_int), ("hidden2", C.c_int), ("leaky_alpha", C.c_float), ("out_bounds", C.c_float * 12),
                ("clamp_outputs", C.c_int), ("no_backscatter", C.c_int)]


def desc(hidden1=20, hidden2=20, alpha=0.0, bounds=None, clamp_outputs=False, no_backscatter=False) -> HbMlpDesc:
    d = HbMlpDesc(hidden1, hidden2, alpha)
    d.clamp_outputs, d.no_backscatter = int(clamp_outputs), int(no_backscatter)
    b = np.zeros(12) if bounds is None else np.asarray(bounds, dtype=np.float64).reshape(12)
    for i in range(12):
        d.out_bounds[i] = float(b[i])
    return d


def num_params(d: HbMlpDesc) -> int:
    n = _load().hb_mlp_num_params(C.byref(d))
    if n < 0:
        raise ValueError(f"unsupported network shape 6-{d.hidden1}-{d.hidden2}-6")
    return n


def read_dat(path) -> np.ndarray:
    """PHASTA ASCII array: a header line `N M`, then N*M values."""
    with open(path) as f:
        head = f.readline().split()
        n = int(head[0]) * (int(head[1]) if len(head) > 1 else 1)
        vals = np.array([float(t) for t in f.read().split()], dtype=np.float64)
    if vals.size != n:
        raise ValueError(f"{path}: expected {n} values, found {vals.size}")
    return vals


def load_reference_model(data_dir, alpha=0.0):
    """(HbMlpDesc, flat float64 parameters) of the reference's 6-20-6 model files b1/b2/w1/w2/OutScaling.dat.
    w1.dat holds [6][20] and w2.dat [20][6]; the reference transposes both into row-major [out][in]."""
    b1, b2 = read_dat(os.path.join(data_dir, "b1.dat")), read_dat(os.path.join(data_dir, "b2.dat"))
    w1, w2 = read_dat(os.path.join(data_dir, "w1.dat")), read_dat(os.path.join(data_dir, "w2.dat"))
    bounds = read_dat(os.path.join(data_dir, "OutScaling.dat"))
    W1 = w1.reshape(6, 20).T
    W2 = w2.reshape(20, 6).T
    flat = np.concatenate([W1.reshape(-1), b1[:20], W2.reshape(-1), b2[:6]])
    return desc(20, 0, alpha, bounds), flat


def sgs_dd_context(newt_ctx_bytes: bytes, flat_params, bounds, alpha=0.0):
    """The SgsDDContext_ blob of a 6-20-6 network (qfunctions/sgs_dd_model.h:16-31) as SgsDDContextFill lays it out
    (problems/sgs_dd_model.c:598-651): num_inputs, num_outputs, num_layers (1), num_neurons, alpha, the Newtonian context,
    the data offsets bias1 0, bias2 20, weight1 40, weight2 160, out_scaling 280 (in doubles; bias2 gets num_neurons
    slots), total_bytes, then data = b1 | b2 | W1 [20][6] | W2 [6][20] | bounds [6][2].  flat_params in the layout of
    load_reference_model.  Returns a ctypes char array (what CeedQFunctionContextSetData is given)."""
    p = np.asarray(flat_params, dtype=np.float64)
    W1, b1, W2, b2 = p[:120], p[120:140], p[140:260], p[260:266]
    data = np.concatenate([b1, np.pad(b2, (0, 14)), W1, W2, np.asarray(bounds, dtype=np.float64).reshape(12)])
    o_data = 256
    total = o_data + 8 * data.size
    buf = bytearray(total)
    np.frombuffer(buf, dtype=np.int32, count=4, offset=0)[:] = [6, 6, 1, 20]
    np.frombuffer(buf, dtype=np.float64, count=1, offset=16)[:] = alpha
    if len(newt_ctx_bytes) != 184:
        raise ValueError("the Newtonian context must be the 184-byte NewtonianIdealGasContext_")
    buf[24:208] = newt_ctx_bytes
    np.frombuffer(buf, dtype=np.uint64, count=6, offset=208)[:] = [0, 20, 40, 160, 280, total]
    np.frombuffer(buf, dtype=np.float64, count=data.size, offset=o_data)[:] = data
    return (C.c_char * total).from_buffer_copy(bytes(buf))


def xavier_init(d: HbMlpDesc, seed=0) -> np.ndarray:
    """Glorot-uniform weights U(-a, a), a = sqrt(6 / (fan_in + fan_out)), zero biases, from a seeded generator."""
    rng = np.random.default_rng(seed)
    dims = [6, d.hidden1] + ([d.hidden2] if d.hidden2 else []) + [6]
    parts = []
    for nin, nout in zip(dims[:-1], dims[1:]):
        a = math.sqrt(6.0 / (nin + nout))
        parts += [rng.uniform(-a, a, size=nout * nin), np.zeros(nout)]
    flat = np.concatenate(parts).astype(np.float32)
    assert flat.size == num_params(d)
    return flat


class Trainer:
    """Adam training of the closure network on device-resident pairs X, Y ([n][6] float32 torch tensors)."""

    def __init__(self, d: HbMlpDesc, params, batch=65536, lr=1e-3, seed=0, device="cuda:0", stream=None):
        import torch
        self.torch = torch
        self.d = d
        self.np = num_params(d)
        dev = torch.device(device)
        self.w = torch.as_tensor(np.asarray(params, dtype=np.float32)).to(dev).contiguous()
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.batch, self.lr, self.seed, self.step_count = batch, lr, seed, 0
        nb = (batch + 255) // 256
        self.work = torch.empty(nb * (self.np + 1) + 16, dtype=torch.float32, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.stream = stream

    def step(self, X, Y, idx=None, lr=None, grad=None):
        """One Adam step (or, with lr=0, the gradient only into `grad`); returns nothing, the loss stays on the device."""
        self.step_count += 1
        n = X.shape[0]
        batch = self.batch if idx is None else idx.numel()
        _chk(_load().hb_mlp_train_step(C.byref(self.d), _addr(self.w), _addr(self.m), _addr(self.v), _addr(X), _addr(Y), C.c_int64(n),
                                       _addr(idx), C.c_int(batch), C.c_uint64(self.seed), C.c_int(self.step_count),
                                       C.c_float(self.lr if lr is None else lr), _addr(self.work), _addr(self.loss), _addr(grad),
                                       _stream(self.stream)), "hb_mlp_train_step")

    def train(self, X, Y, steps, log_every=0):
        hist = []
        for k in range(steps):
            self.step(X, Y)
            if log_every and (k % log_every == 0 or k == steps - 1):
                hist.append((self.step_count, float(self.loss.item())))
        return hist

    def params(self) -> np.ndarray:
        return self.w.cpu().numpy()


def forward(d: HbMlpDesc, w, X, Y, stream=None):
    _chk(_load().hb_mlp_forward(C.byref(d), _addr(w), _addr(X), _addr(Y), C.c_int64(X.shape[0]), _stream(stream)), "hb_mlp_forward")


def target_bounds(Y, work, stream=None) -> np.ndarray:
    b = (C.c_float * 12)()
    _chk(_load().hb_sgs_target_bounds(_addr(Y), C.c_int64(Y.shape[0]), _addr(work), b, _stream(stream)), "hb_sgs_target_bounds")
    return np.array(b[:], dtype=np.float64)


def normalize_targets(Y, bounds, stream=None):
    b = (C.c_float * 12)(*[float(x) for x in np.asarray(bounds).reshape(12)])
    _chk(_load().hb_sgs_normalize_targets(_addr(Y), C.c_int64(Y.shape[0]), b, _stream(stream)), "hb_sgs_normalize_targets")


def point_anisotropy(dXdx, kmA, delta, stream=None):
    _chk(_load().hb_sgs_anisotropy(C.c_int64(dXdx.shape[0]), _addr(dXdx), _addr(kmA), _addr(delta), _stream(stream)), "hb_sgs_anisotropy")


def point_inputs(G, kmA, delta, nu, inputs, E, gmag, stream=None):
    _chk(_load().hb_sgs_inputs(C.c_int64(G.shape[0]), _addr(G), _addr(kmA), _addr(delta), _addr(nu), _addr(inputs), _addr(E), _addr(gmag),
                               _stream(stream)), "hb_sgs_inputs")


def nodal_closure(ctx_blob, state_var, q, G, A, w, km_sgs, stream=None):
    """km_sgs [n][6] += w [n] tau: the closure of an SgsDDContext_ blob at n nodes (hb_sgs_nodal_closure) from q [n][5] in
    state_var, the velocity gradient G [n][9] and the anisotropy tensor with width A [n][7] (device tensors)."""
    n = w.shape[0]
    _chk(_load().hb_sgs_nodal_closure(C.c_int64(n), C.cast(C.pointer(ctx_blob), C.c_void_p), C.c_size_t(C.sizeof(ctx_blob)), C.c_int(state_var),
                                      _addr(q), _addr(G), _addr(A), _addr(w), _addr(km_sgs), _stream(stream)), "hb_sgs_nodal_closure")


def point_stress(out_n, delta, E, gmag, bounds, km_tau, stream=None):
    b = (C.c_float * 12)(*[float(x) for x in np.asarray(bounds).reshape(12)])
    _chk(_load().hb_sgs_stress(C.c_int64(out_n.shape[0]), _addr(out_n), _addr(delta), _addr(E), _addr(gmag), b, _addr(km_tau),
                               _stream(stream)), "hb_sgs_stress")
