"""GPU tests of the Krylov block operations (multi-dot and multi-axpy, FP64 and FP32 storage with FP64 sums) against
torch in FP64, on both the vectorised path (16-byte aligned rows) and the element-wise path (odd row strides), for basis
sizes across the range the GMRES solver uses."""
import ctypes as C
import importlib

import pytest

pytestmark = pytest.mark.gpu


def _lib():
    L = importlib.import_module("honee-4aiad_b200").lib()
    for name in ("hb_krylov_multidot_f64", "hb_krylov_multidot_f32"):
        getattr(L, name).argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    for name in ("hb_krylov_multiaxpy_f64", "hb_krylov_multiaxpy_f32"):
        getattr(L, name).argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_double), C.c_int64, C.c_void_p]
    return L


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("k,n,ldv", [(1, 10, 12), (5, 100_001, 100_004), (16, 333_333, 333_336), (31, 65_537, 65_537),
                                     (32, 4096, 4096), (3, 7, 7)])
def test_multidot_and_multiaxpy_match_torch(dtype, k, n, ldv):
    import torch
    L = _lib()
    dev = torch.device("cuda:0")
    tt = torch.float64 if dtype == "f64" else torch.float32
    g = torch.Generator().manual_seed(k * 7 + n)
    V = torch.randn(k, ldv, generator=g, dtype=torch.float64).to(dev, tt)
    w = torch.randn(n, generator=g, dtype=torch.float64).to(dev, tt)
    partial = torch.empty(512 * 32, dtype=torch.float64, device=dev)
    out = torch.full((k,), float("nan"), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    assert getattr(L, f"hb_krylov_multidot_{dtype}")(V.data_ptr(), ldv, k, w.data_ptr(), n, partial.data_ptr(), out.data_ptr(), s) == 0
    torch.cuda.synchronize()
    ref = V[:, :n].double() @ w.double()
    torch.testing.assert_close(out, ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max()))
    c = [((-1) ** i) * 0.5 / (i + 1) for i in range(k)]
    cc = (C.c_double * k)(*c)
    w0 = w.double().clone()
    assert getattr(L, f"hb_krylov_multiaxpy_{dtype}")(w.data_ptr(), V.data_ptr(), ldv, k, cc, n, s) == 0
    torch.cuda.synchronize()
    ref_w = w0 + (torch.tensor(c, dtype=torch.float64, device=dev)[:, None] * V[:, :n].double()).sum(0)
    tol = 1e-14 if dtype == "f64" else 2e-7  # FP64 sum rounded once to the storage precision
    torch.testing.assert_close(w.double(), ref_w, rtol=tol, atol=tol * float(ref_w.abs().max()))


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("k,n,ldv", [(1, 10, 12), (7, 100_001, 100_004), (30, 65_537, 65_537), (3, 7, 7)])
def test_multiaxpy_with_device_coefficients_equals_the_host_form(dtype, k, n, ldv):
    """hb_krylov_multiaxpy_dev_* (coefficients in device memory times a sign, as the GMRES loop passes the multi-dot's
    result with sign -1) gives the host-coefficient multi-axpy's result bit for bit, on the vectorised and element-wise
    paths."""
    import torch
    L = _lib()
    for name in ("hb_krylov_multiaxpy_dev_f64", "hb_krylov_multiaxpy_dev_f32"):
        getattr(L, name).argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_double, C.c_int64, C.c_void_p]
    dev = torch.device("cuda:0")
    tt = torch.float64 if dtype == "f64" else torch.float32
    g = torch.Generator().manual_seed(k * 11 + n)
    V = torch.randn(k, ldv, generator=g, dtype=torch.float64).to(dev, tt)
    w = torch.randn(n, generator=g, dtype=torch.float64).to(dev, tt)
    h = torch.randn(k, generator=g, dtype=torch.float64)
    s = torch.cuda.current_stream(dev).cuda_stream
    w_host, w_dev = w.clone(), w.clone()
    neg = (C.c_double * k)(*[-float(x) for x in h])
    assert getattr(L, f"hb_krylov_multiaxpy_{dtype}")(w_host.data_ptr(), V.data_ptr(), ldv, k, neg, n, s) == 0
    d_h = h.to(dev)
    assert getattr(L, f"hb_krylov_multiaxpy_dev_{dtype}")(w_dev.data_ptr(), V.data_ptr(), ldv, k, d_h.data_ptr(), -1.0, n, s) == 0
    torch.cuda.synchronize()
    assert torch.equal(w_dev, w_host)
    assert getattr(L, f"hb_krylov_multiaxpy_dev_{dtype}")(w_dev.data_ptr(), V.data_ptr(), ldv, 0, d_h.data_ptr(), -1.0, n, s) != 0
