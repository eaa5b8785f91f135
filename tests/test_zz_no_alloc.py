"""GPU test of hb_krylov_multidot_f64_static, the Krylov multi-dot whose partial sums live in a fixed device array of
the library instead of a caller buffer.  It must give what hb_krylov_multidot_f64 gives on the same inputs, on repeated
calls, and refuse a basis larger than its scratch holds.  Named to run after the other test files and also run alone."""
import ctypes as C
import importlib

import pytest

pytestmark = pytest.mark.gpu

HB_GMRES_MAX_BASIS = 32
HB_ERROR_INVALID = -4


def _lib():
    L = importlib.import_module("honee-4aiad_b200").lib()
    sig = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int64]
    L.hb_krylov_multidot_f64.argtypes = sig + [C.c_void_p, C.c_void_p, C.c_void_p]
    L.hb_krylov_multidot_f64_static.argtypes = sig + [C.c_void_p, C.c_void_p]
    L.hb_krylov_multidot_f64.restype = L.hb_krylov_multidot_f64_static.restype = C.c_int
    return L


@pytest.mark.parametrize("k,n,ldv_pad", [(7, 1_000_003, 5), (HB_GMRES_MAX_BASIS, 4099, 0), (1, 1, 0)])
def test_static_scratch_multidot_matches_buffered_entry_point(k, n, ldv_pad):
    import torch
    L = _lib()
    dev = torch.device("cuda:0")
    g = torch.Generator().manual_seed(k * 1000 + n % 997)
    ldv = n + ldv_pad
    V = torch.randn(k, ldv, generator=g, dtype=torch.float64).to(dev)
    w = torch.randn(n, generator=g, dtype=torch.float64).to(dev)
    partial = torch.empty(512 * HB_GMRES_MAX_BASIS, dtype=torch.float64, device=dev)
    ref = torch.full((k,), float("nan"), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    assert L.hb_krylov_multidot_f64(V.data_ptr(), ldv, k, w.data_ptr(), n, partial.data_ptr(), ref.data_ptr(), s) == 0
    torch.cuda.synchronize()
    exact = (V[:, :n] @ w)
    torch.testing.assert_close(ref, exact, rtol=1e-12, atol=1e-12 * float(exact.abs().max()))
    for _ in range(2):  # two calls in a row reuse the same scratch
        out = torch.full((k,), float("nan"), dtype=torch.float64, device=dev)
        assert L.hb_krylov_multidot_f64_static(V.data_ptr(), ldv, k, w.data_ptr(), n, out.data_ptr(), s) == 0
        torch.cuda.synchronize()
        # same kernels and block order as the buffered call: agreement to the last bits is expected, 1e-14 is the bar
        torch.testing.assert_close(out, ref, rtol=1e-14, atol=0.0)


def test_static_scratch_multidot_refuses_basis_beyond_scratch():
    import torch
    L = _lib()
    dev = torch.device("cuda:0")
    V = torch.zeros(HB_GMRES_MAX_BASIS + 1, 8, dtype=torch.float64, device=dev)
    w = torch.zeros(8, dtype=torch.float64, device=dev)
    out = torch.full((HB_GMRES_MAX_BASIS + 1,), 7.0, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    for k in (HB_GMRES_MAX_BASIS + 1, 0):
        assert L.hb_krylov_multidot_f64_static(V.data_ptr(), 8, k, w.data_ptr(), 8, out.data_ptr(), s) == HB_ERROR_INVALID
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())  # nothing was launched
