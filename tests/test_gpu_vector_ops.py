"""The element-wise vector kernels of the Krylov inner loop through the C ABI (hb_vec_scale_*, hb_vec_pointwise_mult_*,
hb_vec_reduce_*), FP32 and FP64: 16-byte vector loads where every pointer is 16-byte aligned, the scalar kernels on
other views, and a tail of n mod (16 / element size) entries.  Scale and multiply are bit-exact against torch; the FP64
reductions (sum |x|, sum x^2, max |x|, x . y) within 1e-13 relative of an FP64 sum in another order, max exactly."""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

hb = importlib.import_module("honee-4aiad_b200")


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n", [1, 3, 7, 1001, 1_000_003])
@pytest.mark.parametrize("offset", [0, 1])
def test_scale_multiply_reduce(dtype, n, offset):
    import torch
    L = hb.lib()
    T = torch.float32 if dtype == "f32" else torch.float64
    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(n + offset)
    base_x = torch.randn(n + offset, generator=g, dtype=T).to(dev)
    base_y = torch.randn(n + offset, generator=g, dtype=T).to(dev)
    base_w = torch.zeros(n + offset, dtype=T, device=dev)
    x, y, w = base_x[offset:], base_y[offset:], base_w[offset:]  # offset 1: 4- or 8-byte aligned views, the scalar path
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    scalar = C.c_float if dtype == "f32" else C.c_double
    ref_x = x.clone()
    assert getattr(L, f"hb_vec_pointwise_mult_{dtype}")(p(w), p(x), p(y), C.c_int64(n), s) == 0
    assert getattr(L, f"hb_vec_scale_{dtype}")(p(x), C.c_int64(n), scalar(0.75), s) == 0
    torch.cuda.synchronize()
    assert torch.equal(w, ref_x * y)
    assert torch.equal(x, ref_x * 0.75)
    scratch = torch.empty(1024, dtype=torch.float64, device=dev)
    xd, yd = x.double().cpu().numpy(), y.double().cpu().numpy()
    refs = [np.abs(xd).sum(), (xd * xd).sum(), np.abs(xd).max(), (xd * yd).sum()]
    for typ, ref in enumerate(refs):
        out = C.c_double()
        ptr_y = p(y) if typ == 3 else C.c_void_p(0)
        assert getattr(L, f"hb_vec_reduce_{dtype}")(p(x), ptr_y, C.c_int64(n), typ, p(scratch), C.byref(out), s) == 0
        if typ == 2:
            assert out.value == ref
        else:
            assert abs(out.value - ref) <= 1e-13 * max(1.0, np.abs(xd).sum() * max(1.0, np.abs(yd).max()))
