"""The basis-contraction A/B probe (hb_contraction_probe): shared-memory fibre passes (the operator kernels' mechanism)
and warp shuffles compute the same in-plane collocated derivatives, bit for bit, and both equal a numpy restatement
within 1e-13 relative (numpy sums in another order).  The timing of the two variants is `bench.py --contraction-ab`."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

prob = importlib.import_module("honee-4aiad_b200.problem")


def colo_derivative(Q=5):
    qx, _ = prob.gauss_legendre(Q)
    _, D = prob.lagrange_tabulate(qx, qx)
    return D / np.abs(D).sum(1).max()


def numpy_rounds(D, u, reps):
    v = u.reshape(-1, 5, 5, 5, 5).copy()  # [e][c][z][y][x]
    for _ in range(reps):
        v = np.einsum("im,ecjkm->ecjki", D, v) + np.einsum("jm,eczmi->eczji", D, v)
    return v.reshape(u.shape)


@pytest.mark.parametrize("E,reps", [(1, 1), (37, 3), (1000, 2)])
def test_shared_and_shuffle_contractions_agree(E, reps):
    import torch
    kern = importlib.import_module("honee-4aiad_b200.kernels")
    D = colo_derivative()
    rng = np.random.default_rng(E + reps)
    u = rng.normal(size=(E, 5, 125))
    tu = torch.from_numpy(u).cuda()
    outs = []
    for variant in (0, 1):
        for ctas in (0, 3):
            _, fmas, out = kern.contraction_probe(variant, D, tu, reps, ctas_per_sm=ctas, launches=1)
            assert fmas == E * reps * 6250
            outs.append(out.cpu().numpy())
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
    ref = numpy_rounds(D, u, reps)
    assert np.linalg.norm(outs[0] - ref) / np.linalg.norm(ref) < 1e-13
