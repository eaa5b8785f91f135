"""End-to-end GPU test of the learned closure at reduced size: a fine plain run (32^3, degree 2), differential filter,
training pairs, GPU training of the 6-20-20-6 network, the stress scale chosen among four candidates on the first half of
the snapshots, and two coarse runs (8^3, the full study's 4:1 element ratio) from the filtered initial state, with the
closure as the reference evaluates it (no limiter).  The closure must beat the closure-free coarse run against the
filtered fine solution on the kinetic energy, its decay and the resolved dissipation over all snapshots, at no more than a
fifth of the fine run's GPU time."""
import importlib

import pytest

pytestmark = pytest.mark.gpu


def test_learned_closure_beats_the_plain_coarse_run():
    les = importlib.import_module("honee-4aiad_b200.les")
    r = les.study(fine_faces=32, coarse_faces=8, degree=2, t_end=1.0, snaps=4, train_steps=800, batch=16384, lr=1e-3, seed=0, no_backscatter=False,
                  scales=(0.25, 0.5, 0.75, 1.0))
    assert r["coarse_closure"]["diverged"] is None
    e = r["errors_vs_filtered_fine"]
    assert e["closure"]["ke_decay_err"] < e["plain"]["ke_decay_err"], e
    assert e["closure"]["ke_err"] < e["plain"]["ke_err"], e
    assert e["closure"]["dissipation_err"] < e["plain"]["dissipation_err"], e
    assert r["training"]["loss"][-1][1] < 0.1 * r["training"]["loss"][0][1]
    assert r["fine"]["gpu_seconds"] >= 5 * r["coarse_closure"]["gpu_seconds"], (r["fine"]["gpu_seconds"], r["coarse_closure"]["gpu_seconds"])
