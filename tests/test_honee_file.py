"""CPU checks of the HONEE solution-file format (honee-4aiad_b200/honee_file.py, src/honee-file.c:136-232): the reference's own
files (32- and 64-bit-index variants, tests/golden/ref_*.bin) decode to the values, step and time the fixtures record, and
write -> read round-trips, including the legacy bare-Vec form; a checkpoint of an essential-DOF state expands back."""
import importlib
import os

import numpy as np

HF = importlib.import_module("honee-4aiad_b200.honee_file")
prob = importlib.import_module("honee-4aiad_b200.problem")
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_reference_files_decode():
    f = HF.read(os.path.join(GOLD, "ref_channel.bin"))
    G = np.load(os.path.join(GOLD, "channel_be5.npz"))
    assert not f.int64 and f.step == int(G["final_step"]) and f.time == float(G["final_time"])
    np.testing.assert_array_equal(f.values, G["free_state"])
    f = HF.read(os.path.join(GOLD, "ref_taylor-green.bin"))
    G = np.load(os.path.join(GOLD, "taylorgreen_rk4.npz"))
    assert f.step == 3 and abs(f.time - 0.006) < 1e-18
    np.testing.assert_array_equal(f.values, G["final_state"])
    f = HF.read(os.path.join(GOLD, "ref_gaussianwave-explicit.bin"))
    G = np.load(os.path.join(GOLD, "gaussianwave_explicit.npz"))
    assert f.int64 and f.step == 5 and f.values.size == 882
    np.testing.assert_array_equal(f.values, G["free_state"])


def test_write_read_round_trip_and_legacy(tmp_path):
    v = np.random.default_rng(0).normal(size=123)
    for wide in (False, True):
        p = str(tmp_path / f"s{int(wide)}.bin")
        HF.write(p, v, step=7, time=1.25e-3, int64=wide)
        f = HF.read(p)
        assert f.step == 7 and f.time == 1.25e-3 and f.int64 == wide
        np.testing.assert_array_equal(f.values, v)
    # a bare PETSc Vec (32-bit indices), as old regression files were written
    p = str(tmp_path / "legacy.bin")
    with open(p, "wb") as fh:
        fh.write(np.array([HF.VEC_FILE_CLASSID, v.size], dtype=">i4").tobytes() + v.astype(">f8").tobytes())
    f = HF.read(p)
    assert f.step == 0 and f.time == 0.0
    np.testing.assert_array_equal(f.values, v)
    # the 64-bit bare Vec splits its class id over two int32 words
    p = str(tmp_path / "legacy64.bin")
    with open(p, "wb") as fh:
        fh.write(np.array([HF.VEC_FILE_CLASSID, v.size], dtype=">i8").tobytes() + v.astype(">f8").tobytes())
    np.testing.assert_array_equal(HF.read(p).values, v)


def test_checkpoint_of_an_essential_state_expands_back(tmp_path):
    mesh = prob.box_mesh((5, 5, 1), 2, periodic=(1, 0, 0), hi=(0.01, 0.01, 0.001))
    idx = prob.box_essential(mesh, {"y-": (1, 2, 3), "y+": (1, 2, 3), "z-": (3,), "z+": (3,)})
    q = np.random.default_rng(1).normal(size=mesh.l_size)
    q[idx] = 0.0
    p = str(tmp_path / "ckpt.bin")
    HF.write(p, HF.free_values(q, idx), step=5, time=2.5e-5)
    f = HF.read(p)
    assert f.values.size == 200
    np.testing.assert_array_equal(HF.expand(f.values, mesh.l_size, idx), q)
