"""The N > 1 path of bench.py on CPU: two gloo ranks (world_size 2) run the replica timing logic -- every rank takes the
same collective steps, the job time is the maximum over ranks and the job throughput counts every replica's work."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [3.0, 5.0][rank]
        ms = bench.max_over_ranks(local_ms, world, torch.device("cpu"))
        out.put((rank, ms, bench.job_gdofs(world, 1_000_000, ms)))
        torch.distributed.barrier()
    finally:
        torch.distributed.destroy_process_group()


def test_two_replicas_take_the_slowest_rank_and_count_both():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [5.0, 5.0]
    assert res[0][2] == pytest.approx(2 * 1_000_000 / 5e-3 / 1e9)


def test_single_rank_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.0, 1, None) == 4.0
    assert bench.job_gdofs(1, 2_000_000, 2.0) == pytest.approx(1.0)


def test_reference_arm_under_torchrun_prints_one_line_from_rank_zero():
    """`bench.py --impl reference` launched as the driver launches every arm for N > 1 (torchrun, one process per GPU):
    rank 0 alone runs the reference's CPU path and prints the JSON line, the other ranks exit 0 without work.  The arm's
    process group is a CPU (gloo) one, so this runs here; a small box keeps it short."""
    import json
    import subprocess
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--size", "3", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2 and lines[0]["value"] > 0
