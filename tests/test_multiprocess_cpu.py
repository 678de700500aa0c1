"""The N > 1 path of bench.py on the CPU (gloo, world size 2): one process
per replica, the job time is the slowest rank's (MAX over ranks), the
whole-job value counts every rank's node updates, and under
torch.distributed.run only rank 0 prints the reference arm's line while the
other ranks exit 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t_local = 1.5 + rank  # rank 1 is the slow one
    t_max = bench.max_over_ranks(dist, t_local, "cpu")
    value = bench.whole_job_mlups(65536, 2000, world, t_max)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, t_max, value))


def test_max_over_ranks_and_whole_job_value_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]
    assert out[0][2] == out[1][2] == pytest.approx(65536 * 2000 * 2 / 2.5 / 1e6)


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(None, 3.25, "cpu") == 3.25


def test_reference_arm_under_torchrun_two_ranks():
    port = free_port()
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
                        "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
