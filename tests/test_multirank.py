"""The N > 1 path on CPU with gloo, world size 2: the slowest rank's time becomes the job's, the rate
counts every rank's units, and the reference arm runs on rank 0 alone (one JSON line, both exit 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(10.0 + rank, world)           # rank 1 is the slow one
        q.put((rank, slowest, bench.job_rate(1e9, world, 4, slowest)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, rate in got:
        assert slowest == 11.0
        assert rate == pytest.approx(2 * 4 * 1e9 / 11.0e-3 / 1e9)


def test_reference_arm_under_torchrun_prints_once_from_rank_zero():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--recipes", "6"]
    _check_one_reference_line(subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600))


def _check_one_reference_line(out):
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    res = json.loads(lines[0])
    assert res["impl"] == "reference" and res["n_gpus"] == 2 and res["value"] > 0
    assert res["cpu_baseline"]["kind"] == "port" and res["e2e"]["h2d_bytes_per_step"] == 0
    # the step time is the measured time of that step's sample, not a projection
    assert 0 < res["ms_per_step"] < 600_000


def test_gpus_flag_without_torchrun_starts_the_ranks_itself():
    """`bench.py --gpus 2` run directly re-executes itself under torch.distributed.run with two
    ranks; rank 0 alone prints the reference arm's line."""
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--recipes", "6"]
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    _check_one_reference_line(subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600, env=env))
