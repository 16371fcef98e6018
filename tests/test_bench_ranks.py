"""The bench's multi-rank host logic on CPU (gloo, world size 2): one
replica per rank, the step time is the max over ranks, the whole-job value
counts every rank's IAs, and the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = bench.max_over_ranks(times[rank], world)
        with open(os.path.join(out_dir, f"r{rank}"), "w") as f:
            f.write(repr(m))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    times = [12.5, 31.25]  # ms of K steps on rank 0 and rank 1
    mp.start_processes(_rank, args=(2, _free_port(), times, str(tmp_path)), nprocs=2, start_method="spawn",
                       join=True)
    got = [float(open(tmp_path / f"r{r}").read()) for r in range(2)]
    assert got == [31.25, 31.25]
    # the job rate uses the slowest rank's time and every rank's units
    assert bench.job_rate(2, 64009, 10, 31.25e-3) == pytest.approx(2 * 64009 * 10 / 31.25e-3)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(7.0, 1) == 7.0


def test_reference_arm_under_torchrun_prints_once():
    """`torch.distributed.run --nproc-per-node 2 bench.py --impl reference`:
    rank 0 times the CPU restatement and prints one JSON line, rank 1 exits 0
    without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--size", "256", "--steps", "1", "--warmup", "0", "--ref-budget", "0.2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("port", "reference")
