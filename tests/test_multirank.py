"""The multi-rank plumbing of bench.py on CPU: world-size-2 gloo ranks agree on the slowest
rank's time, the job value counts every replica, and the reference arm under torchrun
prints exactly one line (rank 0) while the other rank exits cleanly."""
from __future__ import annotations

import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, times, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        out[rank] = bench.max_over_ranks(dist, torch, times[rank], "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, [3.5, 7.25], out), nprocs=2, start_method="spawn")
        assert out[0] == out[1] == 7.25


def test_job_value_counts_every_replica():
    bench = _bench()
    assert bench.job_gbs(1, 2e9, 1000.0) == pytest.approx(2.0)
    assert bench.job_gbs(4, 2e9, 1000.0) == pytest.approx(8.0)


def test_reference_arm_under_torchrun_prints_one_line(tmp_path):
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--log2n", "16", "--log2sort", "14", "--ref-log2", "16"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
