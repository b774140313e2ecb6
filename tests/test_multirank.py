"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (replicas only -- no data
collective; the one collective is the max over ranks of the timed intervals), and the
reference arm under torchrun, where rank 0 alone runs and prints."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # each rank's own step and end-to-end times; every rank must see the slowest ones
        got = bench.max_over_ranks(dist, [1.0 + rank, 10.0 - rank], "cpu")
        Path(out_dir, f"rank{rank}.json").write_text(json.dumps(got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    mp.start_processes(_rank, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        assert json.loads((tmp_path / f"rank{r}.json").read_text()) == [2.0, 10.0]


def test_max_over_ranks_without_a_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(None, [3.0, 4.0], "cpu") == [3.0, 4.0]


def test_reference_arm_under_torchrun_prints_one_line():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--elements", "2000"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
