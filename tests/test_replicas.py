"""The N > 1 replica path (independent runs, one per GPU) on CPU: two gloo
ranks exchange only timing (barrier, max over ranks) and the whole-job
throughput is the units of all ranks over the slowest rank's time."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    from kh_simulations_b200 import replicas

    r = replicas.init("gloo", timeout_s=60)
    ms = 10.0 + 5.0 * r.rank  # rank 1 is the slow one
    replicas.barrier(r)
    m = replicas.max_over_ranks(ms, r)
    rate = replicas.aggregate_rate(1000.0, m, r)
    replicas.barrier(r)
    replicas.finish(r)
    Path(out, f"rank{rank}.json").write_text(json.dumps({"world": r.world, "max": m, "rate": rate}))


def test_two_gloo_ranks_max_and_aggregate(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.loads((tmp_path / f"rank{i}.json").read_text()) for i in range(2)]
    for r in res:
        assert r["world"] == 2
        assert r["max"] == 15.0
        assert r["rate"] == pytest.approx(1000.0 * 2 / 15e-3)


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, str(ROOT))
    from kh_simulations_b200 import replicas

    r = replicas.init("gloo")
    assert (r.world, r.rank, r.backend) == (1, 0, None)
    assert replicas.max_over_ranks(3.5, r) == 3.5
    assert replicas.aggregate_rate(100.0, 2.0, r) == pytest.approx(5e4)


def test_reference_arm_non_zero_rank_exits_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"], env=env,
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""
