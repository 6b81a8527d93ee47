"""Multi-GPU plumbing of the bench on CPU: world_size-2 gloo process groups.

Replicas are independent (no data-path collective); the timed region is
bracketed by barriers and the whole-job rate uses the slowest rank's time.
A rank that never joins makes the others fail within the group timeout
instead of hanging.  The reference arm under torchrun runs on rank 0 only.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

from hicar_b200 import replicas as R

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    rk = R.from_env()
    R.init(rk, "gloo", timeout_s=30)
    R.barrier(rk)
    my_ms = 10.0 * (rank + 1)                   # per-rank device time of the timed region
    mx = R.max_over_ranks(rk, my_ms)
    rate = R.whole_job_rate(1000.0, rk.world, mx / 1e3)
    R.barrier(rk)
    R.finalize(rk)
    Path(out_dir, f"r{rank}.json").write_text(json.dumps(
        {"rank": rank, "max_ms": mx, "rate": rate, "seed": R.replica_seed(100, rk), "root": rk.is_root}))


def test_two_replicas_take_the_max_time_and_aggregate(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(2)]
    assert [r["max_ms"] for r in res] == [20.0, 20.0]                # both see the slowest rank
    assert all(abs(r["rate"] - 1000.0 * 2 / 0.020) < 1e-6 for r in res)
    assert res[0]["seed"] != res[1]["seed"]                          # independent replicas
    assert [r["root"] for r in res] == [True, False]


def _lonely(rank, port, out_dir):
    # rank 1 of a world of 2 whose rank 0 never starts
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="1", WORLD_SIZE="2", LOCAL_RANK="0")
    rk = R.from_env()
    try:
        R.init(rk, "gloo", timeout_s=3)
        R.barrier(rk)
        status = "joined"
    except Exception as e:                       # the store times out: an error, not a hang
        status = "error:" + type(e).__name__
    Path(out_dir, "lonely.json").write_text(json.dumps({"status": status}))


def test_a_missing_rank_ends_in_an_error_not_a_hang(tmp_path):
    port = _free_port()
    mp.start_processes(_lonely, args=(port, str(tmp_path)), nprocs=1, join=True, start_method="spawn")
    status = json.loads((tmp_path / "lonely.json").read_text())["status"]
    assert status.startswith("error:")


def test_single_rank_needs_no_process_group():
    rk = R.Ranks(0, 1, 0)
    R.init(rk)
    R.barrier(rk)
    assert R.max_over_ranks(rk, 3.5) == 3.5
    assert R.whole_job_rate(10.0, 1, 2.0) == 5.0
    R.finalize(rk)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_prints_one_contract_line():
    """bench.py --impl reference on rank 0: one JSON line with the metric of
    the GPU arm, the CPU baseline it was measured as, and an e2e entry with
    no host-device traffic."""
    import json
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "MPDATA cell-species updates/s"
    assert d["value"] > 0 and d["unit"] == "cell-species updates/s" and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
