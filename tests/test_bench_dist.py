"""The multi-rank timing of bench.py on two gloo ranks (CPU): every rank
ends with the slowest rank's step time, the whole-job rate counts every
rank's units, and the reference arm prints only on rank 0."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local_ms = [3.0, 5.5][rank]
        ms = bench.max_over_ranks(local_ms, device="cpu")
        out[rank] = (ms, bench.whole_job_rate(1_000_000, world, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == out[1]
    ms, rate = out[0]
    assert ms == 5.5
    assert rate == pytest.approx(2 * 1_000_000 / 5.5e-3 / 1e6)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.25, device="cpu") == 4.25
    assert bench.whole_job_rate(10, 1, 2.0) == pytest.approx(10 / 2e-3 / 1e6)


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_issue_roofline_arithmetic():
    # the small kernel's capture on 148 SMs at 1965 MHz: 464.9M warp
    # instructions take 0.400 ms at one per sub-partition per cycle
    sys.path.insert(0, ROOT)
    import bench
    r = bench.issue_roofline(464942099, 0.544, {"sm_mhz": 1965}, sms=148)
    assert r["peak"] == round(148 * 4 * 1965e6 / 1e9, 1)
    assert abs(r["frac"] - 464942099 / 0.544e-3 / (148 * 4 * 1965e6)) < 1e-4
    assert 0.73 < r["frac"] < 0.74
    # the sampled clock missing: the maximum clock; no clock or no time: None
    assert bench.issue_roofline(1000, 1.0, {"sm_max_mhz": 1000}, sms=1)["sm_mhz"] == 1000
    assert bench.issue_roofline(1000, 1.0, {}, sms=1) is None
    assert bench.issue_roofline(1000, 0.0, {"sm_mhz": 1965}, sms=1) is None
