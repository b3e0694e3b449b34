"""Host-side models of bench.py's served-stream legs (no GPU): the first-come-first-served queue that
turns per-request service times into time-to-result for the one-case-at-a-time FP64 path and for the
reference's process pool, and the specified served stream's generator."""
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))

import bench  # noqa: E402


def test_fifo_single_server():
    # arrivals 0, 1, 2; service 2 each: the queue builds up by one unit per request
    assert bench.fifo_latency([0.0, 1.0, 2.0], [2.0, 2.0, 2.0]) == [2.0, 3.0, 4.0]
    # an idle server starts a request when it arrives
    assert bench.fifo_latency([0.0, 10.0], [1.0, 1.0]) == [1.0, 1.0]


def test_fifo_many_servers():
    # two servers: the third request waits for the first to finish
    lat = bench.fifo_latency([0.0, 0.0, 0.0], [4.0, 1.0, 1.0], servers=2)
    assert lat == [4.0, 1.0, 2.0]


def test_c5_stream_is_the_specified_one():
    reqs, gaps = bench.c5_stream(n=400)
    sides = [r["nx"] for r in reqs]
    steps = [r["steps"] for r in reqs]
    assert min(sides) >= 64 and max(sides) <= 2048 and max(sides) > 1024
    assert min(steps) >= 5000 and max(steps) <= 100000
    frac64 = sum(r["fp64"] for r in reqs) / len(reqs)
    strips = sum(r["strip"] for r in reqs) / len(reqs)
    assert 0.05 < frac64 < 0.15 and 0.12 < strips < 0.28
    assert len(gaps) == 400 and all(g > 0 for g in gaps)
    # deterministic from its seed
    assert bench.c5_stream(n=400)[0] == reqs


def test_cpu_estimate_scales_with_processes():
    reqs = [dict(nx=100, steps=1000)] * 8
    arrive = [0.0] * 8
    one = bench.c5_cpu_estimate(reqs, arrive, 1.0, 1)   # 1e7 updates at 1 MLUPS: 10 s each
    four = bench.c5_cpu_estimate(reqs, arrive, 1.0, 4)
    assert one["p99_s"] == pytest.approx(80.0, rel=0.02)
    assert four["p99_s"] == pytest.approx(20.0, rel=0.02)
