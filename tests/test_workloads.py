"""The seeded ensemble and serving workloads on CPU (no device calls).

The ensemble: solves with N drawn from {32, 48, 64, 96, 128} by default_rng(2026), Re
log-uniform in [400, 3200], solve i perturbed with seed i (1 <= |m| <= N/8, amplitude 1e-3),
each with its own CFL 0.5 step.  The serving stream: Poisson arrivals at 20 requests/s from
default_rng(5) for 120 s, N in {64, 128, 256} at {0.6, 0.3, 0.1}, Re log-uniform in
[400, 3200], t_end uniform in [1, 10], seed = request id.  bench.py serves the stream's first
2 s (43 requests) and the first 64 ensemble members.
"""
import math

import numpy as np
import pytest

from spectral_solver_b200.ensemble import SIZES, make_specs
from spectral_solver_b200.serve import make_stream, percentile


def test_ensemble_specs_are_seeded_and_in_range():
    a, b = make_specs(64), make_specs(64)
    assert a == b
    assert [s["seed"] for s in a] == list(range(64))
    assert {s["n"] for s in a} == set(SIZES)
    assert [sum(1 for s in a if s["n"] == n) for n in SIZES] == [15, 15, 13, 12, 9]
    for s in a:
        assert 1.0 / 3200.0 <= s["nu"] <= 1.0 / 400.0
        assert s["pert_kmax"] == max(1, s["n"] // 8) and s["pert_amp"] == 1e-3
        assert s["dt"] == 0.0 and s["cfl"] == 0.5 and s["dt_max"] == 0.5  # CFL step per solve
    assert make_specs(64, seed=7) != a


def test_serving_stream_statistics():
    full = make_stream()
    assert full == make_stream()
    arrivals = [r["arrival"] for r in full]
    assert all(0.0 < x <= 120.0 for x in arrivals)
    assert arrivals == sorted(arrivals)
    # Poisson count at 20/s over 120 s: 2400 +- 5 sigma
    assert abs(len(full) - 2400) < 5 * math.sqrt(2400)
    for n, p in ((64, 0.6), (128, 0.3), (256, 0.1)):
        share = sum(1 for r in full if r["n"] == n) / len(full)
        assert abs(share - p) < 0.03, (n, share)
    for i, r in enumerate(full):
        assert r["seed"] == i
        assert 1.0 <= r["t_end"] <= 10.0
        assert 1.0 / 3200.0 <= r["nu"] <= 1.0 / 400.0
        assert r["pert_kmax"] == max(1, r["n"] // 8)


def test_bench_serves_the_streams_first_two_seconds():
    head = make_stream(2.0)
    assert len(head) == 43
    assert head == make_stream()[:43]


def test_percentile():
    assert percentile([], 50) is None
    xs = list(np.random.default_rng(1).exponential(size=101))
    assert percentile(xs, 50) == pytest.approx(float(np.median(xs)))
    assert percentile(xs, 99) <= max(xs)
