"""Serving stream over the continuous-batching server (``sns_server_*``).

The serving configuration: Poisson arrivals at 20 requests/s (``default_rng(5)``), each with
N in {64, 128, 256}^3 at probabilities {0.6, 0.3, 0.1}, Re log-uniform in [400, 3200],
horizon t_end uniform in [1, 10] and its own seed (the request id) for the k^(-5/3)
perturbation (amplitude 1e-3, 1 <= |m| <= N/8).  Requests are admitted against an HBM budget
(80 GB), fields stay on the device, and all resident solves step together; the FP32
precision form runs first and the FP64 form as a second pass.  Reports solves/s, p50 / p95 /
p99 latency (arrival to result), the offered and served load and the backlog when the
arrivals stop.

    python -m spectral_solver_b200.serve [--seconds 120] [--rate 20] [--budget-gb 80]
                                         [--precision both|fp32|fp64]
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from ._lib import PRECISION_FP32, PRECISION_FP64, Server


def make_stream(seconds: float = 120.0, rate: float = 20.0, seed: int = 5):
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > seconds:
            break
        n = int(rng.choice([64, 128, 256], p=[0.6, 0.3, 0.1]))
        re = float(np.exp(rng.uniform(np.log(400.0), np.log(3200.0))))
        t_end = float(rng.uniform(1.0, 10.0))
        reqs.append(dict(arrival=t, n=n, nu=1.0 / re, t_end=t_end, seed=len(reqs), pert_amp=1e-3,
                         pert_kmax=max(1, n // 8)))
    return reqs


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs), q)) if xs else None


def run(stream, budget_bytes: int, precision: int, max_wall: float | None = None):
    """Replay the stream in real time; returns the report.  With max_wall the run stops
    after that many seconds and reports what finished (the rest is backlog)."""
    seconds = stream[-1]["arrival"] if stream else 0.0
    lat, finished, gpsteps = {}, {}, 0.0
    submitted = {}
    backlog_at_close = None
    tick_s = []
    with Server(budget_bytes, precision) as srv:
        t0 = time.perf_counter()
        nxt = 0
        while len(finished) < len(stream):
            now = time.perf_counter() - t0
            while nxt < len(stream) and stream[nxt]["arrival"] <= now:
                r = stream[nxt]
                rid = srv.submit(r["n"], r["nu"], r["t_end"], r["seed"], r["pert_amp"], r["pert_kmax"], 0.5, 0.5)
                submitted[rid] = nxt
                nxt += 1
            if len(finished) == len(submitted):  # idle: wait for the next arrival
                time.sleep(max(0.0, min(0.01, stream[nxt]["arrival"] - now)))
                continue
            ta = time.perf_counter()
            out, resident, queued, used = srv.step()
            tick_s.append(time.perf_counter() - ta)
            done_at = time.perf_counter() - t0
            for res in out:
                i = submitted[res["id"]]
                finished[i] = res
                lat[i] = done_at - stream[i]["arrival"]
                gpsteps += res["n"] ** 3 * res["steps"]
            if backlog_at_close is None and done_at >= seconds:
                backlog_at_close = resident + queued
            if max_wall is not None and done_at > max_wall:
                break
        wall = time.perf_counter() - t0
        pool = srv.stats()
    lats = list(lat.values())
    offered = sum(r["n"] ** 3 * math.ceil(r["t_end"] / (0.5 * 2 * math.pi / r["n"])) for r in stream) / max(seconds, 1e-9)
    return {"precision": "fp64" if precision == PRECISION_FP64 else "fp32", "requests": len(stream),
            "completed": len(finished), "arrival_seconds": seconds, "wall_seconds": wall,
            "solves_per_s": len(finished) / wall if wall > 0 else None,
            "latency_s": {"p50": percentile(lats, 50), "p95": percentile(lats, 95), "p99": percentile(lats, 99)},
            "served_gpts_per_s": gpsteps / wall / 1e9 if wall > 0 else None,
            "offered_gpts_per_s_estimate": offered / 1e9,
            "backlog_when_arrivals_stop": backlog_at_close,
            "drain_seconds": max(0.0, wall - seconds),
            # host time of a server tick (admission and re-initialisation of new solves,
            # launches, retirement), which does not wait for GPU work
            "tick_ms": {"p50": 1e3 * percentile(tick_s, 50), "p99": 1e3 * percentile(tick_s, 99),
                        "max": 1e3 * max(tick_s)} if tick_s else None,
            "handles_created": pool["handles_created"], "idle_pool_bytes_at_end": pool["idle_bytes"]}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--seconds", type=float, default=120.0, help="length of the arrival stream")
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--budget-gb", type=float, default=80.0)
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "fp64"])
    ap.add_argument("--max-wall", type=float, default=None, help="stop after this many seconds")
    a = ap.parse_args(argv)
    stream = make_stream(a.seconds, a.rate)
    forms = {"both": [PRECISION_FP32, PRECISION_FP64], "fp64": [PRECISION_FP64], "fp32": [PRECISION_FP32]}
    for p in forms[a.precision]:
        print(json.dumps(run(stream, int(a.budget_gb * 1e9), p, a.max_wall)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
