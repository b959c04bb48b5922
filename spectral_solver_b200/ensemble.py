"""Batched ensemble run: many independent Taylor-Green solves of uneven size on one GPU.

The ensemble configuration: solves with N drawn from {32, 48, 64, 96, 128}^3 (radix-2 and
radix-3 plans) by ``numpy.random.default_rng(2026)``, Re log-uniform in [400, 3200], solve i
perturbed with seed i (k^(-5/3), amplitude 1e-3, 1 <= |m| <= N/8), each with its own
CFL-limited step (CFL 0.5) recomputed on the device from its current vmax before every step,
in the FP64 plain form and the FP32 precision form.  Every batch step is one CUDA graph
launch with one branch per solve; launch shapes are autotuned once per (N, precision) and
cached.

    python -m spectral_solver_b200.ensemble [--count 64] [--steps 500] [--warmup 3]
                                            [--precision both|fp64|fp32] [--autotune 2]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

import numpy as np

from ._lib import PRECISION_FP32, PRECISION_FP64, Batch

SIZES = (32, 48, 64, 96, 128)


def make_specs(count: int = 64, precision: int = PRECISION_FP64, seed: int = 2026):
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(rng.choice(SIZES))
        re = float(np.exp(rng.uniform(np.log(400.0), np.log(3200.0))))
        specs.append(dict(n=n, nu=1.0 / re, precision=precision, seed=i, pert_amp=1e-3, pert_kmax=max(1, n // 8),
                          dt=0.0, cfl=0.5, dt_max=0.5))
    return specs


def run(count=64, steps=500, warmup=3, precision=PRECISION_FP64, autotune=2, cache=None):
    specs = make_specs(count, precision)
    with Batch(specs, autotune_trials=autotune, autotune_cache=cache) as b:
        b.step(warmup)
        ms = b.time_steps(steps)
        energies = [b.solver(i).diagnostics(0.0)["kinetic_energy"] for i in range(len(specs))]
    points = sum(sp["n"] ** 3 for sp in specs)
    return {"precision": "fp64" if precision == PRECISION_FP64 else "fp32", "solves": count, "steps": steps,
            "ms": ms, "ms_per_step": ms / steps, "gpts_per_s": points * steps / (ms / 1e3) / 1e9,
            "grid_points": points, "sizes": {str(n): sum(1 for sp in specs if sp["n"] == n) for n in SIZES},
            "all_finite": bool(np.all(np.isfinite(energies)))}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "fp32"])
    ap.add_argument("--autotune", type=int, default=2, help="trial steps per launch shape (0: defaults)")
    ap.add_argument("--cache", default=None, help="autotune cache file (default: a temporary file)")
    a = ap.parse_args(argv)
    cache = a.cache or os.path.join(tempfile.gettempdir(), "sns_autotune_cache.txt")
    forms = {"both": [PRECISION_FP64, PRECISION_FP32], "fp64": [PRECISION_FP64], "fp32": [PRECISION_FP32]}
    for p in forms[a.precision]:
        print(json.dumps(run(a.count, a.steps, a.warmup, p, a.autotune, cache)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
