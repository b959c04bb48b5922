"""Error of the FP32 precision form against the FP64 plain form over a long run.

The precision configuration: the Taylor-Green vortex at Re 1600 with a fixed step (1e-3 at
512^3) run to t = 20 in both forms from the same initial field, E, eps and enstrophy every
`--output-dt`.  Reports, as the target asks:
  * max_t |E32 - E64| and max_t |eps32 - eps64|, absolute and relative to max_t of the FP64
    value;
  * the time of peak dissipation in each form and their difference;
  * the relative L2 error of the final velocity (spectral state, stored half mx <= N/2).
Trajectories separate after the transition (t >~ 9) by the flow's own sensitivity, so the
errors are also reported for t <= 9.

    python -m spectral_solver_b200.precision_report [--n 512] [--dt 1e-3] [--t-end 20]
                                                    [--output-dt 0.1] [--csv out.csv]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from ._lib import PRECISION_FP32, PRECISION_FP64, Solver


def summarize(a, b, state32, state64):
    """The report's figures from the two diagnostic series (rows t, E, eps, enstrophy; `a` the
    FP32 form, `b` the FP64 form, same output times) and the two final spectral states."""
    t = b[:, 0]

    def gaps(mask):
        dE = np.abs(a[mask, 1] - b[mask, 1])
        dEps = np.abs(a[mask, 2] - b[mask, 2])
        return {"max_abs_E": float(dE.max()), "max_rel_E": float(dE.max() / np.abs(b[mask, 1]).max()),
                "max_abs_eps": float(dEps.max()), "max_rel_eps": float(dEps.max() / np.abs(b[mask, 2]).max())}

    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(state32, state64))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in state64)
    ip32, ip64 = int(np.argmax(a[:, 2])), int(np.argmax(b[:, 2]))
    return {"whole_run": gaps(np.ones_like(t, dtype=bool)), "up_to_t9": gaps(t <= 9.0 + 1e-12),
            "peak_eps": {"t_fp64": float(t[ip64]), "t_fp32": float(t[ip32]),
                         "abs_dt": float(abs(t[ip32] - t[ip64])), "eps_fp64": float(b[ip64, 2]),
                         "eps_fp32": float(a[ip32, 2])},
            "final_velocity_rel_l2": (num / den) ** 0.5}


def run(n=512, dt=1e-3, t_end=20.0, output_dt=0.1, reynolds=1600.0, seed=0, pert_amp=0.0, pert_kmax=0):
    per_out = max(1, int(round(output_dt / dt)))
    nsteps = int(round(t_end / dt))
    series = {"t": []}
    states = {}
    walls = {}
    for name, prec in (("fp64", PRECISION_FP64), ("fp32", PRECISION_FP32)):
        # each form starts from the analytic field, initialised in its own precision (as a
        # user runs it)
        with Solver(n, reynolds, seed=seed, pert_amp=pert_amp, pert_kmax=pert_kmax, precision=prec) as s:
            rows = []
            t0 = time.perf_counter()
            done = 0
            d = s.diagnostics(0.0)
            rows.append((0.0, d["kinetic_energy"], d["dissipation"], d["enstrophy"]))
            while done < nsteps:
                k = min(per_out, nsteps - done)
                s.step(dt, k)
                done += k
                d = s.diagnostics(done * dt)
                rows.append((done * dt, d["kinetic_energy"], d["dissipation"], d["enstrophy"]))
            walls[name] = time.perf_counter() - t0
            # keep the stored half (mx in [0, N/2]) of the final state: host memory at 512^3
            states[name] = [np.ascontiguousarray(c[..., : n // 2 + 1]) for c in s.get_state()]
        series[name] = np.array(rows)
    report = summarize(series["fp32"], series["fp64"], states["fp32"], states["fp64"])
    report.update({"n": n, "dt": dt, "t_end": t_end, "steps": nsteps, "reynolds": reynolds, "wall_s": walls})
    return report, series


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--t-end", type=float, default=20.0)
    ap.add_argument("--output-dt", type=float, default=0.1)
    ap.add_argument("--csv", default=None, help="write t, E64, eps64, E32, eps32 to this file")
    a = ap.parse_args(argv)
    report, series = run(a.n, a.dt, a.t_end, a.output_dt)
    if a.csv:
        b, c = series["fp64"], series["fp32"]
        np.savetxt(a.csv, np.column_stack([b[:, 0], b[:, 1], b[:, 2], c[:, 1], c[:, 2]]), delimiter=",",
                   header="t,E_fp64,eps_fp64,E_fp32,eps_fp32", comments="")
    print(json.dumps(report), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
