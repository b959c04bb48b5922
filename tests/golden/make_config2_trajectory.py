"""Generate the seeded 256^3 trajectory fixture of the FP64 drop-in (configuration 2).

Configuration 2 is the Taylor-Green field at N = 256, Re = 1600, with the seeded solenoidal
k^(-5/3) perturbation (seed 0, rms amplitude 1e-3, shell 1 <= |m| <= 8), stepped with the
low-storage RK3 scheme at the fixed dt = 2.5e-3.  This script runs the CPU oracle
(oracle/ref_r2c.py, the half-spectrum restatement of the reference's
src/ava_taylor_green_impl.hpp:767-1179) for 100 steps and writes
tests/golden/config2_256_trajectory.json:

* the diagnostics (E, dissipation, enstrophy, max velocity, max |k.u|) every 10 steps;
* the final state's per-component energy sum(|u_hat|^2) over the half spectrum and a few
  sampled modes, so the GPU test can check the field itself, not only its integrals.

The oracle takes about 20 s per step at 256^3 on 8 cores (~35 min in all), which is why the
GPU test reads this fixture instead of running the oracle on the GPU box.

    python tests/golden/make_config2_trajectory.py [--steps 100] [--every 10]
"""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from oracle.perturbation import perturbation_half  # noqa: E402
from oracle.ref_r2c import TaylorGreenR2C  # noqa: E402

N, RE, DT, SEED, AMP, KMAX = 256, 1600.0, 2.5e-3, 0, 1e-3, 8
# sampled modes (mz, my, mx) with mx on the stored half; signed y/z modes as indices
SAMPLES = [(1, 1, 1), (0, 1, 1), (1, 0, 1), (2, 3, 1), (3, 2, 5), (-4, 7, 3), (0, 0, 8), (8, -8, 8), (-11, 5, 13),
           (20, -30, 40), (64, 64, 64), (-100, 17, 90), (0, 0, 128)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                  "config2_256_trajectory.json"))
    a = ap.parse_args()
    o = TaylorGreenR2C(N, RE)
    p = perturbation_half(N, SEED, AMP, KMAX)
    for c in range(3):
        o.u_hat[c] = o.u_hat[c] + p[c]
    o.project_truncate(o.u_hat)
    rows = []
    keys = ("kinetic_energy", "dissipation", "enstrophy", "max_velocity", "max_spectral_divergence")

    def row(step):
        d = o.diagnostics(step * DT)
        rows.append({"step": step, **{k: d[k] for k in keys}})

    row(0)
    t0 = time.time()
    for s in range(1, a.steps + 1):
        o.step(DT)
        if s % a.every == 0 or s == a.steps:
            row(s)
            print(f"step {s}: E={rows[-1]['kinetic_energy']:.17g} ({time.time() - t0:.0f} s)", flush=True)
    # mx = 0 and mx = N/2 columns hold Hermitian pairs twice; weight them once
    w = np.full(N // 2 + 1, 2.0)
    w[0] = w[-1] = 1.0
    energy = [float(np.sum(w * np.abs(c) ** 2)) for c in o.u_hat]
    samples = []
    for mz, my, mx in SAMPLES:
        v = [o.u_hat[c][mz % N, my % N, mx] for c in range(3)]
        samples.append({"mode": [mz, my, mx], "re": [float(x.real) for x in v], "im": [float(x.imag) for x in v]})
    out = {"what": "configuration 2: seeded Taylor-Green, N=256, Re=1600, dt=2.5e-3, FP64 CPU oracle",
           "n": N, "reynolds": RE, "dt": DT, "seed": SEED, "pert_amp": AMP, "pert_kmax": KMAX,
           "steps": a.steps, "rows": rows, "final_weighted_energy": energy, "final_samples": samples}
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(f"wrote {a.out}")


if __name__ == "__main__":
    main()
