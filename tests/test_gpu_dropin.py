"""The C++ drop-in layer and the configuration-level parity pins, on the GPU.

* the reference's own C++ tests (cpp_tests/spectral_ns_tests.cpp) compiled against
  SpectralNavierStokes over B200Fft3D;
* configuration 1 (64^3, Re 1600, dt 5e-3, 200 steps, a CSV row every step, final
  velocity) through the CLI, against the CPU oracle row by row;
* the reference's published FP64 finals at t = 20 (Benchmark.md:644-649, 749-754,
  777-782) through the CLI with the benchmark's flags;
* configuration 2's seeded field at 256^3: one RHS against the oracle (1e-12 relative L2), and
  its 100-step trajectory against the oracle's (a committed fixture), E and eps within 1e-10;
* 100 steps of the seeded field at 128^3: kinetic energy and dissipation within 1e-10.
"""
import csv
import os
import re
import subprocess

import numpy as np
import pytest

from oracle.ref_r2c import TaylorGreenR2C, half_to_full
from oracle.perturbation import perturbation_half
from oracle.run import RunConfig, run_taylor_green, rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "spectral_solver_b200", "bin")


def run_cli(args, outdir, timeout=900):
    r = subprocess.run([os.path.join(BIN, "taylor_green_b200"), *args, "--output-dir", str(outdir)],
                       capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr + r.stdout
    with open(os.path.join(outdir, "taylor_green_diagnostics.csv")) as f:
        rows = [{k: float(v) for k, v in row.items()} for row in csv.DictReader(f)]
    return rows, r.stdout


def test_reference_cpp_tests_on_b200_backend(tmp_path):
    # the binary writes its vorticity PPMs into the working directory
    r = subprocess.run([os.path.join(BIN, "spectral_ns_b200")], capture_output=True, text=True, timeout=300,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "all C++ spectral tests passed" in r.stdout


def test_config1_cli_matches_oracle(tmp_path):
    rows, _ = run_cli(["--n", "64", "--re", "1600", "--adaptive-cfl", "0", "--dt", "0.005", "--steps", "200",
                       "--output-every", "1", "--dump-final", "1"], tmp_path)
    assert len(rows) == 201
    o = TaylorGreenR2C(64, 1600.0)
    ref, _ = run_taylor_green(o, RunConfig(n=64, steps=200, dt=0.005, output_every=1, reynolds=1600.0))
    assert len(ref) == 201
    for a, b in zip(rows, ref):
        assert abs(a["t"] - b["t"]) < 1e-12
        for key in ("kinetic_energy", "dissipation", "enstrophy", "max_velocity", "cfl"):
            assert rel(a[key], b[key]) <= 1e-10 or abs(a[key] - b[key]) < 1e-300, (key, a["t"], a[key], b[key])
        assert a["max_spectral_divergence"] < 1e-10
    # final velocity dump: header + 3 x 64^3 doubles, against the oracle's physical field
    raw = open(os.path.join(tmp_path, "velocity_final.bin"), "rb").read()
    assert raw[:8] == b"SNSVEL01"
    n = int(np.frombuffer(raw[8:16], np.int64)[0])
    assert n == 64
    vel = np.frombuffer(raw[16:], np.float64).reshape(3, n, n, n)
    ref_vel = o.velocity()
    assert max(float(np.max(np.abs(vel[c] - ref_vel[c]))) for c in range(3)) < 1e-10


@pytest.mark.parametrize("n", [64, 128, 256])
def test_golden_t20_through_cli(tmp_path, n):
    from tests.conftest import golden_finals
    g = golden_finals()[n]  # the reference's published FP64 finals (tests/golden/)
    steps, e, eps, umax = g["steps"], g["kinetic_energy"], g["dissipation"], g["max_velocity"]
    rows, out = run_cli(["--n", str(n), "--re", "1600", "--adaptive-cfl", "1", "--dt", "0.5", "--cfl", "0.5",
                         "--t-end", "20", "--output-dt", "1", "--print-every", "20"], tmp_path, timeout=1800)
    assert len(rows) == 21
    m = re.search(r"step_calls=(\d+)", out)
    assert m and int(m.group(1)) == steps
    last = rows[-1]
    assert abs(last["t"] - 20.0) < 1e-12
    assert rel(last["kinetic_energy"], e) < 1e-10
    assert rel(last["dissipation"], eps) < 1e-10
    assert rel(last["max_velocity"], umax) < 1e-9


def seeded_oracle(n, seed=0, amp=1e-3, kmax=8):
    o = TaylorGreenR2C(n, 1600.0)
    p = perturbation_half(n, seed, amp, kmax)
    for c in range(3):
        o.u_hat[c] = o.u_hat[c] + p[c]
    o.project_truncate(o.u_hat)
    return o


def rel_l2(a, b):
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in b)
    return np.sqrt(num / den)


def test_config2_seeded_rhs_256():
    from spectral_solver_b200 import Solver
    n = 256
    o = seeded_oracle(n)
    with Solver(n, 1600.0, seed=0, pert_amp=1e-3, pert_kmax=8) as s:
        u = s.get_state()
        assert rel_l2(u, [half_to_full(c) for c in o.u_hat]) < 1e-13
        r = s.rhs(u)
    r_ref = [half_to_full(c) for c in o.compute_rhs()]
    assert rel_l2(r, r_ref) < 1e-12


def test_seeded_trajectory_128_100_steps():
    from spectral_solver_b200 import Solver
    n, dt = 128, 2.5e-3
    o = seeded_oracle(n)
    worst = 0.0
    with Solver(n, 1600.0, seed=0, pert_amp=1e-3, pert_kmax=8) as s:
        for k in range(10):
            s.step(dt, 10)
            for _ in range(10):
                o.step(dt)
            d, dr = s.diagnostics(), o.diagnostics(0.0)
            for key in ("kinetic_energy", "dissipation"):
                worst = max(worst, rel(d[key], dr[key]))
    assert worst <= 1e-10, worst


def test_config2_trajectory_256_100_steps():
    """Configuration 2 itself: the seeded 256^3 field, dt = 2.5e-3, 100 steps of the FP64
    drop-in against the CPU oracle's trajectory (tests/golden/config2_256_trajectory.json,
    made by tests/golden/make_config2_trajectory.py; the oracle takes ~35 min for it).
    E, dissipation and enstrophy within 1e-10 relative every 10 steps; the final state's
    per-component energy within 1e-10 relative and sampled modes within 1e-11 of the largest
    mode amplitude."""
    import json
    from spectral_solver_b200 import Solver
    with open(os.path.join(ROOT, "tests", "golden", "config2_256_trajectory.json")) as f:
        gold = json.load(f)
    n, dt = gold["n"], gold["dt"]
    rows = {r["step"]: r for r in gold["rows"]}
    with Solver(n, gold["reynolds"], seed=gold["seed"], pert_amp=gold["pert_amp"], pert_kmax=gold["pert_kmax"]) as s:
        done = 0
        for step in sorted(rows):
            s.step(dt, step - done)
            done = step
            d, ref = s.diagnostics(step * dt), rows[step]
            for key in ("kinetic_energy", "dissipation", "enstrophy"):
                assert rel(d[key], ref[key]) <= 1e-10, (step, key, d[key], ref[key])
            assert rel(d["max_velocity"], ref["max_velocity"]) <= 1e-9
        assert done == gold["steps"] == 100
        u = s.get_state()
    half = [c[..., : n // 2 + 1] for c in u]
    w = np.full(n // 2 + 1, 2.0)
    w[0] = w[-1] = 1.0
    for c in range(3):
        assert rel(float(np.sum(w * np.abs(half[c]) ** 2)), gold["final_weighted_energy"][c]) <= 1e-10
    amax = max(float(np.max(np.abs(c))) for c in half)
    for smp in gold["final_samples"]:
        mz, my, mx = smp["mode"]
        for c in range(3):
            want = complex(smp["re"][c], smp["im"][c])
            assert abs(half[c][mz % n, my % n, mx] - want) <= 1e-11 * amax, (smp["mode"], c)


def test_rhs_512_seeded():
    """The 512^3 pass variants (radix-32 split over lane pairs in the x pass, two TMA
    boxes per tile in the y/z passes) against the oracle: one RHS, 1e-12 relative L2."""
    from spectral_solver_b200 import Solver
    n = 512
    o = seeded_oracle(n, seed=3, amp=1e-2, kmax=16)
    with Solver(n, 1600.0, seed=3, pert_amp=1e-2, pert_kmax=16) as s:
        u = s.get_state()
        assert rel_l2(u, [half_to_full(c) for c in o.u_hat]) < 1e-13
        r = s.rhs(u)
    del u
    r_ref = [half_to_full(c) for c in o.compute_rhs()]
    assert rel_l2(r, r_ref) < 1e-12


@pytest.mark.parametrize("adaptive", [0, 1])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_checkpoint_resume_is_exact(tmp_path, adaptive, precision):
    """A run interrupted at a checkpoint and resumed with --restart writes the same rows as
    the uninterrupted run, bit for bit (the checkpoint holds the exact spectral state)."""
    flags = ["--n", "48", "--re", "800", "--seed", "3", "--pert-amp", "1e-3", "--pert-kmax", "6",
             "--precision", precision]
    if adaptive:
        # the 0.02 cap sets every step (the CFL step is ~0.065): 20 steps reach t = 0.4
        flags += ["--adaptive-cfl", "1", "--dt", "0.02", "--cfl", "0.5", "--t-end", "1.0", "--output-dt", "0.1"]
    else:
        flags += ["--adaptive-cfl", "0", "--dt", "0.01", "--steps", "40", "--output-every", "5"]
    full, _ = run_cli(flags, tmp_path / "full")
    # the interrupted run: stops early, leaving checkpoint.bin at step 20
    part_flags = list(flags)
    if adaptive:
        part_flags[part_flags.index("--t-end") + 1] = "0.45"
    else:
        part_flags[part_flags.index("--steps") + 1] = "23"
    run_cli(part_flags + ["--checkpoint-every", "10"], tmp_path / "part")
    ckpt = tmp_path / "part" / "checkpoint.bin"
    raw = open(ckpt, "rb").read(40)
    assert raw[:8] == b"SNSCKPT1" and int(np.frombuffer(raw[32:40], np.int64)[0]) == 20
    # resume into a copy of the first 20 steps' CSV rows
    os.makedirs(tmp_path / "resumed")
    with open(tmp_path / "part" / "taylor_green_diagnostics.csv") as f:
        lines = f.read().splitlines()
    t_ck = float(np.frombuffer(raw[24:32], np.float64)[0])
    keep = [lines[0]] + [ln for ln in lines[1:] if float(ln.split(",")[0]) < t_ck - 1e-12 or
                         (adaptive and abs(float(ln.split(",")[0]) - t_ck) < 1e-12)]
    with open(tmp_path / "resumed" / "taylor_green_diagnostics.csv", "w") as f:
        f.write("\n".join(keep) + "\n")
    resumed, out = run_cli(flags + ["--restart", str(ckpt)], tmp_path / "resumed")
    assert "resumed from" in out
    assert len(resumed) == len(full)
    for a, b in zip(resumed, full):
        assert a == b
