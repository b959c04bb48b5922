#!/usr/bin/env python
"""Benchmark of the pseudo-spectral Taylor-Green RK3 step on B200.

Workload (one "step" = one low-storage RK3 step over the whole grid): Taylor-Green vortex,
N = 512^3 (the reference's scheme: phase-shift dealiasing, sphere truncation, explicit
viscosity, Williamson RK3), Re = 1600, dt = 1e-3, in two forms measured in the same run:
the FP32 precision ("mixed") form -- fields in FP32, twiddles / phases generated in FP64,
energy / enstrophy / dissipation reductions in FP64 -- is the headline `value`; the FP64
plain drop-in form runs beside it (`fp64_plain`, `mixed_vs_fp64`), and the gap between the
two forms' E and eps after the same steps is reported (`mixed_error_vs_fp64`).  The state
stays resident in HBM (10 GB FP32, 20 GB FP64: far above the 126 MB L2, so no L2 flush).

Metric: grid-point * RK3-steps per second, in units of 1e9 (Gpt*RK3-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--n 512]
                    [--precision both|fp32|fp64]

With --gpus N > 1 (torchrun, one rank per GPU) every rank steps its own replica (the
path does not shard without an all-to-all transpose, so multi-GPU is replicas only);
`value` is the sum over ranks divided by the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "512³ Gpt·RK3-steps/s mixed vs FP64 plain at ε≤1e-6; served solves/s, p50/p99"
UNIT = "Gpt*RK3-steps/s"
RE = 1600.0
DT = 1e-3

# Algorithmic bytes per launch of each pass, in units of S = N^3 * 8 B (one FP64 real field
# or one half-spectrum complex field): every field read or written once.  At N = 128, 256,
# 512 the forward z pass and the sweep are one fused kernel ("p5_sweep": 12 product fields
# + u + g in, u + g out; g is not read in the first stage, hence 23 on average).
PASS_BYTES_S = {"p1_zinv_phase": 9, "p2_yinv": 12, "p3_xpass": 18, "p3_nyq": 0,
                "p4_yfwd": 24, "p5_zfwd": 24, "p5_sweep": 23}


def live_fraction(n, w):
    """Fraction L of the z-pencil column-block tiles (my, mx block of 128 bytes) that hold a
    mode inside the sphere |k| <= N/2; the sphere pruning skips the rest."""
    tw = 128 // (2 * w)
    ncb = (n // 2 + tw - 1) // tw
    live = 0
    for my in range(n):
        m = my if my <= n // 2 else my - n
        live += sum(1 for cb in range(ncb) if 4 * ((cb * tw) ** 2 + m * m) <= n * n)
    return live / (n * ncb)


def pruned_pass_bytes(n, w):
    """Per-launch bytes (units of S) that the sphere-pruned step moves: the fused forward z +
    sweep loads, transforms and sweeps only the live tiles.  Reported beside the canonical
    model (PASS_BYTES_S, 261 per step), which stays the roofline's algorithmic figure."""
    L = live_fraction(n, w)
    b = dict(PASS_BYTES_S)
    b["p5_sweep"] = 23 * L
    return b, L


def step_bytes_s(L):
    """Bytes per RK3 step in units of S: 3 x (P1 9, P2 12, P3 18, P4 24, P5 24L), which is 261
    without pruning (L = 1)."""
    return 189 + 72 * L
# kernels per RK3 stage at N = 512: P1, P2, P3, P4, the (N/2,0,0) mode, fused P5
LAUNCHES_PER_STEP = 3 * 6
# DRAM traffic per launch per grid point (dram__bytes_read.sum + dram__bytes_write.sum).  The
# x pass and the fused P5 were captured on the 512^3 bench workload itself (one-pass metrics;
# profiles/taylor_green_512_dram_traffic.txt; P5 with the sphere pruning); the other passes
# come from single-launch captures at 256^3 (profiles/k_*_256_fp64.txt), scaled by N^3.
TRAFFIC_PER_POINT = {"p5_sweep": (16.716e9 + 5.166e9) / 512 ** 3, "p3_xpass": (6.696e9 + 12.928e9) / 512 ** 3,
                     "p4_yfwd": 3.268e9 / 256 ** 3, "p1_zinv_phase": 1.166e9 / 256 ** 3,
                     "p2_yinv": 1.582e9 / 256 ** 3}
# The same for the FP32 precision form.
TRAFFIC_PER_POINT_FP32 = {"p3_xpass": (3.485e9 + 6.485e9) / 512 ** 3, "p5_sweep": (9.059e9 + 2.983e9) / 512 ** 3}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.path is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args, backend: str = "nccl"):
    """One process per GPU (torchrun's env).  The process group carries only the barriers
    and the max-over-ranks timing: the replicas share no data."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def _reduce_device(pg):
    return "cuda" if pg.get_backend() == "nccl" else "cpu"


def replica_rate(world: int, n: int, steps: int, ms_max: float) -> float:
    """Whole-job Gpt*RK3-steps/s of `world` replicas of an N^3 solve: every rank stepped
    its own grid `steps` times; the slowest rank's device time is the job's time."""
    return world * n ** 3 * steps / (ms_max / 1e3) / 1e9


def barrier_sync(pg):
    if pg is not None and _reduce_device(pg) == "cpu":
        pg.barrier()
        return
    import torch
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()


def max_over_ranks(pg, value: float) -> float:
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class OracleStages:
    """The CPU oracle (oracle/ref_r2c.py: scipy pocketfft and the element-wise work on every
    host thread) advanced one RK3 stage per sample: stages 0, 1, 2, 0, ... with the Williamson
    coefficients, so three consecutive samples are one whole RK3 step (g carried between
    them).  A sample is N^3 / 3 grid-point * RK3-steps of work."""

    def __init__(self, n: int, precision: str):
        from oracle import ref_r2c
        self.threads = os.cpu_count() or 1
        self.n = n
        self.s = ref_r2c.TaylorGreenR2C(n, RE, workers=self.threads, precision=precision)
        self.k = 0

    def sample(self) -> float:
        t0 = time.perf_counter()
        self.s.stage(DT, self.k % 3)
        self.k += 1
        return time.perf_counter() - t0


def cpu_oracle_rate(n: int, precision: str = "fp64", samples: int = 1):
    """Gpt*RK3-steps/s of the CPU oracle over `samples` consecutive stages at N^3; returns
    (rate, seconds, threads)."""
    o = OracleStages(n, precision)
    secs = sum(o.sample() for _ in range(samples))
    return n ** 3 * (samples / 3.0) / secs / 1e9, secs, o.threads


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_oracle_config1(steps: int = 40):
    """The CPU oracle on configuration 1's grid (64^3 FP64, dt 5e-3): `steps` RK3 steps, for
    comparison with the reference's published single-rank FFTW rates at 64^3."""
    from oracle import ref_r2c
    threads = os.cpu_count() or 1
    s = ref_r2c.TaylorGreenR2C(64, RE, workers=threads)
    s.step(5e-3)  # plans and caches
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step(5e-3)
    dt = time.perf_counter() - t0
    return 64 ** 3 * steps / dt, dt, threads


def workload_config(n: int, head: str, world: int) -> dict:
    """The `config` of the JSON line, the same for both arms (the reference arm runs the
    same workload on the host cores)."""
    cb = 16 if head == "fp64" else 8
    pitch = ((n // 2 + 1) + 128 // cb - 1) // (128 // cb) * (128 // cb)
    # 18 half fields, plus the FP32 form's compensation words of u (3 fields of 2 B per value)
    resident = (18 * n * n * pitch * cb + (3 * n * n * pitch * 2 if head == "fp32" else 0)) / 1e9
    return {"workload": f"Taylor-Green RK3 step, {n}^3, "
                        + ("FP32 precision form (mixed)" if head == "fp32" else "FP64 plain drop-in form")
                        + " (phase-shift dealiasing, sphere truncation, explicit viscosity)",
            "n": n, "precision": head, "reynolds": RE, "dt": DT,
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "l2": f"inputs larger than L2 ({resident:.1f} GB resident)"}


def run_reference(args, world, rank, pg):
    """--impl reference: the reference's CPU path on the host cores, on this arm's workload.
    The reference itself cannot be built here (FFTW3, MPI, AVA and FLUPS are absent), so its
    CPU restatement (the oracle) runs, with every host thread, in the headline's precision
    (the reference's single-precision build for the FP32 form).  Each timed "step" is one
    sample: one RK3 stage at N^3 (a third of an RK3 step, stages cycling 0, 1, 2), since a
    whole 512^3 step takes the CPU tens of seconds; `value` counts N^3 / 3 grid-point *
    RK3-steps per sample, and steps * ms_per_step is the timed region.  One FP64 stage is
    timed after the region for the like-for-like ratio of the FP64 drop-in."""
    if rank != 0:
        return 0
    n = args.n
    head = "fp32" if args.precision in ("both", "fp32") else "fp64"
    o = OracleStages(n, head)
    # warm-up (untimed): one stage at N^3 (pocketfft plans, page-in), the rest at 64^3
    for i in range(args.warmup):
        if i == 0:
            o.sample()
        else:
            cpu_oracle_rate(64, head, 1)
    o.k = 0
    secs = [o.sample() for _ in range(args.steps)]
    total_s = sum(secs)
    value = n ** 3 * (args.steps / 3.0) / total_s / 1e9
    del o
    r64 = s64 = None
    if head == "fp32":
        r64, s64, _ = cpu_oracle_rate(n, "fp64", 1)
    threads = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if head == "fp32" else "f64",
        "data": "synthetic: analytic Taylor-Green initial field (Re=1600)",
        "config": workload_config(n, head, world),
        "each_step": f"one RK3 stage at {n}^3 (stages 0, 1, 2 in turn: three samples are one RK3 step)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} consecutive RK3 stages at {n}^3 of the CPU oracle "
                                   f"(oracle/ref_r2c.py, {head}, scipy pocketfft and element-wise work on "
                                   f"{threads} threads); the reference's FFTW path cannot be built here",
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if r64 is not None:
        line["fp64_stage"] = {"value": r64, "unit": UNIT, "seconds": s64,
                              "what": f"one FP64 RK3 stage at {n}^3 (the FP64 drop-in's CPU counterpart)"}
    print(json.dumps(line), flush=True)
    return 0


def measure_form(args, n, precision, local, pg):
    """Time one form (FP64 plain or FP32 precision) of the step on this rank: warm-up, K
    timed steps on the library's stream with CUDA events, per-pass event times.  Returns
    (solver, dict)."""
    from spectral_solver_b200 import Solver
    s = Solver(n, RE, precision=precision)
    s.step(DT, args.warmup)  # warm-up (untimed)
    barrier_sync(pg)
    with ClockSampler(local) as clk:
        ms = s.time_steps(DT, args.steps)  # CUDA events on the library's launching stream
    barrier_sync(pg)
    clocks = clk.summary()
    ms_max = max_over_ranks(pg, ms)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    value = replica_rate(world, n, args.steps, ms_max)
    # Per-pass device times (events between passes, separate from the timed region).
    prof = s.profile_passes(DT, 1)
    w = 8 if precision == 0 else 4
    S = n ** 3 * w
    # roofline.achieved and the model fraction use the canonical per-pass bytes (261 N^3 w per
    # step, fixed); the sphere-pruned bytes that the fused P5 actually moves are reported beside
    pass_bytes, L = pruned_pass_bytes(n, w)
    top = max(prof, key=prof.get)
    achieved = PASS_BYTES_S[top] * S / (prof[top] / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    traffic_table = TRAFFIC_PER_POINT if precision == 0 else TRAFFIC_PER_POINT_FP32
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (traffic_table[top] * n ** 3) if top in traffic_table else None,
            "kernel": top, "peak_source": f"hbm_gbs {peak_kind}",
            "algorithmic_bytes_per_launch": PASS_BYTES_S[top] * S, "mean_launch_ms": prof[top],
            "pruned_bytes_per_launch": pass_bytes[top] * S}
    return s, {"value": value, "ms_per_step": ms_max / args.steps, "clocks": clocks, "roofline": roof,
               "passes_ms_per_stage": prof, "live_tile_fraction": L,
               "model_roofline_frac": value / (peak / (261 * w)),
               "pruned_bytes_per_point_step": step_bytes_s(L) * w,
               "pruned_model_roofline_frac": value / (peak / (step_bytes_s(L) * w)),
               "steps_done": args.warmup + args.steps + 1}


def e2e_solve(args, s, n, pg):
    """End to end through the C ABI with host buffers: upload the initial spectral state from
    pinned host memory, K steps each followed by a diagnostics row read back to the host,
    then the final physical velocity read back -- a whole solve from the user's side."""
    import ctypes as C
    import numpy as np
    import torch
    from spectral_solver_b200 import _lib
    state = s.get_state()
    pin = [torch.empty(2 * n ** 3, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    for c in range(3):
        pin[c].numpy()[:] = state[c].view(np.float64).reshape(-1)
    out = [torch.empty(n ** 3, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    lib = _lib.load()
    DP = C.POINTER(C.c_double)
    ins = (DP * 3)(*[C.cast(p.data_ptr(), DP) for p in pin])
    outs = (DP * 3)(*[C.cast(p.data_ptr(), DP) for p in out])
    diag = _lib.SnsDiag()
    barrier_sync(pg)
    t0 = time.perf_counter()
    rc = lib.sns_set_state(s.h, ins)
    t = 0.0
    for _ in range(args.steps):
        rc |= lib.sns_step(s.h, DT, 1)
        t += DT
        rc |= lib.sns_diagnostics(s.h, t, C.byref(diag))
    rc |= lib.sns_dump_velocity(s.h, outs)
    e2e_s = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError("e2e run failed: " + lib.sns_last_error(s.h).decode())
    e2e_s = max_over_ranks(pg, e2e_s)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    units = world * n ** 3 * args.steps
    return {"value": units / e2e_s / 1e9, "unit": UNIT,
            # set_state copies columns 0..N/2 of each row of the full-layout spectrum
            "h2d_bytes_per_step": 3 * n * n * (n // 2 + 1) * 16 / args.steps,
            "d2h_bytes_per_step": (3 * n ** 3 * 8 + args.steps * 6 * 8) / args.steps,
            "what": "set_state from pinned host + K x (step + diagnostics row to host) + final velocity to host"}


def run_b200(args, world, rank, local, pg):
    import torch

    n = args.n
    torch.cuda.set_device(local)
    forms = {"fp64": 0, "fp32": 1} if args.precision == "both" else {args.precision: 0 if args.precision == "fp64" else 1}
    results, diags = {}, {}
    head = "fp32" if "fp32" in forms else "fp64"
    e2e = None
    for name, prec in forms.items():
        s, r = measure_form(args, n, prec, local, pg)
        # both forms started from the same Taylor-Green field and took the same steps
        diags[name] = s.diagnostics(DT * r["steps_done"])
        if name == head:
            e2e = e2e_solve(args, s, n, pg)
        s.close()
        results[name] = r

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            # the CPU oracle in the headline's precision (3 stages = one RK3 step at N^3), and
            # one FP64 stage for the FP64 drop-in's like-for-like ratio
            rate, secs, threads = cpu_oracle_rate(n, head, 3)
            rate64, secs64, _ = cpu_oracle_rate(n, "fp64", 1) if head != "fp64" else (rate, secs, threads)
            r64, s64, _ = cpu_oracle_config1()
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"one RK3 step (3 stages) at {n}^3 ({secs:.1f} s) of the CPU oracle (oracle/ref_r2c.py, "
                             f"{head}, scipy pocketfft and element-wise work on {threads} threads); the reference's "
                             f"FFTW path cannot be built here",
                   "cpu_model": cpu_model(),
                   "fp64": {"value": rate64, "unit": UNIT, "sample": f"1 FP64 RK3 stage at {n}^3 ({secs64:.1f} s)"},
                   "config1_64": {"value": r64 / 1e9, "unit": UNIT, "gpt_steps_per_s": r64,
                                  "sample": f"40 RK3 steps at 64^3, dt 5e-3 ({s64:.1f} s, {threads} threads)",
                                  "reference_published_gpt_steps_per_s": [1.39e6, 2.47e6]}}
        r = results[head]
        line = {
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 twiddles, IF exponent and reductions)" if head == "fp32" else "f64",
            "data": "synthetic: analytic Taylor-Green initial field (Re=1600)",
            "config": workload_config(n, head, world),
            "clocks": r["clocks"],
            "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "roofline": r["roofline"],
            "passes_ms_per_stage": r["passes_ms_per_stage"],
            "model_roofline_frac": r["model_roofline_frac"],
            "pruned_bytes_per_point_step": r["pruned_bytes_per_point_step"],
            "pruned_model_roofline_frac": r["pruned_model_roofline_frac"],
            "live_tile_fraction": r["live_tile_fraction"],
            "e2e": e2e,
        }
        if "fp64" in results and head != "fp64":
            f64 = results["fp64"]
            line["fp64_plain"] = {k: f64[k] for k in ("value", "ms_per_step", "model_roofline_frac",
                                                        "pruned_model_roofline_frac", "roofline",
                                                        "passes_ms_per_stage", "clocks")}
            line["mixed_vs_fp64"] = r["value"] / f64["value"]
            d32, d64 = diags["fp32"], diags["fp64"]
            line["mixed_error_vs_fp64"] = {
                "after_steps": r["steps_done"],
                "abs_kinetic_energy": abs(d32["kinetic_energy"] - d64["kinetic_energy"]),
                "abs_dissipation": abs(d32["dissipation"] - d64["dissipation"]),
                "rel_enstrophy": abs(d32["enstrophy"] - d64["enstrophy"]) / d64["enstrophy"]}
        if cpu is not None:
            line["cpu_baseline"] = cpu
            if "fp64_plain" in line:
                # like for like: the FP64 drop-in over the FP64 CPU oracle, the FP32 form over
                # the FP32 one
                line["fp64_plain"]["vs_cpu_fp64"] = line["fp64_plain"]["value"] / cpu["fp64"]["value"]
            line["vs_cpu_same_precision"] = r["value"] / cpu["value"]
        extra = run_multi(args) if world == 1 else {}
        line.update(extra)
        print(json.dumps(line), flush=True)
    return 0


def run_multi(args):
    """The batched-ensemble and serving legs of the metric, shortened so the run stays within
    minutes: the 64-solve ensemble for --ensemble-steps graph steps per form, and the
    serving stream's first --serve-seconds of arrivals served to completion per form."""
    out = {}
    if args.ensemble_steps > 0:
        from spectral_solver_b200 import ensemble
        out["ensemble"] = [ensemble.run(64, args.ensemble_steps, 3, p, 2, None) for p in (1, 0)]
    if args.serve_seconds > 0:
        from spectral_solver_b200 import serve
        stream = serve.make_stream(args.serve_seconds, 20.0)
        out["serving"] = [serve.run(stream, int(80e9), p) for p in (1, 0)]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ensemble-steps", type=int, default=50,
                    help="steps of the 64-solve batched ensemble per form (0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=2.0,
                    help="seconds of the serving stream's arrivals served per form (0: skip)")
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "fp64"],
                    help="both: the FP32 precision form is the headline, the FP64 plain form runs beside it")
    args = ap.parse_args()
    if args.impl == "reference":
        # CPU-only arm: no process group; under torchrun rank 0 alone runs
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), None)
    world, rank, local, pg = dist_setup(args)
    try:
        return run_b200(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
