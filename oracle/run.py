"""Run-driver restatement (fixed-dt and adaptive-CFL loops) for the oracle solvers.

TEST INFRASTRUCTURE ONLY.  Restates ``run_taylor_green`` of ovankerm/Spectral_solver
(``src/ava_taylor_green_impl.hpp:1310-1410``) minus the file output: it returns the rows
the reference writes to ``taylor_green_diagnostics.csv`` (columns of :1326).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from .ref_c2c import PI


@dataclass
class RunConfig:
    """Defaults of ``RunConfig`` (``ava_taylor_green.hpp:21-34``)."""
    n: int = 64
    steps: int = 80
    max_steps: int = 10000000
    output_every: int = 1
    print_every: int = 10
    dt: float = 0.0025
    cfl: float = 0.4
    t_end: float = 0.2
    output_dt: float = 0.1
    reynolds: float = 1600.0
    adaptive_cfl: bool = False


COLUMNS = ("t", "kinetic_energy", "dissipation", "enstrophy", "max_spectral_divergence",
           "max_velocity", "dt", "cfl", "main_dt", "main_cfl")


def run_taylor_green(solver, cfg: RunConfig):
    """Return (rows, steps) exactly as the reference loop would produce them."""
    if cfg.dt <= 0.0 or cfg.cfl <= 0.0 or cfg.output_dt <= 0.0:
        raise ValueError("--dt, --cfl, and --output-dt must be positive")  # :1311-1313
    rows = []
    t = 0.0
    step = 0
    dx = 2.0 * PI / float(cfg.n)

    def write_row(time, last_dt, last_cfl, main_dt, main_cfl):
        d = solver.diagnostics(time)
        d.update(dt=last_dt, cfl=last_cfl, main_dt=main_dt, main_cfl=main_cfl)
        rows.append(d)

    if cfg.adaptive_cfl:  # :1355-1388
        next_output = 0.0
        write_row(t, 0.0, 0.0, 0.0, 0.0)
        next_output += cfg.output_dt
        while t < cfg.t_end - 1.0e-14:
            if step >= cfg.max_steps:
                raise RuntimeError("adaptive CFL run exceeded --max-steps before reaching --t-end")
            vmax = solver.max_velocity()
            main_dt = cfg.dt
            if vmax > 1.0e-14:
                main_dt = min(main_dt, cfg.cfl * (2.0 * PI / float(cfg.n)) / vmax)
            main_cfl = vmax * main_dt / dx
            dt_step = main_dt
            dt_step = min(dt_step, cfg.t_end - t)
            if next_output <= cfg.t_end + 1.0e-14:
                dt_step = min(dt_step, next_output - t)
            if dt_step <= 1.0e-14:
                next_output += cfg.output_dt
                continue
            actual_cfl = vmax * dt_step / dx
            solver.step_rk3(dt_step)
            t += dt_step
            step += 1
            if t >= next_output - 1.0e-12 or t >= cfg.t_end - 1.0e-12:
                write_row(t, dt_step, actual_cfl, main_dt, main_cfl)
                while next_output <= t + 1.0e-12:
                    next_output += cfg.output_dt
    else:  # :1389-1401
        for step in range(0, cfg.steps + 1):
            if step % cfg.output_every == 0 or step == cfg.steps:
                fixed_cfl = solver.max_velocity() * cfg.dt / dx
                first = step == 0
                write_row(t, 0.0 if first else cfg.dt, 0.0 if first else fixed_cfl,
                          0.0 if first else cfg.dt, 0.0 if first else fixed_cfl)
            if step != cfg.steps:
                solver.step_rk3(cfg.dt)
                t += cfg.dt
        step = cfg.steps
    return rows, step


def rel(a: float, b: float) -> float:
    return abs(a - b) / max(abs(b), 1e-300)


def isfinite_rows(rows) -> bool:
    return all(math.isfinite(r[c]) for r in rows for c in COLUMNS)
