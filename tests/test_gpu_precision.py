"""The FP32 precision form against the FP64 oracle and the FP64 plain form.

Fields are stored and transformed in FP32 (twiddles and phases generated in FP64 and
rounded; energy, enstrophy, dissipation and Nyquist-plane sums accumulated in FP64).
Tolerances, stated per check:
  * FFT backend: max abs error <= 5e-6 * max|X| against numpy's FP64 transform;
  * one RHS: relative L2 <= 2e-5 against the FP64 oracle (the RHS is a difference of
    products, so its relative error is a few FP32 ulps times the condition of the sum);
  * trajectories: |E32 - E64| <= 1e-6 and |eps32 - eps64| <= 1e-6 (absolute), the
    precision form's accuracy target, at every checked step; max |k.u_hat| <= 1e-7 N^3
    (round-off of modes whose amplitude scales with N^3).
"""
import numpy as np
import pytest

from oracle.ref_r2c import TaylorGreenR2C, half_to_full
from oracle.perturbation import perturbation_half

pytestmark = pytest.mark.gpu

FP32 = 1


def rel_l2(a, b):
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in b)
    return np.sqrt(num / den)


@pytest.fixture(scope="module")
def Solver():
    from spectral_solver_b200 import Solver as S
    return S


@pytest.mark.parametrize("n", [16, 48, 64, 128, 256])
def test_fp32_fft_forward_backward(Solver, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n))
    with Solver(n, precision=FP32) as s:
        X = s.forward(x)
        ref = np.fft.fftn(x)
        assert np.max(np.abs(X - ref)) <= 5e-6 * np.max(np.abs(ref))
        c = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
        y = s.backward(c)
        yref = np.fft.ifftn(c).real
        assert np.max(np.abs(y - yref)) <= 5e-6 * np.max(np.abs(yref))


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256])
def test_fp32_rhs_matches_oracle(Solver, n):
    o = TaylorGreenR2C(n, 1600.0)
    p = perturbation_half(n, 3, 1e-2, max(1, min(8, n // 2 - 1)))
    for c in range(3):
        o.u_hat[c] = o.u_hat[c] + p[c]
    o.project_truncate(o.u_hat)
    r_ref = [half_to_full(c) for c in o.compute_rhs()]
    with Solver(n, 1600.0, precision=FP32) as s:
        r = s.rhs([half_to_full(c) for c in o.u_hat])
    assert rel_l2(r, r_ref) < 2e-5


@pytest.mark.parametrize("n", [32, 48, 96, 128, 256])
def test_fp32_diagnostics_match_oracle(Solver, n):
    """Energy, enstrophy, dissipation and vmax of an FP32 state against the FP64 oracle
    (the FP32 rounding of the state bounds the relative error: 1e-6)."""
    o = TaylorGreenR2C(n, 1600.0)
    p = perturbation_half(n, 9, 3e-2, max(1, min(5, n // 2 - 1)))
    for c in range(3):
        o.u_hat[c] = o.u_hat[c] + p[c]
    o.project_truncate(o.u_hat)
    with Solver(n, 1600.0, seed=9, pert_amp=3e-2, pert_kmax=max(1, min(5, n // 2 - 1)), precision=FP32) as s:
        d = s.diagnostics(0.0)
        vmax = s.max_velocity()
    dr = o.diagnostics(0.0)
    for key in ("kinetic_energy", "dissipation", "enstrophy", "max_velocity"):
        assert abs(d[key] - dr[key]) <= 1e-6 * abs(dr[key]), key
    assert abs(vmax - dr["max_velocity"]) <= 1e-6 * dr["max_velocity"]


@pytest.mark.parametrize("n,dt,steps,amp", [(64, 5e-3, 200, 0.0), (128, 2.5e-3, 100, 1e-3), (256, 2.5e-3, 40, 1e-3)])
def test_fp32_trajectory_vs_fp64(Solver, n, dt, steps, amp):
    kmax = 8 if amp else 0
    with Solver(n, 1600.0, seed=0, pert_amp=amp, pert_kmax=kmax) as s64, \
            Solver(n, 1600.0, seed=0, pert_amp=amp, pert_kmax=kmax, precision=FP32) as s32:
        s32.set_state(s64.get_state())  # identical initial state, rounded to FP32
        worst_e = worst_eps = 0.0
        for k in range(0, steps, 10):
            s64.step(dt, 10)
            s32.step(dt, 10)
            d64 = s64.diagnostics(dt * (k + 10))
            d32 = s32.diagnostics(dt * (k + 10))
            worst_e = max(worst_e, abs(d32["kinetic_energy"] - d64["kinetic_energy"]))
            worst_eps = max(worst_eps, abs(d32["dissipation"] - d64["dissipation"]))
            # spectral amplitudes scale with N^3 (unnormalised forward transform): the FP32
            # divergence is round-off of |k||u_hat|, bounded relative to N^3
            assert d32["max_spectral_divergence"] < 1e-7 * n ** 3
        u32, u64 = s32.get_state(), s64.get_state()
    print(f"N={n}: max|dE|={worst_e:.3e} max|d eps|={worst_eps:.3e} velocity rel L2={rel_l2(u32, u64):.3e}")
    assert worst_e <= 1e-6 and worst_eps <= 1e-6
    assert rel_l2(u32, u64) < 1e-4


def test_fp32_512_steps_track_fp64(Solver):
    """The 512^3 kernels of the precision form (two-row x pass, fused P5) against the FP64
    form: both from the analytic field, 20 steps, E and eps within 1e-6."""
    n, dt = 512, 1e-3
    with Solver(n, 1600.0, precision=FP32) as s32:
        s32.step(dt, 20)
        d32 = s32.diagnostics(20 * dt)
    with Solver(n, 1600.0) as s64:
        s64.step(dt, 20)
        d64 = s64.diagnostics(20 * dt)
    assert abs(d32["kinetic_energy"] - d64["kinetic_energy"]) <= 1e-6
    assert abs(d32["dissipation"] - d64["dissipation"]) <= 1e-6
    assert abs(d32["enstrophy"] - d64["enstrophy"]) <= 1e-6 * d64["enstrophy"] * 10
    assert d32["max_spectral_divergence"] < 1e-7 * n ** 3


def test_fp32_compensated_state_round_trips(Solver):
    """get_state returns the compensated value (FP32 value + int8 remainder) and set_state
    of that value restores both parts exactly: continuing from the reloaded state is bitwise
    the uninterrupted run (what checkpoint/resume relies on)."""
    n, dt = 32, 1e-2
    with Solver(n, 1600.0, seed=1, pert_amp=1e-2, pert_kmax=5, precision=FP32) as s:
        s.step(dt, 5)
        a = s.get_state()
        s.set_state(a)
        assert all(np.array_equal(x, y) for x, y in zip(a, s.get_state()))
        s.step(dt, 3)
        c = s.get_state()
    with Solver(n, 1600.0, precision=FP32) as t:
        t.set_state(a)
        t.step(dt, 3)
        d = t.get_state()
    assert all(np.array_equal(x, y) for x, y in zip(c, d))


def test_fp32_compensation_reduces_drift(Solver):
    """With dt = 1e-3 the RK increment is ~1e-3 of |u|, so FP32 rounding of u drops most of
    its low bits every stage; the compensated state keeps them.  After 600 steps at 64^3 the
    compensated FP32 state is at least 4x closer to the FP64 state than the plain one (7.5x
    measured on B200: what is left is the FP32 round-off of the right-hand side)."""
    n, dt, steps = 64, 1e-3, 600
    with Solver(n, 1600.0, seed=2, pert_amp=1e-3, pert_kmax=8) as s64:
        u0 = s64.get_state()
        s64.step(dt, steps)
        ref = s64.get_state()
    errs = {}
    for comp in (True, False):
        with Solver(n, 1600.0, precision=FP32) as s:
            s.set_compensation(comp)
            s.set_state(u0)
            s.step(dt, steps)
            errs[comp] = rel_l2(s.get_state(), ref)
    print(f"velocity rel L2 vs FP64 after {steps} steps: compensated {errs[True]:.3e}, plain {errs[False]:.3e}")
    assert errs[True] <= 0.25 * errs[False]


def test_fp32_compensation_switch(Solver):
    with Solver(16, 1600.0) as s:
        s.set_compensation(False)  # the FP64 form accepts "off" only
        with pytest.raises(Exception):
            s.set_compensation(True)


def test_config3_schedule_256_to_t20_within_1e6(Solver):
    """Configuration 3's schedule (Taylor-Green, Re 1600, dt = 1e-3, 20 000 steps to t = 20,
    diagnostics every 0.1) at 256^3 in both forms: the precision form's E and eps stay within
    1e-6 (absolute) of the FP64 form over the whole run, and the time of peak eps agrees."""
    from spectral_solver_b200 import precision_report
    report, _ = precision_report.run(n=256, dt=1e-3, t_end=20.0, output_dt=0.1)
    print(report)
    assert report["whole_run"]["max_abs_E"] <= 1e-6
    assert report["whole_run"]["max_abs_eps"] <= 1e-6
    assert report["peak_eps"]["abs_dt"] <= 0.1 + 1e-9
