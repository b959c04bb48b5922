"""The precision-form report's arithmetic (precision_report.summarize) on synthetic series.

Two diagnostic series on the same output times (rows t, E, eps, enstrophy) with known gaps:
the report must give the largest |E32 - E64| and |eps32 - eps64| over the whole run and up to
t = 9 (the output at t = 9 itself included), the times of peak dissipation, and the relative
L2 distance of the final spectral states.
"""
import numpy as np
import pytest

from spectral_solver_b200.precision_report import summarize


def series(t, e, eps):
    return np.column_stack([t, e, eps, 2.0 * eps])


def test_summary_figures():
    t = np.round(np.arange(0, 201) * 0.1, 12)  # 0 .. 20 by 0.1, as the report's outputs
    e64 = 0.125 * np.exp(-0.1 * t)
    eps64 = 0.0128 * np.exp(-((t - 9.0) / 3.0) ** 2)
    de = np.where(t <= 9.0, 1e-8, 0.0)
    de[t == 9.0] = 3e-8                  # the largest gap up to t = 9 sits on t = 9 itself
    de[t == 18.5] = 1.35e-6              # the late-time separation
    deps = np.full_like(t, 2e-9)
    deps[t == 12.0] = -4e-7
    a = series(t, e64 + de, eps64 + deps)
    b = series(t, e64, eps64)
    rng = np.random.default_rng(0)
    s64 = [rng.standard_normal((4, 4, 3)) + 1j * rng.standard_normal((4, 4, 3)) for _ in range(3)]
    s32 = [x * (1 + 1e-3) for x in s64]
    r = summarize(a, b, s32, s64)
    assert r["whole_run"]["max_abs_E"] == pytest.approx(1.35e-6)
    assert r["whole_run"]["max_rel_E"] == pytest.approx(1.35e-6 / 0.125)
    assert r["whole_run"]["max_abs_eps"] == pytest.approx(4e-7)
    assert r["up_to_t9"]["max_abs_E"] == pytest.approx(3e-8)
    assert r["up_to_t9"]["max_abs_eps"] == pytest.approx(2e-9)
    assert r["peak_eps"]["t_fp64"] == 9.0 and r["peak_eps"]["t_fp32"] == 9.0
    assert r["peak_eps"]["abs_dt"] == 0.0
    assert r["final_velocity_rel_l2"] == pytest.approx(1e-3)


def test_peak_time_shift_is_reported():
    t = np.round(np.arange(0, 101) * 0.1, 12)
    eps64 = np.exp(-((t - 5.0) ** 2))
    eps32 = np.exp(-((t - 5.2) ** 2))
    one = [np.ones((2, 2, 2), complex)] * 3
    r = summarize(series(t, np.ones_like(t), eps32), series(t, np.ones_like(t), eps64), one, one)
    assert r["peak_eps"]["t_fp64"] == 5.0 and r["peak_eps"]["t_fp32"] == pytest.approx(5.2)
    assert r["peak_eps"]["abs_dt"] == pytest.approx(0.2)
    assert r["final_velocity_rel_l2"] == 0.0
