"""Oracle pins: the reference's own test assertions and its published FP64 golden run.

The oracle (``oracle/``) is the CPU restatement every GPU parity test compares against;
these tests pin it to ovankerm/Spectral_solver before it is trusted:
  * ``cpp_tests/spectral_ns_tests.cpp:16-51`` (12^3 grid, nu = 0.05): FFT round trip,
    projected TGV energy / divergence, one RK3 step decreasing energy;
  * ``Benchmark.md:644-649`` (FFTW FP64, 64^3, adaptive CFL 0.5, dt cap 0.5, t_end 20,
    output_dt 1): 352 steps, final E / dissipation / enstrophy / max velocity.
"""
import numpy as np
import pytest

from oracle.ref_c2c import TaylorGreenC2C
from oracle.ref_r2c import TaylorGreenR2C, full_to_half, half_to_full
from oracle.perturbation import perturbation_half
from oracle.run import RunConfig, run_taylor_green, rel


def test_reference_fft_roundtrip_12():
    """spectral_ns_tests.cpp:16-32: max |u - B(F(u))| < 1e-10."""
    n = 12
    i = np.arange(n)
    u = np.sin(2 * np.pi * (i[None, None, :] + 0.5) / n) + 0.25 * np.cos(2 * np.pi * (i[None, :, None] + 0.5) / n)
    u = np.broadcast_to(u, (n, n, n))
    s = TaylorGreenC2C(n, 20.0)
    assert np.max(np.abs(u - s.backward_real(s.forward(u)))) < 1e-10


@pytest.mark.parametrize("cls", [TaylorGreenC2C, TaylorGreenR2C])
def test_reference_projection_and_energy_12(cls):
    """spectral_ns_tests.cpp:34-41: divergence < 1e-8 and |E - 0.125| < 1e-12."""
    s = cls(12, 20.0)
    d = s.diagnostics(0.0)
    assert d["max_spectral_divergence"] < 1e-8
    assert abs(d["kinetic_energy"] - 0.125) < 1e-12


@pytest.mark.parametrize("cls", [TaylorGreenC2C, TaylorGreenR2C])
def test_reference_viscous_decay_12(cls):
    """spectral_ns_tests.cpp:43-51: one RK3 step (dt = 1e-3, nu = 0.05) reduces E, div < 1e-7."""
    s = cls(12, 20.0)
    e0 = s.diagnostics(0.0)["kinetic_energy"]
    s.step_rk3(1e-3)
    d = s.diagnostics(1e-3)
    assert d["kinetic_energy"] < e0
    assert d["max_spectral_divergence"] < 1e-7


@pytest.mark.parametrize("n", [12, 16, 24])
def test_half_spectrum_matches_full_spectrum(n):
    """The r2c restatement equals the literal c2c one, including complex Nyquist values."""
    a = TaylorGreenC2C(n, 1600.0)
    b = TaylorGreenR2C(n, 1600.0)
    p = perturbation_half(n, 3, 1e-2, max(1, n // 4 - 1))
    for c in range(3):
        b.u_hat[c] += p[c]
    b.project_truncate(b.u_hat)
    full = [half_to_full(c) for c in b.u_hat]
    h = n // 2
    full[1][0, 0, h] = 0.3 + 0.7j
    full[0][0, h, 0] = 0.5 - 0.4j
    full[2][h, 0, 0] = -0.1 + 0.9j
    a.set_state(full)
    b.u_hat = [full_to_half(c) for c in full]
    ra, rb = a.compute_rhs(), b.compute_rhs()
    num = sum(np.sum(np.abs(full_to_half(ra[c]) - rb[c]) ** 2) for c in range(3))
    den = sum(np.sum(np.abs(ra[c]) ** 2) for c in range(3))
    assert np.sqrt(num / den) < 1e-14
    # the reference's RHS is Hermitian away from the self-conjugate points
    fb = [half_to_full(c) for c in rb]
    num = sum(np.sum(np.abs(ra[c] - fb[c]) ** 2) for c in range(3))
    assert np.sqrt(num / den) < 1e-14
    assert abs(rb[1][0, 0, h].imag) > 0  # RHS is complex at the Nyquist point (N/2, 0, 0)


def test_perturbation_spec():
    n, amp = 32, 1e-3
    p = perturbation_half(n, 0, amp, 8)
    full = [half_to_full(c) for c in p]
    phys = [np.fft.ifftn(c) for c in full]
    assert max(np.max(np.abs(x.imag)) for x in phys) < 1e-18
    rms = np.sqrt(np.mean(sum(x.real ** 2 for x in phys)))
    assert abs(rms - amp) < 1e-15
    # solenoidal
    s = TaylorGreenR2C(n, 1600.0)
    ix, iy, iz = s.kvals
    div = p[0] * ix + p[1] * iy + p[2] * iz
    scale = max(np.max(np.abs(c)) for c in p) * 8.0
    assert np.max(np.abs(div)) < 1e-14 * scale
    # seeds differ, same seed reproduces
    assert np.array_equal(perturbation_half(n, 0, amp, 8)[0], p[0])
    assert not np.array_equal(perturbation_half(n, 1, amp, 8)[0], p[0])


def test_oracle_golden_64_adaptive_t20():
    """Benchmark.md:644-649 (FFTW FP64 64^3 to t = 20): 352 steps, E and eps to <= 1e-11."""
    s = TaylorGreenR2C(64, 1600.0)
    cfg = RunConfig(n=64, adaptive_cfl=True, dt=0.5, cfl=0.5, t_end=20.0, output_dt=1.0)
    rows, steps = run_taylor_green(s, cfg)
    assert steps == 352
    assert len(rows) == 21
    last = rows[-1]
    from tests.conftest import golden_finals
    g = golden_finals()[64]  # Benchmark.md:281, 647-648 via tests/golden/benchmark_finals.json
    assert steps == g["steps"]
    assert rel(last["kinetic_energy"], g["kinetic_energy"]) < 1e-11
    assert rel(last["dissipation"], g["dissipation"]) < 1e-11
    assert rel(last["enstrophy"], g["enstrophy"]) < 1e-11
    assert rel(last["max_velocity"], g["max_velocity"]) < 1e-10
    assert last["max_spectral_divergence"] < 1e-11


def test_integrating_factor_oracle_limits():
    """The oracle's integrating-factor RK3: with nu = 0 the factor is 1 and the explicit
    scheme's viscous term is 0, so the two agree bit for bit; with nu > 0 they differ by the
    schemes' truncation error only (dt = 1e-2, 10 steps at 12^3, nu = 0.05)."""
    import numpy as np
    from oracle.ref_r2c import TaylorGreenR2C
    for nu, tol in ((0.0, 0.0), (0.05, 1e-6)):
        a = TaylorGreenR2C(12, 1.0, workers=1)
        b = TaylorGreenR2C(12, 1.0, workers=1, integrating_factor=True)
        a.nu = b.nu = nu
        for _ in range(10):
            a.step(1e-2)
            b.step(1e-2)
        num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a.u_hat, b.u_hat))
        den = sum(float(np.sum(np.abs(y) ** 2)) for y in a.u_hat)
        assert (num / den) ** 0.5 <= tol
        if nu > 0:
            assert num > 0.0


def test_golden_fixture_is_the_published_record():
    """tests/golden/benchmark_finals.json holds the three FP64 runs the parity tests pin
    (64^3 FFTW, 128^3 and 256^3 cuFFT), with the step counts of the same runs."""
    from tests.conftest import golden_finals
    g = golden_finals()
    assert sorted(g) == [64, 128, 256]
    assert [g[n]["steps"] for n in (64, 128, 256)] == [352, 740, 1527]
    assert g[64]["kinetic_energy"] == 0.016877965072920623 and g[256]["dissipation"] == 0.0019036857700047299
    for r in g.values():
        assert all(v.startswith("Benchmark.md:") for v in r["source"].values())
