"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (FP64 throughout, from the performance target's parity bar):
  * FFT backend: max abs error <= 1e-12 * max|input| * log2(N)-ish (1e-12 relative here);
  * one RHS evaluation: relative L2 <= 1e-12 against the literal c2c oracle;
  * trajectories: kinetic energy and dissipation within 1e-10 relative.
"""
import numpy as np
import pytest

from oracle.ref_c2c import TaylorGreenC2C
from oracle.ref_r2c import TaylorGreenR2C, full_to_half, half_to_full
from oracle.perturbation import perturbation_half

pytestmark = pytest.mark.gpu

SIZES_SMALL = [8, 12, 16, 24, 32, 48, 64]


def rel_l2(a, b):
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in b)
    return np.sqrt(num / den)


def oracle_state(n, seed=0, amp=0.0, kmax=0):
    s = TaylorGreenR2C(n, 1600.0)
    if amp > 0:
        p = perturbation_half(n, seed, amp, kmax)
        for c in range(3):
            s.u_hat[c] = s.u_hat[c] + p[c]
        s.project_truncate(s.u_hat)
    return s


@pytest.fixture(scope="module")
def Solver():
    from spectral_solver_b200 import Solver as S
    return S


@pytest.mark.parametrize("n", SIZES_SMALL + [96, 128])
def test_fft_forward_backward(Solver, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n))
    with Solver(n) as s:
        X = s.forward(x)
        ref = np.fft.fftn(x)
        assert np.max(np.abs(X - ref)) <= 1e-12 * np.max(np.abs(ref))
        # backward of an arbitrary (non-Hermitian) spectrum = Re(IDFT)
        c = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
        y = s.backward(c)
        yref = np.fft.ifftn(c).real
        assert np.max(np.abs(y - yref)) <= 1e-12 * np.max(np.abs(yref))
        # reference test cpp_tests/spectral_ns_tests.cpp:16-32 round trip
        assert np.max(np.abs(s.backward(s.forward(x)) - x)) < 1e-10


@pytest.mark.parametrize("n", SIZES_SMALL)
@pytest.mark.parametrize("amp", [0.0, 1e-2])
def test_initial_state(Solver, n, amp):
    kmax = max(1, min(8, n // 2 - 1)) if amp else 0
    o = oracle_state(n, 5, amp, kmax)
    with Solver(n, 1600.0, seed=5, pert_amp=amp, pert_kmax=kmax) as s:
        u = s.get_state()
    ref = [half_to_full(c) for c in o.u_hat]
    assert rel_l2(u, ref) < 1e-13


@pytest.mark.parametrize("n", SIZES_SMALL)
def test_rhs_matches_reference_c2c(Solver, n):
    """One RHS evaluation against the literal full-spectrum restatement, 1e-12 relative L2."""
    o = oracle_state(n, 11, 5e-2, max(1, min(6, n // 2 - 1)))
    full = [half_to_full(c) for c in o.u_hat]
    h = n // 2
    # complex values at the self-conjugate Nyquist points, as the reference state carries them
    full[1][0, 0, h] += 0.01 + 0.02j
    full[2][0, h, 0] += -0.03 + 0.01j
    full[0][h, 0, 0] += 0.02 - 0.05j
    ref = TaylorGreenC2C(n, 1600.0)
    ref.set_state(full)
    r_ref = ref.compute_rhs()
    with Solver(n, 1600.0) as s:
        r = s.rhs(full)
    assert rel_l2(r, r_ref) < 1e-12


@pytest.mark.parametrize("n", [96, 128])
def test_rhs_matches_oracle_r2c(Solver, n):
    o = oracle_state(n, 2, 1e-2, 8)
    r_ref = [half_to_full(c) for c in o.compute_rhs()]
    with Solver(n, 1600.0) as s:
        r = s.rhs([half_to_full(c) for c in o.u_hat])
    assert rel_l2(r, r_ref) < 1e-12


@pytest.mark.parametrize("n", [12, 32, 48])
def test_steps_match_oracle(Solver, n):
    o = oracle_state(n, 1, 1e-2, max(1, min(4, n // 2 - 1)))
    with Solver(n, 1600.0, seed=1, pert_amp=1e-2, pert_kmax=max(1, min(4, n // 2 - 1))) as s:
        for k in range(5):
            o.step(0.01)
            s.step(0.01)
            d_ref = o.diagnostics(0.01 * (k + 1))
            d = s.diagnostics(0.01 * (k + 1))
            for key in ("kinetic_energy", "dissipation", "enstrophy", "max_velocity"):
                assert abs(d[key] - d_ref[key]) <= 1e-12 * abs(d_ref[key]), (key, d[key], d_ref[key])
            assert d["max_spectral_divergence"] < 1e-9
        u = s.get_state()
    assert rel_l2(u, [half_to_full(c) for c in o.u_hat]) < 1e-12


@pytest.mark.parametrize("n", [12, 48, 64, 96, 128])
def test_diagnostics_match_oracle(Solver, n):
    o = oracle_state(n, 9, 3e-2, max(1, min(5, n // 2 - 1)))
    with Solver(n, 1600.0, seed=9, pert_amp=3e-2, pert_kmax=max(1, min(5, n // 2 - 1))) as s:
        d = s.diagnostics(0.0)
        vmax = s.max_velocity()
        phys = s.dump_velocity()
    dr = o.diagnostics(0.0)
    for key in ("kinetic_energy", "dissipation", "enstrophy", "max_velocity"):
        assert abs(d[key] - dr[key]) <= 1e-13 * abs(dr[key]), key
    assert abs(vmax - dr["max_velocity"]) <= 1e-13 * dr["max_velocity"]
    pr = o.velocity()
    assert max(float(np.max(np.abs(a - b))) for a, b in zip(phys, pr)) < 1e-13


@pytest.mark.parametrize("n", [8, 12, 16])
def test_rhs_unmasked_state_with_nyquist_plane(Solver, n):
    """An arbitrary (unmasked) state: Hermitian away from the planes mx = 0, N/2 and
    arbitrary on them, so the Nyquist plane carries content off (N/2,0,0)."""
    rng = np.random.default_rng(100 + n)
    full = [np.fft.fftn(rng.standard_normal((n, n, n))) * 0.05 for _ in range(3)]
    h = n // 2
    for c in range(3):
        full[c][:, :, 0] += 0.3 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        full[c][:, :, h] += 0.3 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    ref = TaylorGreenC2C(n, 1600.0)
    ref.set_state([c.copy() for c in full])
    r_ref = ref.compute_rhs()
    with Solver(n, 1600.0) as s:
        r = s.rhs(full)
        # and the state path: set, one step, compare with the reference's step
        s.set_state(full)
        d = s.diagnostics(0.0)
        s.step(1e-3)
        u = s.get_state()
    assert rel_l2(r, r_ref) < 1e-12
    dr = ref.diagnostics(0.0)
    for key in ("kinetic_energy", "enstrophy", "max_velocity", "max_spectral_divergence"):
        assert abs(d[key] - dr[key]) <= 1e-12 * abs(dr[key]), key
    ref.step(1e-3)
    assert rel_l2(u, ref.get_state()) < 1e-12
