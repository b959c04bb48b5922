"""The generic-shape device path (sns_fft3d_*) against numpy and the legacy-solver oracle.

FftwFft3D accepts any grid with every n > 1 and any box lengths (src/fftw_fft.cpp:8-36), and
SpectralNavierStokes has a plain-product branch (src/spectral_solver.cpp:160-240).  Here:
* forward / backward on anisotropic and odd shapes (radices up to 16 and a prime above 16 as
  a direct DFT) against numpy's fftn / ifftn, max error <= 1e-12 * max|X|;
* rhs, nonlinear_rhs (phase-shift pair and plain product), step_rk3, the diagnostics,
  product_dealiased and the vorticity slice against oracle/legacy.py with L = (1, 2, 3):
  relative L2 (or relative) <= 1e-12;
* the transform-only handle's device bytes: one complex + one real field plus the twiddles.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.legacy import LegacyNS

pytestmark = pytest.mark.gpu

SHAPES = [(12, 16, 24), (32, 48, 64), (10, 15, 7), (17, 8, 6), (2, 3, 5), (100, 30, 9), (256, 4, 2)]


def rel_l2(a, b):
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in b)
    return np.sqrt(num / den)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("shape", SHAPES)
def test_forward_backward_any_shape(shape):
    from spectral_solver_b200 import Fft3D
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 1000 + ny * 10 + nz)
    x = rng.standard_normal((nz, ny, nx))
    with Fft3D(shape, (1.0, 2.0, 3.0)) as f:
        X = f.forward(x)
        ref = np.fft.fftn(x)
        assert np.max(np.abs(X - ref)) <= 1e-12 * np.max(np.abs(ref))
        c = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
        y = f.backward(c)
        yref = np.fft.ifftn(c).real
        assert np.max(np.abs(y - yref)) <= 1e-12 * np.max(np.abs(yref))
        assert f.device_bytes() == 24 * nx * ny * nz + 16 * (nx + ny + nz)


def seeded_state(s, seed=5):
    rng = np.random.default_rng(seed)
    return s.truncate(s.project([s.forward(rng.standard_normal(s.shape_zyx)) for _ in range(3)]))


@pytest.mark.parametrize("dealias", [True, False])
@pytest.mark.parametrize("shape,lengths", [((12, 16, 24), (1.0, 2.0, 3.0)), ((20, 10, 14), (2 * np.pi, 1.5, 4.0)),
                                           ((16, 16, 16), (2 * np.pi,) * 3)])
def test_rhs_and_nonlinear_match_oracle(shape, lengths, dealias):
    from spectral_solver_b200 import Fft3D
    nu = 0.01
    o = LegacyNS(shape, lengths, nu, dealias=dealias)
    u = seeded_state(o)
    with Fft3D(shape, lengths) as f:
        assert rel_l2(f.rhs(u, nu, dealias, full=True), o.rhs(u)) <= 1e-12
        assert rel_l2(f.rhs(u, nu, dealias, full=False), o.nonlinear_rhs(u)) <= 1e-12


@pytest.mark.parametrize("dealias", [True, False])
def test_step_and_diagnostics_match_oracle(dealias):
    from spectral_solver_b200 import Fft3D
    shape, lengths, nu, dt = (12, 16, 24), (1.0, 2.0, 3.0), 0.02, 1e-3
    o = LegacyNS(shape, lengths, nu, dealias=dealias)
    u = seeded_state(o, 7)
    ref = u
    for _ in range(3):
        ref = o.step_rk3(ref, dt)
    with Fft3D(shape, lengths) as f:
        got = f.step(u, nu, dt, 3, dealias)
        assert rel_l2(got, ref) <= 1e-12
        d, dr = f.diagnostics(got, nu), o.diagnostics(ref)
    for key in ("kinetic_energy", "enstrophy", "dissipation", "max_velocity"):
        assert rel(d[key], dr[key]) <= 1e-12, key
    assert d["max_spectral_divergence"] <= 1e-10 * max(float(np.max(np.abs(c))) for c in ref)


def test_product_and_vorticity_slice_match_oracle():
    from spectral_solver_b200 import Fft3D
    shape, lengths = (12, 16, 24), (1.0, 2.0, 3.0)
    o = LegacyNS(shape, lengths, 0.01)
    u = seeded_state(o, 9)
    with Fft3D(shape, lengths) as f:
        p = f.product(u[0], u[1])
        assert rel_l2([p], [o.product_dealiased(u[0], u[1])]) <= 1e-12
        for iz in (0, 12, 23):
            w = f.vorticity_slice(u, iz)
            wr = o.vorticity_slice(u, iz)
            assert np.max(np.abs(w - wr)) <= 1e-12 * np.max(np.abs(wr))


def test_rejects_bad_shapes(lib):
    from spectral_solver_b200 import _lib
    h = C.c_void_p()
    assert lib.sns_fft3d_create(1, 8, 8, 1.0, 1.0, 1.0, C.byref(h)) == _lib.SNS_ERR_INVALID
    assert lib.sns_fft3d_create(8, 8, 8, 1.0, -1.0, 1.0, C.byref(h)) == _lib.SNS_ERR_INVALID
    assert lib.sns_fft3d_create(8, 8, 7000, 1.0, 1.0, 1.0, C.byref(h)) == _lib.SNS_ERR_UNSUPPORTED
    assert b"6400" in lib.sns_last_error(None)
