"""The legacy-solver oracle (oracle/legacy.py) pinned on CPU.

* On the benchmark domain (cubic, L = 2 pi, phase-shift pair) its rhs equals the AVA-path
  restatement's compute_rhs (oracle/ref_c2c.py), which the reference's golden runs pin: the
  reference's two solvers compute the same right-hand side.
* The reference's own C++ tests (cpp_tests/spectral_ns_tests.cpp, 12^3, nu = 0.05) hold on
  it: round trip < 1e-10, projected Taylor-Green E = 0.125 +- 1e-12 and divergence < 1e-8,
  one RK3 step at dt = 1e-3 lowers E with divergence < 1e-7.
* On other domains (anisotropic grids, L = (1, 2, 3), the plain product) its rhs is
  divergence-free and masked.
"""
import numpy as np
import pytest

from oracle.legacy import LegacyNS
from oracle.ref_c2c import TaylorGreenC2C


def test_matches_ava_restatement_on_benchmark_domain():
    n = 16
    ref = TaylorGreenC2C(n, 1600.0)
    rng = np.random.default_rng(4)
    u = [c + 1e-3 * (rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)) * np.abs(c).max()
         for c in ref.u_hat]
    ref.project_truncate(u)
    leg = LegacyNS((n, n, n), (2 * np.pi,) * 3, 1.0 / 1600.0, dealias=True)
    r_ref = ref.compute_rhs(u)
    r = leg.rhs(u)
    num = sum(float(np.sum(np.abs(a - b) ** 2)) for a, b in zip(r, r_ref))
    den = sum(float(np.sum(np.abs(b) ** 2)) for b in r_ref)
    assert (num / den) ** 0.5 < 1e-13


def test_reference_cpp_assertions():
    n = 12
    s = LegacyNS((n, n, n), (2 * np.pi,) * 3, 0.05)
    rng = np.random.default_rng(0)
    f = rng.standard_normal((n, n, n))
    assert np.max(np.abs(s.backward(s.forward(f)) - f)) < 1e-10
    u = s.truncate(s.project([s.forward(c) for c in s.taylor_green()]))
    d = s.diagnostics(u)
    assert abs(d["kinetic_energy"] - 0.125) < 1e-12
    assert d["max_spectral_divergence"] < 1e-8
    d1 = s.diagnostics(s.step_rk3(u, 1e-3))
    assert d1["kinetic_energy"] < d["kinetic_energy"]
    assert d1["max_spectral_divergence"] < 1e-7


@pytest.mark.parametrize("shape,lengths,dealias", [((12, 16, 24), (1.0, 2.0, 3.0), True),
                                                   ((10, 6, 14), (2 * np.pi, 1.5, 4.0), False)])
def test_general_domains_are_consistent(shape, lengths, dealias):
    s = LegacyNS(shape, lengths, 0.01, dealias=dealias)
    rng = np.random.default_rng(1)
    u = s.truncate(s.project([s.forward(rng.standard_normal(s.shape_zyx)) for _ in range(3)]))
    r = s.rhs(u)
    div = s.kx * r[0] + s.ky * r[1] + s.kz * r[2]
    assert np.max(np.abs(div)) < 1e-10 * max(float(np.max(np.abs(c))) for c in r)
    nl = s.nonlinear_rhs(u)
    outside = ~np.broadcast_to(s.keep, s.shape_zyx)
    assert all(np.all(c[outside] == 0) for c in nl)
