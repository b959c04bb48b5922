"""Sphere pruning of the RK update (sns_set_sphere_pruning, on by default).

A z-pencil column-block tile (my, mx block) whose smallest |(mx, my)| already lies outside
the sphere |k| <= N/2 holds only modes that the reference's sweep zeroes.  With the state
zero there, the fused forward z + sweep neither loads, transforms nor updates those tiles.
Every value that is computed is computed exactly as without pruning, so the bar is bitwise
equality with pruning off:

* seeded, perturbed fields at 128^3 and 256^3 in both precisions, 3 steps;
* a state set with content outside the sphere (stage 0 must then run unpruned and zero it);
* 512^3 FP32 through the diagnostics (fixed-order reductions of the physical field).
"""
import numpy as np
import pytest

from spectral_solver_b200 import Solver

pytestmark = pytest.mark.gpu

DT = 1e-3


def run(n, precision, prune, steps, u0=None, seed=5):
    with Solver(n, 1600.0, seed=seed, pert_amp=1e-2, pert_kmax=n // 3, precision=precision) as s:
        s.set_sphere_pruning(prune)
        if u0 is not None:
            s.set_state(u0)
        s.step(DT, steps)
        return s.get_state(), s.diagnostics(steps * DT)


def signed_k2(n):
    k = np.fft.fftfreq(n, 1.0 / n)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    return kx ** 2 + ky ** 2 + kz ** 2


@pytest.mark.parametrize("n", [128, 256])
@pytest.mark.parametrize("precision", [0, 1])
def test_pruned_steps_are_bitwise_the_full_steps(n, precision):
    full, d_full = run(n, precision, False, 3)
    pruned, d_pruned = run(n, precision, True, 3)
    for a, b in zip(full, pruned):
        assert np.array_equal(a, b)
    assert d_full == d_pruned


def test_state_with_content_outside_the_sphere():
    n = 128
    with Solver(n, 1600.0, seed=2, pert_amp=1e-2, pert_kmax=20) as s:
        u = s.get_state()
    outside = 4.0 * signed_k2(n) > n * n
    rng = np.random.default_rng(7)
    for c in range(3):
        u[c] = u[c] + outside * 1e-3 * (rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n)))
    full, _ = run(n, 0, False, 2, u0=u)
    pruned, _ = run(n, 0, True, 2, u0=u)
    for a, b in zip(full, pruned):
        assert np.array_equal(a, b)
        assert not np.any(a[outside])  # the first stage zeroed what lay outside


def test_pruned_512_fp32_diagnostics_bitwise():
    n = 512
    d = []
    for prune in (False, True):
        with Solver(n, 1600.0, precision=1) as s:
            s.set_sphere_pruning(prune)
            s.step(DT, 2)
            d.append(s.diagnostics(2 * DT))
    assert d[0] == d[1]


def test_pruning_switch_rejects_bad_values():
    with Solver(16) as s:
        assert s.lib.sns_set_sphere_pruning(s.h, 3) == 1  # SNS_ERR_INVALID
        s.set_sphere_pruning(False)
        s.set_sphere_pruning(True)
