"""Seeded solenoidal k^(-5/3) perturbation: the oracle's restatement of the spec.

TEST INFRASTRUCTURE ONLY (used by tests and the CPU legs of ``bench.py``).

The reference has no perturbed initial condition (its AVA path starts from the pure
Taylor-Green field, ``ava_taylor_green_impl.hpp:796-817``).  The perturbation is new in
this project and is specified once; the device library implements the same definition
(``perturbation_entries`` in ``spectral_solver_b200/csrc/sns_api.cu``) and the tests check the two agree.

Specification (half spectrum, reference full-layout flat index):
  * modes m = (mx, my, mz), mx in [0, N/2], my, mz signed in (-N/2, N/2], with
    1 <= |m|^2 <= kmax^2;
  * in the plane mx = 0 only the canonical half (my > 0, or my == 0 and mz > 0) draws
    random numbers; its mirror (0, -my, -mz) receives the complex conjugate;
  * component c of mode m: amplitude |m|^(-5/3), phase 2*pi*theta with
    theta = (splitmix64(splitmix64(seed) ^ (3*flat + c)) >> 11) * 2^-53 and
    flat = mx + N*((my mod N) + N*(mz mod N));
  * the vector is Leray-projected, u -= m (m.u)/|m|^2;
  * the whole field is scaled so that sqrt(<|u'|^2>) over the physical grid equals
    ``amp`` (Parseval: <|u'|^2> = sum over the full spectrum of |u'_m|^2 / N^6).
"""
from __future__ import annotations

import numpy as np

from .ref_c2c import signed_mode

M64 = (1 << 64) - 1


def splitmix64_np(x: np.ndarray) -> np.ndarray:
    """SplitMix64 output function (Steele, Lea, Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)).astype(np.uint64)
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)).astype(np.uint64)
        return z ^ (z >> np.uint64(31))


def perturbation_half(n: int, seed: int, amp: float, kmax: int) -> list[np.ndarray]:
    """Return the 3 perturbation components on the half spectrum ``[iz, iy, mx]``."""
    out = [np.zeros((n, n, n // 2 + 1), np.complex128) for _ in range(3)]
    if amp == 0.0 or kmax < 1:
        return out
    if 2 * kmax >= n:
        raise ValueError("perturbation kmax must be below N/2")
    m = signed_mode(np.arange(n), n).astype(np.int64)
    mx = np.arange(n // 2 + 1, dtype=np.int64)
    MZ, MY, MX = np.meshgrid(m, m, mx, indexing="ij")
    k2 = MX * MX + MY * MY + MZ * MZ
    sel = (k2 >= 1) & (k2 <= kmax * kmax)
    canon = (MX > 0) | (MY > 0) | ((MY == 0) & (MZ > 0))
    gen = sel & canon
    iz, iy, ix = np.nonzero(gen)
    gx, gy, gz = MX[gen], MY[gen], MZ[gen]
    flat = (gx + n * ((gy % n) + n * (gz % n))).astype(np.uint64)
    kk = k2[gen].astype(np.float64)
    a = np.sqrt(kk) ** (-5.0 / 3.0)
    h = splitmix64_np(np.array([seed], dtype=np.uint64))[0]
    vals = []
    for c in range(3):
        r = splitmix64_np(h ^ (np.uint64(3) * flat + np.uint64(c)))
        theta = (r >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
        ang = 2.0 * np.pi * theta
        vals.append(a * (np.cos(ang) + 1j * np.sin(ang)))
    fx, fy, fz = gx.astype(np.float64), gy.astype(np.float64), gz.astype(np.float64)
    dot = (vals[0] * fx + vals[1] * fy) + vals[2] * fz
    fac = dot / kk
    vals = [vals[0] - fac * fx, vals[1] - fac * fy, vals[2] - fac * fz]
    # Parseval over the full spectrum: every generated mode has a distinct mirror -m there
    # (kmax < N/2 excludes every self-conjugate point), so each counts twice.
    total = 2.0 * float(np.sum(np.abs(vals[0]) ** 2 + np.abs(vals[1]) ** 2 + np.abs(vals[2]) ** 2))
    rms = np.sqrt(total / float(n) ** 6)
    s = amp / rms
    for c in range(3):
        out[c][iz, iy, ix] = vals[c] * s
        zero_plane = gx == 0
        out[c][(-gz[zero_plane]) % n, (-gy[zero_plane]) % n, 0] = np.conj(vals[c][zero_plane] * s)
    return out
