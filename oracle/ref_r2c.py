"""CPU oracle, half-spectrum (r2c/c2r) restatement of the reference TGV time step.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` use it.

Same numerics as :mod:`oracle.ref_c2c` (``src/ava_taylor_green_impl.hpp:658-1179`` of
ovankerm/Spectral_solver) but the spectral state is stored on the half spectrum
``mx in [0, N/2]`` with SciPy's pocketfft r2c/c2r (multithreaded through ``workers``),
which makes 256^3 parity checks and the CPU baseline affordable.

Why this is exact.  The reference consumes only the real part of every inverse transform
(``:904-905, :1114, :1131, :1165``), i.e. it computes IDFT(H(c)) with H(c)_m =
(c_m + conj(c_-m))/2.  Away from the planes mx = 0 and mx = N/2 the reference state is
Hermitian, so H(c) = c there; pocketfft's c2r along x takes the real part of the mx = 0
and mx = N/2 bins after the complex y/z inverse transforms, which is exactly H restricted
to those planes.  The three self-conjugate Nyquist points (N/2,0,0), (0,N/2,0), (0,0,N/2)
survive the sphere mask and carry complex values in the reference (``signed_mode`` maps
index N/2 to +N/2, :123-125); the half spectrum stores each of them once, with its full
complex value, so nothing is lost.  ``tests/test_oracle.py`` checks this module against
the literal c2c restatement to round-off.

Arrays are indexed ``[iz, iy, mx]`` (x fastest, as the reference layout).
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft as sfft

from .ref_c2c import PI, signed_mode

WORKERS = int(os.environ.get("SNS_ORACLE_WORKERS", os.cpu_count() or 1))


def half_mode_grids(n: int):
    m = signed_mode(np.arange(n), n).astype(np.int64)
    mxh = np.arange(n // 2 + 1, dtype=np.int64)  # index n/2 -> +n/2
    return mxh[None, None, :], m[None, :, None], m[:, None, None]


def full_to_half(c: np.ndarray) -> np.ndarray:
    """Keep mx in [0, N/2] of a reference full spectrum (indexed [iz, iy, ix])."""
    n = c.shape[-1]
    return np.ascontiguousarray(c[..., : n // 2 + 1])


def half_to_full(h: np.ndarray) -> np.ndarray:
    """Rebuild the reference's full layout: mx < 0 from conj of the mirror mode."""
    n = h.shape[0]
    full = np.zeros((n, n, n), np.complex128)
    full[..., : n // 2 + 1] = h
    ix = np.arange(n // 2 + 1, n)
    src = n - ix  # -mx
    iy = (-np.arange(n)) % n
    iz = (-np.arange(n)) % n
    full[..., n // 2 + 1:] = np.conj(h[iz][:, iy][:, :, src])
    return full


class TaylorGreenR2C:
    """Half-spectrum restatement of ``TaylorGreenSolver::Impl`` with identical numerics."""

    def __init__(self, n: int, reynolds: float, u_hat0=None, workers: int | None = None,
                 integrating_factor: bool = False, rotational: bool = False, precision: str = "fp64"):
        """precision "fp32" runs the same arithmetic on complex64/float32 arrays, as the
        reference's single-precision build does (``Real = float``,
        ``ava_taylor_green_impl.hpp:48-51``); it times the CPU path of the FP32 form and is
        not a parity reference."""
        if n <= 0:
            raise ValueError("grid size must be positive")
        if reynolds <= 0.0:
            raise ValueError("Reynolds number must be positive")
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be fp64 or fp32")
        self.n = n
        self.nu = 1.0 / reynolds
        self.integrating_factor = integrating_factor
        self.rotational = rotational
        self.global_size = n * n * n
        self.workers = WORKERS if workers is None else workers
        self.precision = precision
        self.rdtype = np.float64 if precision == "fp64" else np.float32
        self.cdtype = np.complex128 if precision == "fp64" else np.complex64
        self._pool = None
        mx, my, mz = half_mode_grids(n)
        msum = (mx + my + mz).astype(np.float64)
        angle = (msum * PI) / float(n)  # initialize_metadata :782-783
        self.phase = (np.cos(angle) + 1j * np.sin(angle)).astype(self.cdtype)
        h = 0.5 * float(n)
        m2 = (mx * mx + my * my + mz * mz).astype(np.float64)
        self.keep = (m2 / (h * h)) <= 1.0  # keep_mode_host :131-134
        self.k2 = m2.astype(self.rdtype)
        self.kvals = tuple(k.astype(self.rdtype) for k in (mx, my, mz))
        self.g = [None, None, None]
        if u_hat0 is None:
            self.initialize_velocity()
        else:
            self.u_hat = [np.array(c, self.cdtype, copy=True) for c in u_hat0]

    def _slabs(self, fn):
        """Run fn(s) over z-slabs s that cover axis 0, on the worker threads (numpy releases
        the GIL inside its loops).  Every element is computed by the same expression whatever
        the split, so the results do not depend on the thread count."""
        k = max(1, min(self.workers, self.n))
        if k == 1:
            fn(slice(None))
            return
        if self._pool is None:
            self._pool = ThreadPoolExecutor(k)
        b = np.linspace(0, self.n, k + 1).astype(int)
        list(self._pool.map(fn, [slice(b[i], b[i + 1]) for i in range(k)]))

    def forward(self, phys):
        return sfft.rfftn(phys, workers=self.workers)

    def backward_real(self, spec):
        n = self.n
        return sfft.irfftn(spec, s=(n, n, n), workers=self.workers)

    def initialize_velocity(self):
        n = self.n
        i = np.arange(n, dtype=np.float64)
        c = (i + 0.5) * 2.0 * PI / float(n)
        x, y, z = c[None, None, :], c[None, :, None], c[:, None, None]
        p0 = np.broadcast_to(np.sin(x) * np.cos(y) * np.cos(z), (n,) * 3)
        p1 = np.broadcast_to(-np.cos(x) * np.sin(y) * np.cos(z), (n,) * 3)
        p2 = np.zeros((n, n, n))
        self.u_hat = [self.forward(np.ascontiguousarray(p, dtype=self.rdtype)) for p in (p0, p1, p2)]
        self.project_truncate(self.u_hat)

    def project_truncate(self, f):
        ix, iy, iz = self.kvals
        k2 = self.k2
        ok = (k2 > 0.0) & self.keep
        inv = np.where(k2 > 0.0, 1.0 / np.where(k2 > 0.0, k2, 1.0), 0.0)
        dot = (f[0] * ix + f[1] * iy) + f[2] * iz
        factor = dot * inv
        f[0][...] = np.where(ok, f[0] - factor * ix, 0.0)
        f[1][...] = np.where(ok, f[1] - factor * iy, 0.0)
        f[2][...] = np.where(ok, f[2] - factor * iz, 0.0)

    def nonlinear(self, u_hat):
        """Masked conservative-form nonlinear term only (before viscosity and projection).
        The element-wise work runs on z-slabs in the worker threads (``_slabs``); per element
        it is the reference's expression: value = (c0 + cs conj(phase)) / 2, masked, then
        r_a -= i k_b value and r_b -= i k_a value (:926-936)."""
        phys = [self.backward_real(u) for u in u_hat]
        shift = [self.backward_real(u * self.phase) for u in u_hat]
        rhs = [np.zeros_like(u_hat[0]) for _ in range(3)]
        shape = rhs[0].shape
        keep = np.broadcast_to(self.keep, shape)
        kvb = [np.broadcast_to(k, shape) for k in self.kvals]
        ph = np.broadcast_to(np.conj(self.phase), shape)
        p = np.empty_like(phys[0])
        for a, b in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)):
            def mul0(s):
                np.multiply(phys[a][s], phys[b][s], out=p[s])
            self._slabs(mul0)
            c0 = self.forward(p)

            def muls(s):
                np.multiply(shift[a][s], shift[b][s], out=p[s])
            self._slabs(muls)
            cs = self.forward(p)

            def combine(s):
                value = 0.5 * (c0[s] + cs[s] * ph[s])
                value = np.where(keep[s], value, 0.0)
                rhs[a][s] = rhs[a][s] + (-1j) * kvb[b][s] * value
                if a != b:
                    rhs[b][s] = rhs[b][s] + (-1j) * kvb[a][s] * value
            self._slabs(combine)
        return rhs

    def nonlinear_rotational(self, u_hat):
        """Rotational-form nonlinear term u x omega, omega_hat = i k x u_hat, with the same
        phase-shift dealiasing and sphere mask as the conservative form.  The two forms
        differ by a gradient (removed by the projection) and by their aliasing residue.
        The reference implements only the conservative form; this is the project's own
        specification of the alternative."""
        kx, ky, kz = self.kvals
        w_hat = [1j * (ky * u_hat[2] - kz * u_hat[1]), 1j * (kz * u_hat[0] - kx * u_hat[2]),
                 1j * (kx * u_hat[1] - ky * u_hat[0])]
        u0 = [self.backward_real(u) for u in u_hat]
        w0 = [self.backward_real(w) for w in w_hat]
        us = [self.backward_real(u * self.phase) for u in u_hat]
        ws = [self.backward_real(w * self.phase) for w in w_hat]

        def cross(a, b):
            return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]

        c0, cs = cross(u0, w0), cross(us, ws)
        cphase = np.conj(self.phase)
        return [np.where(self.keep, 0.5 * (self.forward(a) + self.forward(b) * cphase), 0.0) for a, b in zip(c0, cs)]

    def compute_rhs(self, u_hat=None):
        if u_hat is None:
            u_hat = self.u_hat
        rhs = self.nonlinear_rotational(u_hat) if self.rotational else self.nonlinear(u_hat)
        if not self.integrating_factor:
            for c in range(3):
                rhs[c] = rhs[c] - u_hat[c] * (self.nu * self.k2)
        self.project_truncate(rhs)
        return rhs

    def _if_advance(self, u, g, tau):
        # Integrating-factor variant (an option the reference's method notes list, doc.md:325-343,
        # but do not implement): u and g are carried to the next stage time by exp(-nu k^2 tau).
        if self.integrating_factor:
            f = np.exp(-self.nu * self.k2 * tau)
            for c in range(3):
                u[c] = u[c] * f
                g[c] = g[c] * f

    def stage(self, dt: float, s: int):
        """Stage s (0, 1, 2) of the Williamson low-storage RK3 step (``Impl::step``,
        ``ava_taylor_green_impl.hpp:979-1045``): g = a_s g + H(u); u += b_s dt g; P(u)."""
        u, g = self.u_hat, self.g
        r = self.compute_rhs()
        if s == 0:
            for c in range(3):
                g[c] = r[c].copy()
                u[c] = u[c] + g[c] * (dt / 3.0)
            self._if_advance(u, g, dt / 3.0)
        elif s == 1:
            for c in range(3):
                g[c] = g[c] * (-5.0 / 9.0) + r[c]
                u[c] = u[c] + g[c] * (15.0 * dt / 16.0)
            self._if_advance(u, g, 5.0 * dt / 12.0)
        else:
            for c in range(3):
                g[c] = g[c] * (-153.0 / 128.0) + r[c]
                u[c] = u[c] + g[c] * (8.0 * dt / 15.0)
            self._if_advance(u, g, dt / 4.0)
        self.project_truncate(u)

    def step(self, dt: float):
        for s in range(3):
            self.stage(dt, s)

    step_rk3 = step

    def velocity(self):
        return [self.backward_real(u) for u in self.u_hat]

    def max_velocity(self) -> float:
        p = self.velocity()
        return float(np.sqrt(np.max(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])))

    def vorticity_hat(self, u):
        ix, iy, iz = self.kvals
        return [1j * (iy * u[2] - iz * u[1]), 1j * (iz * u[0] - ix * u[2]), 1j * (ix * u[1] - iy * u[0])]

    def diagnostics(self, t: float) -> dict:
        u = self.u_hat
        p = [self.backward_real(c) for c in u]
        s2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2]
        energy = float(np.sum(0.5 * s2)) / self.global_size
        vmax2 = float(np.max(s2))
        w = [self.backward_real(c) for c in self.vorticity_hat(u)]
        enstrophy = float(np.sum(0.5 * (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]))) / self.global_size
        ix, iy, iz = self.kvals
        div = (u[0] * ix + u[1] * iy) + u[2] * iz
        maxdiv = float(np.max(np.sqrt(div.real * div.real + div.imag * div.imag)))
        return dict(t=t, kinetic_energy=energy, dissipation=2.0 * self.nu * enstrophy,
                    enstrophy=enstrophy, max_spectral_divergence=maxdiv, max_velocity=float(np.sqrt(vmax2)))

    def get_state_full(self):
        return [half_to_full(c) for c in self.u_hat]
