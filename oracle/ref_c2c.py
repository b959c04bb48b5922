"""CPU oracle, literal full-spectrum (c2c) restatement of the reference TGV time step.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path imports this module; only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` use it, and only as the checker or the timed CPU baseline.

This module restates, in NumPy FP64, the benchmarked AVA path of
ovankerm/Spectral_solver (``src/ava_taylor_green_impl.hpp``) with the FFTW backend's
semantics: full N^3 complex storage, unnormalised forward DFT of sign -1, inverse DFT
scaled by 1/N^3 of which only the real part is consumed.  numpy.fft (pocketfft) uses the
same conventions as FFTW (``fftw_plan_dft_3d`` FORWARD/BACKWARD), so the only difference
from the reference is round-off of the FFT algorithm.  FFTW itself (the third-party
dependency, pinned only through the nixpkgs revision in ``flake.lock:9``) is absent from
this machine; its published definition of the DFT is what is restated here.

Arrays are indexed ``[iz, iy, ix]`` so that C order is the reference's x-fastest layout
``id = ix + N*(iy + N*iz)`` (``ava_taylor_green_impl.hpp:127-129``, ``fftw_fft.hpp:30-40``).
"""
from __future__ import annotations

import numpy as np

PI = 3.141592653589793238462643383279502884


def signed_mode(i: np.ndarray | int, n: int):
    """Index -> signed mode; index n/2 maps to +n/2 (``ava_taylor_green_impl.hpp:123-125``)."""
    return np.where(np.asarray(i) <= n // 2, i, np.asarray(i) - n)


def mode_grids(n: int):
    """Integer mode arrays broadcast to ``[iz, iy, ix]`` (``fill_spectral_modes`` :377-412)."""
    m = signed_mode(np.arange(n), n).astype(np.int64)
    mz = m[:, None, None]
    my = m[None, :, None]
    mx = m[None, None, :]
    return mx, my, mz


class TaylorGreenC2C:
    """Full-spectrum restatement of ``TaylorGreenSolver::Impl`` (ava_taylor_green_impl.hpp:658-1179)."""

    def __init__(self, n: int, reynolds: float):
        if n <= 0:
            raise ValueError("grid size must be positive")  # :704-706
        if reynolds <= 0.0:
            raise ValueError("Reynolds number must be positive")  # :707-709
        self.n = n
        self.nu = 1.0 / reynolds  # :703
        self.global_size = n * n * n
        mx, my, mz = mode_grids(n)
        self.mx, self.my, self.mz = mx, my, mz
        msum = (mx + my + mz).astype(np.float64)
        # initialize_metadata :779-785: phase exp(i*pi*(mx+my+mz)/n), mask |m|^2/(n/2)^2 <= 1
        angle = (msum * PI) / float(n)
        self.phase = np.cos(angle) + 1j * np.sin(angle)
        h = 0.5 * float(n)
        m2 = (mx * mx + my * my + mz * mz).astype(np.float64)
        self.keep = (m2 / (h * h)) <= 1.0
        self.k2 = m2
        self.kvals = (mx.astype(np.float64), my.astype(np.float64), mz.astype(np.float64))
        self.u_hat = [None, None, None]
        self.g = [np.zeros((n, n, n), np.complex128) for _ in range(3)]
        self.initialize_velocity()

    # -- FFT backend (FftPlan FFTW branch :414-561) ------------------------------------
    def forward(self, phys: np.ndarray) -> np.ndarray:
        return np.fft.fftn(phys)

    def backward_real(self, spec: np.ndarray) -> np.ndarray:
        """``backward`` + ``scale_inverse``; callers consume only ``.x`` (:904-905, :1114)."""
        return np.fft.ifftn(spec).real

    # -- kernels -----------------------------------------------------------------------
    def physical_coordinates(self):
        n = self.n
        i = np.arange(n, dtype=np.float64)
        c = (i + 0.5) * 2.0 * PI / float(n)  # initialize_velocity :806-808
        return c[None, None, :], c[None, :, None], c[:, None, None]

    def initialize_velocity(self):
        """TGV at cell centres, 3 forward FFTs, project_truncate (:796-817)."""
        x, y, z = self.physical_coordinates()
        p0 = np.sin(x) * np.cos(y) * np.cos(z)
        p1 = -np.cos(x) * np.sin(y) * np.cos(z)
        p2 = np.zeros((self.n, self.n, self.n))
        p0 = np.broadcast_to(p0, (self.n,) * 3)
        p1 = np.broadcast_to(p1, (self.n,) * 3)
        self.u_hat = [self.forward(p) for p in (p0, p1, p2)]
        self.project_truncate(self.u_hat)

    def project_truncate(self, f):
        """Leray projection with integer k, zero k=0 and outside-sphere modes (:819-845)."""
        ix, iy, iz = self.kvals
        k2 = self.k2
        ok = (k2 > 0.0) & self.keep
        inv = np.where(k2 > 0.0, 1.0 / np.where(k2 > 0.0, k2, 1.0), 0.0)
        dot = (f[0] * ix + f[1] * iy) + f[2] * iz
        factor = dot * inv
        f[0][...] = np.where(ok, f[0] - factor * ix, 0.0)
        f[1][...] = np.where(ok, f[1] - factor * iy, 0.0)
        f[2][...] = np.where(ok, f[2] - factor * iz, 0.0)

    def compute_rhs(self, u_hat=None):
        """Conservative-form dealiased RHS (:847-977)."""
        if u_hat is None:
            u_hat = self.u_hat
        phys = [self.backward_real(u) for u in u_hat]  # :850-852
        shift = [self.backward_real(u * self.phase) for u in u_hat]  # :866-879
        rhs = [np.zeros_like(u_hat[0]) for _ in range(3)]
        kv = self.kvals
        for a, b in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)):  # :881-886
            c0 = self.forward(phys[a] * phys[b])  # :903-911
            cs = self.forward(shift[a] * shift[b])
            value = 0.5 * (c0 + cs * np.conj(self.phase))  # :928
            value = np.where(self.keep, value, 0.0)  # :929-931
            rhs[a] = rhs[a] + (-1j) * kv[b] * value  # minus_i_k :118-121, :932
            if a != b:
                rhs[b] = rhs[b] + (-1j) * kv[a] * value  # :933-935
        # add_viscous_project :955-974
        for c in range(3):
            rhs[c] = rhs[c] - u_hat[c] * (self.nu * self.k2)
        self.project_truncate(rhs)
        return rhs

    def step(self, dt: float):
        """Williamson low-storage RK3 (:979-1045); coefficient products formed as the reference does."""
        u, g = self.u_hat, self.g
        r = self.compute_rhs()
        for c in range(3):
            g[c] = r[c].copy()
            u[c] = u[c] + g[c] * (dt / 3.0)
        self.project_truncate(u)
        r = self.compute_rhs()
        for c in range(3):
            g[c] = g[c] * (-5.0 / 9.0) + r[c]
            u[c] = u[c] + g[c] * (15.0 * dt / 16.0)
        self.project_truncate(u)
        r = self.compute_rhs()
        for c in range(3):
            g[c] = g[c] * (-153.0 / 128.0) + r[c]
            u[c] = u[c] + g[c] * (8.0 * dt / 15.0)
        self.project_truncate(u)

    def step_rk3(self, dt: float):
        self.step(dt)

    # -- diagnostics (:1105-1179) ------------------------------------------------------
    def max_velocity(self) -> float:
        p = [self.backward_real(u) for u in self.u_hat]
        return float(np.sqrt(np.max(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])))

    def vorticity_hat(self, u):
        ix, iy, iz = self.kvals
        return [1j * (iy * u[2] - iz * u[1]), 1j * (iz * u[0] - ix * u[2]), 1j * (ix * u[1] - iy * u[0])]

    def diagnostics(self, t: float) -> dict:
        u = self.u_hat
        p = [self.backward_real(c) for c in u]
        energy = float(np.sum(0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]))) / self.global_size
        vmax2 = float(np.max(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]))
        w = [self.backward_real(c) for c in self.vorticity_hat(u)]
        enstrophy = float(np.sum(0.5 * (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]))) / self.global_size
        ix, iy, iz = self.kvals
        div = (u[0] * ix + u[1] * iy) + u[2] * iz
        maxdiv = float(np.max(np.sqrt(div.real * div.real + div.imag * div.imag)))
        return dict(t=t, kinetic_energy=energy, dissipation=2.0 * self.nu * enstrophy,
                    enstrophy=enstrophy, max_spectral_divergence=maxdiv, max_velocity=float(np.sqrt(vmax2)))

    # -- state exchange in the reference's full-complex layout -------------------------
    def get_state(self):
        return [c.copy() for c in self.u_hat]

    def set_state(self, u_full):
        self.u_hat = [np.array(c, dtype=np.complex128, copy=True) for c in u_full]
