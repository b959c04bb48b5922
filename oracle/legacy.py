"""CPU oracle of the legacy host-vector solver for any grid and box.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path imports this module; only ``tests/``
uses it.

Restates ``SpectralNavierStokes`` of ovankerm/Spectral_solver (``src/spectral_solver.cpp``)
over the FftwFft3D backend (``src/fftw_fft.cpp``) in NumPy FP64, for any shape
(nx, ny, nz) > 1, box lengths L > 0 and either product form:

* modes m = i <= n/2 ? i : i - n on each axis, k = 2 pi m / L (``fftw_fft.hpp:45-71``);
* forward: unnormalised c2c DFT of the real field, sign -1; backward: Re(IDFT) / N
  (``fftw_fft.cpp:53-85``);
* phase exp(i (kx dx + ky dy + kz dz)) with d = L / (2 n) (``spectral_solver.cpp:48-54``);
  keep mask (mx/(nx/2))^2 + (my/(ny/2))^2 + (mz/(nz/2))^2 <= 1 (``:392-398``);
* project (k2 > 0) then zero mean (``:94-109, 400-409``); truncate (``:111-120``);
* product_dealiased (``:122-158``); nonlinear_rhs with or without the phase-shift pair
  (``:160-240``); rhs (``:242-260``); step_rk3 (``:262-309``); the diagnostics
  (``:311-386``); the vorticity slice behind write_vorticity_ppm (``:421-486``).

Arrays are indexed [iz, iy, ix] (x fastest, the reference's id = ix + nx (iy + ny iz)).
"""
from __future__ import annotations

import numpy as np

TWO_PI = 6.283185307179586476925286766559005768


def signed(n: int) -> np.ndarray:
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n)


class LegacyNS:
    def __init__(self, shape, lengths, nu: float, dealias: bool = True):
        self.nx, self.ny, self.nz = (int(v) for v in shape)
        self.lx, self.ly, self.lz = (float(v) for v in lengths)
        self.nu = float(nu)
        self.dealias = bool(dealias)
        mx, my, mz = signed(self.nx), signed(self.ny), signed(self.nz)
        self.mx, self.my, self.mz = mx[None, None, :], my[None, :, None], mz[:, None, None]
        self.kx = TWO_PI * self.mx / self.lx
        self.ky = TWO_PI * self.my / self.ly
        self.kz = TWO_PI * self.mz / self.lz
        self.k2 = self.kx * self.kx + self.ky * self.ky + self.kz * self.kz
        dx, dy, dz = 0.5 * self.lx / self.nx, 0.5 * self.ly / self.ny, 0.5 * self.lz / self.nz
        self.phase = np.exp(1j * (self.kx * dx + self.ky * dy + self.kz * dz))
        ex = (self.mx * self.mx) / (self.nx / 2.0) ** 2
        ey = (self.my * self.my) / (self.ny / 2.0) ** 2
        ez = (self.mz * self.mz) / (self.nz / 2.0) ** 2
        self.keep = (ex + ey + ez) <= 1.0
        self.size = self.nx * self.ny * self.nz

    @property
    def shape_zyx(self):
        return (self.nz, self.ny, self.nx)

    def forward(self, f):
        return np.fft.fftn(f)

    def backward(self, c):
        return np.fft.ifftn(c).real

    def project(self, u):
        k2 = np.broadcast_to(self.k2, self.shape_zyx)
        ok = k2 != 0.0
        f = (self.kx * u[0] + self.ky * u[1] + self.kz * u[2]) / np.where(ok, k2, 1.0)
        out = [np.where(ok, u[0] - self.kx * f, u[0]), np.where(ok, u[1] - self.ky * f, u[1]),
               np.where(ok, u[2] - self.kz * f, u[2])]
        for c in out:
            c[0, 0, 0] = 0.0  # zero_mean
        return out

    def truncate(self, u):
        return [np.where(self.keep, c, 0.0) for c in u]

    def product_dealiased(self, a_hat, b_hat):
        c0 = self.forward(self.backward(a_hat) * self.backward(b_hat))
        cs = self.forward(self.backward(a_hat * self.phase) * self.backward(b_hat * self.phase))
        return np.where(self.keep, 0.5 * (c0 + cs * np.conj(self.phase)), 0.0)

    def nonlinear_rhs(self, u_hat):
        u = [self.backward(c) for c in u_hat]
        us = [self.backward(c * self.phase) for c in u_hat] if self.dealias else None
        P = {}
        for a in range(3):
            for b in range(a, 3):
                v = self.forward(u[a] * u[b])
                if self.dealias:
                    v = 0.5 * (v + self.forward(us[a] * us[b]) * np.conj(self.phase))
                P[(a, b)] = P[(b, a)] = np.where(self.keep, v, 0.0)
        rhs = [-1j * (self.kx * P[(0, i)] + self.ky * P[(1, i)] + self.kz * P[(2, i)]) for i in range(3)]
        return self.truncate(rhs)

    def rhs(self, u_hat):
        r = self.nonlinear_rhs(u_hat)
        r = [r[c] - self.nu * self.k2 * u_hat[c] for c in range(3)]
        return self.truncate(self.project(r))

    def step_rk3(self, u_hat, dt):
        u = [c.copy() for c in u_hat]
        g = self.rhs(u)
        u = [u[c] + (dt / 3.0) * g[c] for c in range(3)]
        u = self.truncate(self.project(u))
        h = self.rhs(u)
        g = [-(5.0 / 9.0) * g[c] + h[c] for c in range(3)]
        u = [u[c] + (15.0 / 16.0) * dt * g[c] for c in range(3)]
        u = self.truncate(self.project(u))
        h = self.rhs(u)
        g = [-(153.0 / 128.0) * g[c] + h[c] for c in range(3)]
        u = [u[c] + (8.0 / 15.0) * dt * g[c] for c in range(3)]
        return self.truncate(self.project(u))

    def vorticity_hat(self, u):
        return [1j * (self.ky * u[2] - self.kz * u[1]), 1j * (self.kz * u[0] - self.kx * u[2]),
                1j * (self.kx * u[1] - self.ky * u[0])]

    def diagnostics(self, u_hat):
        p = [self.backward(c) for c in u_hat]
        s2 = p[0] ** 2 + p[1] ** 2 + p[2] ** 2
        w = [self.backward(c) for c in self.vorticity_hat(u_hat)]
        ens = 0.5 * float(np.sum(w[0] ** 2 + w[1] ** 2 + w[2] ** 2)) / self.size
        div = self.kx * u_hat[0] + self.ky * u_hat[1] + self.kz * u_hat[2]
        return {"kinetic_energy": float(np.sum(0.5 * s2)) / self.size, "enstrophy": ens,
                "dissipation": 2.0 * self.nu * ens, "max_spectral_divergence": float(np.max(np.abs(div))),
                "max_velocity": float(np.sqrt(np.max(s2)))}

    def vorticity_slice(self, u_hat, iz):
        w = [self.backward(c) for c in self.vorticity_hat(u_hat)]
        return np.sqrt(w[0][iz] ** 2 + w[1][iz] ** 2 + w[2][iz] ** 2)

    def taylor_green(self, amplitude=1.0, mode=1):
        x = (np.arange(self.nx) + 0.5) * self.lx / self.nx
        y = (np.arange(self.ny) + 0.5) * self.ly / self.ny
        z = (np.arange(self.nz) + 0.5) * self.lz / self.nz
        ax = (TWO_PI * mode * x / self.lx)[None, None, :]
        ay = (TWO_PI * mode * y / self.ly)[None, :, None]
        az = (TWO_PI * mode * z / self.lz)[:, None, None]
        u = amplitude * np.sin(ax) * np.cos(ay) * np.cos(az)
        v = -amplitude * np.cos(ax) * np.sin(ay) * np.cos(az)
        return [np.broadcast_to(u, self.shape_zyx).copy(), np.broadcast_to(v, self.shape_zyx).copy(),
                np.zeros(self.shape_zyx)]
