"""ctypes binding of the C ABI in ``include/sns_b200.h`` (``libsns_b200.so``).

The library is built in-tree (``spectral_solver_b200/build.py``); loading fails loudly if
it is missing — there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
# SNS_B200_LIB=check loads the index-checked debug build (libsns_b200_check.so)
LIB_PATH = os.path.join(_PKG, "libsns_b200_check.so" if os.environ.get("SNS_B200_LIB") == "check"
                        else "libsns_b200.so")

SNS_OK = 0
SNS_ERR_INVALID = 1
SNS_ERR_UNSUPPORTED = 2
SNS_ERR_CUDA = 3
SNS_ERR_NOMEM = 4
SNS_ERR_NO_DEVICE = 5
SNS_ERR_INJECTED = 6
PRECISION_FP64 = 0
PRECISION_FP32 = 1
VISCOUS_EXPLICIT = 0

# Every symbol include/sns_b200.h declares, with its ctypes signature.
_DP = C.POINTER(C.c_double)
_DPP = C.POINTER(_DP)
_H = C.c_void_p


class SnsDiag(C.Structure):
    _fields_ = [("t", C.c_double), ("kinetic_energy", C.c_double), ("dissipation", C.c_double),
                ("enstrophy", C.c_double), ("max_spectral_divergence", C.c_double),
                ("max_velocity", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolveSpec(C.Structure):
    _fields_ = [("n", C.c_int), ("nu", C.c_double), ("precision", C.c_int), ("viscous_mode", C.c_int),
                ("seed", C.c_uint64), ("pert_amp", C.c_double), ("pert_kmax", C.c_int), ("dt", C.c_double),
                ("cfl", C.c_double), ("dt_max", C.c_double)]


class Request(C.Structure):
    _fields_ = [("n", C.c_int), ("nu", C.c_double), ("t_end", C.c_double), ("seed", C.c_uint64),
                ("pert_amp", C.c_double), ("pert_kmax", C.c_int), ("cfl", C.c_double), ("dt_max", C.c_double)]


class Result(C.Structure):
    _fields_ = [("id", C.c_int64), ("n", C.c_int), ("steps", C.c_int), ("dt", C.c_double), ("final", SnsDiag)]


SIGNATURES = {
    "sns_version": (C.c_char_p, []),
    "sns_bytes_required": (C.c_size_t, [C.c_int, C.c_int]),
    "sns_create": (C.c_int, [C.c_int, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_int,
                             C.POINTER(_H)]),
    "sns_destroy": (C.c_int, [_H]),
    "sns_last_error": (C.c_char_p, [_H]),
    "sns_forward_r2c": (C.c_int, [_H, _DP, _DP]),
    "sns_backward_c2r": (C.c_int, [_H, _DP, _DP]),
    "sns_set_state": (C.c_int, [_H, _DPP]),
    "sns_get_state": (C.c_int, [_H, _DPP]),
    "sns_rhs": (C.c_int, [_H, _DPP, _DPP]),
    "sns_nonlinear": (C.c_int, [_H, _DPP, _DPP]),
    "sns_step": (C.c_int, [_H, C.c_double, C.c_int]),
    "sns_diagnostics": (C.c_int, [_H, C.c_double, C.POINTER(SnsDiag)]),
    "sns_max_velocity": (C.c_int, [_H, _DP]),
    "sns_dump_velocity": (C.c_int, [_H, _DPP]),
    "sns_set_viscosity": (C.c_int, [_H, C.c_double]),
    "sns_set_nonlinear_form": (C.c_int, [_H, C.c_int]),
    "sns_set_sphere_pruning": (C.c_int, [_H, C.c_int]),
    "sns_set_compensation": (C.c_int, [_H, C.c_int]),
    "sns_launch_config": (C.c_int, [_H, C.POINTER(C.c_int), C.c_int]),
    "sns_grid_size": (C.c_int, [_H]),
    "sns_device_bytes": (C.c_size_t, [_H]),
    "sns_time_steps": (C.c_int, [_H, C.c_double, C.c_int, _DP]),
    "sns_debug_fail_after": (C.c_int, [_H, C.c_int]),
    "sns_debug_set_error_word": (C.c_int, [_H, C.c_int]),
    "sns_debug_bounded_wait": (C.c_int, [C.c_uint, C.POINTER(C.c_int)]),
    "sns_debug_bounds": (C.c_int, [C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "sns_dft16_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, _DP]),
    "sns_profile_passes": (C.c_int, [_H, C.c_double, C.c_int, _DP]),
    "sns_forward_r2c_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sns_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.POINTER(C.c_void_p), _DP]),
    "sns_batch_destroy": (C.c_int, [C.c_void_p]),
    "sns_batch_step": (C.c_int, [C.c_void_p, C.c_int]),
    "sns_batch_time_steps": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "sns_batch_handle": (C.c_void_p, [C.c_void_p, C.c_int]),
    "sns_batch_size": (C.c_int, [C.c_void_p]),
    "sns_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "sns_autotune": (C.c_int, [_H, C.c_int, C.c_char_p, C.POINTER(C.c_int)]),
    "sns_server_create": (C.c_int, [C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]),
    "sns_server_destroy": (C.c_int, [C.c_void_p]),
    "sns_server_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]),
    "sns_server_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
    "sns_server_last_error": (C.c_char_p, [C.c_void_p]),
    "sns_grid_supported": (C.c_int, [C.c_int]),
    "sns_set_clock": (C.c_int, [_H, C.c_double, C.c_double, C.c_double, C.c_double]),
    "sns_step_cfl": (C.c_int, [_H, C.c_int]),
    "sns_get_clock": (C.c_int, [_H, _DP, C.c_int]),
    "sns_server_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_longlong)]),
    "sns_fft3d_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.POINTER(C.c_void_p)]),
    "sns_fft3d_destroy": (C.c_int, [C.c_void_p]),
    "sns_fft3d_last_error": (C.c_char_p, [C.c_void_p]),
    "sns_fft3d_device_bytes": (C.c_size_t, [C.c_void_p]),
    "sns_fft3d_forward": (C.c_int, [C.c_void_p, _DP, _DP]),
    "sns_fft3d_backward": (C.c_int, [C.c_void_p, _DP, _DP]),
    "sns_fft3d_rhs": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, _DPP, _DPP]),
    "sns_fft3d_step": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_int, _DPP]),
    "sns_fft3d_diagnostics": (C.c_int, [C.c_void_p, C.c_double, _DPP, C.c_double, C.POINTER(SnsDiag)]),
    "sns_fft3d_product": (C.c_int, [C.c_void_p, _DP, _DP, _DP]),
    "sns_fft3d_vorticity_slice": (C.c_int, [C.c_void_p, _DPP, C.c_int, _DP]),
}

PASS_NAMES = ("p1_zinv_phase", "p2_yinv", "p3_xpass", "p3_nyq", "p4_yfwd", "p5_zfwd", "p5_sweep")

_lib = None


def load(path: str = LIB_PATH):
    """Load libsns_b200.so and attach signatures.  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: run __graft_entry__.build() (no CPU fallback exists)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class SnsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _arr3(arrs):
    return (_DP * 3)(*[_dptr(a) for a in arrs])


def full_to_interleaved(c: np.ndarray) -> np.ndarray:
    """complex [iz, iy, ix] -> 2*N^3 doubles (the reference's interleaved storage)."""
    return np.ascontiguousarray(c, dtype=np.complex128).view(np.float64).reshape(-1)


def interleaved_to_full(d: np.ndarray, n: int) -> np.ndarray:
    return d.view(np.complex128).reshape(n, n, n)


class Solver:
    """Thin RAII wrapper of an ``sns_handle`` (Python mirror of TaylorGreenSolver)."""

    def __init__(self, n: int, reynolds: float = 1600.0, seed: int = 0, pert_amp: float = 0.0,
                 pert_kmax: int = 0, nu: float | None = None, precision: int = PRECISION_FP64,
                 viscous_mode: int = VISCOUS_EXPLICIT):
        self.lib = load()
        self.n = n
        self.precision = precision
        self.nu = (1.0 / reynolds) if nu is None else nu
        h = _H()
        rc = self.lib.sns_create(n, self.nu, precision, viscous_mode, seed, pert_amp, pert_kmax, C.byref(h))
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.sns_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # FFT-backend contract
    def forward(self, phys: np.ndarray) -> np.ndarray:
        n = self.n
        x = np.ascontiguousarray(phys, dtype=np.float64).reshape(-1)
        out = np.empty(2 * n ** 3, np.float64)
        self._check(self.lib.sns_forward_r2c(self.h, _dptr(x), _dptr(out)))
        return interleaved_to_full(out, n)

    def backward(self, spec: np.ndarray) -> np.ndarray:
        n = self.n
        x = full_to_interleaved(spec)
        out = np.empty(n ** 3, np.float64)
        self._check(self.lib.sns_backward_c2r(self.h, _dptr(x), _dptr(out)))
        return out.reshape(n, n, n)

    def set_state(self, u_full):
        arrs = [full_to_interleaved(c) for c in u_full]
        self._check(self.lib.sns_set_state(self.h, _arr3(arrs)))

    def get_state(self):
        n = self.n
        arrs = [np.empty(2 * n ** 3, np.float64) for _ in range(3)]
        self._check(self.lib.sns_get_state(self.h, _arr3(arrs)))
        return [interleaved_to_full(a, n) for a in arrs]

    def rhs(self, u_full):
        n = self.n
        ins = [full_to_interleaved(c) for c in u_full]
        outs = [np.empty(2 * n ** 3, np.float64) for _ in range(3)]
        self._check(self.lib.sns_rhs(self.h, _arr3(ins), _arr3(outs)))
        return [interleaved_to_full(a, n) for a in outs]

    def nonlinear(self, u_full):
        n = self.n
        ins = [full_to_interleaved(c) for c in u_full]
        outs = [np.empty(2 * n ** 3, np.float64) for _ in range(3)]
        self._check(self.lib.sns_nonlinear(self.h, _arr3(ins), _arr3(outs)))
        return [interleaved_to_full(a, n) for a in outs]

    def step(self, dt: float, nsteps: int = 1):
        self._check(self.lib.sns_step(self.h, dt, nsteps))

    step_rk3 = step

    def set_clock(self, t: float = 0.0, t_end: float = float("inf"), cfl: float = 0.5, dt_max: float = 0.5):
        """Start the device clock for adaptive CFL steps (sns_step_cfl)."""
        self._check(self.lib.sns_set_clock(self.h, t, t_end, cfl, dt_max))

    def step_cfl(self, nsteps: int = 1):
        """nsteps adaptive CFL steps taken on the device (no-ops once the horizon is reached)."""
        self._check(self.lib.sns_step_cfl(self.h, nsteps))

    def clock(self) -> dict:
        out = (C.c_double * 4)()
        self._check(self.lib.sns_get_clock(self.h, out, 4))
        return {"t": out[0], "dt": out[1], "steps": int(out[2]), "stopped": bool(out[3])}

    def time_steps(self, dt: float, nsteps: int) -> float:
        ms = C.c_double()
        self._check(self.lib.sns_time_steps(self.h, dt, nsteps, C.byref(ms)))
        return ms.value

    def diagnostics(self, t: float = 0.0) -> dict:
        d = SnsDiag()
        self._check(self.lib.sns_diagnostics(self.h, t, C.byref(d)))
        return d.as_dict()

    def max_velocity(self) -> float:
        v = C.c_double()
        self._check(self.lib.sns_max_velocity(self.h, C.byref(v)))
        return v.value

    def dump_velocity(self):
        n = self.n
        arrs = [np.empty(n ** 3, np.float64) for _ in range(3)]
        self._check(self.lib.sns_dump_velocity(self.h, _arr3(arrs)))
        return [a.reshape(n, n, n) for a in arrs]

    def profile_passes(self, dt: float, nsteps: int) -> dict:
        out = (C.c_double * len(PASS_NAMES))()
        self._check(self.lib.sns_profile_passes(self.h, dt, nsteps, out))
        return dict(zip(PASS_NAMES, list(out)))

    def launch_config(self) -> dict:
        out = (C.c_int * 4)()
        self._check(self.lib.sns_launch_config(self.h, out, 4))
        return dict(tma_grid=out[0], xpass_grid=out[1], p5_grid=out[2], sms=out[3])

    def set_nonlinear_form(self, form: int):
        """0: the reference's conservative form (default), 1: the rotational form u x omega."""
        self._check(self.lib.sns_set_nonlinear_form(self.h, form))

    def set_sphere_pruning(self, enabled: bool):
        """Skip the z-pencil tiles outside the sphere |k| <= N/2 (default on; bitwise neutral)."""
        self._check(self.lib.sns_set_sphere_pruning(self.h, 1 if enabled else 0))

    def set_compensation(self, enabled: bool):
        """FP32 form: carry u as its FP32 value plus an int8 remainder per part (1/255 of an
        FP32 ulp), the RK update formed in FP64 (default on; the FP64 form accepts False
        only)."""
        self._check(self.lib.sns_set_compensation(self.h, 1 if enabled else 0))

    def device_bytes(self) -> int:
        return int(self.lib.sns_device_bytes(self.h))

    def autotune(self, trial_steps: int = 2, cache_path: str | None = None) -> dict:
        """Pick the fastest launch shape for this handle (the state advances by the trials)."""
        out = (C.c_int * 3)()
        self._check(self.lib.sns_autotune(self.h, trial_steps, cache_path.encode() if cache_path else None, out))
        return dict(tma_grid=out[0], xpass_grid=out[1], p5_grid=out[2])



class Fft3D:
    """Generic-shape transforms and the legacy solver's numerics (``sns_fft3d_*``): any
    nx, ny, nz > 1, box lengths lx, ly, lz > 0, the reference's full complex layout (arrays
    indexed [iz, iy, ix])."""

    def __init__(self, shape, lengths=(2 * np.pi, 2 * np.pi, 2 * np.pi)):
        self.lib = load()
        self.shape = tuple(int(v) for v in shape)  # (nx, ny, nz)
        self.lengths = tuple(float(v) for v in lengths)
        h = C.c_void_p()
        rc = self.lib.sns_fft3d_create(*self.shape, *self.lengths, C.byref(h))
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_last_error(None).decode())
        self.h = h

    @property
    def zyx(self):
        nx, ny, nz = self.shape
        return (nz, ny, nx)

    def _check(self, rc):
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_fft3d_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.sns_fft3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def device_bytes(self) -> int:
        return int(self.lib.sns_fft3d_device_bytes(self.h))

    def _cplx(self, d):
        return d.view(np.complex128).reshape(self.zyx)

    def forward(self, phys: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(phys, dtype=np.float64).reshape(-1)
        out = np.empty(2 * x.size, np.float64)
        self._check(self.lib.sns_fft3d_forward(self.h, _dptr(x), _dptr(out)))
        return self._cplx(out)

    def backward(self, spec: np.ndarray) -> np.ndarray:
        x = full_to_interleaved(spec)
        out = np.empty(x.size // 2, np.float64)
        self._check(self.lib.sns_fft3d_backward(self.h, _dptr(x), _dptr(out)))
        return out.reshape(self.zyx)

    def rhs(self, u_full, nu: float, dealias: bool = True, full: bool = True):
        ins = [full_to_interleaved(c) for c in u_full]
        outs = [np.empty_like(a) for a in ins]
        self._check(self.lib.sns_fft3d_rhs(self.h, nu, int(dealias), int(full), _arr3(ins), _arr3(outs)))
        return [self._cplx(a) for a in outs]

    def step(self, u_full, nu: float, dt: float, nsteps: int = 1, dealias: bool = True):
        arrs = [full_to_interleaved(c).copy() for c in u_full]
        self._check(self.lib.sns_fft3d_step(self.h, nu, int(dealias), dt, nsteps, _arr3(arrs)))
        return [self._cplx(a) for a in arrs]

    def diagnostics(self, u_full, nu: float, t: float = 0.0) -> dict:
        ins = [full_to_interleaved(c) for c in u_full]
        d = SnsDiag()
        self._check(self.lib.sns_fft3d_diagnostics(self.h, nu, _arr3(ins), t, C.byref(d)))
        return d.as_dict()

    def product(self, a_hat, b_hat):
        a, b = full_to_interleaved(a_hat), full_to_interleaved(b_hat)
        out = np.empty_like(a)
        self._check(self.lib.sns_fft3d_product(self.h, _dptr(a), _dptr(b), _dptr(out)))
        return self._cplx(out)

    def vorticity_slice(self, u_full, iz: int) -> np.ndarray:
        ins = [full_to_interleaved(c) for c in u_full]
        nx, ny, _ = self.shape
        out = np.empty(nx * ny, np.float64)
        self._check(self.lib.sns_fft3d_vorticity_slice(self.h, _arr3(ins), iz, _dptr(out)))
        return out.reshape(ny, nx)


class _BorrowedSolver(Solver):
    """A Solver view of a handle owned by a batch (closing it does nothing)."""

    def __init__(self, lib, h, n, precision):
        self.lib = lib
        self.h = C.c_void_p(h)
        self.n = n
        self.precision = precision

    def close(self):
        self.h = None


class Batch:
    """Many independent solves stepped together: one CUDA graph launch per batch step."""

    def __init__(self, specs, autotune_trials: int = 0, autotune_cache: str | None = None):
        self.lib = load()
        arr = (SolveSpec * len(specs))()
        for i, sp in enumerate(specs):
            arr[i] = SolveSpec(sp["n"], sp["nu"], sp.get("precision", PRECISION_FP64),
                               sp.get("viscous_mode", VISCOUS_EXPLICIT), sp.get("seed", 0), sp.get("pert_amp", 0.0),
                               sp.get("pert_kmax", 0), sp.get("dt", 0.0), sp.get("cfl", 0.5), sp.get("dt_max", 0.5))
        self.specs = list(specs)
        dts = (C.c_double * len(specs))()
        b = C.c_void_p()
        rc = self.lib.sns_batch_create(C.cast(arr, C.c_void_p), len(specs), autotune_trials,
                                       autotune_cache.encode() if autotune_cache else None, C.byref(b), dts)
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_last_error(None).decode())
        self.b = b
        self.dt = list(dts)

    def _check(self, rc):
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_batch_last_error(self.b).decode())

    def step(self, nsteps: int = 1):
        self._check(self.lib.sns_batch_step(self.b, nsteps))

    def time_steps(self, nsteps: int) -> float:
        ms = C.c_double()
        self._check(self.lib.sns_batch_time_steps(self.b, nsteps, C.byref(ms)))
        return ms.value

    def solver(self, i: int) -> Solver:
        h = self.lib.sns_batch_handle(self.b, i)
        if not h:
            raise IndexError(i)
        sp = self.specs[i]
        return _BorrowedSolver(self.lib, h, sp["n"], sp.get("precision", PRECISION_FP64))

    def __len__(self):
        return int(self.lib.sns_batch_size(self.b))

    def close(self):
        if getattr(self, "b", None):
            self.lib.sns_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Server:
    """Continuous-batching server: admission by HBM budget, all resident solves stepped together."""

    def __init__(self, hbm_budget_bytes: int, precision: int = PRECISION_FP32):
        self.lib = load()
        s = C.c_void_p()
        rc = self.lib.sns_server_create(int(hbm_budget_bytes), precision, C.byref(s))
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_last_error(None).decode())
        self.s = s
        self.precision = precision

    def _check(self, rc):
        if rc != SNS_OK:
            raise SnsError(rc, self.lib.sns_server_last_error(self.s).decode())

    def submit(self, n, nu, t_end, seed=0, pert_amp=0.0, pert_kmax=0, cfl=0.5, dt_max=0.5) -> int:
        r = Request(n, nu, t_end, seed, pert_amp, pert_kmax, cfl, dt_max)
        rid = C.c_int64()
        self._check(self.lib.sns_server_submit(self.s, C.byref(r), C.byref(rid)))
        return rid.value

    def step(self, max_done: int = 256):
        done = (Result * max_done)()
        nd, res, q = C.c_int(), C.c_int(), C.c_int()
        used = C.c_size_t()
        self._check(self.lib.sns_server_step(self.s, C.cast(done, C.c_void_p), max_done, C.byref(nd), C.byref(res),
                                             C.byref(q), C.byref(used)))
        out = [dict(id=done[i].id, n=done[i].n, steps=done[i].steps, dt=done[i].dt, final=done[i].final.as_dict())
               for i in range(nd.value)]
        return out, res.value, q.value, used.value

    def stats(self) -> dict:
        """Idle-pool bytes and the number of handles the server has allocated."""
        idle, made = C.c_size_t(), C.c_longlong()
        self._check(self.lib.sns_server_stats(self.s, C.byref(idle), C.byref(made)))
        return {"idle_bytes": idle.value, "handles_created": made.value}

    def close(self):
        if getattr(self, "s", None):
            self.lib.sns_server_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
