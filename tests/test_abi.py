"""The drop-in boundary without a GPU: the C ABI loads, exports every symbol the header
declares, and rejects bad arguments with the documented codes; the C++ layer and its
executables are built and fail cleanly when no device is visible."""
import ctypes as C
import os
import re
import subprocess

import pytest

from tests.conftest import has_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "spectral_solver_b200")


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "sns_b200.h")).read()
    return sorted(set(re.findall(r"\b(sns_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(lib):
    from spectral_solver_b200 import _lib
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), "binding and header disagree"


def test_version_and_sizes(lib):
    assert b"sm_100a" in lib.sns_version()
    b512 = lib.sns_bytes_required(512, 0)
    assert 18e9 < b512 < 22e9  # 18 half-spectrum fields at 512^3
    b512f = lib.sns_bytes_required(512, 1)
    # the same 18 fields in FP32 (rows padded to 16 complex floats) plus the compensation
    # words of u (3 fields of 2 bytes per complex value)
    assert 10.4e9 < b512f < 11.2e9
    assert lib.sns_bytes_required(0, 0) == 0
    assert lib.sns_bytes_required(64, 7) == 0


@pytest.mark.parametrize("args,code", [
    ((0, 1e-3, 0, 0, 0, 0.0, 0), 1),     # n <= 0
    ((64, -1.0, 0, 0, 0, 0.0, 0), 1),    # negative viscosity (Re <= 0)
    ((64, 1e-3, 7, 0, 0, 0.0, 0), 2),    # unknown precision
    ((64, 1e-3, 0, 5, 0, 0.0, 0), 2),    # unknown viscous mode
    ((10, 1e-3, 0, 0, 0, 0.0, 0), 2),    # no FFT plan for 10
    ((64, 1e-3, 0, 0, 0, 1e-3, 32), 1),  # perturbation kmax >= N/2
])
def test_create_rejects_bad_arguments(lib, args, code):
    h = C.c_void_p()
    rc = lib.sns_create(*args, C.byref(h))
    assert rc == code
    assert not h.value
    assert len(lib.sns_last_error(None)) > 0


def test_null_handle_calls(lib):
    assert lib.sns_destroy(None) == 1
    assert lib.sns_step(None, 1e-3, 1) == 1
    assert lib.sns_debug_fail_after(None, 1) == 1
    assert lib.sns_set_viscosity(None, 1.0) == 1
    assert lib.sns_set_sphere_pruning(None, 1) == 1
    assert lib.sns_grid_size(None) == 0
    assert lib.sns_autotune(None, 1, None, None) == 1
    assert lib.sns_batch_step(None, 1) == 1
    assert lib.sns_batch_destroy(None) == 1
    assert lib.sns_batch_size(None) == 0
    assert lib.sns_batch_handle(None, 0) is None
    assert lib.sns_server_destroy(None) == 1
    assert lib.sns_server_step(None, None, 0, None, None, None, None) == 1
    assert lib.sns_server_submit(None, None, None) == 1


def test_batch_and_server_reject_bad_arguments(lib):
    from spectral_solver_b200 import _lib
    b = C.c_void_p()
    assert lib.sns_batch_create(None, 0, 0, None, C.byref(b), None) == 1
    assert not b.value
    s = C.c_void_p()
    assert lib.sns_server_create(0, 1, C.byref(s)) == 1  # zero budget
    assert lib.sns_server_create(1 << 30, 7, C.byref(s)) == 1  # unknown precision
    assert not s.value
    assert len(lib.sns_last_error(None)) > 0


def test_dft16_batch_rejects_bad_arguments(lib):
    buf = C.c_void_p(1 << 20)  # never dereferenced: the arguments are refused first
    assert lib.sns_dft16_batch(None, buf, 128, 1, None, None) == 1
    assert lib.sns_dft16_batch(buf, buf, 100, 1, None, None) == 1  # not a multiple of 128
    assert lib.sns_dft16_batch(buf, buf, 128, 2, None, None) == 1  # unknown method
    assert lib.sns_dft16_batch(C.c_void_p((1 << 20) + 4), buf, 128, 0, None, None) == 1  # unaligned
    assert b"sns_dft16_batch" in lib.sns_last_error(None)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_is_reported(lib):
    h = C.c_void_p()
    rc = lib.sns_create(16, 1e-3, 0, 0, 0, 0.0, 0, C.byref(h))
    assert rc == 5
    assert b"no CUDA device" in lib.sns_last_error(None)


def test_cpp_layer_built():
    so = os.path.join(PKG, "libspectral_b200.so")
    assert os.path.exists(so)
    out = subprocess.run(["nm", "-DC", so], capture_output=True, text=True).stdout
    for sym in ("spectral::B200Fft3D::forward", "spectral::B200Fft3D::backward",
                "spectral::SpectralNavierStokes::step_rk3", "spectral::SpectralNavierStokes::rhs",
                "spectral::ava_solver::TaylorGreenSolver::step_rk3",
                "spectral::ava_solver::run_taylor_green"):
        assert sym in out, sym


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_cli_fails_cleanly_without_device(tmp_path):
    exe = os.path.join(PKG, "bin", "taylor_green_b200")
    r = subprocess.run([exe, "--n", "12", "--steps", "1", "--output-dir", str(tmp_path)], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1
    assert "error:" in r.stderr
