"""sns_forward_r2c_noalloc: the forward transform for callers that cannot let a library
allocate device memory (applications that reserve the GPU's memory up front and serve it
from their own pool, runs near the HBM limit, loops that cannot take the synchronisation
an allocation may cause).  Its scratch is a fixed __device__ array inside the library, so
it serves grids up to N = 64 only.

The GPU tests call it through the C ABI on device buffers and check it against the
handle-based sns_forward_r2c and against numpy's fftn, on two calls in a row (the second
reuses the shared scratch that the first one left behind), to the FFT tolerance of the other
GPU tests: max abs error <= 1e-12 * max|X|; and once more on a caller's own non-default
stream.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from spectral_solver_b200 import _lib

MAX_N = 64
TOL = 1e-12


def test_noalloc_rejects_bad_sizes_and_pointers(lib):
    dummy = C.c_void_p(0x1000)
    assert lib.sns_forward_r2c_noalloc(MAX_N * 2, dummy, dummy, None) == _lib.SNS_ERR_UNSUPPORTED
    assert b"N <= 64" in lib.sns_last_error(None)
    assert lib.sns_forward_r2c_noalloc(10, dummy, dummy, None) == _lib.SNS_ERR_UNSUPPORTED
    assert lib.sns_forward_r2c_noalloc(0, dummy, dummy, None) == _lib.SNS_ERR_INVALID
    assert lib.sns_forward_r2c_noalloc(16, None, dummy, None) == _lib.SNS_ERR_INVALID


@pytest.mark.gpu
def test_noalloc_forward_matches_handle_forward(lib):
    import torch

    from spectral_solver_b200 import Solver

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(2026)
    # two calls in a row at the largest size, then a smaller one on the same scratch
    for n in (MAX_N, MAX_N, 24):
        x = rng.standard_normal((n, n, n))
        with Solver(n) as s:
            want = s.forward(x)
        d_in = torch.from_numpy(x).to(dev)
        d_out = torch.full((2 * n ** 3,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = lib.sns_forward_r2c_noalloc(n, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), None)
        assert rc == _lib.SNS_OK, lib.sns_last_error(None)
        got = d_out.cpu().numpy().view(np.complex128).reshape(n, n, n)
        assert np.max(np.abs(got - want)) <= TOL * np.max(np.abs(want)), n
        # and directly against numpy (x fastest: the array is indexed [iz, iy, ix])
        ref = np.fft.fftn(x)
        assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref)), n


@pytest.mark.gpu
def test_noalloc_forward_on_callers_stream(lib):
    """The documented use on a stream the caller owns: the call enqueues its work there and
    returns after that stream finished."""
    import torch

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(7)
    n = 48
    x = rng.standard_normal((n, n, n))
    side = torch.cuda.Stream(device=dev)
    d_in = torch.from_numpy(x).to(dev)
    d_out = torch.full((2 * n ** 3,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    for _ in range(2):
        rc = lib.sns_forward_r2c_noalloc(n, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()),
                                         C.c_void_p(side.cuda_stream))
        assert rc == _lib.SNS_OK, lib.sns_last_error(None)
        got = d_out.cpu().numpy().view(np.complex128).reshape(n, n, n)
        ref = np.fft.fftn(x)
        assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref))


@pytest.mark.gpu
def test_noalloc_rejects_host_and_misaligned_buffers(lib):
    import torch

    n = 16
    host = np.zeros(2 * n ** 3)
    d_in = torch.zeros(n ** 3, dtype=torch.float64, device="cuda:0")
    assert lib.sns_forward_r2c_noalloc(n, C.c_void_p(d_in.data_ptr()), host.ctypes.data_as(C.c_void_p),
                                       None) == _lib.SNS_ERR_INVALID
    assert b"device memory" in lib.sns_last_error(None)
    # misaligned output (a double2 store needs 16 bytes)
    d_out = torch.zeros(2 * n ** 3 + 2, dtype=torch.float64, device="cuda:0")
    assert lib.sns_forward_r2c_noalloc(n, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr() + 8),
                                       None) == _lib.SNS_ERR_INVALID
