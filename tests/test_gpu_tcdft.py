"""Tensor-core DFT sub-block against the register butterflies and a float64 DFT.

Batches of 16-point complex DFTs (sign -1, unnormalised) run as tcgen05.mma kind::tf32 tiles
with the 3xTF32 split and as the register butterflies the pass kernels use; both must match
numpy's float64 FFT within FP32 accuracy (max error relative to the largest output
magnitude <= 2e-6 for 3xTF32, which keeps about 21 mantissa bits, <= 1e-6 for the FP32
butterflies).  The kernel times are printed for the design notes' comparison.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from spectral_solver_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(lib, x, tensor_cores):
    dev_in = torch.from_numpy(x).cuda()
    dev_out = torch.zeros_like(dev_in)
    ms = C.c_double(-1.0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.sns_dft16_batch(dev_in.data_ptr(), dev_out.data_ptr(), x.shape[0], int(tensor_cores),
                             C.c_void_p(stream), C.byref(ms))
    assert rc == _lib.SNS_OK, lib.sns_last_error(None)
    return dev_out.cpu().numpy(), ms.value


@pytest.mark.parametrize("count", [128, 128 * 148 * 4 + 128 * 37])
def test_dft16_both_methods_match_float64(lib, count):
    rng = np.random.default_rng(count)
    x = rng.uniform(-1.0, 1.0, size=(count, 32)).astype(np.float32)
    ref = np.fft.fft(x[:, 0::2].astype(np.float64) + 1j * x[:, 1::2].astype(np.float64), axis=1)
    scale = np.abs(ref).max()
    for tc, tol in ((1, 2e-6), (0, 1e-6)):
        y, ms = _run(lib, x, tc)
        got = y[:, 0::2].astype(np.float64) + 1j * y[:, 1::2].astype(np.float64)
        err = np.abs(got - ref).max() / scale
        print(f"count {count} tensor_cores {tc}: rel err {err:.2e}, {ms:.4f} ms")
        assert err <= tol, (tc, err)


def test_dft16_rate(lib):
    """Both methods on 2^22 sequences (512 MiB in + out, well above L2): report the
    per-sequence rates; the solver keeps the butterflies."""
    count = 1 << 22
    x = np.random.default_rng(1).uniform(-1, 1, size=(count, 32)).astype(np.float32)
    times = {}
    for tc in (0, 1, 0, 1):
        _, ms = _run(lib, x, tc)
        times[tc] = ms
    gbs = {tc: 2 * count * 32 * 4 / (ms * 1e-3) / 1e9 for tc, ms in times.items()}
    print(f"dft16 x {count}: butterflies {times[0]:.3f} ms ({gbs[0]:.0f} GB/s), "
          f"tcgen05 3xTF32 {times[1]:.3f} ms ({gbs[1]:.0f} GB/s)")
    assert times[0] > 0 and times[1] > 0
