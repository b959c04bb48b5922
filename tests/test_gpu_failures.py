"""The device failure paths, exercised without a GPU fault.

* A pass kernel whose bounded wait runs out records code 1 in the handle's device error
  word and returns; the host checks the word after every synchronisation.  Here the host
  plants that code (sns_debug_set_error_word): the next call must fail with SNS_ERR_CUDA and
  the "gave up waiting for its TMA tile" message, and the call after it must run normally.
* The bounded wait itself: a probe kernel polls a barrier that nothing will complete (armed
  for bytes no copy delivers; nothing is in flight) with a short poll limit and must report
  the timeout instead of spinning.
"""
import ctypes as C

import numpy as np
import pytest

from spectral_solver_b200 import _lib

pytestmark = pytest.mark.gpu


def test_error_word_reported_then_cleared(lib):
    from spectral_solver_b200 import Solver
    with Solver(16, 1600.0) as s:
        before = s.get_state()
        assert lib.sns_debug_set_error_word(s.h, 1) == _lib.SNS_OK
        rc = lib.sns_step(s.h, 1e-3, 1)
        assert rc == _lib.SNS_ERR_CUDA
        assert b"gave up waiting for its TMA tile" in lib.sns_last_error(s.h)
        # the word was cleared: the handle keeps working
        assert lib.sns_step(s.h, 1e-3, 1) == _lib.SNS_OK
        after = s.get_state()
        assert all(np.all(np.isfinite(a)) for a in after)
        assert any(not np.array_equal(a, b) for a, b in zip(after, before))


@pytest.mark.parametrize("polls", [1, 64, 4096])
def test_bounded_wait_runs_out(lib, polls):
    status = C.c_int(-1)
    rc = lib.sns_debug_bounded_wait(polls, C.byref(status))
    assert rc == _lib.SNS_OK, lib.sns_last_error(None)
    assert status.value == 1  # the pass kernels' timeout code
    # the context is still usable
    from spectral_solver_b200 import Solver
    with Solver(8, 1600.0) as s:
        s.step(1e-3, 1)


def test_bounded_wait_rejects_bad_arguments(lib):
    status = C.c_int(0)
    assert lib.sns_debug_bounded_wait(0, C.byref(status)) == _lib.SNS_ERR_INVALID
    assert lib.sns_debug_bounded_wait(1 << 23, C.byref(status)) == _lib.SNS_ERR_INVALID
    assert lib.sns_debug_bounded_wait(16, None) == _lib.SNS_ERR_INVALID
