"""The sphere-pruning tile rule on CPU, against the oracle's mode mask.

The fused forward-z + sweep pass skips a z-pencil tile (my, column block cb of TW = 128 bytes
of complex values) when 4 ((cb * TW)^2 + my^2) > N^2.  Pruning is exact only if such a tile
holds no mode the reference keeps (keep_mode_host, ava_taylor_green_impl.hpp:131-134, as the
oracle states it) and every other tile holds at least one.  bench.py's byte model uses the
same rule for its live fraction.
"""
import numpy as np
import pytest

import bench
from oracle.ref_r2c import half_mode_grids


@pytest.mark.parametrize("n", [16, 24, 32, 64, 128, 256])
@pytest.mark.parametrize("w", [8, 4])  # FP64 (8 complex per tile row) and FP32 (16)
def test_dead_tiles_hold_only_masked_modes(n, w):
    tw = 128 // (2 * w)
    ncb = (n // 2 + tw - 1) // tw
    mx, my, mz = half_mode_grids(n)
    h = 0.5 * n
    keep = ((mx * mx + my * my + mz * mz) / (h * h)) <= 1.0  # the oracle's mask, [mz, my, mx]
    live = 0
    for y in range(n):
        m = y if y <= n // 2 else y - n
        for cb in range(ncb):
            rule_live = 4 * ((cb * tw) ** 2 + m * m) <= n * n
            cols = slice(cb * tw, min(cb * tw + tw, n // 2))  # data columns mx < N/2
            assert rule_live == bool(keep[:, y, cols].any()), (y, cb)
            live += rule_live
    assert bench.live_fraction(n, w) == pytest.approx(live / (n * ncb), rel=0, abs=1e-15)


def test_byte_model_without_pruning_is_the_full_model():
    assert bench.step_bytes_s(1.0) == 261
    b, L = bench.pruned_pass_bytes(512, 4)
    assert 0.80 < L < 0.82
    assert b["p5_sweep"] == pytest.approx(23 * L)
    assert b["p1_zinv_phase"] == 9 and b["p4_yfwd"] == 24
