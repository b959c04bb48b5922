"""The encoding of the FP32 precision form's compensated state, restated in numpy (CPU).

The sweep kernels carry each real part of u as hi + lo: hi = round-to-nearest FP32 of the
FP64 update U, lo = U - hi rounded toward zero, first to FP32 and then to bf16 by dropping
the low 16 bits, a zero remainder always stored as +0 (comp_encode in
spectral_solver_b200/csrc/sns_kernels.cu).  Two properties
make the scheme exact through the host: decoding hi + lo in FP64 and encoding again gives the
same pair (get_state -> set_state, checkpoint -> resume), and hi + lo is within 2^-30 |U|
of U (the error the FP32 form keeps per stage, against 2^-24 without lo).
"""
import numpy as np


def encode(U):
    hi = U.astype(np.float32)
    rem = U - hi.astype(np.float64)  # exact
    lo32 = rem.astype(np.float32)
    # round toward zero: step back where round-to-nearest went up in magnitude
    up = np.abs(lo32.astype(np.float64)) > np.abs(rem)
    lo32 = np.where(up, np.nextafter(lo32, np.float32(0)), lo32)
    bits = lo32.view(np.uint32) & np.uint32(0xFFFF0000)
    bits = np.where(bits & np.uint32(0x7FFFFFFF), bits, np.uint32(0))  # no negative zeros
    return hi, bits.view(np.float32)


def decode(hi, lo):
    return hi.astype(np.float64) + lo.astype(np.float64)


def cases():
    rng = np.random.default_rng(11)
    mags = 10.0 ** rng.uniform(-30, 3, 200000)
    U = mags * rng.choice([-1.0, 1.0], mags.size) * rng.uniform(0.5, 2.0, mags.size)
    # values next to FP32 binade edges and exact FP32 ties
    p2 = 2.0 ** rng.integers(-40, 10, 4000).astype(np.float64)
    edges = np.concatenate([p2 * (1 - 2.0 ** -25), p2 * (1 + 2.0 ** -24), p2 * (1 - 2.0 ** -26),
                            p2 * (1 + 3 * 2.0 ** -25), p2 * (1 + 2.0 ** -30)])
    return np.concatenate([U, edges, -edges, [0.0]])


def test_round_trip_is_exact():
    U = cases()
    hi, lo = encode(U)
    hi2, lo2 = encode(decode(hi, lo))
    assert np.array_equal(hi, hi2)
    assert np.array_equal(lo.view(np.uint32), lo2.view(np.uint32))


def test_hi_is_round_to_nearest_of_the_pair():
    U = cases()
    hi, lo = encode(U)
    assert np.array_equal(decode(hi, lo).astype(np.float32), hi)


def test_error_bound():
    U = cases()
    hi, lo = encode(U)
    err = np.abs(decode(hi, lo) - U)
    tiny = np.abs(U) < 1e-36  # FP32 subnormals: bounded by the smallest FP32 step instead
    assert np.all(err[~tiny] <= 2.0 ** -30 * np.abs(U[~tiny]))
    assert np.all(err[tiny] <= 2.0 ** -149)
    # against FP32 alone: the remainder carries the next 8 bits
    e32 = np.abs(hi.astype(np.float64) - U)
    big = np.abs(U) > 1e-30
    assert np.median(err[big] / np.maximum(e32[big], 1e-300)) < 2.0 ** -7
