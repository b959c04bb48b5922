"""The encoding of the FP32 precision form's compensated state, restated in numpy (CPU).

The sweep kernels carry each real part of u as hi + lo: hi = round-to-nearest FP32 of the
FP64 update U, and the remainder U - hi as an int8 q, in units of ulp(hi) / 255, truncated
toward zero after a nudge of 1e-6 away from it (comp_encode / comp_decode in
spectral_solver_b200/csrc/sns_kernels.cu; ulp(hi) = 2^(E - 150) for the biased exponent E,
taken as at least 1; multiplications by exact powers of two and by 255 or 1/255, no
division).  Three properties make the scheme work:
* decoding hi + q ulp / 255 in FP64 and encoding again gives the same pair (get_state ->
  set_state, checkpoint -> resume are exact);
* round-to-nearest FP32 of the decoded value is hi (the stored FP32 value is the nearest
  one, including just below a power of two, where the lower neighbour is half an ulp away);
* the decoded value is within ulp(hi) / 255 of U (about 2^-31 relative, against 2^-24 for
  FP32 alone).
"""
import numpy as np


def exp_of(hi):
    return np.maximum(((hi.view(np.uint32) >> 23) & 0xFF).astype(np.int64), 1)


def ulp_of(hi):
    return np.ldexp(1.0, exp_of(hi) - 150)


def encode(U):
    hi = U.astype(np.float32)
    r = (U - hi.astype(np.float64)) * np.ldexp(1.0, 150 - exp_of(hi)) * 255.0
    q = np.trunc(r + np.copysign(1e-6, r)).astype(np.int64)
    assert np.all(np.abs(q) <= 127)
    return hi, q


def decode(hi, q):
    return hi.astype(np.float64) + q * ulp_of(hi) * (1.0 / 255.0)


def cases():
    rng = np.random.default_rng(11)
    mags = 10.0 ** rng.uniform(-40, 3, 200000)
    U = mags * rng.choice([-1.0, 1.0], mags.size) * rng.uniform(0.5, 2.0, mags.size)
    # values next to FP32 binade edges, exact FP32 ties and the subnormal range
    p2 = 2.0 ** rng.integers(-140, 10, 4000).astype(np.float64)
    edges = np.concatenate([p2 * (1 - 2.0 ** -25), p2 * (1 + 2.0 ** -24), p2 * (1 - 2.0 ** -26),
                            p2 * (1 + 3 * 2.0 ** -25), p2 * (1 + 2.0 ** -30), p2 * (1 - 2.0 ** -26 + 2.0 ** -40)])
    return np.concatenate([U, edges, -edges, [0.0, 1e-45, -3e-46]])


def test_round_trip_is_exact():
    hi, q = encode(cases())
    hi2, q2 = encode(decode(hi, q))
    assert np.array_equal(hi, hi2)
    assert np.array_equal(q, q2)


def test_hi_is_round_to_nearest_of_the_pair():
    hi, q = encode(cases())
    assert np.array_equal(decode(hi, q).astype(np.float32), hi)


def test_error_bound():
    U = cases()
    hi, q = encode(U)
    err = np.abs(decode(hi, q) - U)
    assert np.all(err <= ulp_of(hi) / 255.0 * 1.001)
    # against FP32 alone: the remainder carries about 8 more bits
    e32 = np.abs(hi.astype(np.float64) - U)
    big = np.abs(U) > 1e-30
    assert np.median(err[big] / np.maximum(e32[big], 1e-300)) < 2.0 ** -6
