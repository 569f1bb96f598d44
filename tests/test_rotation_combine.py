"""CPU check of the rotation epilogue's arithmetic (rot_i8_kernel): the four
INT32 slice accumulators D0..D3 of an output element, combined as one exact
integer D0 2^21 + D1 2^14 + D2 2^7 + D3 (in units of 2^-21), rounded once to
FP32 and scaled by the column's power of two, give the same FP32 bits as the
exact FP64 sum D0 + D1 2^-7 + D2 2^-14 + D3 2^-21 times the scale rounded to
FP32 -- the form it replaced -- for accumulators up to the bounds of K <= 1152
(|D_l| <= (l + 1) 64^2 K)."""
import numpy as np


def test_integer_combination_is_bit_identical_to_the_fp64_one():
    rng = np.random.default_rng(11)
    n = 200000
    K = 1152
    D = [rng.integers(-(l + 1) * 4096 * K, (l + 1) * 4096 * K + 1, n, dtype=np.int64) for l in range(4)]
    # also small values, where the low slices decide the rounding
    D[0][: n // 4] = rng.integers(-3, 4, n // 4)
    e = rng.integers(-40, 10, n)
    scale = np.ldexp(1.0, e)
    v64 = D[0].astype(np.float64) + D[1] * 2.0 ** -7 + D[2] * 2.0 ** -14 + D[3] * 2.0 ** -21
    old = (v64 * scale).astype(np.float32)
    iv = D[0] * 2097152 + D[1] * 16384 + D[2] * 128 + D[3]
    new = iv.astype(np.float32) * (scale * 2.0 ** -21).astype(np.float32)
    np.testing.assert_array_equal(old.view(np.uint32), new.view(np.uint32))
