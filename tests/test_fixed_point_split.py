"""The FP64 tile spreader's exact three-word split, restated on the host.

k_spread_t (curig_b200/csrc/kernels.cu, split_fix3) adds a scaled term x
(|x| <= 2^54) to three int32 planes as x = h 2^36 + m 2^18 + l: adding
1.5 * 2^70 rounds x to a multiple of 2^18 whose quotient X is the difference of
the bit patterns, h = X >> 18, m = X & (2^18 - 1), and the remainder
x - X 2^18 (exact) is rounded to the integer l by adding 1.5 * 2^52.  The same
IEEE double additions in Python reproduce it bit for bit; this checks the
ranges that keep the planes' sums of up to 4096 terms inside int32 and that
the only rounding is l's (at most 1/2)."""
import struct

import numpy as np

M18 = 1.5 * 2.0 ** 70
M0 = 1.5 * 2.0 ** 52


def _bits(d):
    return struct.unpack("<q", struct.pack("<d", d))[0]


def split3(x):
    t1 = x + M18
    t2 = (x - (t1 - M18)) + M0
    X = _bits(t1) - _bits(M18)
    return X >> 18, X & 0x3FFFF, _bits(t2) - _bits(M0)


def test_split_is_exact_up_to_the_last_rounding():
    rng = np.random.default_rng(3)
    xs = list(rng.uniform(-1, 1, 20000) * 2.0 ** rng.uniform(-40, 54, 20000))
    xs += [2.0 ** 54, -2.0 ** 54, 2.0 ** 54 * (1 - 2.0 ** -52), 0.5, -0.5, 1.5, -1.5, 2.0 ** 17 + 0.5, 0.0]
    for x in xs:
        h, m, l = split3(float(x))
        assert -2 ** 18 <= h <= 2 ** 18
        assert 0 <= m < 2 ** 18
        assert -2 ** 17 <= l <= 2 ** 17
        # h, m, l are integers, x a double: the comparison is exact
        assert abs(x - (h * 2 ** 36 + m * 2 ** 18 + l)) <= 0.5


def test_plane_sums_of_4096_terms_stay_in_int32():
    n = 4096
    worst_h = n * 2 ** 18
    worst_m = n * (2 ** 18 - 1)
    worst_l = n * 2 ** 17
    assert worst_h <= 2 ** 31 - 1 and worst_m <= 2 ** 31 - 1 and worst_l <= 2 ** 31 - 1
    # and a random accumulation reconstructs the exact integer sum
    rng = np.random.default_rng(4)
    xs = rng.uniform(-2.0 ** 54, 2.0 ** 54, n)
    H = M = L = 0
    exact = 0
    for x in xs:
        h, m, l = split3(float(x))
        H, M, L = H + h, M + m, L + l
        exact += h * 2 ** 36 + m * 2 ** 18 + l
    assert H * 2 ** 36 + M * 2 ** 18 + L == exact
    assert abs(H) < 2 ** 31 and 0 <= M < 2 ** 31 and abs(L) < 2 ** 31
