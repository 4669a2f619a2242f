"""Exactness of the arithmetic the int8 product kernels rely on, restated in Python doubles
(IEEE binary64, as on the device):

* slicing: the digits cut from v = rint(x 2^(7S - e)) in FP64 (t = rint(r 2^-k), r -= t 2^k)
  equal the integer digits (round half to even at every level), ties included, and stay in
  [-127, 127];
* epilogue: x 2^k computed as x 2^(k >> 1) 2^(k - (k >> 1)) equals ldexp(x, k) whenever the
  result is a normal number.
"""
import math

import numpy as np

S = 5
LIM = int(127.5 * 2 ** 28) - 1   # |v| < 127.5 2^28: the row exponent is raised when 128 m >= 127.5


def _int_digits(r):
    out = []
    for q in range(S):
        if q < S - 1:
            k = 7 * (S - 1 - q)
            half = 1 << (k - 1)
            t = (r + half) >> k
            if ((r + half) & ((1 << k) - 1)) == 0 and (t & 1):
                t -= 1
            out.append(t)
            r -= t << k
        else:
            out.append(r)
    return out


def _fp_digits(r):
    r = float(r)
    out = []
    for q in range(S):
        if q < S - 1:
            k = 7 * (S - 1 - q)
            t = float(np.rint(r * 2.0 ** -k))
            r = r - t * 2.0 ** k
            out.append(int(t))
        else:
            out.append(int(r))
    return out


def test_fp64_digits_equal_integer_digits():
    rng = np.random.default_rng(0)
    vals = [int(v) for v in rng.integers(-LIM, LIM, 40000)]
    for k in (28, 21, 14, 7):   # exact ties at every level
        q = LIM // (1 << (k - 1))
        vals += [int(m) * (1 << (k - 1)) for m in rng.integers(-q, q, 4000)]
    vals += list(range(-3000, 3000)) + [LIM, -LIM]
    for v in vals:
        d = _fp_digits(v)
        assert d == _int_digits(v), v
        assert all(-127 <= x <= 127 for x in d), v
        assert sum(x * 2 ** (7 * (S - 1 - i)) for i, x in enumerate(d)) == v


def _pow2_normal(k):
    if k > 1023:
        return math.inf
    if k < -1022:
        return 0.0
    return math.ldexp(1.0, k)


def test_two_product_power_of_two_scaling_equals_ldexp():
    rng = np.random.default_rng(1)
    checked = 0
    for _ in range(50000):
        x = float(rng.uniform(-1, 1)) * 2.0 ** int(rng.integers(-60, 90))
        k = int(rng.integers(-2162, 2035))
        try:
            ref = math.ldexp(x, k)
        except OverflowError:
            continue
        if abs(ref) < 2.0 ** -1022:
            continue
        k1 = k >> 1
        assert x * _pow2_normal(k1) * _pow2_normal(k - k1) == ref, (x, k)
        checked += 1
    assert checked > 1000
