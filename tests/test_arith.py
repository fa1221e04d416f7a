"""The integer arithmetic the kernels rely on, restated in Python and checked
on the CPU (the GPU tests check the device code against the oracle):

* the double-precision quotient estimate of mod_p_f64 (gb_device.cuh):
  within 1 of floor(x / p) whenever x / p < 2^51;
* the sieve's G0 mod p from one FMA of G0 / 2^64 by the Barrett magic as
  a double (near_mod, kernels/sieve6.cuh), for 0 <= G0 < 2^53, p < 2^31;
* the windows' large-prime remainder from one FMA of g0 (a double) by a
  reciprocal built from the single-precision one and a Newton step
  (large_prime / large_pair, kernels/windows.cu), for g0 < 2^62,
  2^20 < p < 2^31;
* the 32-bit-limb Montgomery product of mont_mul32 (gb_device.cuh), step by
  step with its carries, against a * b * 2^-64 mod n;
* R mod n without division (mont32_init, kernels/single.cu) and the
  Newton inverse -n^-1 mod 2^32;
* the exact-division test of the single-n filter: r | x iff
  x * r^-1 mod 2^32 <= (2^32 - 1) / r for odd r.
"""
import random
from fractions import Fraction

import numpy as np

M32 = (1 << 32) - 1


def test_double_quotient_estimate_within_one():
    rng = random.Random(5)
    cases = []
    for _ in range(20000):
        p = rng.choice([rng.randrange(1 << 13, 1 << 32), rng.randrange(1 << 17, 1 << 30), (1 << 32) - 5])
        x = rng.choice([rng.randrange(0, 1 << 64), (1 << 64) - 1 - rng.randrange(1 << 20),
                        p * rng.randrange(1, ((1 << 64) - 1) // p), p * rng.randrange(1, ((1 << 64) - 1) // p) - 1])
        cases.append((x, p))
    for x, p in cases:
        assert x // p < 1 << 51
        q = int(float(x) * (1.0 / p))  # round-to-nearest conversions and product, truncation
        assert abs(q - x // p) <= 1
        r = x - q * p
        assert -p < r < 2 * p


def _fma(a, b, c):
    """a * b + c with one rounding to the nearest double."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _low32_of_rounded(est):
    """The low 32 bits of the integer held by a double in [2^52, 2^53)."""
    assert 2.0**52 <= est < 2.0**53
    return int(est) & M32


def test_sieve_remainder_from_the_barrett_magic_as_a_double():
    rng = random.Random(11)
    for _ in range(20000):
        p = rng.choice([71, 73, 1009, 999983, (1 << 31) - 1, rng.randrange(71, 1 << 31) | 1])
        g0 = rng.choice([rng.randrange(0, 1 << 53), rng.randrange(0, 1 << 40),
                         (rng.randrange(0, (1 << 53) // p) * p + rng.choice([0, 1, p - 1])) % (1 << 53)])
        magic = ((1 << 64) - 1) // p
        est = _fma(g0 * 2.0**-64, float(magic), 1.5 * 2.0**52)
        r = (g0 - _low32_of_rounded(est) * p) & M32
        r = min(r, (r + p) & M32)
        assert r == g0 % p, (g0, p)


def test_window_remainder_from_the_newton_reciprocal():
    rng = random.Random(13)
    for _ in range(20000):
        p = rng.choice([(1 << 20) + 7, (1 << 31) - 1, rng.randrange((1 << 20) + 1, 1 << 31) | 1])
        g0 = rng.choice([rng.randrange(1 << 30, 1 << 62), (1 << 62) - 1 - rng.randrange(1 << 20),
                         p * rng.randrange(1, ((1 << 62) - 1) // p) + rng.choice([0, 1, p - 1])])
        g0 = min(g0, (1 << 62) - 1)
        pd = float(p)
        r0 = float(np.float32(1.0) / np.float32(p))  # __frcp_rn((float)p)
        inv = _fma(r0, _fma(-pd, r0, 1.0), r0)
        est = _fma(float(g0), inv, 1.5 * 2.0**52)
        r = (g0 - _low32_of_rounded(est) * p) & M32
        r = min(r, (r + p) & M32)
        assert r == g0 % p, (g0, p)


def _mont_mul32(a, b, n, ninv0):
    """mont_mul32's steps: the 128-bit a*b on 32-bit limbs, two reduction
    steps with m = t_i * ninv0 mod 2^32, one conditional subtraction."""
    t = [0] * 5
    T = a * b
    for i in range(4):
        t[i] = (T >> (32 * i)) & M32

    def add_at(i, v):
        s = sum(t[j] << (32 * j) for j in range(5)) + (v << (32 * i))
        assert s >> 160 == 0
        for j in range(5):
            t[j] = (s >> (32 * j)) & M32

    n0, n1 = n & M32, n >> 32
    for i in range(2):
        m = (t[i] * ninv0) & M32
        add_at(i, m * n0)
        add_at(i + 1, m * n1)
        assert t[i] == 0
    r = t[2] | (t[3] << 32) | (t[4] << 64)
    assert r < 2 * n
    return r - n if r >= n else r


def test_montgomery_product_on_32bit_limbs():
    rng = random.Random(7)
    for _ in range(20000):
        n = rng.randrange(3, 1 << 64) | 1
        if rng.random() < 0.3:
            n = (1 << 64) - 1 - 2 * rng.randrange(1 << 20)
        a, b = rng.randrange(n), rng.randrange(n)
        ninv0 = (-pow(n & M32, -1, 1 << 32)) & M32
        assert _mont_mul32(a, b, n, ninv0) == a * b * pow(1 << 64, -1, n) % n


def test_r_mod_n_by_doubling_and_newton_inverse():
    rng = random.Random(9)
    for _ in range(20000):
        n = rng.randrange(1 << 20, 1 << 64) | 1
        k = n.bit_length() - 1
        x = (1 << 64) - n if k == 63 else (2 << k) - n
        for _ in range(k + 1, 64):
            x = x + x - n if x + x >= n else x + x
        assert x == (1 << 64) % n
        r = n & M32
        y = r
        for _ in range(4):  # 3 -> 6 -> 12 -> 24 -> 48 correct bits
            y = (y * (2 - r * y)) & M32
        assert (r * y) & M32 == 1


def test_exact_division_filter():
    rng = random.Random(11)
    for r in (3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61):
        inv = pow(r, -1, 1 << 32)
        lim = M32 // r
        for x in [0, r, r - 1, M32 - M32 % r, M32] + [rng.randrange(1 << 28) for _ in range(3000)]:
            assert ((x * inv) & M32 <= lim) == (x % r == 0)
