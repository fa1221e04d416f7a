"""The integer arithmetic the kernels rely on, restated in Python and checked
on the CPU (the GPU tests check the device code against the oracle):

* the double-precision quotient estimate of mod_p_f64 (gb_device.cuh):
  within 1 of floor(x / p) whenever x / p < 2^51;
* the 32-bit-limb Montgomery product of mont_mul32 (gb_device.cuh), step by
  step with its carries, against a * b * 2^-64 mod n;
* R mod n without division (mont32_init, kernels/single.cu) and the
  Newton inverse -n^-1 mod 2^32;
* the exact-division test of the single-n filter: r | x iff
  x * r^-1 mod 2^32 <= (2^32 - 1) / r for odd r.
"""
import random

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
