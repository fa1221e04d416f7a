"""CPU ORACLE for even n beyond 2^64 -- TEST INFRASTRUCTURE ONLY.

Restates, in plain Python big integers, the scan of the reference's
big_check (src/big_check.cpp:35-144: candidate primes p ascending, q = n - p,
a probable-prime test of q) with the minimal-p rule of
src/cpu_goldbach.cpp:14-24 (the first p that works is the answer) and the
strong probable-prime test to the 12 prime bases 2..37 of the reference's
Miller-Rabin (src/goldbach.cu:333-360).  Only tests/ use it, as the checker
of gb_check_big; the product never imports it.
"""
BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def small_primes(limit):
    sieve = bytearray([1]) * (limit + 1)
    sieve[0:2] = b"\0\0"
    for i in range(2, int(limit ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = bytearray(len(range(i * i, limit + 1, i)))
    return [i for i in range(limit + 1) if sieve[i]]


_TRIAL = small_primes(4096)


def sprp(q, a):
    """Strong probable prime to base a (q odd, q > a)."""
    d, s = q - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    x = pow(a, d, q)
    if x == 1 or x == q - 1:
        return True
    for _ in range(s - 1):
        x = x * x % q
        if x == q - 1:
            return True
        if x == 1:
            return False
    return False


def is_probable_prime(q):
    """No prime below 4096 divides q (q itself excepted), and q passes the
    strong test to all 12 bases (a primality proof for q < 3.3e24)."""
    if q < 2:
        return False
    for r in _TRIAL:
        if q == r:
            return True
        if q % r == 0:
            return False
    if q < 4096 * 4096:
        return True
    return all(sprp(q, a) for a in BASES)


def minimal_p(n, p_limit=10**8, primes=None):
    """Smallest prime p <= min(p_limit, n / 2) with n - p a probable prime;
    0 if none.  n even, n >= 4."""
    if n == 4:
        return 2
    primes = primes if primes is not None else small_primes(min(p_limit, 10**6))
    for p in primes[1:]:
        if p > p_limit or p > n // 2:
            break
        if is_probable_prime(n - p):
            return p
    return 0
