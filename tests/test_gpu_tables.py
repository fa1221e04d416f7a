"""Device prime tables, the bitset sieve and 64-bit primality against the
oracle and the reference's own outputs."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_prime_table_matches_oracle(ctx, oracle):
    p = ctx.primes_upto(10**8)
    assert len(p) == 5_761_455  # src/test_sieve.cpp:39
    np.testing.assert_array_equal(p.astype(np.uint64), oracle.primes(10**8))


@pytest.mark.parametrize("n,expected", [(10, 4), (100, 25), (1000, 168), (10**4, 1229),
                                        (10**5, 9592), (10**6, 78498), (10**7, 664579)])
def test_pi_known_answers(ctx, n, expected):
    assert len(ctx.primes_upto(n)) == expected


@pytest.mark.parametrize("q_lo,nbits", [(3, 1 << 20), (1, 1000), (10**9 + 1, 1 << 19),
                                        (10**12 + 1, (1 << 20) + 7), (10**15 + 1, 1 << 17),
                                        (2**40 + 1, 123457)])
def test_sieve_bitset_matches_oracle(ctx, oracle, q_lo, nbits):
    np.testing.assert_array_equal(ctx.sieve_bitset(q_lo, nbits), oracle.odd_bitset(q_lo, nbits))


def test_window_prime_counts_match_reference(ctx):
    g = json.load(open(os.path.join(GOLD, "ref_window_pi.json")))
    for w in g["windows"]:
        lo, hi = w["low"], w["high"]
        q_lo = lo | 1
        nbits = (hi - q_lo) // 2 + 1
        bits = ctx.sieve_bitset(q_lo, nbits)
        c = int(np.unpackbits(bits.view(np.uint8)).sum()) + (1 if lo <= 2 <= hi else 0)
        assert c == w["count"], w


def test_is_prime_matches_reference_mr(ctx):
    g = json.load(open(os.path.join(GOLD, "ref_mr.json")))
    n = np.array([int(x) for x in g["n"]], dtype=np.uint64)
    np.testing.assert_array_equal(ctx.is_prime(n), np.array(g["prime"], bool))


def test_is_prime_exhaustive_small(ctx, oracle):
    n = np.arange(0, 1 << 20, dtype=np.uint64)
    ps = np.zeros(1 << 20, bool)
    ps[oracle.primes((1 << 20) - 1).astype(np.int64)] = True
    np.testing.assert_array_equal(ctx.is_prime(n), ps)


def test_is_prime_random_64bit(ctx, oracle):
    rng = np.random.default_rng(7)
    n = rng.integers(0, 2**63, size=20000, dtype=np.uint64) * 2 + 1
    got = ctx.is_prime(n)
    want = np.array([oracle.mr7(int(x)) for x in n])
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("q_lo,nbits", [(2**64 - 2**21 + 1, 2**20), (2**63 + 1, 100003),
                                        (2**62 + 2**31 + 1, 65536)])
def test_sieve_bitset_near_the_top_of_uint64(ctx, q_lo, nbits):
    """Windows that need sieving primes above 2^31 (q > 2^62) against the
    device Miller-Rabin (itself checked against the reference's MR)."""
    bits = ctx.sieve_bitset(q_lo, nbits)
    got = np.unpackbits(bits.view(np.uint8), bitorder="little")[:nbits].astype(bool)
    q = q_lo + 2 * np.arange(nbits, dtype=np.uint64)
    np.testing.assert_array_equal(got, ctx.is_prime(q))
