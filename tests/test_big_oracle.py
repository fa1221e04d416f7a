"""The big-n oracle (oracle/big_oracle.py) against the C oracle's 12-base
Miller-Rabin and against known primes and factorisations."""
import importlib.util
import os

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def big_oracle():
    spec = importlib.util.spec_from_file_location("big_oracle", os.path.join(ROOT, "oracle", "big_oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_agrees_with_c_oracle_below_2_64(oracle):
    B = big_oracle()
    rng = np.random.default_rng(31)
    xs = [int(x) | 1 for x in rng.integers(2**40, 2**63, size=3000, dtype=np.uint64)]
    xs += [2047, 3277, 4033, 25326001, 3215031751, 2152302898747, 3474749660383,
           341550071728321, 3825123056546413051, (1 << 61) - 1, (1 << 64) - 59]
    for x in xs:
        assert B.is_probable_prime(x) == oracle.mr12(x), x


def test_known_large_primes_and_composites():
    B = big_oracle()
    assert B.is_probable_prime(2**89 - 1) and B.is_probable_prime(2**127 - 1)
    assert B.is_probable_prime(2**521 - 1)
    assert not B.is_probable_prime(2**128 + 1)        # 59649589127497217 * 5704689200685129054721
    assert not B.is_probable_prime((2**61 - 1) * (2**89 - 1))
    # 3825123056546413051 is a strong pseudoprime to bases 2..23 but not to 29..37
    assert not B.is_probable_prime(3825123056546413051)


def test_minimal_p_matches_the_c_oracle_below_2_64(oracle):
    B = big_oracle()
    rng = np.random.default_rng(32)
    ns = (rng.integers(2, 2**62, size=300, dtype=np.uint64) * 2).astype(np.uint64)
    pr = B.small_primes(10**5)
    want = oracle.single_minp(ns)
    for n, w in zip(ns, want):
        assert B.minimal_p(int(n), primes=pr) == int(w)
