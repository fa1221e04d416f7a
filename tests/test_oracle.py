"""The CPU oracle pinned against the reference's own tests and outputs.

Known answers: src/test_sieve.cpp:31-40, src/test_bitset.cpp:17-74.
Fixtures: tests/golden/*.json, produced by tests/golden/make_golden.py from
the reference's code compiled from its sources (oracle/_ref).
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def gold(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


# pi(n) table of src/test_sieve.cpp:31-40 (and test_bitset.cpp:43-50)
PI = [(10, 4), (100, 25), (1000, 168), (10_000, 1229), (100_000, 9592), (1_000_000, 78498),
      (10_000_000, 664579), (100_000_000, 5761455)]


@pytest.mark.parametrize("n,expected", PI)
def test_pi_known_answers(oracle, n, expected):
    assert oracle.count_primes(0, n) == expected


def test_primes_up_to_30(oracle):  # src/test_bitset.cpp:19
    assert oracle.primes(30).tolist() == [2, 3, 5, 7, 11, 13, 17, 19, 23, 29]


def test_odd_bitset_matches_byte_sieve(oracle):
    q_lo, nbits = 10**12 + 1, 5000
    w = oracle.odd_bitset(q_lo, nbits)
    bits = np.unpackbits(w.view(np.uint8), bitorder="little")[:nbits]
    byte = np.zeros(2 * nbits, np.uint8)
    oracle.L.gbo_segmented_sieve(q_lo, q_lo + 2 * nbits - 1, byte.ctypes.data)
    assert (bits == byte[::2]).all()


def test_window_prime_counts_match_reference(oracle):
    for w in gold("ref_window_pi.json")["windows"]:
        assert oracle.count_primes(w["low"], w["high"]) == w["count"], w


def test_miller_rabin_matches_reference(oracle):
    g = gold("ref_mr.json")
    for s, p in zip(g["n"], g["prime"]):
        n = int(s)
        assert oracle.mr12(n) == bool(p), n
        assert oracle.mr7(n) == bool(p), n


def test_mr7_exhaustive_small(oracle):
    ps = set(oracle.primes(200_000).tolist())
    for n in range(0, 200_000):
        assert oracle.mr7(n) == (n in ps), n


def test_goldbach_count_matches_reference(oracle):
    g = gold("ref_goldbach_count.json")
    for j, c in enumerate(g["counts"][:600]):
        assert oracle.goldbach_count(4 + 2 * j) == c


def test_cpu_goldbach_summary_matches_reference(oracle):
    for r in gold("ref_cpu_goldbach.json")["runs"]:
        s, _ = oracle.verify_range(4, r["limit"])
        assert s["checked"] == r["checked"]
        assert s["failures"] == r["failures"] == 0
        assert "satisfy Goldbach" in r["final"]


def test_minp_small_brute_force_fixture(oracle):
    g = gold("minp_small.json")
    mp = oracle.minp(4, len(g["min_p"]))
    assert mp.tolist() == g["min_p"]


def test_minp_windows_match_reference_scan(oracle):
    import hashlib
    for w in gold("ref_window_minp.json")["windows"]:
        mp = oracle.minp(w["start"], w["count"])
        assert hashlib.sha256(mp.tobytes()).hexdigest() == w["sha256"], w["start"]
        assert w["unverified"] == 0


def test_phase2_check_matches_reference(oracle):
    g = gold("ref_phase2.json")
    for s, ok in zip(g["n"], g["verified"]):
        assert (oracle.phase2_minp(int(s)) > 0) == bool(ok)


def test_phase2_and_window_paths_agree(oracle):
    # src/goldbach.cu:362-373 and the window scan give the same minimal p
    start = 10**13 + 40
    mp = oracle.minp(start, 500)
    for j in range(0, 500, 7):
        assert oracle.phase2_minp(start + 2 * j) == mp[j]


def test_single_minp_is_window_minp(oracle):
    start = 10**15 + 2
    mp = oracle.minp(start, 300)
    ns = start + 2 * np.arange(300, dtype=np.uint64)
    assert (oracle.single_minp(ns) == mp).all()


def test_oracle_hist_1e9_fixture_small_prefix(oracle):
    # the [4, 1e9] fixture (validation_gpu.sh:48-54 asserts 0 Phase-2
    # fallbacks at p_small = 1e5); recompute the summary for a prefix
    g = gold("oracle_hist_1e9.json")
    assert g["fallbacks"] == 0 and g["failures"] == 0 and g["checked"] == 499_999_999
    assert g["max_minp"] == 1789 and g["max_minp_n"] == 721_013_438
    s, h = oracle.verify_range(4, 10**7, p_small=10**5)
    assert s["fallbacks"] == 0 and s["checked"] == 4_999_999
    assert int(h.sum()) == 4_999_999


def test_oracle_failure_semantics(oracle):
    # with bounds 3 the first n whose minimal p exceeds 3 is 12 (= 5 + 7)
    s, _ = oracle.verify_range(4, 100, p_small=3, phase2=3)
    assert s["first_failure"] == 12
    mp = oracle.minp(4, 49, p_limit=3)
    fails = [4 + 2 * j for j in range(49) if mp[j] == 0]
    assert fails[0] == 12 and s["failures"] == len(fails)


def test_published_single_check_partitions_bound_minp(oracle):
    # RESULTS.md:112-121 (valid, not minimal): minimal p <= published p
    pub = {10**12: 194267, 10**13: 90059, 10**14: 145391, 10**15: 152639, 10**16: 56687,
           10**17: 91967, 10**18: 14831, 10**19: 226283}
    ns = np.array(list(pub), dtype=np.uint64)
    mp = oracle.single_minp(ns)
    for n, p in zip(pub, mp):
        assert 0 < p <= pub[n]
        assert oracle.mr7(int(p)) and oracle.mr7(n - int(p))


def test_minp_over_c1_matches_reference_hash(oracle):
    # [4, 1e9] whole (C1): the oracle's minimal p of all 499,999,999 n and the
    # verified bitmap hash to what the reference's own scan produced
    import hashlib
    g = gold("ref_c1_1e9.json")
    count = g["checked"]
    mp = oracle.minp(4, count)
    assert hashlib.sha256(mp.tobytes()).hexdigest() == g["min_p_sha256"]
    bits = np.packbits(mp > 0, bitorder="little")
    bits = np.concatenate([bits, np.zeros(4 * ((count + 31) // 32) - len(bits), np.uint8)])
    assert hashlib.sha256(bits.tobytes()).hexdigest() == g["verified_bits_sha256"]
    assert int(mp.max()) == g["max_minp"] and g["cpu_goldbach_failures"] == 0
