"""The benchmark configurations in full, against the CPU oracle.

C1: every even n in [4, 1e9] with SEG_SIZE 2^26 and P_SMALL 1e8, the
    per-n outputs of the whole range (minimal p as uint32, 2 GB; the
    verified bitmap, 62.5 MB) hashed and compared with the oracle and with
    the hash of the reference's own segmented_sieve + cpu_goldbach scan rule
    (tests/golden/ref_c1_1e9.json), and the summary with cpu_goldbach's
    own output for LIMIT = 1e9.
C3: the benchmark's seeded windows in [1e15, 1e18] (seed 1), the widest
    (about 2^24 even n) among them, in both pipelines.
C4: the benchmark's whole batch of 1e6 seeded single n (seed 2).
"""
import hashlib
import importlib.util
import json
import os

import numpy as np
import pytest

from oracle_lib import hist_of

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _bench():
    spec = importlib.util.spec_from_file_location("gb_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_c1_full_range_per_n_outputs(ctx, oracle):
    g = json.load(open(os.path.join(GOLD, "ref_c1_1e9.json")))
    start, limit = 4, 10**9
    count = (limit - start) // 2 + 1
    r = ctx.verify_range(start, limit, seg_size=1 << 26, p_small=10**8, want_minp=True,
                         want_bits=True, want_hist=True, want_seg=True)
    res = r.result
    assert res["checked"] == count == g["checked"]
    assert res["num_segments"] == 8
    # the reference's own scan over the whole range, hashed
    assert _sha(r.min_p) == g["min_p_sha256"]
    assert _sha(r.verified_bits) == g["verified_bits_sha256"]
    # and the oracle, computed here on all host cores
    mp = oracle.minp(start, count, p_limit=10**8)
    if _sha(r.min_p) != _sha(mp):
        bad = np.nonzero(r.min_p != mp)[0]
        raise AssertionError(("first mismatch", int(start + 2 * bad[0]), int(r.min_p[bad[0]]),
                              int(mp[bad[0]])))
    bits = np.packbits(mp > 0, bitorder="little")
    bits = np.concatenate([bits, np.zeros(4 * len(r.verified_bits) - len(bits), np.uint8)])
    assert _sha(bits.view(np.uint32)) == _sha(r.verified_bits)
    # cpu_goldbach's summary for LIMIT = 1e9 (the reference binary's output)
    assert res["failures"] == g["cpu_goldbach_failures"] == 0
    assert res["verified"] == count
    assert res["phase2_fallbacks"] == 0  # every minimal p is below P_SMALL = 1e8
    assert res["max_minp"] == int(mp.max()) == g["max_minp"]
    assert not r.seg_fallbacks.any() and not r.seg_failures.any()
    np.testing.assert_array_equal(r.hist, hist_of(mp, oracle.primes(10**6)))


@pytest.fixture(scope="module")
def c3_windows(oracle):
    """The 8 widest of the benchmark's 4096 windows, 24 others drawn by seed
    (narrow ones among them take the Miller-Rabin path), and windows of
    width 2^18, 2^20 and 2^22 ending near 1e18; with the oracle's minimal p."""
    starts, counts = _bench().seeded_windows()
    order = np.argsort(counts)[::-1]
    rng = np.random.default_rng(0xC3)
    pick = np.concatenate([order[:8], rng.choice(order[8:], size=24, replace=False)])
    s = list(starts[pick]) + [10**18 - 2 * (1 << 18), 10**18 - 2 * (1 << 20) - 10**6,
                              10**18 - 2 * (1 << 22) - 10**9]
    c = list(counts[pick]) + [1 << 18, 1 << 20, 1 << 22]
    s = np.array(s, dtype=np.uint64)
    c = np.array(c, dtype=np.uint64)
    assert c.max() >= 1 << 23 and c.min() < 1 << 14
    return s, c, oracle.minp_windows(s, c)


@pytest.mark.parametrize("mode", [0, 1])
def test_c3_wide_windows(ctx, c3_windows, mode):
    s, c, want = c3_windows
    per, minp, summ = ctx.verify_windows(s, c, mode=mode, want_minp=True)
    bad = np.nonzero(minp != want)[0]
    assert bad.size == 0, (bad[:8], minp[bad[:8]], want[bad[:8]])
    off = 0
    for i, k in enumerate(c):
        w = want[off:off + int(k)]
        assert per[i]["verified"] == k and per[i]["failures"] == 0
        assert per[i]["max_minp"] == int(w.max())
        assert per[i]["minp_sum"] == int(w.astype(np.uint64).sum())
        off += int(k)
    assert summ["total_n"] == int(c.sum()) and summ["failures"] == 0


@pytest.mark.parametrize("mr_below", [1, 1 << 21])
def test_c3_sieve_and_miller_rabin_paths_on_wide_windows(ctx, c3_windows, mr_below):
    """Every window sieved (mr_below = 1), or every window up to 2^21 n on
    the Miller-Rabin path: the same minimal p."""
    s, c, want = c3_windows
    keep = c <= (1 << 21)
    offs = np.concatenate([[0], np.cumsum(c.astype(np.int64))])
    sub = np.concatenate([want[offs[i]:offs[i + 1]] for i in np.nonzero(keep)[0]])
    _, minp, _ = ctx.verify_windows(s[keep], c[keep], want_minp=True, mr_below=mr_below)
    np.testing.assert_array_equal(minp, sub)


def test_c4_full_batch(ctx, oracle):
    rng = np.random.default_rng(2)
    n = (rng.integers(2, 2**63, size=10**6, dtype=np.uint64) * 2).astype(np.uint64)
    p, q, r = ctx.check_single(n)
    want = oracle.single_minp(n)
    bad = np.nonzero(p != want)[0]
    assert bad.size == 0, (n[bad[:8]], p[bad[:8]], want[bad[:8]])
    np.testing.assert_array_equal(q, n - p)
    assert r.found == len(n) and r.max_p == int(want.max())
