"""Range verification on the GPU against the CPU oracle, bit for bit.

Per n: the minimal p (src/cpu_goldbach.cpp:14-24 rule) and the verified
bit; per call: the reference's summary figures (checked, Phase-2 fallbacks
of src/goldbach.cu:799, failures, first failing n) and the minimal-p
histogram; per segment: fallbacks, failures and histograms.
"""
import numpy as np
import pytest

from oracle_lib import hist_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def primes(oracle):
    return oracle.primes(2_000_000)


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x, z ^ (z >> 31)


def run_and_check(ctx, oracle, primes, start, count, p_small=10**6, phase2_limit=10**8, **kw):
    limit = start + 2 * (count - 1)
    r = ctx.verify_range(start, limit, p_small=p_small, phase2_limit=phase2_limit,
                         want_minp=True, want_bits=True, want_hist=True, **kw)
    mp = oracle.minp(start, count, p_limit=max(p_small, phase2_limit))
    bad = np.nonzero(r.min_p != mp)[0]
    assert bad.size == 0, (start, bad[:8], r.min_p[bad[:8]], mp[bad[:8]])
    bits = np.unpackbits(r.verified_bits.view(np.uint8), bitorder="little")
    assert (bits[:count] == (mp > 0)).all()
    assert not bits[count:].any()
    np.testing.assert_array_equal(r.hist, hist_of(mp, primes))
    res = r.result
    assert res["checked"] == count
    assert res["failures"] == int((mp == 0).sum())
    assert res["verified"] == int((mp > 0).sum())
    assert res["phase2_fallbacks"] == int(((mp == 0) | (mp > p_small)).sum())
    assert res["max_minp"] == int(mp.max())
    fails = np.nonzero(mp == 0)[0]
    assert res["first_failure_n"] == (start + 2 * int(fails[0]) if fails.size else 0)
    return r, mp


@pytest.mark.parametrize("start,count", [
    (4, 1 << 21),                         # from the bottom: n = 4, p <= n/2 masking
    (10**9 - (1 << 21), 1 << 20),          # below 1e9
    (10**12 - (1 << 21), 1 << 20),         # below 1e12 (sieving primes to 1e6)
    (10**15 + 2, 1 << 17),                 # sieving primes to 3.2e7
    (123456789012, 777777),                # ragged count
])
def test_minp_bit_exact(ctx, oracle, primes, start, count):
    run_and_check(ctx, oracle, primes, start, count)


def test_reference_fixture_windows(ctx, oracle, primes):
    # windows whose minimal p the reference's own code produced
    import hashlib
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_window_minp.json")))
    for w in g["windows"]:
        r = ctx.verify_range(w["start"], w["start"] + 2 * (w["count"] - 1), want_minp=True)
        assert hashlib.sha256(r.min_p.tobytes()).hexdigest() == w["sha256"], w["start"]
        assert r.result["failures"] == w["unverified"] == 0


@pytest.mark.parametrize("chunk", [8192, 32768, 1 << 20])
def test_chunk_sizes(ctx, oracle, primes, chunk):
    run_and_check(ctx, oracle, primes, 10**11 + 2, 300_001, chunk=chunk)


@pytest.mark.parametrize("halo", [128, 1024, 1 << 17])
def test_halo_sizes_and_phase2_path(ctx, oracle, primes, halo):
    r, mp = run_and_check(ctx, oracle, primes, 10**9 + 2, 1 << 16, halo=halo)
    if halo == 128:
        # the window search covers the primes p <= H - 13 (every q = n - p
        # then lies inside the chunk's q-window); larger minimal p go to
        # the device Phase 2
        assert r.result["queued"] == int((mp > halo - 13).sum()) > 0


def test_bounds_force_failures(ctx, oracle, primes):
    # with P_SMALL = phase2 = 3 every n whose minimal p exceeds 3 fails; the
    # first is 12 (src/goldbach.cu:476-479 reports the first failing n)
    r, mp = run_and_check(ctx, oracle, primes, 4, 500, p_small=3, phase2_limit=3)
    assert r.result["first_failure_n"] == 12 and r.result["failures"] > 0


def test_fallback_count_small_p_small(ctx, oracle, primes):
    r, mp = run_and_check(ctx, oracle, primes, 10**10, 1 << 18, p_small=100)
    assert r.result["phase2_fallbacks"] == int((mp > 100).sum()) > 0


def test_single_n_and_normalisation(ctx, oracle, primes):
    run_and_check(ctx, oracle, primes, 4, 1)
    run_and_check(ctx, oracle, primes, 1000, 1)
    # odd limit -> limit-1, start < 4 -> 4, odd start -> start+1
    r = ctx.verify_range(1, 101, want_minp=True)
    assert r.result["checked"] == 49
    np.testing.assert_array_equal(r.min_p, oracle.minp(4, 49))
    r = ctx.verify_range(7, 20, want_minp=True)
    np.testing.assert_array_equal(r.min_p, oracle.minp(8, 7))


def test_start_after_limit_is_an_error(ctx, gbmod):
    with pytest.raises(gbmod.GbError):
        ctx.verify_range(100, 98)


def test_segments_and_shards(ctx, oracle, primes):
    start, count, seg = 10**12 + 6, 1_000_003, 100_003
    limit = start + 2 * (count - 1)
    mp = oracle.minp(start, count)
    nseg = (count + seg - 1) // seg
    merged = np.zeros(count, np.uint32)
    fb = np.zeros(nseg, np.uint32)
    tot = 0
    for si in range(3):
        r = ctx.verify_range(start, limit, seg_size=seg, p_small=300, shard_index=si,
                             shard_count=3, want_minp=True, want_seg=True, want_seg_hist=True)
        tot += r.result["checked"]
        mine = [s for s in range(nseg) if s % 3 == si]
        for s in range(nseg):
            lo, hi = s * seg, min(count, (s + 1) * seg)
            if s in mine:
                np.testing.assert_array_equal(r.min_p[lo:hi], mp[lo:hi])
                assert r.seg_fallbacks[s] == int((mp[lo:hi] > 300).sum())
                np.testing.assert_array_equal(r.seg_hist[s], hist_of(mp[lo:hi], primes))
                fb[s] = r.seg_fallbacks[s]
            else:
                assert not r.min_p[lo:hi].any() and r.seg_fallbacks[s] == 0
        merged |= r.min_p
    assert tot == count
    np.testing.assert_array_equal(merged, mp)


def test_seeded_sample_segments_near_1e12(ctx, oracle, primes):
    # 64 segments of seg-size 2^24 in [4, 1e12], chosen by splitmix64(0xB200);
    # the first 2^16 n of each are compared per n
    seg = 1 << 24
    total = (10**12 - 4) // 2 + 1
    nseg = (total + seg - 1) // seg
    state = 0xB200
    for _ in range(64):
        state, z = splitmix64(state)
        s = z % nseg
        start = 4 + 2 * seg * s
        count = min(1 << 16, total - seg * s)
        run_and_check(ctx, oracle, primes, start, count)


def test_full_segment_histograms(ctx, oracle, primes):
    # two whole 2^24 segments, per-segment histograms against the oracle
    start = 4 + 2 * (1 << 24) * 29000
    count = 2 << 24
    r = ctx.verify_range(start, start + 2 * (count - 1), seg_size=1 << 24, want_seg_hist=True,
                         want_seg=True)
    for s in range(2):
        mp = oracle.minp(start + 2 * (1 << 24) * s, 1 << 24)
        np.testing.assert_array_equal(r.seg_hist[s], hist_of(mp, primes))
        assert r.seg_failures[s] == 0
    assert r.result["failures"] == 0


def test_summary_1e9_matches_oracle_fixture(ctx):
    # [4, 1e9] with P_SMALL = 1e5: the validation_gpu.sh:48-54 case
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_hist_1e9.json")))
    r = ctx.verify_range(4, 10**9, seg_size=1 << 26, p_small=10**5)
    assert r.result["checked"] == g["checked"]
    assert r.result["phase2_fallbacks"] == g["fallbacks"] == 0
    assert r.result["failures"] == 0
    assert r.result["max_minp"] == g["max_minp"]
    h = {str(i): int(c) for i, c in enumerate(r.hist) if c}
    assert h == g["hist_nonzero"]


@pytest.mark.parametrize("count", [1, 2, 3, 97, 1 << 16])
def test_range_ending_at_the_top_of_uint64(ctx, oracle, count):
    """Chunks whose last n is 2^64 - 2 (limit 2^64 - 1 normalises to it):
    sieving primes up to 2^32, and no chunk arithmetic may pass 2^64.
    Checked against the oracle's single-n search (7-base MR on each q)."""
    limit = 2**64 - 1
    start = 2**64 - 2 - 2 * (count - 1)
    r = ctx.verify_range(start, limit, want_minp=True, want_bits=True)
    ns = np.array([start + 2 * j for j in range(count)], np.uint64)
    want = oracle.single_minp(ns, p_limit=10**8).astype(np.uint32)
    bad = np.nonzero(r.min_p != want)[0]
    assert bad.size == 0, (ns[bad[:8]], r.min_p[bad[:8]], want[bad[:8]])
    assert r.result["checked"] == count and r.result["failures"] == 0
    bits = np.unpackbits(r.verified_bits.view(np.uint8), bitorder="little")
    assert bits[:count].all()
