"""Batched windows (persistent and plain pipelines) against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def seeded_windows(seed, nwin, lo=10**15, hi=10**18, wmin=10, wmax=14):
    rng = np.random.default_rng(seed)
    starts = rng.integers(lo // 2, hi // 2, size=nwin, dtype=np.uint64) * 2
    widths = np.exp2(rng.uniform(wmin, wmax, size=nwin)).astype(np.uint64)
    return starts, widths


@pytest.mark.parametrize("mode", [0, 1])
def test_windows_bit_exact(ctx, oracle, gbmod, mode):
    starts, counts = seeded_windows(1, 48)
    per, minp, summ = ctx.verify_windows(starts, counts, mode=mode, want_minp=True)
    allw = oracle.minp_windows(starts, counts)
    np.testing.assert_array_equal(minp, allw)
    off = 0
    for i, (s, c) in enumerate(zip(starts, counts)):
        want = allw[off:off + int(c)]
        got = minp[off:off + int(c)]
        np.testing.assert_array_equal(got, want)
        assert per[i]["failures"] == 0 and per[i]["verified"] == c
        assert per[i]["max_minp"] == int(want.max())
        assert per[i]["minp_sum"] == int(want.astype(np.uint64).sum())
        off += int(c)
    assert summ["total_n"] == int(counts.sum())


def test_windows_small_starts_and_tiny_halo(ctx, oracle):
    starts = np.array([4, 1000, 10**6, 10**9 + 2, 4 + 2 * 70000], dtype=np.uint64)
    counts = np.array([5000, 1, 3000, 20000, 100], dtype=np.uint64)
    for halo in (0, 256):
        per, minp, _ = ctx.verify_windows(starts, counts, halo=halo, want_minp=True)
        np.testing.assert_array_equal(minp, oracle.minp_windows(starts, counts))


def test_windows_modes_agree_large(ctx):
    starts, counts = seeded_windows(3, 256, wmin=10, wmax=18)
    a, _, sa = ctx.verify_windows(starts, counts, mode=0)
    b, _, sb = ctx.verify_windows(starts, counts, mode=1)
    assert a == b
    assert sa["failures"] == sb["failures"] == 0


@pytest.mark.parametrize("mode", [0, 1])
def test_windows_at_the_top_of_uint64(ctx, oracle, mode):
    """Windows ending at 2^64 - 2 and just below it (sieving primes to 2^32),
    against the oracle's MR-based single-n search."""
    top = 2**64 - 2
    counts = np.array([1, 2, 97, 5000], dtype=np.uint64)
    starts = np.array([top, top - 2, top - 2 * 96 - 10**6, top - 2 * 4999 - 10**9],
                      dtype=np.uint64)
    per, minp, _ = ctx.verify_windows(starts, counts, mode=mode, want_minp=True)
    ns = np.concatenate([s + 2 * np.arange(int(c), dtype=np.uint64) for s, c in zip(starts, counts)])
    want = oracle.single_minp(ns, p_limit=10**8).astype(np.uint32)
    bad = np.nonzero(minp != want)[0]
    assert bad.size == 0, (ns[bad[:8]], minp[bad[:8]], want[bad[:8]])
    assert all(p["failures"] == 0 for p in per)


@pytest.mark.parametrize("mr_below", [1, 1 << 40])
@pytest.mark.parametrize("mode", [0, 1])
def test_sieve_and_miller_rabin_paths_agree(ctx, oracle, mr_below, mode):
    """mr_below = 1: every window sieved; 2^40: every window on the
    Miller-Rabin path; the default splits by width.  Same minimal p."""
    starts, counts = seeded_windows(7, 24, wmin=10, wmax=13)
    per, minp, summ = ctx.verify_windows(starts, counts, mode=mode, want_minp=True,
                                         mr_below=mr_below)
    want = oracle.minp_windows(starts, counts)
    np.testing.assert_array_equal(minp, want)
    off = 0
    for i, c in enumerate(counts):
        w = want[off:off + int(c)]
        assert per[i]["verified"] == c and per[i]["failures"] == 0
        assert per[i]["max_minp"] == int(w.max()) and per[i]["minp_sum"] == int(w.astype(np.uint64).sum())
        off += int(c)
    assert summ["total_n"] == int(counts.sum())
