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
