"""Batched single-n checks: the minimal partition p + q of every n, against
the oracle's 7-base Miller-Rabin scan (bit-exact)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PUBLISHED = {10**12: 194267, 10**13: 90059, 10**14: 145391, 10**15: 152639, 10**16: 56687,
             10**17: 91967, 10**18: 14831, 10**19: 226283}  # RESULTS.md:112-121


def test_seeded_uniform_64bit(ctx, oracle):
    rng = np.random.default_rng(2)
    n = (rng.integers(2, 2**63, size=20000, dtype=np.uint64) * 2).astype(np.uint64)
    p, q, r = ctx.check_single(n)
    want = oracle.single_minp(n)
    np.testing.assert_array_equal(p, want)
    np.testing.assert_array_equal(q, n - p)
    assert r.found == len(n)


def test_small_and_edge_n(ctx, oracle):
    n = np.array([4, 6, 8, 10, 12, 98, 2 * 10**6, (1 << 21) - 2, 1 << 21, (1 << 21) + 2,
                  2**64 - 2, 2**63, 2**63 + 2, 2**32, 2**32 + 2] +
                 list(range(14, 4000, 2)), dtype=np.uint64)
    p, q, _ = ctx.check_single(n)
    np.testing.assert_array_equal(p, oracle.single_minp(n))
    assert p[0] == 2 and q[0] == 2
    for a, b in zip(p[:15], q[:15]):
        assert oracle.mr7(int(a)) and oracle.mr7(int(b))


def test_published_partitions_bound_minimal_p(ctx, oracle):
    n = np.array(list(PUBLISHED), dtype=np.uint64)
    p, q, _ = ctx.check_single(n)
    for ni, pi, qi in zip(n, p, q):
        assert 0 < pi <= PUBLISHED[int(ni)]
        assert oracle.mr7(int(pi)) and oracle.mr7(int(qi)) and pi + qi == ni
    np.testing.assert_array_equal(p, oracle.single_minp(n))


def test_p_limit_bound(ctx, oracle):
    n = np.array([10**12 + 2 * i for i in range(2000)], dtype=np.uint64)
    p, q, _ = ctx.check_single(n, p_limit=50)
    want = oracle.single_minp(n, p_limit=50)
    np.testing.assert_array_equal(p, want)
    assert (p == 0).any() and (q[p == 0] == 0).all()


def test_agrees_with_range_path(ctx):
    start = 10**14 + 2
    r = ctx.verify_range(start, start + 2 * 4095, want_minp=True)
    n = start + 2 * np.arange(4096, dtype=np.uint64)
    p, _, _ = ctx.check_single(n)
    np.testing.assert_array_equal(p, r.min_p.astype(np.uint64))


def test_small_and_large_batches_agree(ctx, oracle):
    """Batches below 8192 queries take the warp-per-query kernel, larger ones
    the lane-per-query kernel: the same n give the same (p, q) either way."""
    rng = np.random.default_rng(11)
    n = (rng.integers(2, 2**63, size=12000, dtype=np.uint64) * 2).astype(np.uint64)
    n[:40] = np.arange(4, 84, 2, dtype=np.uint64)  # the plain path for small n too
    p_big, q_big, r = ctx.check_single(n)
    parts = [ctx.check_single(n[i:i + 1000]) for i in range(0, len(n), 1000)]
    p_small = np.concatenate([x[0] for x in parts])
    q_small = np.concatenate([x[1] for x in parts])
    np.testing.assert_array_equal(p_big, p_small)
    np.testing.assert_array_equal(q_big, q_small)
    np.testing.assert_array_equal(p_big, oracle.single_minp(n))
    assert r.found == len(n) and sum(x[2].found for x in parts) == len(n)
