"""Tuning knobs never change results: block shapes and chunk sizes of the
range kernel, the windows pipeline's Miller-Rabin split divisor, large-prime
grid and block shape, and whatever the two autotuners pick."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("threads,chunk", [(256, 1 << 18), (256, 1 << 19), (512, 1 << 20),
                                           (1024, 1 << 19), (1024, 1 << 20)])
def test_block_shapes_match_the_oracle(ctx, oracle, threads, chunk):
    start, count = 10**12 - 2 * 1_500_000, 1_400_001
    r = ctx.verify_range(start, start + 2 * (count - 1), chunk=chunk, block_threads=threads,
                         want_minp=True)
    np.testing.assert_array_equal(r.min_p, oracle.minp(start, count))
    assert r.result["failures"] == 0 and r.result["checked"] == count


def test_bad_block_shape_is_rejected(ctx, gbmod):
    with pytest.raises(gbmod.GbError):
        ctx.verify_range(10**9, 10**9 + 1000, block_threads=384)


def test_range_autotuner_choice_gives_identical_results(ctx):
    start, limit = 10**11, 10**11 + 2 * (1 << 24)
    t = ctx.autotune_range(start, limit)
    assert t["block_threads"] in (256, 512, 1024) and t["candidates"] >= 27
    again = ctx.autotune_range(start, limit)
    assert again["cached"] == 1 and again["block_threads"] == t["block_threads"]
    tuned = ctx.verify_range(start, limit, chunk=t["chunk_evens"], halo=t["halo"],
                             block_threads=t["block_threads"], want_seg=True)
    plain = ctx.verify_range(start, limit, want_seg=True)
    np.testing.assert_array_equal(tuned.hist, plain.hist)
    np.testing.assert_array_equal(tuned.seg_fallbacks, plain.seg_fallbacks)
    for k in ("checked", "verified", "failures", "phase2_fallbacks", "max_minp"):
        assert tuned.result[k] == plain.result[k]


def _windows(seed, nwin):
    rng = np.random.default_rng(seed)
    starts = rng.integers(10**15 // 2, 10**18 // 2, size=nwin, dtype=np.uint64) * 2
    counts = np.exp2(rng.uniform(10, 19, size=nwin)).astype(np.uint64)
    return starts, counts


@pytest.mark.parametrize("knobs", [dict(mr_divisor=700), dict(mr_divisor=20000),
                                   dict(large_ctas_per_sm=8), dict(block_threads=256, chunk=1 << 19),
                                   dict(block_threads=1024)])
def test_windows_knobs_agree(ctx, oracle, knobs):
    starts, counts = _windows(17, 40)
    per, minp, _ = ctx.verify_windows(starts, counts, want_minp=True, **knobs)
    np.testing.assert_array_equal(minp, oracle.minp_windows(starts, counts))
    assert all(p["failures"] == 0 for p in per)


def test_windows_autotuner_choice_gives_identical_results(ctx):
    starts, counts = _windows(19, 300)
    t = ctx.autotune_windows(starts, counts)
    assert t["candidates"] == 24 and t["sample_windows"] == 300
    assert ctx.autotune_windows(starts, counts)["cached"] == 1
    tuned, mt, _ = ctx.verify_windows(starts, counts, want_minp=True, chunk=t["chunk_evens"],
                                      mr_divisor=t["mr_divisor"],
                                      large_ctas_per_sm=t["large_ctas_per_sm"],
                                      block_threads=t["block_threads"])
    plain, mp, _ = ctx.verify_windows(starts, counts, want_minp=True)
    assert tuned == plain
    np.testing.assert_array_equal(mt, mp)
