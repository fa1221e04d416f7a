"""Serving with continuous batching: every response equals the same request
run alone (single n: gb_check_single_batch; range: gb_verify_range), while
requests of both kinds are queued, batched and overlapped on the GPU."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _alone(ctx, kind, a, count):
    if kind == 0:
        p, q, _ = ctx.check_single(np.array([a], np.uint64))
        return {"p": int(p[0]), "q": int(q[0]), "verified": int(p[0] > 0),
                "failures": int(p[0] == 0), "max_minp": int(p[0]), "minp_sum": int(p[0])}
    r = ctx.verify_range(a, a + 2 * (count - 1), want_minp=True)
    m = r.min_p.astype(np.uint64)
    return {"verified": int((m > 0).sum()), "failures": int((m == 0).sum()),
            "max_minp": int(m.max()), "minp_sum": int(m.sum())}


def test_mixed_stream_matches_requests_run_alone(gbmod):
    with gbmod.Context(0, max_n=10**13) as ctx:
        ctx.serve_start(max_n=10**13, small_range=2000, max_single_batch=1 << 16)
        rng = np.random.default_rng(3)
        reqs = []
        for _ in range(3):  # three waves: later ones arrive while earlier run
            for _ in range(200):
                reqs.append((0, int(rng.integers(2, 5 * 10**12)) * 2, 1))
            for _ in range(30):
                reqs.append((1, int(rng.integers(2, 5 * 10**12)) * 2, int(rng.integers(1, 2000))))
            for _ in range(8):
                reqs.append((1, int(rng.integers(2, 5 * 10**12)) * 2, int(rng.integers(2001, 300000))))
        tickets = []
        for w in range(3):
            part = reqs[w * 238:(w + 1) * 238]
            k, a, c = zip(*part)
            tickets += list(ctx.submit(k, a, c))
            time.sleep(0.002)
        got = [ctx.wait(t, 120000) for t in tickets]
        st = ctx.serve_stats()
        assert st["completed"] == st["submitted"] == len(reqs)
        assert st["rejected"] == 0 and st["p99_us"] >= st["p50_us"] > 0
        lanes = {g["lane"] for g in got}
        assert 0 in lanes and lanes - {0} and lanes <= {0, 1, 2}
        for (kind, a, count), g in zip(reqs, got):
            assert g["status"] == 0
            want = _alone(ctx, kind, a, count)
            for key, v in want.items():
                assert g[key] == v, (kind, a, count, key, g[key], v)
        ctx.serve_stop()


def test_invalid_requests_are_rejected_not_run(gbmod):
    with gbmod.Context(0, max_n=10**12) as ctx:
        ctx.serve_start(max_n=10**12)
        t = ctx.submit([0, 0, 1, 0], [7, 2, 10, 2 * 10**12], [1, 1, 0, 1])
        res = [ctx.wait(x, 10000) for x in t]
        assert [r["status"] for r in res] == [gbmod.GB_EINVAL] * 4
        ok = ctx.submit([0], [100])[0]
        r = ctx.wait(ok, 10000)
        assert r["status"] == 0 and r["p"] + r["q"] == 100 and r["p"] == 3
        assert ctx.serve_stats()["rejected"] == 4
        ctx.serve_stop()


def test_high_offsets_match_the_oracle(gbmod, oracle):
    """Requests near 1e19 and the top of uint64 (both lanes) against the
    oracle's MR-based minimal-p search."""
    with gbmod.Context(0, max_n=2**64 - 1) as ctx:
        ctx.serve_start(max_n=2**64 - 1, small_range=500)
        rng = np.random.default_rng(5)
        reqs = [(0, int(rng.integers(5 * 10**17, 2**63 - 1)) * 2, 1) for _ in range(64)]
        reqs += [(0, 2**64 - 2, 1), (1, 2**64 - 2 - 2 * 99, 100), (1, 2**64 - 2 - 2 * 2999, 3000)]
        reqs += [(1, int(rng.integers(5 * 10**18, 9 * 10**18)) * 2, int(rng.integers(1, 4000)))
                 for _ in range(12)]
        k, a, c = zip(*reqs)
        got = [ctx.wait(t, 120000) for t in ctx.submit(k, a, c)]
        assert 0 in {g["lane"] for g in got} and {g["lane"] for g in got} - {0}
        for (kind, a0, count), g in zip(reqs, got):
            ns = np.array([a0 + 2 * j for j in range(count)], np.uint64)
            m = oracle.single_minp(ns, p_limit=10**8)
            assert g["status"] == 0
            if kind == 0:
                assert g["p"] == int(m[0]) and g["q"] == a0 - int(m[0])
            assert g["verified"] == int((m > 0).sum()) and g["failures"] == int((m == 0).sum())
            assert g["max_minp"] == int(m.max()) and g["minp_sum"] == int(m.sum()), (kind, a0, count)
        ctx.serve_stop()


def test_graph_and_stream_launches_agree(gbmod):
    """Small single-lane batches run as one CUDA graph (copy sizes and kernel
    arguments updated per batch); with no_graph the same requests run as
    plain stream launches; with spin_us the lanes poll their queues before
    blocking.  All give the same responses, one request at a time (one batch
    each) and as a burst, and the single n match gb_check_single_batch."""
    rng = np.random.default_rng(21)
    a = [int(x) * 2 for x in rng.integers(2, 2**62, size=60)] + [4, 6, 8, 100]
    out = {}
    with gbmod.Context(0) as ctx:
        for no_graph, spin in ((False, 0), (True, 0), (False, 2000)):
            ctx.serve_start(small_range=2000, no_graph=no_graph, spin_us=spin)
            got = []
            for x in a[:20]:  # one at a time: one batch per request
                got.append(ctx.wait(ctx.submit([0], [x], [1])[0], 60000))
            kinds = [0] * (len(a) - 20) + [1]
            burst = ctx.submit(kinds, a[20:] + [10**12], [1] * (len(a) - 20) + [500])
            got += [ctx.wait(t, 60000) for t in burst]
            assert all(g["status"] == 0 for g in got)
            out[(no_graph, spin)] = [(g["p"], g["q"], g["verified"], g["minp_sum"]) for g in got]
            ctx.serve_stop()
        p, _, _ = ctx.check_single(np.array(a, np.uint64))
    assert out[(False, 0)] == out[(True, 0)] == out[(False, 2000)]
    assert [o[0] for o in out[(False, 0)][:len(a)]] == [int(x) for x in p]


def test_backpressure_and_a_small_pool(gbmod):
    """A pool of 256 KB holds only a few ranges at a time: the rest wait in the
    queue for memory (deferred, not failed).  With max_pending_n at 2^23 a
    burst of wide ranges is partly refused with GB_EBUSY at once; everything
    admitted completes with the result it has alone; three range lanes."""
    with gbmod.Context(0, max_n=10**13) as ctx:
        ctx.serve_start(max_n=10**13, small_range=2000, range_lanes=3, pool_bytes=256 << 10,
                        max_pending_n=1 << 23)
        rng = np.random.default_rng(9)
        reqs = [(1, int(rng.integers(2, 5 * 10**12)) * 2, int(rng.integers(100000, 400000)))
                for _ in range(60)]
        reqs += [(0, int(rng.integers(2, 5 * 10**12)) * 2, 1) for _ in range(50)]
        k, a, c = zip(*reqs)
        got = [ctx.wait(t, 120000) for t in ctx.submit(k, a, c)]
        st = ctx.serve_stats()
        busy = [g for g in got if g["status"] == gbmod.GB_EBUSY]
        assert busy and st["busy"] == len(busy) and st["rejected"] == len(busy)
        assert all(g["kind"] == 1 for g in busy)  # the single lane's queue was never full
        assert st["pool_bytes"] == 256 << 10 and 0 < st["pool_peak_bytes"] <= 256 << 10
        assert st["batches_range"] >= 3  # the admitted ranges did not fit one batch
        done = [(r, g) for r, g in zip(reqs, got) if g["status"] == 0]
        assert len(done) + len(busy) == len(reqs)
        assert {g["lane"] for r, g in done if r[0] == 1} <= {1, 2, 3}
        for (kind, a0, count), g in done:
            want = _alone(ctx, kind, a0, count)
            for key, v in want.items():
                assert g[key] == v, (kind, a0, count, key)
        # the queue drains: a later request is admitted again
        r = ctx.wait(ctx.submit([1], [10**12], [300000])[0], 120000)
        assert r["status"] == 0
        ctx.serve_stop()
