"""Multi-rank host logic on CPU: two gloo ranks split a range by segments
(the library's shard rule) and merge their summaries and histograms; the
merged figures must equal the single-process result.  Each rank's device
call is stood in for by the CPU oracle on its own segments."""
import importlib.util
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _load_multi():
    spec = importlib.util.spec_from_file_location(
        "gb_multi", os.path.join(ROOT, "goldbach-gpu_b200", "multi.py"))
    m = importlib.util.module_from_spec(spec)
    sys.modules["gb_multi"] = m
    spec.loader.exec_module(m)
    return m


def _rank_summary(oracle, primes, start, total, seg, segs, p_small):
    from oracle_lib import hist_of
    res = {k: 0 for k in ("checked", "verified", "phase2_fallbacks", "failures", "queued",
                          "kernel_launches")}
    res.update({"max_minp": 0, "device_ms": 0.0, "kernel_ms": 0.0, "first_failure_n": 0})
    hist = np.zeros(4096, np.int64)
    for s in segs:
        cnt = min(seg, total - s * seg)
        a = start + 2 * s * seg
        mp_ = oracle.minp(a, cnt, p_limit=10**8)
        res["checked"] += cnt
        res["verified"] += int((mp_ > 0).sum())
        res["failures"] += int((mp_ == 0).sum())
        res["phase2_fallbacks"] += int(((mp_ == 0) | (mp_ > p_small)).sum())
        res["max_minp"] = max(res["max_minp"], int(mp_.max()))
        hist += hist_of(mp_, primes).astype(np.int64)
    return res, hist


def _worker(rank, world, port, start, limit, seg, p_small, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(__file__))
    import oracle_lib
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    multi = _load_multi()
    oracle = oracle_lib.Oracle()
    primes = oracle.primes(2_000_000)
    total = (limit - start) // 2 + 1
    nseg = (total + seg - 1) // seg
    segs = multi.shard_segments(nseg, rank, world)
    res, hist = _rank_summary(oracle, primes, start, total, seg, segs, p_small)
    assert res["checked"] == multi.shard_even_count(total, seg, rank, world)
    h = torch.from_numpy(hist)
    merged = multi.merge_results(res, h, dist)
    slow = multi.max_over_ranks(float(rank + 1), dist)
    if rank == 0:
        q.put((merged, h.numpy().copy(), slow))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_two_rank_merge_equals_single_process(oracle, world):
    from oracle_lib import hist_of
    start, limit, seg, p_small = 10**9, 10**9 + 2 * 300_000, 7919, 150
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, start, limit, seg, p_small, q))
             for r in range(world)]
    for p in procs:
        p.start()
    merged, hist, slow = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    total = (limit - start) // 2 + 1
    mp_ = oracle.minp(start, total)
    assert merged["checked"] == total
    assert merged["failures"] == 0
    assert merged["phase2_fallbacks"] == int((mp_ > p_small).sum())
    assert merged["max_minp"] == int(mp_.max())
    np.testing.assert_array_equal(hist, hist_of(mp_, oracle.primes(2_000_000)).astype(np.int64))
    assert slow == float(world)
