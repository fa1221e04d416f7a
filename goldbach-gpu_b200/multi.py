"""Multi-GPU plumbing for range verification (one process per GPU).

Segments of a range are independent (the reference hands them to GPU
threads with a host atomic counter, src/goldbach.cu:422).  Here the split
is static: rank r of W takes the segments s with s % W == r -- the rule
gb_range_opts.shard_index / shard_count applies inside the library -- and
the only exchange is the final merge of the per-rank summaries and
minimal-p histograms (a few KB), done with torch.distributed collectives.
"""
from __future__ import annotations

import torch


def shard_segments(nseg: int, rank: int, world: int) -> list[int]:
    """Segment indices of one rank (same rule as the C library)."""
    return list(range(rank, nseg, world))


def shard_even_count(total: int, seg_size: int, rank: int, world: int) -> int:
    """Number of even n a rank verifies."""
    nseg = (total + seg_size - 1) // seg_size
    return sum(min(seg_size, total - s * seg_size) for s in shard_segments(nseg, rank, world))


# summary fields and how they combine across ranks
_SUM = ("checked", "verified", "phase2_fallbacks", "failures", "queued", "kernel_launches")
_MAX = ("max_minp", "device_ms", "kernel_ms")


def merge_results(local: dict, hist: torch.Tensor | None, dist, group=None) -> dict:
    """All-reduces one rank's range summary (and, in place, its minimal-p
    histogram) so that every rank ends with the whole-range figures.  The
    first failing n is the minimum over the ranks that saw a failure."""
    dev = hist.device if hist is not None else torch.device("cpu")
    s = torch.tensor([int(local[k]) for k in _SUM], dtype=torch.int64, device=dev)
    m = torch.tensor([float(local[k]) for k in _MAX], dtype=torch.float64, device=dev)
    ff = int(local.get("first_failure_n", 0))
    f = torch.tensor([ff if ff else (1 << 63) - 1], dtype=torch.int64, device=dev)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(f, op=dist.ReduceOp.MIN, group=group)
    if hist is not None:
        dist.all_reduce(hist, op=dist.ReduceOp.SUM, group=group)
    out = dict(local)
    out.update({k: int(v) for k, v in zip(_SUM, s.tolist())})
    out.update({k: float(v) for k, v in zip(_MAX, m.tolist())})
    fv = int(f.item())
    out["first_failure_n"] = 0 if fv == (1 << 63) - 1 else fv
    return out


def max_over_ranks(value: float, dist, device=None, group=None) -> float:
    """The slowest rank's time (multi-GPU timings are max over ranks)."""
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
