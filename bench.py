#!/usr/bin/env python3
"""bench.py -- even n verified per second, [4, 1e12], on B200.

One step = one gb_verify_range call over every even n in [4, LIMIT] (the
range split over the ranks for N > 1: strong scaling), outputs (minimal-p
histogram, per-segment fallback and failure counts) resident on the device.
`value` times the steps with CUDA events on the library's launch stream
(L2 flushed between steps, outside the timed events).  `e2e` repeats the
steps through the same C-ABI call with pinned host output buffers, the
device-to-host copies inside the timed region.

--impl reference times the reference's own CPU code (oracle/_ref, built from
the reference sources: its segmented_sieve plus the cpu_goldbach scan rule)
on a bounded sample of the same workload (the top 2^24 even n below LIMIT
per step) with all host threads.
"""
import argparse
import ctypes
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "even n verified/s to 1e12 on 1 B200"
UNIT = "even n/s"


def load_gb():
    spec = importlib.util.spec_from_file_location(
        "goldbach_gpu_b200", os.path.join(ROOT, "goldbach-gpu_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["goldbach_gpu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.path = os.path.join("/tmp", f"gb_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1])]
        mx = [num(r[2]) for r in rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline_oracle(limit, sample_log2=28):
    """The oracle port (C, OpenMP, all host threads) on the top 2^k even n
    below LIMIT.  Test infrastructure used only as the reported baseline."""
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    L = ctypes.CDLL(lib)
    L.gbo_minp_range.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                 ctypes.c_void_p, ctypes.c_int]
    import numpy as np
    cnt = 1 << sample_log2
    start = limit - 2 * (cnt - 1)
    buf = np.zeros(cnt, np.uint32)
    L.gbo_minp_range(start, 1 << 16, 10**8, buf.ctypes.data, 0)  # warm the prime tables
    t0 = time.perf_counter()
    L.gbo_minp_range(start, cnt, 10**8, buf.ctypes.data, 0)
    dt = time.perf_counter() - t0
    return {"value": cnt / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"{cnt} even n ending at {limit} (top of the range), oracle gbo_minp_range, "
                      f"{os.cpu_count()} OpenMP threads, {dt:.2f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    so = os.path.join(ROOT, "oracle", "_ref", "libgbref.so")
    if not os.path.exists(so):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libgbref.so not built"}))
        return 0
    L = ctypes.CDLL(so)
    L.gbref_window_verify.restype = ctypes.c_uint64
    L.gbref_window_verify.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                      ctypes.c_void_p, ctypes.c_int]
    cnt = 1 << args.ref_sample_log2
    start = args.limit - 2 * (cnt - 1)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        L.gbref_window_verify(start, cnt, 1 << 16, None, threads)
    times = []
    unver = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        unver += L.gbref_window_verify(start, cnt, 1 << 16, None, threads)
        times.append(time.perf_counter() - t0)
    ms = 1000 * statistics.mean(times)
    value = cnt / (ms / 1000)
    sample = (f"top {cnt} even n below {args.limit} per step; reference segmented_sieve "
              f"(src/segmented_sieve.cpp) + cpu_goldbach scan rule (src/cpu_goldbach.cpp:19-21), "
              f"{threads} threads; unverified={unver}")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"range [4, {args.limit}] sampled", "sample_even_n": cnt},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--limit", type=int, default=10**12)
    ap.add_argument("--seg-size", type=int, default=1 << 27)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--halo", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-sample-log2", type=int, default=24)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    gb = load_gb()
    ctx = gb.Context(local, max_n=args.limit)
    stream = torch.cuda.Stream()
    start, limit = 4, args.limit - (args.limit & 1)
    total = (limit - start) // 2 + 1
    nseg = gb.load().gb_num_segments(start, limit, args.seg_size)
    dev = torch.device("cuda", local)
    hist = torch.zeros(4096, dtype=torch.int64, device=dev)
    segfb = torch.zeros(nseg, dtype=torch.int32, device=dev)
    segfail = torch.zeros(nseg, dtype=torch.int32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    kw = dict(seg_size=args.seg_size, chunk=args.chunk, halo=args.halo, shard_index=rank,
              shard_count=world, stream=stream.cuda_stream)

    def step_dev():
        r = ctx.verify_range(start, limit, device_out={"minp_hist": hist, "seg_fallbacks": segfb,
                                                       "seg_failures": segfail}, **kw)
        if dist is not None:
            with torch.cuda.stream(stream):
                dist.all_reduce(hist)
        return r

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step_dev()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    times, kms, launches, results = [], [], 0, []
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i & 0xff)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = step_dev()
        e1.record(stream)
        barrier()
        times.append(e0.elapsed_time(e1))
        kms.append(r.result["kernel_ms"])
        launches += r.result["kernel_launches"]
        results.append(r.result)
    clk = clocks.stop()
    ms = statistics.mean(times)
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = total / (ms / 1000)

    # e2e: the same call with pinned host output buffers (D2H inside)
    h_hist = torch.zeros(4096, dtype=torch.int64).pin_memory()
    h_fb = torch.zeros(nseg, dtype=torch.int32).pin_memory()
    h_fail = torch.zeros(nseg, dtype=torch.int32).pin_memory()
    L = gb.load()

    def step_host():
        o = gb.RangeOpts(args.seg_size, 10**6, 0, args.chunk, args.halo, rank, world, 0,
                         stream.cuda_stream)
        out = gb.RangeOut(None, None, h_hist.data_ptr(), h_fb.data_ptr(), h_fail.data_ptr(), None)
        res = gb.RangeResult()
        st = L.gb_verify_range(ctx._h, start, limit, ctypes.byref(o), ctypes.byref(res), ctypes.byref(out))
        if st != 0:
            raise RuntimeError(f"gb_verify_range failed: {st}")
        return res

    for _ in range(max(1, args.warmup // 2)):
        step_host()
    etimes = []
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i & 0xff)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step_host()
        e1.record(stream)
        barrier()
        etimes.append(e0.elapsed_time(e1))
    ems = statistics.mean(etimes)
    if dist is not None:
        t = torch.tensor([ems], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e_value = total / (ems / 1000)
    d2h = 4096 * 8 + nseg * 8 + 8 * 8

    # roofline of the fused sieve+search kernel: algorithmic
    # bytes = the odd-only q-bitset the search consumes (one bit per odd q of
    # every chunk window incl. its halo), written once and read once if it
    # were staged through HBM; the fused kernel keeps it in shared memory.
    halo = args.halo or 32768
    chunk = args.chunk or (1 << 19)
    n_mine = sum(min(args.seg_size, total - s * args.seg_size) for s in range(rank, nseg, world))
    chunks = sum(math.ceil(min(args.seg_size, total - s * args.seg_size) / chunk)
                 for s in range(rank, nseg, world))
    bitset_bytes = 2 * (n_mine + chunks * halo // 2) / 8
    k_ms = statistics.mean(kms)
    hbm_peak, peak_kind = peaks()
    achieved = bitset_bytes / (k_ms / 1000) / 1e9
    res0 = results[-1]
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"range [4, {limit}] (every even n)", "seg_size": args.seg_size,
                   "chunk_evens": chunk, "halo": halo, "p_small": 10**6, "phase2_limit": 10**8,
                   "l2": "flushed (512 MB write) between steps", "parallelism": f"segments sharded over {world} GPU(s)"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": None,
                     "note": f"peak {peak_kind}; kernel range_kernel avg {k_ms:.3f} ms"},
        "clocks": clk,
        "result": {"checked": res0["checked"], "failures": res0["failures"],
                   "phase2_fallbacks": res0["phase2_fallbacks"], "max_minp": res0["max_minp"]},
    }
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_oracle(limit)
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
