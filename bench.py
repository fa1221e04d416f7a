#!/usr/bin/env python3
"""bench.py -- even n verified per second, [4, 1e12], on B200.

Headline (config C2): one step = one gb_verify_range call over every even n
in [4, LIMIT], split over the ranks by segments for N > 1 (strong scaling),
outputs (minimal-p histogram, per-segment fallback and failure counts)
resident on the device.  `value` times the steps with CUDA events on the
library's launch stream (L2 flushed by a 512 MB write between steps, outside
the events).  `e2e` repeats the steps through the same C-ABI call with
pinned host output buffers, the device-to-host copies inside the timed
region (the inputs are two scalars, so there is no bulk host-to-device copy).

Secondary figures in the same line (rank 0, N = 1, skipped with
--no-extras): `windows` (C3: 4096 seeded windows in [1e15, 1e18], one
persistent pipeline vs the plain per-window pipeline), `single` (C4: 1e6
seeded n in [4, 2^64-2]), `serving` (C5: seeded Poisson arrivals, p50/p99).

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
METRIC = "even n verified/s to 1e12 on 1 B200, batched vs plain; p50/p99 query latency"
UNIT = "even n/s"

# Algorithmic work of the range workload, in layout-independent units (the
# odd-only problem statement):
#  * search: sum over n of pi(p_min(n)) scalar (n, p) tests, 32 per word
#    operation of 5 ALU ops (shift, and, xor, popc, add); 14.85 tests per n
#    is the oracle's mean over [4, 1e12] (32 strata of 2^16 n);
#  * sieve: wheel pattern words for the primes 3..67 (7 ANDs of 2 ops per 32
#    odd q) and Eratosthenes marks of the primes 71..sqrt(n) per odd q of
#    each chunk's q-window (sum of 1/p = 1.1225 for sqrt(n) = 1e6), one
#    shared-memory atomic each;
#  * one first-multiple reduction (8 ALU ops) per sieving prime per chunk.
SEARCH_TESTS_PER_N = 14.85
# DRAM bytes of range6_kernel per even n: one ncu capture of 2^30 even n
# ending at 1e12 read 1.97 MB and wrote 13.51 MB (the search's survivor
# lists spilling out of L2, the prime tables' first touch)
DRAM_BYTES_PER_N = (1.972480e6 + 13.508352e6) / 2**30
SEARCH_OPS_PER_WORD = 5
WHEEL_OPS_PER_ODD_Q = 14 / 32
MARKS_PER_ODD_Q = 1.1225
OPS_PER_OFFSET = 8


def sieving_primes(limit):
    """pi(isqrt(limit)): the primes that sieve each chunk's q-window."""
    r = math.isqrt(limit)
    sieve = bytearray([1]) * (r + 1)
    sieve[0:2] = b"\0\0"
    for i in range(2, math.isqrt(r) + 1):
        if sieve[i]:
            sieve[i * i::i] = bytearray(len(range(i * i, r + 1, i)))
    return sum(sieve)


def search_floor(ctx, limit, strata=32, width=1 << 16):
    """The word-parallel floor of the range search, from the kernel's own
    per-n minimal p on `strata` seeded slices of `width` even n spread over
    [4, limit]: the even n of a class rho = n mod 6 are searched 32 to a word
    against the class's candidate sequence (rho 0: every prime >= 5; rho 2:
    3, then the primes = 1 mod 6; rho 4: 3, then the primes = 5 mod 6), and
    a word is done after the entries of its slowest n.  Returns (mean
    sum-of-pi(p_min) tests per n, floor word-steps per n)."""
    import numpy as np
    top = 1 << 20
    primes = ctx.primes_upto(top).astype(np.int64)
    k0 = np.arange(len(primes), dtype=np.int64)
    pi = np.zeros(top + 1, np.int64)  # prime -> its index (2 -> 0)
    pi[primes] = k0
    entry = {0: np.zeros(top + 1, np.int64)}  # prime -> entry index in the class sequence
    entry[0][primes[2:]] = k0[2:] - 2
    for rho, resid in ((2, 1), (4, 5)):
        sel = primes[primes % 6 == resid]
        entry[rho] = np.zeros(top + 1, np.int64)
        entry[rho][sel] = np.arange(1, len(sel) + 1)
    rng = np.random.default_rng(0xB200)
    tests = steps = count = 0
    for j in range(strata):
        lo = 4 + (limit - 4 - 2 * width - (1 << 22)) * j // strata
        a = lo - lo % 2 + 2 * int(rng.integers(0, 1 << 20))
        r = ctx.verify_range(a, a + 2 * (width - 1), want_minp=True, want_hist=False)
        mp = r.min_p.astype(np.int64)
        n = a + 2 * np.arange(width, dtype=np.int64)
        tests += int((pi[mp] + 1).sum())  # pi(p_min): the primes 2 .. p_min tried
        for rho in (0, 2, 4):
            e = entry[rho][mp[n % 6 == rho]] + 1
            e = np.concatenate([e, np.zeros((-len(e)) % 32, np.int64)]).reshape(-1, 32)
            steps += int(e.max(axis=1).sum())
        count += width
    return tests / count, steps / count


def load_gb():
    spec = importlib.util.spec_from_file_location(
        "goldbach_gpu_b200", os.path.join(ROOT, "goldbach-gpu_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["goldbach_gpu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_multi():
    spec = importlib.util.spec_from_file_location(
        "gb_multi", os.path.join(ROOT, "goldbach-gpu_b200", "multi.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gb_multi"] = mod
    spec.loader.exec_module(mod)
    return mod


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)).get("hbm_gbs", 6650.0), "measured"
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
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
        rows = [[x.strip() for x in line.split(",")] for line in open(self.path)]
        rows = [r for r in rows if len(r) >= 9]
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
    below LIMIT: the reported CPU baseline (test infrastructure)."""
    import numpy as np
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    L.gbo_minp_range.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                 ctypes.c_void_p, ctypes.c_int]
    cnt = 1 << sample_log2
    start = limit - 2 * (cnt - 1)
    buf = np.zeros(cnt, np.uint32)
    L.gbo_minp_range(start, 1 << 16, 10**8, buf.ctypes.data, 0)  # builds its prime tables
    t0 = time.perf_counter()
    L.gbo_minp_range(start, cnt, 10**8, buf.ctypes.data, 0)
    dt = time.perf_counter() - t0
    return {"value": cnt / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"{cnt} even n ending at {limit} (top of the range), oracle gbo_minp_range, "
                      f"{os.cpu_count()} OpenMP threads, {dt:.2f} s"}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
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
    times, unver = [], 0
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


# --------------------------------------------------------------------------
def seeded_windows(seed=1, count=4096, lo=10**15, hi=10**18, wlo=10, whi=24):
    import numpy as np
    rng = np.random.default_rng(seed)
    starts = rng.integers(lo // 2, hi // 2, size=count, dtype=np.uint64) * 2
    widths = np.exp2(rng.uniform(wlo, whi, size=count)).astype(np.uint64)
    return starts, np.maximum(widths, 1)


def measure_windows(gb, ctx, nwin=4096, plain=True, tune=True):
    """C3: the whole batch in one persistent pipeline, and the plain
    per-window pipeline on the same 4096 windows; the per-window results of
    the two must be identical.  (nwin < 4096 and plain=False: the first nwin
    seeded windows, persistent only -- a small case for profiling.)"""
    starts, counts = seeded_windows()
    starts, counts = starts[:nwin], counts[:nwin]
    ctx.verify_windows(starts[:64], counts[:64])  # warm-up (tables to 1e9)
    knobs = {}
    if tune:  # the batch class's knobs (timed on a sample)
        tune = ctx.autotune_windows(starts, counts)
        knobs = {k: tune[k] for k in ("mr_divisor", "large_ctas_per_sm", "block_threads")}
        knobs["chunk"] = tune["chunk_evens"]
    if plain:
        ctx.verify_windows(starts[:64], counts[:64], mode=gb.GB_WINDOWS_PLAIN)
    t0 = time.perf_counter()
    per, _, s = ctx.verify_windows(starts, counts, mode=gb.GB_WINDOWS_PERSISTENT, **knobs)
    wall = time.perf_counter() - t0
    total = int(counts.sum())
    t1 = time.perf_counter()
    per_p, _, sp = (ctx.verify_windows(starts, counts, mode=gb.GB_WINDOWS_PLAIN, **knobs) if plain
                    else (per, None, s))
    wall_p = time.perf_counter() - t1
    same = per == per_p
    pv = total / (sp["device_ms"] / 1e3)
    v = total / (s["device_ms"] / 1e3)
    # roofline of the large-prime pass: one first-multiple computation (the
    # range model's OPS_PER_OFFSET ALU ops) per (prime, window) pair it visits
    alu_peak, _ = ctx.probe_peaks()
    large_s = s["large_ms"] / 1e3
    ops = s["large_pairs"] * OPS_PER_OFFSET
    return {"windows": len(starts), "even_n": total, "persistent_ms": s["device_ms"],
            "persistent_value": v, "persistent_launches": s["kernel_launches"],
            "plain_windows": len(starts), "plain_ms": sp["device_ms"], "plain_value": pv,
            "plain_launches": sp["kernel_launches"], "batched_over_plain": v / pv,
            "identical_results": bool(same), "failures": s["failures"],
            "autotuned": tune, "sieved_windows": s["sieved_windows"], "large_pairs": s["large_pairs"],
            "large_ms": s["large_ms"], "search_ms": s["search_ms"],
            "roofline": {"bound": "int", "kernel": "win_large_kernel",
                         "achieved": ops / large_s / 1e12 if large_s else None,
                         "peak": alu_peak / 1e12, "unit": "Top/s",
                         "frac": ops / large_s / alu_peak if large_s else None,
                         "pairs_per_s": s["large_pairs"] / large_s if large_s else None,
                         "work_source": "(prime, window) pairs x 8 ALU ops per first-multiple computation",
                         "peak_source": "measured in-process: gb_probe_peaks (32-bit ALU ops/s)"},
            "wall_s": wall, "plain_wall_s": wall_p, "unit": UNIT}


_MR7_BASES = (2, 325, 9375, 28178, 450775, 9780504, 1795265022)
_SMALL = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31)


def _mr7_products(q):
    """(is q prime, modular products) of the oracle's 7-base Miller-Rabin
    (trial division by the primes <= 31, then per base a binary powmod of
    bitlen(d) squarings and popcount(d) products, then the squaring tail with
    its early exit, stopping at the first failing base)."""
    if q < 2:
        return False, 0
    for sp in _SMALL:
        if q == sp:
            return True, 0
        if q % sp == 0:
            return False, 0
    if q < 37 * 37:
        return True, 0
    d, s = q - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    work = 0
    for b in _MR7_BASES:
        a = b % q
        if a == 0:
            continue
        work += d.bit_length() + bin(d).count("1")
        x = pow(a, d, q)
        if x == 1 or x == q - 1:
            continue
        ok = False
        for _ in range(1, s):
            work += 1
            x = x * x % q
            if x == q - 1:
                ok = True
                break
        if not ok:
            return False, work
    return True, work


def single_mr_products(ns, primes):
    """Mean modular products per query of the oracle's minimal-p scan (p
    ascending from 3, q = n - p by the 7-base test): the Miller-Rabin work
    unit, one Montgomery product each."""
    tot = 0
    for n in ns:
        n = int(n)
        if n == 4:
            continue
        for p in primes[1:]:
            p = int(p)
            if p > n // 2:
                break
            ok, w = _mr7_products(n - p)
            tot += w
            if ok:
                break
    return tot / len(ns)


def measure_single(gb, ctx, count=10**6):
    """C4: 1e6 seeded even n uniform in [4, 2^64-2], minimal (p, q)."""
    import numpy as np
    import torch
    rng = np.random.default_rng(2)
    n = (rng.integers(2, 2**63, size=count, dtype=np.uint64) * 2).astype(np.uint64)
    dev = torch.device("cuda", torch.cuda.current_device())
    n_d = torch.from_numpy(n.view(np.int64)).to(dev)
    p_d = torch.empty_like(n_d)
    q_d = torch.empty_like(n_d)
    st = torch.cuda.Stream()
    for _ in range(2):
        _, _, r = ctx.check_single(None, device_ptrs=(n_d, p_d, q_d), stream=st.cuda_stream)
    times = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        _, _, r = ctx.check_single(None, device_ptrs=(n_d, p_d, q_d), stream=st.cuda_stream)
        e1.record(st)
        st.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.mean(times)
    # host buffers through the public call (H2D + D2H inside): one warm-up
    # call, then the mean of three
    p, q, r2 = ctx.check_single(n)
    walls = []
    for _ in range(3):
        t0 = time.perf_counter()
        p, q, r2 = ctx.check_single(n)
        walls.append(time.perf_counter() - t0)
    e2e = statistics.mean(walls)
    # roofline: Montgomery products of the oracle's scan (seeded sample of
    # the batch) against the measured Montgomery-product peak
    sample = n[np.random.default_rng(5).choice(count, size=1 << 13, replace=False)]
    per_q = single_mr_products(sample, ctx.primes_upto(100000))
    mont = ctx.probe_mont_products()
    achieved = per_q * count / (ms / 1e3)
    return {"queries": count, "ms": ms, "value": count / (ms / 1e3), "unit": "queries/s",
            "e2e_value": count / e2e, "e2e_h2d_bytes": count * 8, "e2e_d2h_bytes": count * 16,
            "found": int(r2.found), "max_p": int(r2.max_p),
            "checksum_p": int(p.astype(np.uint64).sum()),
            "roofline": {"bound": "int-mul", "kernel": "single_kernel",
                         "achieved": achieved / 1e9, "peak": mont / 1e9, "unit": "G Montgomery products/s",
                         "frac": achieved / mont, "products_per_query": per_q,
                         "work_source": "modular products of the oracle's 7-base scan (base order, "
                                        "early exit) on 8192 seeded queries of the batch",
                         "peak_source": "measured in-process: gb_probe_mont_products"}}


def measure_counts(gb, ctx, points=((10**9, 4096), (10**10, 1024))):
    """Partition counts c(n) (gb_goldbach_counts) for `count` consecutive even
    n from n0; one call each (its odd-prime bitset sieve included), the mean
    of three after a warm-up."""
    out = []
    for n0, count in points:
        ctx.goldbach_counts(n0, 32)
        walls = []
        for _ in range(3):
            t0 = time.perf_counter()
            c = ctx.goldbach_counts(n0, count)
            walls.append(time.perf_counter() - t0)
        w = statistics.mean(walls)
        # scalar (n, p) tests the reference's goldbach_count makes: n/2 - 1 per n
        tests = sum((n0 + 2 * j) // 2 - 1 for j in range(count))
        out.append({"n0": n0, "count": count, "ms": w * 1e3, "value": count / w, "unit": "n/s",
                    "pair_tests_per_s": tests / w, "c_first": int(c[0])})
    return out


def measure_c1(gb, ctx, device):
    """C1 as stated: every even n in [4, 1e9], SEG_SIZE 2^26, P_SMALL 1e8, the
    per-n outputs (minimal p as uint32, 2 GB; the verified bitmap) -- on the
    device (kernel + device time), and end to end through the C-ABI into
    pinned host buffers (the 2 GB device-to-host copy inside the timing)."""
    import numpy as np
    import torch
    lim, seg = 10**9, 1 << 26
    count = (lim - 4) // 2 + 1
    words = (count + 31) // 32
    dev = torch.device("cuda", device)
    d_minp = torch.empty(count, dtype=torch.int32, device=dev)
    d_bits = torch.empty(words, dtype=torch.int32, device=dev)
    d_hist = torch.zeros(4096, dtype=torch.int64, device=dev)
    kw = dict(seg_size=seg, p_small=10**8)
    ctx.verify_range(4, lim, device_out={"min_p": d_minp, "verified_bits": d_bits,
                                         "minp_hist": d_hist}, **kw)  # warm
    r = ctx.verify_range(4, lim, device_out={"min_p": d_minp, "verified_bits": d_bits,
                                             "minp_hist": d_hist}, **kw).result
    del d_minp, d_bits
    h_minp = torch.empty(count, dtype=torch.int32).pin_memory()
    h_bits = torch.empty(words, dtype=torch.int32).pin_memory()
    h_hist = torch.empty(4096, dtype=torch.int64).pin_memory()
    L = gb.load()
    o = gb.RangeOpts(seg, 10**8, 0, 0, 0, 0, 1, 0, None, 0)
    out = gb.RangeOut(h_bits.data_ptr(), h_minp.data_ptr(), h_hist.data_ptr(), None, None, None)
    res = gb.RangeResult()
    walls = []
    for _ in range(3):
        t0 = time.perf_counter()
        st = L.gb_verify_range(ctx._h, 4, lim, ctypes.byref(o), ctypes.byref(res), ctypes.byref(out))
        walls.append(time.perf_counter() - t0)
        if st != 0:
            raise RuntimeError(f"gb_verify_range failed: {st}")
    e2e = min(walls)
    mp = h_minp.numpy()
    return {"workload": "[4, 1e9], seg 2^26, P_SMALL 1e8, per-n minimal p + verified bitmap",
            "even_n": count, "kernel_ms": r["kernel_ms"], "device_ms": r["device_ms"],
            "value": count / (r["device_ms"] / 1e3), "e2e_value": count / e2e, "e2e_ms": e2e * 1e3,
            "d2h_bytes_per_step": count * 4 + words * 4 + 4096 * 8, "unit": UNIT,
            "failures": res.failures, "max_minp": int(mp.max()),
            "min_p_sha256": __import__("hashlib").sha256(mp.tobytes()).hexdigest()}


# the reference's published flags for its GPU verifier (RESULTS.md:39-41)
REF_GPU_FLAGS = ["--seg-size=200000000", "--p-small=1000000", "--batch-size=2000000"]


def measure_reference_gpu(gb, ctx, device, limits=(10**9, 10**10, 10**11)):
    """The reference's own GPU verifier (src/goldbach.cu built unmodified for
    sm_100a into oracle/_ref/goldbach) on this B200 with its published flags:
    its printed "Total computation time" (the worker threads' span), beside
    the wall time and device time of this build's gb_verify_range over the
    same [4, LIMIT].  Timing only: the reference's tiled sieve updates shared
    memory without synchronisation, so its answers are not a check."""
    import re
    exe = os.path.join(ROOT, "oracle", "_ref", "goldbach")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/goldbach not built (oracle/build_ref.sh)"}
    out = []
    for lim in limits:
        clk = ClockSampler(device)
        clk.start()
        try:
            r = subprocess.run([exe, str(lim)] + REF_GPU_FLAGS, capture_output=True, text=True,
                               timeout=600)
            txt, rc = r.stdout, r.returncode
        except subprocess.TimeoutExpired:
            txt, rc = "", "timeout"
        clocks = clk.stop()
        m = re.search(r"Total computation time : ([0-9.eE+-]+) seconds", txt)
        fb = re.search(r"Phase 2 fallbacks\s+: (\d+)", txt)
        ctx.verify_range(4, lim)  # warm (tables)
        t0 = time.perf_counter()
        ours = ctx.verify_range(4, lim).result
        wall = time.perf_counter() - t0
        ref_s = float(m.group(1)) if m else None
        out.append({"limit": lim, "flags": " ".join(REF_GPU_FLAGS), "rc": rc,
                    "reference_s": ref_s, "reference_fallbacks": int(fb.group(1)) if fb else None,
                    "reference_says_verified": "satisfy Goldbach" in txt, "reference_clocks": clocks,
                    "ours_wall_s": wall, "ours_device_s": ours["device_ms"] / 1e3,
                    "ours_failures": ours["failures"],
                    "speedup_wall": (ref_s / wall) if ref_s else None})
    return out


# serving lanes poll their queues this long before blocking (one host core
# per lane kept busy; single-request p50 at 1e3 requests/s 58 against 74 us)
SERVE_SPIN_US = 20000


def measure_serving(gb, device, rates=(1e2, 1e3, 1e4, 1e5), seconds=2.0, max_requests=10000,
                    range_lanes=0, max_range_batch=0):
    """C5: Poisson arrivals (seed 3) per rate; 70% single n uniform in
    [4, 2^64-2], 30% ranges of log-uniform width 2^8..2^26 even n at
    offsets uniform in [4, 1e19]; latency from scheduled arrival.  The
    load generator polls the clock for the last 200 us before each arrival
    (a sleep there would submit late by the timer slack, ~50-100 us)."""
    import numpy as np
    out = []
    with gb.Context(device) as ctx:
        ctx.serve_start(max_n=2**64 - 1, spin_us=SERVE_SPIN_US, range_lanes=range_lanes,
                        max_range_batch=max_range_batch)
        for rate in rates:
            rng = np.random.default_rng(3)
            m = int(min(max_requests, rate * seconds))
            gaps = rng.exponential(1.0 / rate, size=m)
            t_arr = np.cumsum(gaps)
            single = rng.random(m) < 0.7
            kinds = np.where(single, 0, 1).astype(np.int32)
            a = np.where(single, rng.integers(2, 2**63, size=m, dtype=np.uint64) * 2,
                         rng.integers(2, 5 * 10**18, size=m, dtype=np.uint64) * 2).astype(np.uint64)
            cnt = np.where(single, 1, np.exp2(rng.uniform(8, 26, size=m))).astype(np.uint64)
            ctx.serve_stats(reset=True)
            base = ctx.now_ns() + 2_000_000
            arr = (base + (t_arr * 1e9)).astype(np.uint64)
            tickets = []
            i = 0
            while i < m:  # submit every request whose arrival time has come
                now = ctx.now_ns()
                j = i
                while j < m and arr[j] <= now:
                    j += 1
                if j > i:
                    tickets += list(ctx.submit(kinds[i:j], a[i:j], cnt[i:j], arr[i:j]))
                    i = j
                else:  # sleep until 200 us before the next arrival, then poll
                    ahead = (int(arr[i]) - now) / 1e9
                    if ahead > 300e-6:
                        time.sleep(min(0.0005, ahead - 200e-6))
            res = [ctx.wait(t, 600000) for t in tickets]
            st = ctx.serve_stats()
            lat_s = np.array([r["latency_us"] for r, k in zip(res, kinds) if k == 0 and r["status"] == 0])
            lat_r = np.array([r["latency_us"] for r, k in zip(res, kinds) if k == 1 and r["status"] == 0])
            span = (max(int(arr[-1]), ctx.now_ns()) - int(arr[0])) / 1e9
            out.append({"rate_rps": rate, "lane_spin_us": SERVE_SPIN_US, "requests": m,
                        "completed": sum(r["status"] == 0 for r in res),
                        "rejected": st["rejected"], "busy": st["busy"],
                        "range_lanes": range_lanes or 2, "max_range_batch": max_range_batch or 4096,
                        "pool_bytes": st["pool_bytes"],
                        "pool_peak_bytes": st["pool_peak_bytes"],
                        "p50_us": st["p50_us"], "p99_us": st["p99_us"],
                        "single_p50_us": float(np.percentile(lat_s, 50)) if lat_s.size else None,
                        "single_p99_us": float(np.percentile(lat_s, 99)) if lat_s.size else None,
                        "range_p50_us": float(np.percentile(lat_r, 50)) if lat_r.size else None,
                        "range_p99_us": float(np.percentile(lat_r, 99)) if lat_r.size else None,
                        "throughput_rps": m / span, "batches_single": st["batches_single"],
                        "batches_range": st["batches_range"],
                        "even_n_served": int(sum(int(c) for c in cnt))})
        ctx.serve_stop()
    return out


# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--limit", type=int, default=10**12)
    ap.add_argument("--count", type=int, default=0,
                    help="time only the top COUNT even n below --limit (default: all of [4, limit])")
    ap.add_argument("--seg-size", type=int, default=1 << 27)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--halo", type=int, default=0)
    ap.add_argument("--block-threads", type=int, default=0)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default chunk / halo / block shape instead of the autotuner's")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--ref-sample-log2", type=int, default=24)
    ap.add_argument("--extra", choices=["windows", "single", "counts", "serving", "reference_gpu", "c1"],
                    help="run only this secondary measurement and print its JSON (profiling)")
    ap.add_argument("--windows", type=int, default=4096,
                    help="--extra windows: the first N seeded windows only")
    ap.add_argument("--no-windows-plain", action="store_true",
                    help="--extra windows: skip the plain per-window pipeline")
    ap.add_argument("--serve-rates", default="100,1000,10000,100000",
                    help="--extra serving: request rates (comma-separated)")
    ap.add_argument("--serve-lanes", type=int, default=0, help="--extra serving: range lanes (0: default)")
    ap.add_argument("--serve-range-batch", type=int, default=0,
                    help="--extra serving: requests per range-lane batch (0: default)")
    ap.add_argument("--no-windows-tune", action="store_true",
                    help="--extra windows: default knobs instead of the windows autotuner's")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.extra:
        gb = load_gb()
        if args.extra == "serving":
            rates = tuple(float(x) for x in args.serve_rates.split(","))
            print(json.dumps(measure_serving(gb, 0, rates, range_lanes=args.serve_lanes,
                                             max_range_batch=args.serve_range_batch)))
        else:
            with gb.Context(0) as c:
                if args.extra == "windows":
                    print(json.dumps(measure_windows(gb, c, args.windows, not args.no_windows_plain,
                                                     not args.no_windows_tune)))
                elif args.extra == "reference_gpu":
                    print(json.dumps(measure_reference_gpu(gb, c, 0)))
                elif args.extra == "c1":
                    print(json.dumps(measure_c1(gb, c, 0)))
                else:
                    f = {"single": measure_single, "counts": measure_counts}
                    print(json.dumps(f[args.extra](gb, c)))
        return 0

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
    multi = load_multi()
    ctx = gb.Context(local, max_n=args.limit)
    stream = torch.cuda.Stream()
    limit = args.limit - (args.limit & 1)
    start = max(4, limit - 2 * (args.count - 1)) if args.count else 4
    total = (limit - start) // 2 + 1
    nseg = gb.load().gb_num_segments(start, limit, args.seg_size)
    dev = torch.device("cuda", local)
    hist = torch.zeros(4096, dtype=torch.int64, device=dev)
    segfb = torch.zeros(nseg, dtype=torch.int32, device=dev)
    segfail = torch.zeros(nseg, dtype=torch.int32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    # chunk, halo and block shape: the autotuner's choice for this range class
    # (timed once on the top 2^28 n, outside the timed region), unless given
    tune = {}
    if not (args.chunk or args.halo or args.no_autotune):
        tune = ctx.autotune_range(start, limit, seg_size=args.seg_size)
        args.chunk, args.halo = tune["chunk_evens"], tune["halo"]
        args.block_threads = tune["block_threads"]
    kw = dict(seg_size=args.seg_size, chunk=args.chunk, halo=args.halo, shard_index=rank,
              block_threads=args.block_threads,
              shard_count=world, stream=stream.cuda_stream)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def step_dev():
        r = ctx.verify_range(start, limit, device_out={"minp_hist": hist, "seg_fallbacks": segfb,
                                                       "seg_failures": segfail}, **kw)
        res = r.result
        if dist is not None:  # the only exchange: the 32 KB histogram + summary
            with torch.cuda.stream(stream):
                res = multi.merge_results(res, hist, dist)
        return res

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
        res = step_dev()
        e1.record(stream)
        barrier()
        times.append(e0.elapsed_time(e1))
        kms.append(res["kernel_ms"])
        launches += res["kernel_launches"]
        results.append(res)
    clk = clocks.stop()
    ms = statistics.mean(times)
    if dist is not None:
        ms = multi.max_over_ranks(ms, dist, device=dev)
    value = total / (ms / 1000)

    # e2e: the same call with pinned host output buffers (D2H inside)
    h_hist = torch.zeros(4096, dtype=torch.int64).pin_memory()
    h_fb = torch.zeros(nseg, dtype=torch.int32).pin_memory()
    h_fail = torch.zeros(nseg, dtype=torch.int32).pin_memory()
    L = gb.load()

    def step_host():
        o = gb.RangeOpts(args.seg_size, 10**6, 0, args.chunk, args.halo, rank, world, 0,
                         stream.cuda_stream, args.block_threads)
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
        ems = multi.max_over_ranks(ems, dist, device=dev)
    e2e_value = total / (ems / 1000)
    d2h = 4096 * 8 + nseg * 8 + 8 * 8

    # roofline of range6_kernel (the dominant kernel, ~100% of the device
    # time): algorithmic integer work of this rank's share over its average
    # launch time, against ALU and shared-memory-atomic peaks measured here.
    halo = args.halo or 32768
    chunk = args.chunk or (1 << 20)
    n_mine = multi.shard_even_count(total, args.seg_size, rank, world)
    odd_q_per_n = 1 + (halo // 2) / chunk
    chunks = math.ceil(n_mine / chunk)
    offsets = chunks * sieving_primes(limit)
    alu_ops = (n_mine * (SEARCH_TESTS_PER_N / 32 * SEARCH_OPS_PER_WORD
                         + WHEEL_OPS_PER_ODD_Q * odd_q_per_n) + offsets * OPS_PER_OFFSET)
    marks = n_mine * MARKS_PER_ODD_Q * odd_q_per_n
    alu_peak, atom_peak = ctx.probe_peaks()
    k_s = statistics.mean(kms) / 1000
    sol_s = alu_ops / alu_peak + marks / atom_peak
    achieved = (alu_ops + marks * alu_peak / atom_peak) / k_s
    # the word-parallel floor: the search's SOL term counts one word op per 32
    # (n, p) tests, but a word of 32 n runs until its slowest n is resolved
    tests_per_n, floor_steps_per_n = search_floor(ctx, limit)
    floor_ops = (alu_ops - n_mine * SEARCH_TESTS_PER_N / 32 * SEARCH_OPS_PER_WORD
                 + n_mine * floor_steps_per_n * SEARCH_OPS_PER_WORD)
    floor_s = floor_ops / alu_peak + marks / atom_peak
    hbm, hbm_kind = hbm_peak()
    hbm_bytes = 2 * n_mine * odd_q_per_n / 8  # the q-bitset, had it gone through HBM
    res0 = results[-1]
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"range [{start}, {limit}] (every even n)", "seg_size": args.seg_size,
                   "chunk_evens": chunk, "halo": halo, "block_threads": args.block_threads or 512,
                   "autotuned": tune or None, "p_small": 10**6, "phase2_limit": 10**8,
                   "l2": "flushed (512 MB write) between steps",
                   "parallelism": f"segments sharded over {world} GPU(s)"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {
            "bound": "int", "achieved": achieved / 1e12, "peak": alu_peak / 1e12, "unit": "Top/s",
            "frac": achieved / alu_peak, "traffic": DRAM_BYTES_PER_N * n_mine,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of range6_kernel "
                               "on 2^30 even n ending at 1e12 (15.5 MB), scaled by the n of the "
                               "launch (the survivor lists' spill out of L2 grows with n)"),
            "kernel": "range6_kernel", "kernel_ms": k_s * 1e3,
            "peak_source": "measured in-process: gb_probe_peaks (32-bit ALU ops/s; shared-memory atomicAnd/s)",
            "smem_atomic_peak": atom_peak, "alu_ops_per_launch": alu_ops,
            "smem_marks_per_launch": marks, "offsets_per_launch": offsets,
            "speed_of_light_ms": sol_s * 1e3,
            "word_parallel_floor": {
                "frac": floor_s / k_s, "floor_ms": floor_s * 1e3,
                "floor_word_steps_per_n": floor_steps_per_n,
                "sol_word_ops_per_n": SEARCH_TESTS_PER_N / 32,
                "sampled_tests_per_n": tests_per_n,
                "source": ("search term at the word-parallel floor (each word of 32 same-class n "
                           "runs to its slowest n), from the kernel's per-n minimal p on 32 seeded "
                           "slices of 2^16 even n over the range; sieve terms as in the SOL")},
            "hbm": {"achieved": hbm_bytes / k_s / 1e9, "peak": hbm, "unit": "GB/s",
                    "frac": hbm_bytes / k_s / 1e9 / hbm, "peak_source": hbm_kind,
                    "note": "q-bitset bytes a staged design would move; the fused kernel keeps them on chip"}},
        "clocks": clk,
        "result": {"checked": res0["checked"], "failures": res0["failures"],
                   "phase2_fallbacks": res0["phase2_fallbacks"], "max_minp": res0["max_minp"]},
    }
    # C2's SEG_SIZE sweep: the segment is only the reporting unit here, so
    # every size runs the same kernel over the same chunks (one call each)
    sweep = []
    if world == 1 and not args.no_extras:
        for lg in range(24, 31):
            segs = gb.load().gb_num_segments(start, limit, 1 << lg)
            fb = torch.zeros(segs, dtype=torch.int32, device=dev)
            kw2 = dict(kw, seg_size=1 << lg)
            r = ctx.verify_range(start, limit, device_out={"minp_hist": hist, "seg_fallbacks": fb,
                                                           "seg_failures": fb}, **kw2)
            sweep.append({"seg_size": 1 << lg, "segments": segs, "kernel_ms": r.result["kernel_ms"],
                          "device_ms": r.result["device_ms"],
                          "value": total / (r.result["device_ms"] / 1e3),
                          "failures": r.result["failures"]})
        out["seg_size_sweep"] = sweep
    ctx.close()
    if world == 1 and rank == 0:
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline_oracle(limit)
        if not args.no_extras:
            with gb.Context(local) as c2:
                out["reference_gpu"] = measure_reference_gpu(gb, c2, local)
                out["c1"] = measure_c1(gb, c2, local)
                out["windows"] = measure_windows(gb, c2)
                out["single"] = measure_single(gb, c2)
                out["counts"] = measure_counts(gb, c2)
            out["serving"] = measure_serving(gb, local)
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
