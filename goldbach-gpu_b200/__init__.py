"""goldbach-gpu_b200 -- Python binding over libgoldbach_b200.so (ctypes).

The product is the sm_100a CUDA library behind include/gb/gb.h and the CLIs
built on it (bin/goldbach, bin/single_check).  This module is the thin Python
view of that C-ABI used by the tests and by bench.py.  There is no fallback:
if the shared library is missing, importing the binding's `load()` raises.

Loading by path (the directory name is not a Python identifier):
    spec = importlib.util.spec_from_file_location(
        "goldbach_gpu_b200", "<repo>/goldbach-gpu_b200/__init__.py")
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgoldbach_b200.so")
BIN_DIR = os.path.join(HERE, "bin")

GB_OK, GB_EINVAL, GB_ENOMEM, GB_ECUDA, GB_ETIMEOUT = 0, -1, -2, -3, -4
GB_ECANCELED, GB_ENODEV, GB_EOVERFLOW, GB_EAGAIN, GB_EBUSY = -5, -6, -7, -8, -9
GB_HIST_BINS = 4096
GB_PHASE2_LIMIT_DEFAULT = 100_000_000
GB_WINDOWS_PERSISTENT, GB_WINDOWS_PLAIN = 0, 1

u64, u32, i32, vp = C.c_uint64, C.c_uint32, C.c_int, C.c_void_p


class GbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"gb status {status}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("device_mem_budget", u64), ("max_n", u64), ("cand_limit", u64)]


class RangeOpts(C.Structure):
    _fields_ = [("seg_size", u64), ("p_small", u64), ("phase2_limit", u64),
                ("chunk_evens", u32), ("halo", u32), ("shard_index", u32),
                ("shard_count", u32), ("on_device", i32), ("stream", vp),
                ("block_threads", u32)]


class AutotuneResult(C.Structure):
    _fields_ = [("chunk_evens", u32), ("halo", u32), ("block_threads", u32),
                ("even_n_per_s", C.c_double), ("candidates", u32), ("sample_evens", u64),
                ("cached", i32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class RangeResult(C.Structure):
    _fields_ = [("checked", u64), ("verified", u64), ("phase2_fallbacks", u64),
                ("failures", u64), ("first_failure_n", u64), ("max_minp", u64),
                ("num_segments", u64), ("queued", u64), ("kernel_launches", u64),
                ("device_ms", C.c_double), ("kernel_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class RangeOut(C.Structure):
    _fields_ = [("verified_bits", vp), ("min_p", vp), ("minp_hist", vp),
                ("seg_fallbacks", vp), ("seg_failures", vp), ("seg_hist", vp)]


class CountOpts(C.Structure):
    _fields_ = [("on_device", C.c_int), ("stream", C.c_void_p)]


class SingleOpts(C.Structure):
    _fields_ = [("p_limit", u64), ("on_device", i32), ("stream", vp)]


class SingleResult(C.Structure):
    _fields_ = [("found", u64), ("max_p", u64), ("kernel_launches", u64),
                ("device_ms", C.c_double)]


class BigResult(C.Structure):
    _fields_ = [("candidates", u64), ("mr_tests", u64), ("device_ms", C.c_double)]


GB_BIG_MAX_LIMBS = 128


class Window(C.Structure):
    _fields_ = [("start", u64), ("count", u64)]


class WindowsOpts(C.Structure):
    _fields_ = [("mode", i32), ("chunk_evens", u32), ("halo", u32),
                ("phase2_limit", u64), ("on_device", i32), ("stream", vp), ("mr_below", u64),
                ("mr_divisor", u32), ("large_ctas_per_sm", u32), ("block_threads", u32),
                ("gpu_share_pct", u32)]


class WindowsTune(C.Structure):
    _fields_ = [("mr_divisor", u32), ("chunk_evens", u32), ("large_ctas_per_sm", u32),
                ("block_threads", u32), ("even_n_per_s", C.c_double), ("candidates", u32),
                ("sample_windows", u32), ("cached", i32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class WindowResult(C.Structure):
    _fields_ = [("verified", u64), ("failures", u64), ("max_minp", u64), ("minp_sum", u64)]


class WindowsSummary(C.Structure):
    _fields_ = [("total_n", u64), ("failures", u64), ("kernel_launches", u64),
                ("device_ms", C.c_double), ("sieved_windows", u64), ("large_pairs", u64),
                ("large_ms", C.c_double), ("search_ms", C.c_double)]


class Request(C.Structure):
    _fields_ = [("kind", i32), ("a", u64), ("count", u64), ("arrival_ns", u64)]


class Response(C.Structure):
    _fields_ = [("status", i32), ("kind", i32), ("p", u64), ("q", u64), ("verified", u64),
                ("failures", u64), ("max_minp", u64), ("minp_sum", u64), ("latency_us", C.c_double),
                ("lane", u32), ("batch", u32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServeOpts(C.Structure):
    _fields_ = [("max_n", u64), ("max_single_batch", u32), ("max_range_batch", u32),
                ("range_arena_bytes", u64), ("small_range", u64), ("no_graph", u32),
                ("spin_us", u32), ("range_lanes", u32), ("pool_bytes", u64),
                ("max_pending", u64), ("max_pending_n", u64)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", u64), ("completed", u64), ("pending", u64), ("rejected", u64),
                ("batches_single", u64), ("batches_range", u64), ("p50_us", C.c_double),
                ("p99_us", C.c_double), ("max_us", C.c_double), ("mean_us", C.c_double),
                ("elapsed_s", C.c_double), ("completed_per_s", C.c_double), ("busy", u64),
                ("pool_bytes", u64), ("pool_peak_bytes", u64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


GB_REQ_SINGLE, GB_REQ_RANGE = 0, 1

_lib = None


def load(path: str = LIB_PATH):
    """Loads the CUDA library (raises FileNotFoundError / OSError if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built: run `make -C goldbach-gpu_b200`")
    L = C.CDLL(path)
    P = C.POINTER
    sig = {
        "gb_device_count": (i32, []),
        "gb_device_info": (i32, [i32, C.c_char_p, C.c_size_t, P(u64)]),
        "gb_estimate_device_bytes": (u64, [P(Config)]),
        "gb_create": (i32, [i32, P(Config), P(vp)]),
        "gb_destroy": (None, [vp]),
        "gb_strerror": (C.c_char_p, [i32]),
        "gb_last_error": (C.c_char_p, [vp]),
        "gb_mem_info": (i32, [vp, P(u64), P(u64)]),
        "gb_num_segments": (u64, [u64, u64, u64]),
        "gb_verify_range": (i32, [vp, u64, u64, P(RangeOpts), P(RangeResult), P(RangeOut)]),
        "gb_sieve_bitset": (i32, [vp, u64, u64, vp, i32, vp]),
        "gb_goldbach_counts": (i32, [vp, u64, u64, vp, P(CountOpts)]),
        "gb_autotune_range": (i32, [vp, u64, u64, P(RangeOpts), P(RangeOpts), P(AutotuneResult)]),
        "gb_autotune_windows": (i32, [vp, P(Window), C.c_size_t, P(WindowsOpts), P(WindowsOpts),
                                      P(WindowsTune)]),
        "gb_primes_upto": (i32, [vp, u64, vp, u64, P(u64)]),
        "gb_is_prime_batch": (i32, [vp, vp, C.c_size_t, vp, i32, vp]),
        "gb_check_big": (i32, [vp, vp, u32, u64, P(u64), vp, P(BigResult)]),
        "gb_check_single_batch": (i32, [vp, vp, C.c_size_t, vp, vp, P(SingleOpts), P(SingleResult)]),
        "gb_verify_windows": (i32, [vp, P(Window), C.c_size_t, P(WindowsOpts), P(WindowResult),
                                    vp, P(WindowsSummary)]),
        "gb_now_ns": (u64, []),
        "gb_probe_peaks": (i32, [vp, P(C.c_double), P(C.c_double)]),
        "gb_probe_mont_products": (i32, [vp, P(C.c_double)]),
        "gb_serve_start": (i32, [vp, P(ServeOpts)]),
        "gb_submit": (i32, [vp, P(Request), C.c_size_t, P(u64)]),
        "gb_poll": (i32, [vp, u64, P(Response)]),
        "gb_wait": (i32, [vp, u64, P(Response), u64]),
        "gb_serve_stats_get": (i32, [vp, P(ServeStats), i32]),
        "gb_serve_stop": (i32, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name, None)
        if f is None:  # entry point not in this build; calling it raises
            continue
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):  # torch tensor
        return a.data_ptr()
    return int(a)


def device_count() -> int:
    return load().gb_device_count()


@dataclass
class RangeRun:
    result: dict
    min_p: np.ndarray | None = None
    verified_bits: np.ndarray | None = None
    hist: np.ndarray | None = None
    seg_fallbacks: np.ndarray | None = None
    seg_failures: np.ndarray | None = None
    seg_hist: np.ndarray | None = None


class Context:
    """One gb_ctx: a CUDA device with its resident prime tables."""

    def __init__(self, device: int = 0, budget: int = 0, max_n: int = 0, cand_limit: int = 0):
        self.L = load()
        self._h = vp()
        cfg = Config(budget, max_n, cand_limit)
        st = self.L.gb_create(device, C.byref(cfg), C.byref(self._h))
        if st != GB_OK:
            raise GbError(st, self.L.gb_strerror(st).decode())

    def close(self):
        if self._h:
            self.L.gb_destroy(self._h)
            self._h = vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != GB_OK:
            raise GbError(st, f"{self.L.gb_strerror(st).decode()}: "
                              f"{self.L.gb_last_error(self._h).decode()}")

    def mem_info(self):
        held, budget = u64(), u64()
        self._check(self.L.gb_mem_info(self._h, C.byref(held), C.byref(budget)))
        return held.value, budget.value

    # -- range -------------------------------------------------------------
    def autotune_range(self, start: int, limit: int, *, seg_size: int = 10_000_000,
                       p_small: int = 1_000_000, phase2_limit: int = 0) -> dict:
        """gb_autotune_range: the chunk_evens and halo to use for [start, limit]
        (timed on a sample at the top of the range, cached per range class)."""
        base = RangeOpts(seg_size, p_small, phase2_limit, 0, 0, 0, 1, 0, None, 0)
        tuned = RangeOpts()
        r = AutotuneResult()
        self._check(self.L.gb_autotune_range(self._h, start, limit, C.byref(base), C.byref(tuned),
                                             C.byref(r)))
        return r.as_dict()

    def verify_range(self, start: int, limit: int, *, seg_size: int = 10_000_000,
                     p_small: int = 1_000_000, phase2_limit: int = 0, chunk: int = 0,
                     halo: int = 0, shard_index: int = 0, shard_count: int = 1,
                     want_minp=False, want_bits=False, want_hist=True, want_seg=False,
                     want_seg_hist=False, stream=None, device_out: dict | None = None,
                     check: bool = True, block_threads: int = 0) -> RangeRun:
        """Verifies every even n in [start, limit].  Host numpy outputs are
        allocated on request; `device_out` maps RangeOut field names to device
        pointers (torch tensors) and switches the call to on_device mode."""
        L = self.L
        lim = limit - (limit & 1)
        st0 = max(4, start + (start & 1))
        count = (lim - st0) // 2 + 1 if lim >= st0 else 0
        nseg = L.gb_num_segments(start, limit, seg_size)
        o = RangeOpts(seg_size, p_small, phase2_limit, chunk, halo, shard_index, shard_count,
                      0, stream or None, block_threads)
        run = RangeRun(result={})
        out = RangeOut()
        if device_out is not None:
            o.on_device = 1
            for k, v in device_out.items():
                setattr(out, k, _ptr(v))
        else:
            if want_minp:
                run.min_p = np.zeros(count, np.uint32)
                out.min_p = run.min_p.ctypes.data
            if want_bits:
                run.verified_bits = np.zeros((count + 31) // 32, np.uint32)
                out.verified_bits = run.verified_bits.ctypes.data
            if want_hist:
                run.hist = np.zeros(GB_HIST_BINS, np.uint64)
                out.minp_hist = run.hist.ctypes.data
            if want_seg:
                run.seg_fallbacks = np.zeros(nseg, np.uint32)
                run.seg_failures = np.zeros(nseg, np.uint32)
                out.seg_fallbacks = run.seg_fallbacks.ctypes.data
                out.seg_failures = run.seg_failures.ctypes.data
            if want_seg_hist:
                run.seg_hist = np.zeros((nseg, GB_HIST_BINS), np.uint64)
                out.seg_hist = run.seg_hist.ctypes.data
        res = RangeResult()
        st = L.gb_verify_range(self._h, start, limit, C.byref(o), C.byref(res), C.byref(out))
        if check:
            self._check(st)
        run.result = res.as_dict()
        run.result["status"] = st
        return run

    # -- tables / primality --------------------------------------------------
    def sieve_bitset(self, q_lo: int, nbits: int) -> np.ndarray:
        w = np.zeros((nbits + 31) // 32, np.uint32)
        self._check(self.L.gb_sieve_bitset(self._h, q_lo, nbits, w.ctypes.data, 0, None))
        return w

    def goldbach_counts(self, start: int, count: int, device_out=None, stream=None) -> np.ndarray:
        """c(n) = #{p <= n/2 : p, n - p prime} for n = start, start + 2, ...
        (count values; gb_goldbach_counts).  device_out: a device buffer
        (torch int64 tensor) to fill instead of returning a host array."""
        o = CountOpts(1 if device_out is not None else 0, stream)
        if device_out is not None:
            self._check(self.L.gb_goldbach_counts(self._h, start, count, _ptr(device_out), C.byref(o)))
            return device_out
        out = np.zeros(count, np.uint64)
        self._check(self.L.gb_goldbach_counts(self._h, start, count, out.ctypes.data, C.byref(o)))
        return out

    def primes_upto(self, limit: int) -> np.ndarray:
        n = u64()
        self._check(self.L.gb_primes_upto(self._h, limit, None, 0, C.byref(n)))
        a = np.zeros(n.value, np.uint32)
        self._check(self.L.gb_primes_upto(self._h, limit, a.ctypes.data, n.value, C.byref(n)))
        return a

    def is_prime(self, ns) -> np.ndarray:
        ns = np.ascontiguousarray(ns, dtype=np.uint64)
        out = np.zeros(len(ns), np.uint8)
        self._check(self.L.gb_is_prime_batch(self._h, ns.ctypes.data, len(ns), out.ctypes.data,
                                             0, None))
        return out.astype(bool)

    def check_single(self, ns, p_limit: int = 0, device_ptrs=None, stream=None):
        """Minimal (p, q) for each even n.  device_ptrs=(n, p, q) runs on
        device buffers (torch tensors) instead of host arrays."""
        r = SingleResult()
        if device_ptrs is not None:
            n_t, p_t, q_t = device_ptrs
            o = SingleOpts(p_limit, 1, stream or None)
            self._check(self.L.gb_check_single_batch(self._h, _ptr(n_t), n_t.numel(), _ptr(p_t),
                                                     _ptr(q_t), C.byref(o), C.byref(r)))
            return None, None, r
        ns = np.ascontiguousarray(ns, dtype=np.uint64)
        p = np.zeros(len(ns), np.uint64)
        q = np.zeros(len(ns), np.uint64)
        o = SingleOpts(p_limit, 0, stream or None)
        self._check(self.L.gb_check_single_batch(self._h, ns.ctypes.data, len(ns), p.ctypes.data,
                                                 q.ctypes.data, C.byref(o), C.byref(r)))
        return p, q, r

    def check_big(self, n: int, p_limit: int = 0):
        """gb_check_big: the minimal p <= p_limit with n - p a probable prime
        (12-base strong test; deterministic below 3.3e24) for an even n of up
        to 4096 bits.  Returns (p, q, result dict); p = q = 0: none."""
        nl = max(1, (n.bit_length() + 31) // 32)
        limbs = np.array([(n >> (32 * i)) & 0xFFFFFFFF for i in range(nl)], dtype=np.uint32)
        q = np.zeros(nl, np.uint32)
        p = u64()
        r = BigResult()
        self._check(self.L.gb_check_big(self._h, limbs.ctypes.data, nl, p_limit, C.byref(p),
                                        q.ctypes.data, C.byref(r)))
        qv = sum(int(x) << (32 * i) for i, x in enumerate(q))
        return p.value, qv, {f: getattr(r, f) for f, _ in BigResult._fields_}

    # -- windows -------------------------------------------------------------
    @staticmethod
    def _windows(starts, counts):
        starts = np.asarray(starts, dtype=np.uint64)
        counts = np.asarray(counts, dtype=np.uint64)
        w = (Window * len(starts))()
        for i in range(len(starts)):
            w[i].start = int(starts[i])
            w[i].count = int(counts[i])
        return w

    def autotune_windows(self, starts, counts, phase2_limit=0) -> dict:
        """gb_autotune_windows: the Miller-Rabin split divisor, chunk, large-prime
        grid and block shape for this batch (timed on a sample, cached per
        batch class); the dict carries the choice and the opts to pass on."""
        w = self._windows(starts, counts)
        base = WindowsOpts(GB_WINDOWS_PERSISTENT, 0, 0, phase2_limit, 0, None, 0, 0, 0, 0, 0)
        tuned = WindowsOpts()
        r = WindowsTune()
        self._check(self.L.gb_autotune_windows(self._h, w, len(w), C.byref(base), C.byref(tuned),
                                               C.byref(r)))
        return r.as_dict()

    def verify_windows(self, starts, counts, *, mode=GB_WINDOWS_PERSISTENT, chunk=0, halo=0,
                       phase2_limit=0, want_minp=False, stream=None, mr_below=0, mr_divisor=0,
                       large_ctas_per_sm=0, block_threads=0, gpu_share_pct=0):
        counts = np.asarray(counts, dtype=np.uint64)
        w = self._windows(starts, counts)
        nw = len(w)
        res = (WindowResult * nw)()
        minp = np.zeros(int(counts.sum()), np.uint32) if want_minp else None
        s = WindowsSummary()
        o = WindowsOpts(mode, chunk, halo, phase2_limit, 0, stream or None, mr_below, mr_divisor,
                        large_ctas_per_sm, block_threads, gpu_share_pct)
        self._check(self.L.gb_verify_windows(self._h, w, nw, C.byref(o), res,
                                             _ptr(minp), C.byref(s)))
        per = [{f: getattr(res[i], f) for f, _ in WindowResult._fields_} for i in range(nw)]
        return per, minp, {f: getattr(s, f) for f, _ in WindowsSummary._fields_}

    # -- serving ---------------------------------------------------------------
    def serve_start(self, max_n: int = 0, max_single_batch: int = 0, max_range_batch: int = 0,
                    range_arena_bytes: int = 0, small_range: int = 0, no_graph: bool = False,
                    spin_us: int = 0, range_lanes: int = 0, pool_bytes: int = 0,
                    max_pending: int = 0, max_pending_n: int = 0):
        o = ServeOpts(max_n, max_single_batch, max_range_batch, range_arena_bytes, small_range,
                      1 if no_graph else 0, spin_us, range_lanes, pool_bytes, max_pending,
                      max_pending_n)
        self._check(self.L.gb_serve_start(self._h, C.byref(o)))

    def submit(self, kinds, a, counts=None, arrival_ns=None) -> np.ndarray:
        """Queues requests (kind GB_REQ_SINGLE / GB_REQ_RANGE); returns tickets."""
        kinds = np.asarray(kinds, dtype=np.int32)
        a = np.asarray(a, dtype=np.uint64)
        m = len(kinds)
        counts = np.ones(m, np.uint64) if counts is None else np.asarray(counts, dtype=np.uint64)
        arr = np.zeros(m, np.uint64) if arrival_ns is None else np.asarray(arrival_ns, dtype=np.uint64)
        reqs = np.zeros(m, dtype=[("kind", "<i4"), ("pad", "<i4"), ("a", "<u8"), ("count", "<u8"),
                                  ("arrival_ns", "<u8")])
        reqs["kind"], reqs["a"], reqs["count"], reqs["arrival_ns"] = kinds, a, counts, arr
        t = np.zeros(m, np.uint64)
        self._check(self.L.gb_submit(self._h, reqs.ctypes.data_as(C.POINTER(Request)), m,
                                     t.ctypes.data_as(C.POINTER(u64))))
        return t

    def poll(self, ticket: int):
        r = Response()
        st = self.L.gb_poll(self._h, int(ticket), C.byref(r))
        if st == GB_EAGAIN:
            return None
        self._check(st)
        return r.as_dict()

    def wait(self, ticket: int, timeout_ms: int = 60000):
        r = Response()
        self._check(self.L.gb_wait(self._h, int(ticket), C.byref(r), timeout_ms))
        return r.as_dict()

    def serve_stats(self, reset: bool = False) -> dict:
        s = ServeStats()
        self._check(self.L.gb_serve_stats_get(self._h, C.byref(s), int(reset)))
        return s.as_dict()

    def serve_stop(self):
        self._check(self.L.gb_serve_stop(self._h))

    def probe_peaks(self) -> tuple[float, float]:
        """(32-bit ALU ops/s, shared-memory atomicAnd/s) measured on this GPU."""
        a, m = C.c_double(), C.c_double()
        self._check(self.L.gb_probe_peaks(self._h, C.byref(a), C.byref(m)))
        return a.value, m.value

    def probe_mont_products(self) -> float:
        """64-bit Montgomery products per second measured on this GPU."""
        v = C.c_double()
        self._check(self.L.gb_probe_mont_products(self._h, C.byref(v)))
        return v.value

    def now_ns(self) -> int:
        return self.L.gb_now_ns()
