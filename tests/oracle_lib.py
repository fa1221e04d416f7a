"""ctypes view of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is test infrastructure: a plain-C restatement of the reference's
CPU algorithm used only as the checker.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
u64 = C.c_uint64


class Summary(C.Structure):
    _fields_ = [("checked", u64), ("fallbacks", u64), ("failures", u64),
                ("first_failure", u64), ("max_minp", u64), ("max_minp_n", u64)]


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                           capture_output=True)
        L = C.CDLL(ORACLE_SO)
        L.gbo_isqrt.restype = u64
        L.gbo_isqrt.argtypes = [u64]
        L.gbo_count_primes.restype = u64
        L.gbo_count_primes.argtypes = [u64, u64, C.c_int]
        L.gbo_simple_sieve.restype = C.c_size_t
        L.gbo_simple_sieve.argtypes = [u64, C.c_void_p, C.c_size_t]
        L.gbo_segmented_sieve.argtypes = [u64, u64, C.c_void_p]
        L.gbo_odd_bitset.argtypes = [u64, u64, C.c_void_p]
        L.gbo_mr12.argtypes = [u64]
        L.gbo_mr7.argtypes = [u64]
        L.gbo_phase2_minp.restype = u64
        L.gbo_phase2_minp.argtypes = [u64, u64]
        L.gbo_minp_range.argtypes = [u64, u64, u64, C.c_void_p, C.c_int]
        L.gbo_minp_windows.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, u64, C.c_void_p, C.c_int]
        L.gbo_single_minp.restype = u64
        L.gbo_single_minp.argtypes = [u64, u64]
        L.gbo_single_minp_batch.argtypes = [C.c_void_p, C.c_size_t, u64, C.c_void_p, C.c_int]
        L.gbo_goldbach_count.restype = u64
        L.gbo_goldbach_count.argtypes = [u64]
        L.gbo_verify_range.argtypes = [u64, u64, u64, u64, C.c_void_p, C.c_size_t,
                                       C.POINTER(Summary), C.c_int]
        L.gbo_prime_index.restype = u64
        L.gbo_prime_index.argtypes = [u64]
        self.L = L

    def isqrt(self, n):
        return self.L.gbo_isqrt(n)

    def count_primes(self, lo, hi, threads=0):
        return self.L.gbo_count_primes(lo, hi, threads)

    def primes(self, limit):
        n = self.L.gbo_simple_sieve(limit, None, 0)
        a = np.zeros(n, np.uint64)
        self.L.gbo_simple_sieve(limit, a.ctypes.data, n)
        return a

    def odd_bitset(self, q_lo, nbits):
        w = np.zeros((nbits + 31) // 32, np.uint32)
        self.L.gbo_odd_bitset(q_lo, nbits, w.ctypes.data)
        return w

    def mr7(self, n):
        return bool(self.L.gbo_mr7(n))

    def mr12(self, n):
        return bool(self.L.gbo_mr12(n))

    def minp(self, start, count, p_limit=10**8, threads=0):
        a = np.zeros(count, np.uint32)
        assert self.L.gbo_minp_range(start, count, p_limit, a.ctypes.data, threads) == 0
        return a

    def minp_windows(self, starts, counts, p_limit=10**8, threads=0):
        starts = np.ascontiguousarray(starts, dtype=np.uint64)
        counts = np.ascontiguousarray(counts, dtype=np.uint64)
        out = np.zeros(int(counts.sum()), np.uint32)
        assert self.L.gbo_minp_windows(starts.ctypes.data, counts.ctypes.data, len(starts), p_limit,
                                       out.ctypes.data, threads) == 0
        return out

    def single_minp(self, ns, p_limit=10**8, threads=0):
        ns = np.ascontiguousarray(ns, dtype=np.uint64)
        out = np.zeros(len(ns), np.uint64)
        self.L.gbo_single_minp_batch(ns.ctypes.data, len(ns), p_limit, out.ctypes.data, threads)
        return out

    def phase2_minp(self, n, limit=10**8):
        return self.L.gbo_phase2_minp(n, limit)

    def goldbach_count(self, n):
        return self.L.gbo_goldbach_count(n)

    def verify_range(self, start, limit, p_small=10**6, phase2=10**8, nbins=4096, threads=0):
        h = np.zeros(nbins, np.uint64)
        s = Summary()
        assert self.L.gbo_verify_range(start, limit, p_small, phase2, h.ctypes.data, nbins,
                                       C.byref(s), threads) == 0
        return {f: getattr(s, f) for f, _ in Summary._fields_}, h

    def prime_index(self, p):
        return self.L.gbo_prime_index(p)


def hist_of(minp, primes_sorted, nbins=4096):
    """Histogram of minimal p by prime index (failures, p = 0, excluded)."""
    m = minp[minp > 0].astype(np.uint64)
    idx = np.searchsorted(primes_sorted, m)
    idx = np.minimum(idx, nbins - 1)
    return np.bincount(idx, minlength=nbins).astype(np.uint64)
