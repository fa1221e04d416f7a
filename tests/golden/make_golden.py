#!/usr/bin/env python3
"""Generates the golden fixtures under tests/golden/ (run in the build
container, where the reference sources exist).

Sources of truth, in order of authority:
  * the reference's own code, compiled from its sources by oracle/build_ref.sh
    into oracle/_ref/: the cpu_goldbach binary, segmented_sieve /
    goldbach_count / goldbach_verify (libgbref.so) and the Phase-2
    cpu_miller_rabin of src/goldbach.cu (libgbref_p2.so);
  * the reference's published single_check partitions (RESULTS.md:112-121);
  * the CPU oracle (oracle/liboracle.so), used only where the reference has
    no runnable equivalent (minimal p over [4, 1e9]) and itself pinned by the
    fixtures above.

Usage: python tests/golden/make_golden.py [c1]   (needs oracle/_ref built;
"c1" writes only ref_c1_1e9.json, about a minute of reference CPU time)
"""
import ctypes as C
import hashlib
import json
import os
import re
import subprocess
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
GOLD = os.path.join(ROOT, "tests", "golden")
REF = os.path.join(ROOT, "oracle", "_ref")


def lib(path):
    return C.CDLL(path)


def main():
    R = lib(os.path.join(REF, "libgbref.so"))
    P2 = lib(os.path.join(REF, "libgbref_p2.so"))
    O = lib(os.path.join(ROOT, "oracle", "liboracle.so"))
    u64 = C.c_uint64
    R.gbref_count_primes.restype = u64
    R.gbref_count_primes.argtypes = [u64, u64]
    R.gbref_goldbach_counts.argtypes = [u64, C.c_void_p]
    R.gbref_window_verify.restype = u64
    R.gbref_window_verify.argtypes = [u64, u64, u64, C.c_void_p, C.c_int]
    P2.gbref_cpu_miller_rabin_batch.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
    P2.gbref_cpu_optimized_check.argtypes = [u64]
    O.gbo_verify_range.argtypes = [u64, u64, u64, u64, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int]
    O.gbo_minp_range.argtypes = [u64, u64, u64, C.c_void_p, C.c_int]

    # 1. prime counts of windows by the reference segmented_sieve
    windows = [(0, 10**6), (10**9, 10**9 + 10**6), (10**12 - 10**6, 10**12),
               (10**13, 10**13 + 2 * 10**5), (10**15, 10**15 + 10**5)]
    pi = [{"low": lo, "high": hi, "count": R.gbref_count_primes(lo, hi)} for lo, hi in windows]
    json.dump({"source": "reference segmented_sieve (src/segmented_sieve.cpp:29-50) via oracle/_ref/libgbref.so",
               "windows": pi}, open(os.path.join(GOLD, "ref_window_pi.json"), "w"), indent=1)

    # 2. Miller-Rabin verdicts of the reference's cpu_miller_rabin
    rng = np.random.default_rng(0xB200)
    xs = list(map(int, rng.integers(0, 2**63, size=4096, dtype=np.uint64) * 2 + 1))
    special = [1, 2, 3, 4, 5, 9, 561, 1105, 1729, 2047, 3277, 4033, 25326001, 3215031751,
               2152302898747, 3474749660383, 341550071728321, 3825123056546413051,
               (1 << 61) - 1, (1 << 64) - 59, (1 << 64) - 1, (1 << 64) - 3, (1 << 63) + 29,
               1000000007, 999999999989, 10**18 + 3, 10**18 + 9]
    vals = np.array(special + xs, dtype=np.uint64)
    out = np.zeros(len(vals), np.uint8)
    P2.gbref_cpu_miller_rabin_batch(vals.ctypes.data, len(vals), out.ctypes.data)
    json.dump({"source": "reference cpu_miller_rabin (src/goldbach.cu:333-360) via oracle/_ref/libgbref_p2.so",
               "n": [str(int(v)) for v in vals], "prime": out.tolist()},
              open(os.path.join(GOLD, "ref_mr.json"), "w"))

    # 3. goldbach_count(n) for n = 4..4000 (src/cpu_goldbach.cpp:29-36)
    lim = 4000
    cnt = np.zeros((lim - 4) // 2 + 1, np.uint64)
    R.gbref_goldbach_counts(lim, cnt.ctypes.data)
    json.dump({"source": "reference goldbach_count via oracle/_ref/libgbref.so", "first_n": 4,
               "counts": cnt.tolist()}, open(os.path.join(GOLD, "ref_goldbach_count.json"), "w"))

    # 4. the reference cpu_goldbach binary's own summary
    runs = []
    for L in (10**5, 10**6, 10**7):
        txt = subprocess.run([os.path.join(REF, "cpu_goldbach"), str(L)], capture_output=True,
                             text=True, check=True).stdout
        runs.append({"limit": L,
                     "checked": int(re.search(r"Even numbers checked : (\d+)", txt).group(1)),
                     "failures": int(re.search(r"Failures found\s+: (\d+)", txt).group(1)),
                     "final": [l for l in txt.splitlines() if "satisfy Goldbach" in l][0]})
    json.dump({"source": "oracle/_ref/cpu_goldbach (src/cpu_goldbach.cpp)", "runs": runs},
              open(os.path.join(GOLD, "ref_cpu_goldbach.json"), "w"), indent=1)

    # 5. minimal p of windows by the reference's segmented_sieve + the
    #    goldbach_verify scan rule (oracle/ref_shim.cpp gbref_window_verify)
    wins = []
    for start, count in [(4, 1 << 16), (10**9 - 2 * (1 << 16), 1 << 16),
                         (10**12 - 2 * (1 << 18), 1 << 18), (10**13 + 123456, 1 << 16),
                         (10**15 + 2, 1 << 14)]:
        mp = np.zeros(count, np.uint32)
        unver = R.gbref_window_verify(start, count, 1 << 16, mp.ctypes.data, 8)
        hist = np.bincount(mp, minlength=1).tolist()
        wins.append({"start": start, "count": count, "unverified": int(unver),
                     "sha256": hashlib.sha256(mp.tobytes()).hexdigest(),
                     "first": mp[:64].tolist(), "max": int(mp.max()),
                     "hist_nonzero": {str(i): int(c) for i, c in enumerate(hist) if c}})
    json.dump({"source": "reference segmented_sieve + cpu_goldbach.cpp:19-21 scan rule "
                         "(oracle/_ref/libgbref.so gbref_window_verify); min_p as uint32 little-endian",
               "windows": wins}, open(os.path.join(GOLD, "ref_window_minp.json"), "w"), indent=1)

    # 6. reference Phase 2 (cpu_optimized_check) on even n near the top of
    #    the 64-bit range: every one verified
    ns = [10**12, 10**15, 10**18, 10**19, (1 << 64) - 2, (1 << 63) + 2]
    ok = [P2.gbref_cpu_optimized_check(n) for n in ns]
    json.dump({"source": "reference cpu_optimized_check (src/goldbach.cu:362-373)",
               "n": [str(n) for n in ns], "verified": ok},
              open(os.path.join(GOLD, "ref_phase2.json"), "w"))

    # 7. oracle histogram over [4, 1e9] (pinned by the fixtures above)
    hist = np.zeros(4096, np.uint64)
    summ = (u64 * 6)()
    assert O.gbo_verify_range(4, 10**9, 10**5, 10**8, hist.ctypes.data, 4096, summ, 0) == 0
    nz = {str(i): int(c) for i, c in enumerate(hist) if c}
    json.dump({"source": "oracle gbo_verify_range(4, 1e9, p_small=1e5, phase2=1e8)",
               "checked": summ[0], "fallbacks": summ[1], "failures": summ[2],
               "max_minp": summ[4], "max_minp_n": summ[5], "hist_nonzero": nz},
              open(os.path.join(GOLD, "oracle_hist_1e9.json"), "w"))

    # 8. minimal p for n = 4..40000 (oracle) cross-checked by brute force
    n_hi = 40000
    cnt = (n_hi - 4) // 2 + 1
    mp = np.zeros(cnt, np.uint32)
    O.gbo_minp_range(4, cnt, 10**8, mp.ctypes.data, 0)
    sieve = bytearray([1]) * (n_hi + 1)
    sieve[0] = sieve[1] = 0
    for i in range(2, int(n_hi**0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = bytearray(len(sieve[i * i::i]))
    for j in range(cnt):
        n = 4 + 2 * j
        p = next(p for p in range(2, n // 2 + 1) if sieve[p] and sieve[n - p])
        assert mp[j] == p, (n, mp[j], p)
    json.dump({"source": "oracle gbo_minp_range, checked against a brute-force scan",
               "first_n": 4, "min_p": mp.tolist()},
              open(os.path.join(GOLD, "minp_small.json"), "w"))
    print("golden fixtures written to", GOLD)


def make_c1():
    """C1 as the benchmark states it: every even n in [4, 1e9].  The minimal p
    of all 499,999,999 n by the reference's segmented_sieve + the
    goldbach_verify scan rule (gbref_window_verify, halo 2^16: every minimal
    p below 1e9 is under 2^11), hashed as uint32 little-endian, and the
    verified bitmap (bit j <-> n = 4 + 2j, packed into uint32 words); plus the
    summary the reference's cpu_goldbach binary prints for LIMIT = 1e9."""
    R = lib(os.path.join(REF, "libgbref.so"))
    R.gbref_window_verify.restype = C.c_uint64
    R.gbref_window_verify.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_int]
    count = (10**9 - 4) // 2 + 1
    mp = np.zeros(count, np.uint32)
    unver = R.gbref_window_verify(4, count, 1 << 16, mp.ctypes.data, os.cpu_count() or 1)
    bits = np.packbits(mp > 0, bitorder="little")
    words = (count + 31) // 32
    bits = np.concatenate([bits, np.zeros(4 * words - len(bits), np.uint8)])
    txt = subprocess.run([os.path.join(REF, "cpu_goldbach"), str(10**9)], capture_output=True,
                         text=True, check=True).stdout
    json.dump({"source": "reference segmented_sieve + cpu_goldbach.cpp:19-21 scan rule over [4, 1e9] "
                         "(oracle/_ref/libgbref.so gbref_window_verify); cpu_goldbach 1000000000 summary",
               "start": 4, "limit": 10**9, "checked": count, "unverified": int(unver),
               "min_p_sha256": hashlib.sha256(mp.tobytes()).hexdigest(),
               "verified_bits_sha256": hashlib.sha256(bits.tobytes()).hexdigest(),
               "max_minp": int(mp.max()),
               "cpu_goldbach_checked": int(re.search(r"Even numbers checked : (\d+)", txt).group(1)),
               "cpu_goldbach_failures": int(re.search(r"Failures found\s+: (\d+)", txt).group(1)),
               "cpu_goldbach_final": [l for l in txt.splitlines() if "satisfy Goldbach" in l][0]},
              open(os.path.join(GOLD, "ref_c1_1e9.json"), "w"), indent=1)
    print("C1 fixture written to", GOLD)


if __name__ == "__main__":
    # no argument: every fixture; "c1": only the [4, 1e9] per-n fixture
    sys.exit(make_c1() if sys.argv[1:] == ["c1"] else (main() or make_c1()))
