/*
 * gb_oracle.h -- CPU ORACLE for the Goldbach range / single-n path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, in plain C, the
 * algorithm of the reference project (isaac-6/goldbach-gpu) so that the
 * GPU product can be checked bit for bit.  Only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline leg of bench.py may load it.  The
 * product library (libgoldbach_b200.so) never links or calls it.
 *
 * Every function names the reference file:line it follows.  Conventions:
 *   - even n are verified by the rule of src/cpu_goldbach.cpp:14-24: scan
 *     p = 2, 3, 4, ... <= n/2 ascending and stop at the first p with p and
 *     n-p prime.  The oracle returns that first (minimal) prime p, or 0.
 *   - odd-only bitsets use the index rule of include/prime_bitset.hpp:7-8,
 *     generalised to a window start: bit i <-> odd number q_lo + 2*i.
 *
 * Parity pins: the known-answer tables of src/test_sieve.cpp:31-40 and
 * src/test_bitset.cpp:17-74, and fixtures produced by the reference's own
 * functions compiled from its sources (oracle/build_ref.sh -> oracle/_ref).
 */
#ifndef GB_ORACLE_H
#define GB_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Exact floor(sqrt(n)) by binary search; src/goldbach.cu:637-646. */
uint64_t gbo_isqrt(uint64_t n);

/* All primes <= limit, ascending; src/segmented_sieve.cpp:13-26.
 * Writes up to cap primes into out (out may be NULL) and returns the count. */
size_t gbo_simple_sieve(uint64_t limit, uint64_t* out, size_t cap);

/* Byte primality table of [low, high]: is_prime[i] = 1 iff low+i is prime;
 * src/segmented_sieve.cpp:29-50.  is_prime must hold high-low+1 bytes. */
void gbo_segmented_sieve(uint64_t low, uint64_t high, uint8_t* is_prime);

/* Number of primes in [low, high] (pi(high) - pi(low-1)); the counting
 * helper of src/test_sieve.cpp:11-17, run in blocks over nthreads threads
 * (nthreads <= 0: all). */
uint64_t gbo_count_primes(uint64_t low, uint64_t high, int nthreads);

/* Odd-only window bitset: bit i of the uint32 word array <-> odd q_lo+2*i,
 * set iff prime (include/prime_bitset.hpp:7-8 with q_lo = 3).  q_lo must be
 * odd; nbits bits are written into ceil(nbits/32) words. */
void gbo_odd_bitset(uint64_t q_lo, uint64_t nbits, uint32_t* words);

/* Deterministic Miller-Rabin with the 12 prime bases {2..37};
 * src/goldbach.cu:333-360 (identical to single_check.cu:67-88). */
int gbo_mr12(uint64_t n);

/* Deterministic Miller-Rabin with the 7-base set {2, 325, 9375, 28178,
 * 450775, 9780504, 1795265022} (J. Sinclair), valid for all n < 2^64 when a
 * base that is 0 mod n is skipped. */
int gbo_mr7(uint64_t n);

/* Phase-2 check of src/goldbach.cu:362-373 (cpu_optimized_check), returning
 * the first prime p <= min(limit, n/2) with n-p prime, or 0.  q <= limit is
 * looked up in a prime table, larger q by gbo_mr12, as the reference does. */
uint64_t gbo_phase2_minp(uint64_t n, uint64_t limit);

/* Minimal Goldbach prime for every even n = start + 2*j, j < count, searched
 * over primes p <= min(p_limit, n/2) by the rule of src/cpu_goldbach.cpp:
 * 14-24; 0 where no such p exists.  start must be even and >= 4.  Primality
 * of q = n-p comes from a restated segmented sieve of the q-window
 * (segmented_sieve.cpp:29-50), or from gbo_mr12 for p beyond the window
 * halo.  Runs over nthreads OpenMP threads (<= 0: all).  Returns 0, or -1 on
 * bad arguments / allocation failure. */
int gbo_minp_range(uint64_t start, uint64_t count, uint64_t p_limit,
                   uint32_t* minp_out, int nthreads);

/* gbo_minp_range over many windows at once: window i covers start[i] +
 * 2j, j < count[i]; results are concatenated in window order.  Windows are
 * split into blocks and all blocks run in parallel (nthreads). */
int gbo_minp_windows(const uint64_t* start, const uint64_t* count, size_t nwin,
                     uint64_t p_limit, uint32_t* minp_out, int nthreads);

/* Minimal prime p with n-p prime for one even n >= 4 (n = 4 -> 2), primes
 * ascending from 2 up to min(p_limit, n/2), q tested by gbo_mr7; 0 if none.
 * This is the answer single-n queries must return (a minimal refinement of
 * the first-finisher partition of src/single_check.cu:95-122). */
uint64_t gbo_single_minp(uint64_t n, uint64_t p_limit);

/* Same for a batch, over nthreads threads. */
void gbo_single_minp_batch(const uint64_t* n, size_t count, uint64_t p_limit,
                           uint64_t* p_out, int nthreads);

/* Number of unordered Goldbach partitions of even n;
 * src/cpu_goldbach.cpp:29-36. */
uint64_t gbo_goldbach_count(uint64_t n);

/* Reference-style range run (src/goldbach.cu:420-485 semantics) for tests:
 * minimal p for every even n in [start, limit] with the phase bounds of the
 * reference, folded into the summary figures the verifier prints.
 *   fallbacks     = #{n : minimal p > p_small}        ("Phase 2 fallbacks")
 *   failures      = #{n : no p <= max(p_small, phase2_limit)}
 *   first_failure = smallest failing n (0 if none)
 * hist (nullable, nbins entries) counts n by the index of their minimal p in
 * the ascending prime list (2 -> 0, 3 -> 1, ...); indexes >= nbins-1 and
 * failures are not binned (failures are counted separately; indexes >=
 * nbins-1 land in the last bin). */
typedef struct gbo_range_summary {
  uint64_t checked;
  uint64_t fallbacks;
  uint64_t failures;
  uint64_t first_failure;
  uint64_t max_minp;
  uint64_t max_minp_n;
} gbo_range_summary;

int gbo_verify_range(uint64_t start, uint64_t limit, uint64_t p_small,
                     uint64_t phase2_limit, uint64_t* hist, size_t nbins,
                     gbo_range_summary* out, int nthreads);

/* Index of prime p in the ascending list of all primes (2 -> 0); p must be
 * prime and <= 2^32. */
uint64_t gbo_prime_index(uint64_t p);

#ifdef __cplusplus
}
#endif
#endif
