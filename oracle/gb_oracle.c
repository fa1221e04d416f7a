/*
 * gb_oracle.c -- CPU ORACLE (test infrastructure only; see gb_oracle.h).
 *
 * Plain C restatement of the reference's CPU algorithm for the Goldbach
 * range and single-n path.  Used only as the checker by tests/, by the smoke
 * check and by the cpu_baseline leg of bench.py.  Never linked by the
 * product library.
 */
#include "gb_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

static int pick_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) return omp_get_max_threads();
  return nthreads;
#else
  (void)nthreads;
  return 1;
#endif
}

/* ---------------------------------------------------------------------- */
/* src/goldbach.cu:637-646 -- exact integer square root by bisection.      */
uint64_t gbo_isqrt(uint64_t n) {
  uint64_t lo = 1, hi = n, r = 0;
  if (n == 0) return 0;
  if (hi > (1ULL << 32)) hi = 1ULL << 32;
  while (lo <= hi) {
    uint64_t mid = lo + (hi - lo) / 2;
    if (mid <= n / mid) {
      r = mid;
      lo = mid + 1;
    } else {
      hi = mid - 1;
    }
  }
  return r;
}

/* ---------------------------------------------------------------------- */
/* src/segmented_sieve.cpp:13-26 -- byte sieve of Eratosthenes to limit.   */
size_t gbo_simple_sieve(uint64_t limit, uint64_t* out, size_t cap) {
  if (limit < 2) return 0;
  uint8_t* mark = (uint8_t*)malloc(limit + 1);
  if (!mark) return 0;
  memset(mark, 1, limit + 1);
  mark[0] = mark[1] = 0;
  for (uint64_t i = 2; i * i <= limit; i++)
    if (mark[i])
      for (uint64_t j = i * i; j <= limit; j += i) mark[j] = 0;
  size_t n = 0;
  for (uint64_t i = 2; i <= limit; i++)
    if (mark[i]) {
      if (out && n < cap) out[n] = i;
      n++;
    }
  free(mark);
  return n;
}

/* Windowed marking shared by the segmented sieve and its callers: clears
 * multiples of each base prime from max(2p, first multiple >= low)
 * (src/segmented_sieve.cpp:38-47). */
static void sieve_window(uint64_t low, uint64_t high, const uint64_t* base,
                         size_t nbase, uint8_t* is_prime) {
  uint64_t len = high - low + 1;
  memset(is_prime, 1, len);
  if (low == 0) is_prime[0] = 0;
  if (low <= 1 && high >= 1) is_prime[1 - low] = 0;
  for (size_t k = 0; k < nbase; k++) {
    uint64_t p = base[k];
    if (p > high / p) break; /* p*p > high: no composite left to clear */
    uint64_t start = (low / p) * p;
    if (start < low) start += p;
    if (start < 2 * p) start = 2 * p;
    for (uint64_t j = start; j <= high && j >= start; j += p) is_prime[j - low] = 0;
  }
}

/* ---------------------------------------------------------------------- */
/* Prime list cache (ascending, uint64) shared by the helpers below.       */
static pthread_mutex_t g_cache_mu = PTHREAD_MUTEX_INITIALIZER;
static uint64_t* g_primes = NULL;
static size_t g_nprimes = 0;
static uint64_t g_primes_limit = 0;

/* Returns a prime list covering at least [2, limit]. */
static const uint64_t* prime_cache(uint64_t limit, size_t* count) {
  pthread_mutex_lock(&g_cache_mu);
  if (g_primes_limit < limit) {
    uint64_t lim = limit < 1000000 ? 1000000 : limit;
    size_t n = gbo_simple_sieve(lim, NULL, 0);
    uint64_t* v = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
    if (v) {
      gbo_simple_sieve(lim, v, n);
      /* the previous list is deliberately kept alive: other threads may
       * still be reading it (a few MB at most over a test run) */
      g_primes = v;
      g_nprimes = n;
      g_primes_limit = lim;
    }
  }
  const uint64_t* r = g_primes;
  /* primes <= limit only */
  size_t lo = 0, hi = g_nprimes;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (g_primes[mid] <= limit) lo = mid + 1; else hi = mid;
  }
  *count = lo;
  pthread_mutex_unlock(&g_cache_mu);
  return r;
}

/* src/segmented_sieve.cpp:29-50 */
void gbo_segmented_sieve(uint64_t low, uint64_t high, uint8_t* is_prime) {
  if (high < low) return;
  size_t nbase = 0;
  const uint64_t* base = prime_cache(gbo_isqrt(high), &nbase);
  sieve_window(low, high, base, nbase, is_prime);
}

/* src/test_sieve.cpp:11-17, blocked over threads */
uint64_t gbo_count_primes(uint64_t low, uint64_t high, int nthreads) {
  if (high < low) return 0;
  size_t nbase = 0;
  const uint64_t* base = prime_cache(gbo_isqrt(high), &nbase);
  const uint64_t BLK = 1ULL << 22;
  uint64_t nblk = (high - low) / BLK + 1;
  uint64_t total = 0;
  int nt = pick_threads(nthreads);
#pragma omp parallel num_threads(nt) reduction(+ : total)
  {
    uint8_t* buf = (uint8_t*)malloc(BLK);
#pragma omp for schedule(dynamic, 1)
    for (long long b = 0; b < (long long)nblk; b++) {
      uint64_t lo = low + (uint64_t)b * BLK;
      uint64_t hi = (high - lo < BLK - 1) ? high : lo + BLK - 1;
      sieve_window(lo, hi, base, nbase, buf);
      uint64_t c = 0;
      for (uint64_t i = 0; i <= hi - lo; i++) c += buf[i];
      total += c;
    }
    free(buf);
  }
  return total;
}

/* include/prime_bitset.hpp:7-8 index rule at a window start q_lo */
void gbo_odd_bitset(uint64_t q_lo, uint64_t nbits, uint32_t* words) {
  uint64_t nwords = (nbits + 31) / 32;
  memset(words, 0, nwords * 4);
  if (nbits == 0) return;
  uint64_t hi = q_lo + 2 * (nbits - 1);
  size_t nbase = 0;
  const uint64_t* base = prime_cache(gbo_isqrt(hi), &nbase);
  uint8_t* buf = (uint8_t*)malloc(hi - q_lo + 1);
  if (!buf) return;
  sieve_window(q_lo, hi, base, nbase, buf);
  for (uint64_t i = 0; i < nbits; i++)
    if (buf[2 * i]) words[i >> 5] |= 1u << (i & 31);
  free(buf);
}

/* ---------------------------------------------------------------------- */
/* Miller-Rabin.                                                           */
static inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) {
  return (uint64_t)((u128)a * b % m);
}
static inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t m) {
  uint64_t r = 1;
  a %= m;
  while (e) {
    if (e & 1) r = mulmod(r, a, m);
    a = mulmod(a, a, m);
    e >>= 1;
  }
  return r;
}

/* one strong-probable-prime round; n odd > 2, n-1 = d*2^s */
static int sprp(uint64_t n, uint64_t a, uint64_t d, unsigned s) {
  uint64_t x = powmod(a, d, n);
  if (x == 1 || x == n - 1) return 1;
  for (unsigned i = 1; i < s; i++) {
    x = mulmod(x, x, n);
    if (x == n - 1) return 1;
  }
  return 0;
}

/* src/goldbach.cu:333-360: 12 prime bases, skip a >= n */
int gbo_mr12(uint64_t n) {
  static const uint64_t W[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return 0;
  if (n == 2 || n == 3) return 1;
  if ((n & 1) == 0) return 0;
  uint64_t d = n - 1;
  unsigned s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    s++;
  }
  for (int i = 0; i < 12; i++) {
    if (W[i] >= n) continue;
    if (!sprp(n, W[i], d, s)) return 0;
  }
  return 1;
}

/* 7-base deterministic set for n < 2^64; small factors are removed first
 * so that no base is 0 mod n for a composite n that reaches the loop. */
int gbo_mr7(uint64_t n) {
  static const uint64_t B[7] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
  static const uint32_t SMALL[11] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31};
  if (n < 2) return 0;
  for (int i = 0; i < 11; i++) {
    if (n == SMALL[i]) return 1;
    if (n % SMALL[i] == 0) return 0;
  }
  if (n < 37 * 37) return 1; /* no factor <= 31 and n < 37^2 */
  uint64_t d = n - 1;
  unsigned s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    s++;
  }
  for (int i = 0; i < 7; i++) {
    uint64_t a = B[i] % n;
    if (a == 0) continue;
    if (!sprp(n, a, d, s)) return 0;
  }
  return 1;
}

/* ---------------------------------------------------------------------- */
static int bsearch_u64(const uint64_t* v, size_t n, uint64_t x) {
  size_t lo = 0, hi = n;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (v[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo < n && v[lo] == x;
}

/* src/goldbach.cu:362-373 (cpu_optimized_check), returning the prime found */
uint64_t gbo_phase2_minp(uint64_t n, uint64_t limit) {
  size_t np = 0;
  const uint64_t* pr = prime_cache(limit, &np);
  for (size_t i = 0; i < np; i++) {
    uint64_t p = pr[i];
    if (p > n / 2) break;
    uint64_t q = n - p;
    if (q <= limit) {
      if (bsearch_u64(pr, np, q)) return p;
    } else if (gbo_mr12(q)) {
      return p;
    }
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* src/cpu_goldbach.cpp:14-24 over a block of evens, with the primality of
 * q = n - p taken from a sieved q-window [A - H, B] (the same window idea as
 * src/goldbach.cu:428-431).  Primes beyond the window halo fall back to
 * exact MR (src/goldbach.cu:362-373 semantics). */
#define ORACLE_HALO 65536ULL
#define ORACLE_BLOCK 65536ULL

/* Evens per block: 2^16, doubled while the block is under a quarter of the
 * sieving-prime count (up to 2^23), so that far from 0 (primes to 1e9
 * near 1e18) the per-prime offset of segmented_sieve.cpp:39-43 is paid once
 * per 2^23 n and not per 2^16.  Results do not depend on the block size. */
static uint64_t oracle_block(uint64_t nbase) {
  uint64_t blk = ORACLE_BLOCK;
  while (blk < (1ULL << 23) && blk < nbase / 4) blk <<= 1;
  return blk;
}

int gbo_minp_range(uint64_t start, uint64_t count, uint64_t p_limit,
                   uint32_t* minp_out, int nthreads) {
  if (count == 0) return 0;
  if (start < 4 || (start & 1) || !minp_out) return -1;
  uint64_t last = start + 2 * (count - 1);
  if (last < start) return -1;
  uint64_t H = p_limit < ORACLE_HALO ? p_limit : ORACLE_HALO;
  uint64_t need = p_limit > ORACLE_HALO ? p_limit : ORACLE_HALO;
  if (gbo_isqrt(last) > need) need = gbo_isqrt(last);
  size_t nall = 0, nbase = 0, nbig = 0, nbig_lim = 0;
  const uint64_t* big = prime_cache(need, &nall); /* one list serves all */
  prime_cache(gbo_isqrt(last), &nbase);
  prime_cache(p_limit > ORACLE_HALO ? p_limit : ORACLE_HALO, &nbig);
  prime_cache(p_limit, &nbig_lim);
  const uint64_t* base = big;
  const uint64_t BLK = oracle_block(nbase);
  uint64_t nblk = (count + BLK - 1) / BLK;
  int nt = pick_threads(nthreads);
  int err = 0;
#pragma omp parallel num_threads(nt)
  {
    uint8_t* win = (uint8_t*)malloc(2 * BLK + ORACLE_HALO + 8);
    if (!win) {
#pragma omp atomic write
      err = 1;
    }
#pragma omp for schedule(dynamic, 1)
    for (long long b = 0; b < (long long)nblk; b++) {
      if (!win) continue;
      uint64_t j0 = (uint64_t)b * BLK;
      uint64_t cnt = count - j0 < BLK ? count - j0 : BLK;
      uint64_t A = start + 2 * j0;
      uint64_t B = A + 2 * (cnt - 1);
      uint64_t wlo = A > H + 2 ? A - H : 2;
      sieve_window(wlo, B, base, nbase, win);
      for (uint64_t j = 0; j < cnt; j++) {
        uint64_t n = A + 2 * j;
        uint64_t half = n / 2;
        uint32_t found = 0;
        size_t i = 0;
        for (; i < nbig; i++) {
          uint64_t p = big[i];
          if (p > H || p > half || p > p_limit) break;
          if (win[n - p - wlo]) {
            found = (uint32_t)p;
            break;
          }
        }
        if (!found && i < nbig && big[i] > H) {
          for (; i < nbig_lim; i++) {
            uint64_t p = big[i];
            if (p > half) break;
            if (gbo_mr12(n - p)) {
              found = (uint32_t)p;
              break;
            }
          }
        }
        minp_out[j0 + j] = found;
      }
    }
    free(win);
  }
  return err ? -1 : 0;
}

int gbo_minp_windows(const uint64_t* start, const uint64_t* count, size_t nwin,
                     uint64_t p_limit, uint32_t* minp_out, int nthreads) {
  uint64_t qmax = 0, nblk = 0;
  for (size_t i = 0; i < nwin; i++) {
    if (start[i] < 4 || (start[i] & 1) || !count[i]) return -1;
    uint64_t last = start[i] + 2 * (count[i] - 1);
    if (last < start[i]) return -1;
    if (last > qmax) qmax = last;
  }
  uint64_t need = p_limit > ORACLE_HALO ? p_limit : ORACLE_HALO;
  if (gbo_isqrt(qmax) > need) need = gbo_isqrt(qmax);
  size_t tmp = 0;
  prime_cache(need, &tmp); /* build the shared tables once, before the threads */
  /* each window in blocks of gbo_minp_range's own size for its top */
  uint64_t* wblk = (uint64_t*)malloc((nwin ? nwin : 1) * sizeof(uint64_t));
  if (!wblk) return -1;
  for (size_t i = 0; i < nwin; i++) {
    size_t nb = 0;
    prime_cache(gbo_isqrt(start[i] + 2 * (count[i] - 1)), &nb);
    wblk[i] = oracle_block(nb);
    nblk += (count[i] + wblk[i] - 1) / wblk[i];
  }
  uint64_t* bw = (uint64_t*)malloc(nblk * sizeof(uint64_t) * 3);
  if (!bw) {
    free(wblk);
    return -1;
  }
  uint64_t b = 0, off = 0;
  for (size_t i = 0; i < nwin; i++) {
    for (uint64_t j0 = 0; j0 < count[i]; j0 += wblk[i], b++) {
      bw[3 * b] = start[i] + 2 * j0;
      bw[3 * b + 1] = count[i] - j0 < wblk[i] ? count[i] - j0 : wblk[i];
      bw[3 * b + 2] = off + j0;
    }
    off += count[i];
  }
  free(wblk);
  int err = 0;
  int nt = pick_threads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1) reduction(| : err)
  for (long long k = 0; k < (long long)nblk; k++)
    err |= gbo_minp_range(bw[3 * k], bw[3 * k + 1], p_limit, minp_out + bw[3 * k + 2], 1) != 0;
  free(bw);
  return err ? -1 : 0;
}

/* ---------------------------------------------------------------------- */
uint64_t gbo_single_minp(uint64_t n, uint64_t p_limit) {
  if (n < 4 || (n & 1)) return 0;
  if (n == 4) return 2;
  size_t np = 0;
  const uint64_t* pr = prime_cache(p_limit < 1000000 ? p_limit : 1000000, &np);
  size_t i = 1; /* skip p = 2: n - 2 is even and > 2 */
  for (;; i++) {
    if (i >= np) {
      if (pr[np - 1] >= p_limit) break;
      pr = prime_cache(p_limit, &np);
      if (i >= np) break;
    }
    uint64_t p = pr[i];
    if (p > n / 2 || p > p_limit) break;
    if (gbo_mr7(n - p)) return p;
  }
  return 0;
}

void gbo_single_minp_batch(const uint64_t* n, size_t count, uint64_t p_limit,
                           uint64_t* p_out, int nthreads) {
  size_t np = 0;
  prime_cache(p_limit < 1000000 ? p_limit : 1000000, &np); /* warm the cache */
  int nt = pick_threads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
  for (long long i = 0; i < (long long)count; i++) p_out[i] = gbo_single_minp(n[i], p_limit);
}

/* src/cpu_goldbach.cpp:29-36 */
uint64_t gbo_goldbach_count(uint64_t n) {
  if (n < 4) return 0;
  uint8_t* t = (uint8_t*)malloc(n + 1);
  if (!t) return 0;
  gbo_segmented_sieve(0, n, t);
  uint64_t c = 0;
  for (uint64_t p = 2; p <= n / 2; p++)
    if (t[p] && t[n - p]) c++;
  free(t);
  return c;
}

uint64_t gbo_prime_index(uint64_t p) {
  size_t np = 0;
  const uint64_t* pr = prime_cache(p, &np);
  size_t lo = 0, hi = np;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (pr[mid] < p) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* ---------------------------------------------------------------------- */
/* src/goldbach.cu:420-485 summary semantics over [start, limit]. */
int gbo_verify_range(uint64_t start, uint64_t limit, uint64_t p_small,
                     uint64_t phase2_limit, uint64_t* hist, size_t nbins,
                     gbo_range_summary* out, int nthreads) {
  if (!out || start < 4 || (start & 1) || limit < start) return -1;
  if (limit & 1) limit--;
  memset(out, 0, sizeof(*out));
  if (hist) memset(hist, 0, nbins * sizeof(uint64_t));
  uint64_t count = (limit - start) / 2 + 1;
  uint64_t p_lim = p_small > phase2_limit ? p_small : phase2_limit;
  const uint64_t PIECE = 1ULL << 24;
  uint32_t* buf = (uint32_t*)malloc(PIECE * sizeof(uint32_t));
  if (!buf) return -1;
  size_t np = 0;
  const uint64_t* pr = prime_cache(ORACLE_HALO, &np);
  /* index table for small primes (minimal p is almost always tiny) */
  uint32_t* idx = (uint32_t*)calloc(ORACLE_HALO + 1, sizeof(uint32_t));
  for (size_t i = 0; i < np && pr[i] <= ORACLE_HALO; i++) idx[pr[i]] = (uint32_t)i;
  int nt = pick_threads(nthreads);
  for (uint64_t j0 = 0; j0 < count; j0 += PIECE) {
    uint64_t cnt = count - j0 < PIECE ? count - j0 : PIECE;
    if (gbo_minp_range(start + 2 * j0, cnt, p_lim, buf, nt) != 0) {
      free(buf);
      free(idx);
      return -1;
    }
    for (uint64_t j = 0; j < cnt; j++) {
      uint64_t n = start + 2 * (j0 + j);
      uint32_t p = buf[j];
      out->checked++;
      if (p == 0 || p > p_small) out->fallbacks++;
      if (p == 0) {
        out->failures++;
        if (!out->first_failure) out->first_failure = n;
        continue;
      }
      if (p > out->max_minp) {
        out->max_minp = p;
        out->max_minp_n = n;
      }
      if (hist && nbins) {
        uint64_t k = p <= ORACLE_HALO ? idx[p] : gbo_prime_index(p);
        if (k >= nbins - 1) k = nbins - 1;
        hist[k]++;
      }
    }
  }
  free(buf);
  free(idx);
  return 0;
}
