// windows.cu -- batched verification of many independent windows of even n:
// the large-prime pass, and the expansion of narrow windows for the
// Miller-Rabin path.
//
// The reference verifies one contiguous range at a time with a host loop of
// launches per segment (src/goldbach.cu:420-485).  Windows far out (starts
// up to 1e18) need sieving primes up to 1e9, and every one of those primes
// needs its first multiple in every window: about 1e11 (prime, window)
// pairs for the 4096 seeded windows in [1e15, 1e18], of which only a few
// percent have a multiple in the window at all.  The batch is therefore
// split by prime size:
//   1. this pass: one thread per prime p above the chunk sieve's bound walks
//      the windows (sorted by their top, so only those with p^2 <= top are
//      visited) and clears p's multiples in each window's two class masks
//      (mod-6 layout, bit t <-> q = 6(g0 + t) + c, c in {1, 5}) with global
//      atomicAnd;
//   2. range6_kernel in windows mode: every (window, chunk) item sieves its
//      q-window in shared memory with the wheel and the primes up to the
//      bound, ANDs in the window's masks, and runs the levelled search;
//   3. the device Phase 2 (range.cu fallback_kernel) for minimal p beyond
//      the halo.
//
// Cost of a pair.  With r = g0 mod p, the first marks of the two classes
// are t_c = (a_c - r) mod p (a_1 = -1/6, a_5 = -5/6 mod p, from the a15
// table).  r comes from a double-precision quotient estimate: g0 < 2^62 and
// p > 2^20, so the fused multiply-add of the window's g0 (as a double) by
// 1/p, added to 1.5 * 2^52, rounds to round(g0 / p) with an error far below
// 1/2 -- floor(g0 / p) or one more -- and the low 32 bits of that double are
// round(g0 / p) mod 2^32.  r = low32(g0) - p * round(g0 / p) (mod 2^32) then
// lies in (-p, p), so 32-bit arithmetic finishes it (p < 2^31).  One 16-byte
// record per window holds g0 as a double, its low 32 bits and the mask
// length; the descriptor is read only on a hit.  The pass marks every
// multiple of p in the window, those below p^2 included (they are
// composite); only p itself must stay, and it can lie in a window only when
// the window starts below 2^32, so those windows (g0 < 2^30) take an exact
// path with the p^2 rule.
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_device.cuh"
#include "../gb_internal.h"
#include "gb/gb.h"
#include "sieve6.cuh"

namespace gb {

constexpr int kWinLargeThreads = 256;

// Exact marks of p in window w: first marks from the signed base with the
// p^2 rule (sieve6.cuh), then every p-th bit of both class masks.
__device__ __noinline__ void win_mark_exact(const WinLargeArgs& a, uint32_t w, uint32_t p, uint32_t k) {
  const WinDesc6 d = a.win[w];
  const uint32_t lbits = d.lwords * 32;
  uint32_t t1, t5;
  first_marks6(d.g0, p, __ldg(a.a15 + k), base_mod(d.g0, p, __ldg(a.magic + k)), lbits, t1, t5);
  uint32_t* L1 = a.lmask + d.lbase;
  uint32_t* L5 = L1 + d.lwords;
  for (uint64_t i = t1; i < lbits; i += p) atomicAnd(&L1[i >> 5], ~(1u << (i & 31)));
  for (uint64_t i = t5; i < lbits; i += p) atomicAnd(&L5[i >> 5], ~(1u << (i & 31)));
}

// Marks from the fast path's first marks t1, t5 (< p < 2^31) up to lbits.
__device__ __noinline__ void win_mark_from(const WinLargeArgs& a, uint32_t w, uint32_t p, uint32_t t1,
                                           uint32_t t5, uint32_t lbits) {
  const uint64_t lbase = a.win[w].lbase;
  const uint32_t lwords = a.win[w].lwords;
  uint32_t* L1 = a.lmask + lbase;
  uint32_t* L5 = L1 + lwords;
  for (uint32_t i = t1; i < lbits; i += p) atomicAnd(&L1[i >> 5], ~(1u << (i & 31)));
  for (uint32_t i = t5; i < lbits; i += p) atomicAnd(&L5[i >> 5], ~(1u << (i & 31)));
}

// First window w in [w_lo, w_hi) whose top reaches p^2 (windows sorted by
// q_top).
__device__ __forceinline__ uint32_t first_window(const WinLargeArgs& a, uint64_t pp) {
  uint32_t lo = a.w_lo, hi = a.w_hi;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a.win[mid].q_top < pp) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Per-prime constants of the fast path.
struct LargePrime {
  uint32_t p, a1, dl;  // prime, -1/6 mod p, (a5 - a1) mod p
  double inv;
};

// The class offsets: from the a15 table when many windows share the pass
// (its cost is per pair), or from p alone when few do (the pass is then paid
// per prime, and the table's 8 bytes per prime are two thirds of what it
// streams): 6 divides p - 1 or p + 1, so -1/6 = (p - 1)/6 for p = 1 (mod 6)
// and p - (p + 1)/6 for p = 5 (mod 6), and a5 - a1 = 4 a1 (mod p).
// Measured: 1.227 -> 1.073 ms for one 2^26-n window near 1e19, but
// 119.3 -> 121.7 ms for the 4096 seeded windows without the table.
constexpr uint32_t kLargeTableWindows = 64;

__device__ __forceinline__ LargePrime large_prime(const WinLargeArgs& a, uint32_t k) {
  LargePrime q;
  q.p = __ldg(a.primes + k);
  if (a.w_hi - a.w_lo >= kLargeTableWindows) {
    const uint2 ac = __ldg(a.a15 + k);
    q.a1 = ac.x;
    q.dl = ac.y >= ac.x ? ac.y - ac.x : ac.y + q.p - ac.x;
  } else {
    const uint32_t q6 = __umulhi(q.p, 0xAAAAAAABu) >> 2;  // floor(p / 6)
    q.a1 = q.p - 6 * q6 == 1 ? q6 : q.p - q6 - 1;
    uint32_t d = q.a1 + q.a1;  // 4 a1 mod p in two doublings (p < 2^31)
    d = min(d, d - q.p);
    d = d + d;
    q.dl = min(d, d - q.p);
  }
  // 1/p to a relative error near 2^-47: the single-precision reciprocal
  // (2^-23 with the rounding of p to a float) and one Newton step in double
  // precision.  The quotient estimate needs |g0/p| * error < 1/4 with
  // g0/p < 2^42, i.e. 2^-44; a correctly rounded division costs several
  // times more and is paid once per prime, which dominates when few
  // windows share the pass.
  const double pd = (double)q.p;
  const double r0 = (double)__frcp_rn((float)q.p);
  q.inv = fma(r0, fma(-pd, r0, 1.0), r0);
  return q;
}

// One (prime, window) pair on the fast path (p < 2^31): the first marks of
// both classes from the quotient estimate, and the marking when one falls
// inside the mask (or the exact path for a window flagged for it).
__device__ __forceinline__ void large_pair(const WinLargeArgs& a, const WinLarge& v, uint32_t w,
                                           const LargePrime& q, uint32_t k) {
  const double kRound = 6755399441055744.0;  // 1.5 * 2^52
  const uint32_t qe = (uint32_t)__double_as_longlong(fma(v.gd, q.inv, kRound));
  uint32_t r = v.gl - qe * q.p;  // g0 - p round(g0 / p), in (-p, p)
  r = min(r, r + q.p);           // [0, p)
  uint32_t t1 = q.a1 - r;
  t1 = min(t1, t1 + q.p);
  uint32_t t5 = t1 + q.dl;
  t5 = min(t5, t5 - q.p);
  if (min(t1, t5) < v.lbits) {  // a mark in the window, or the exact path
    if (v.lbits == 0xffffffffu) win_mark_exact(a, w, q.p, k);
    else win_mark_from(a, w, q.p, t1, t5, v.lbits);
  }
}

// One thread per prime, grid-stride over the primes.  (Four consecutive
// primes per thread sharing each window record measured slower: 146.5
// against 95 ms on the 4096 seeded windows, with 21.7 of 32 lanes active.)
__global__ void __launch_bounds__(kWinLargeThreads) win_large_kernel(const __grid_constant__ WinLargeArgs a) {
  const uint32_t stride = gridDim.x * kWinLargeThreads;
  for (uint32_t k = a.k0 + blockIdx.x * kWinLargeThreads + threadIdx.x; k < a.k1; k += stride) {
    const uint32_t p = __ldg(a.primes + k);
    const uint32_t lo = first_window(a, (uint64_t)p * p);
    if (p >= 0x80000000u) {  // windows near 2^64 only: every pair exact
      for (uint32_t w = lo; w < a.w_hi; ++w) win_mark_exact(a, w, p, k);
      continue;
    }
    const LargePrime q = large_prime(a, k);
#pragma unroll 4
    for (uint32_t w = lo; w < a.w_hi; ++w) large_pair(a, a.wl[w], w, q, k);
  }
}

cudaError_t launch_win_large(const WinLargeArgs& a, int grid, cudaStream_t s) {
  if (a.k1 <= a.k0 || a.w_hi <= a.w_lo || grid < 1) return cudaSuccess;
  win_large_kernel<<<grid, kWinLargeThreads, 0, s>>>(a);
  return cudaGetLastError();
}

// (prime, window) pairs the large-prime pass visits: for each window the
// primes in [k0, pi(isqrt(q_top))), summed into *pairs.
__global__ void win_pairs_kernel(const WinDesc6* __restrict__ win, uint32_t nwin,
                                 const uint32_t* __restrict__ primes, uint64_t nprimes, uint32_t k0,
                                 unsigned long long* pairs) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < nwin) {
    const uint64_t q = win[w].q_top;
    uint64_t r = (uint64_t)sqrt((double)q);
    while (r > 0 && (r > 0xffffffffull || r * r > q)) --r;
    while (r < 0xffffffffull && (r + 1) * (r + 1) <= q) ++r;
    uint64_t lo = 0, hi = nprimes;  // first index with primes[i] > r
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (primes[mid] <= r) lo = mid + 1;
      else hi = mid;
    }
    if (lo > k0) atomicAdd(pairs, (unsigned long long)(lo - k0));
  }
}

cudaError_t launch_win_pairs(const WinDesc6* win, uint32_t nwin, const uint32_t* primes, uint64_t nprimes,
                             uint32_t k0, unsigned long long* pairs, cudaStream_t s) {
  if (!nwin) return cudaSuccess;
  win_pairs_kernel<<<(nwin + 255) / 256, 256, 0, s>>>(win, nwin, primes, nprimes, k0, pairs);
  return cudaGetLastError();
}

// Narrow windows on the Miller-Rabin path: the n of each window, laid out
// window after window at off[i], for the single-n kernel.
__global__ void win_expand_kernel(const gb_window* __restrict__ w, const uint64_t* __restrict__ off,
                                  uint32_t nw, uint64_t* __restrict__ n) {
  for (uint32_t i = blockIdx.x; i < nw; i += gridDim.x) {
    const uint64_t s = w[i].start, c = w[i].count, o = off[i];
    for (uint64_t j = threadIdx.x; j < c; j += blockDim.x) n[o + j] = s + 2 * j;
  }
}

cudaError_t launch_win_expand(const gb_window* w, const uint64_t* off, uint32_t nw, uint64_t* n,
                              cudaStream_t s) {
  if (!nw) return cudaSuccess;
  win_expand_kernel<<<nw < 4096 ? nw : 4096, 256, 0, s>>>(w, off, nw, n);
  return cudaGetLastError();
}

}  // namespace gb
