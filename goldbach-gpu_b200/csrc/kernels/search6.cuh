// search6.cuh -- word-parallel minimal-p search on the mod-6 layout.
//
// Same job as search.cuh (and as goldbach_phase1_kernel, src/goldbach.cu:
// 288-311): the first prime p, ascending, with n - p prime.  The even n of
// a chunk are split by n mod 6 = rho in {0, 2, 4}; a U word holds 32 n of
// one class, bit m <-> n = n_rho + 6m.  q = n - p must avoid 0 (mod 3), so
//   rho = 2: p = 3 (q in class 5), then primes p = 1 (mod 6) (q in class 1);
//   rho = 4: p = 3 (class 1), then primes p = 5 (mod 6) (class 5);
//   rho = 0: every prime p >= 5 (p = 1 -> class 5, p = 5 -> class 1);
// every other candidate gives q divisible by 3 and is skipped, so a class 2
// or 4 word steps through about half the primes (and class 0, whose n have
// the most partitions, finishes early).  With the class bitsets of
// sieve6.cuh (bit t <-> q = 6(G0+t)+c), q = n - p of class c sits at
//     t = m + (X - p) / 6,   X = n_rho - c - 6 G0   (an exact division),
// uniform per warp, so 32 n are tested against one p with one funnel shift.
//
// Within a class, p mod 6 is fixed by q's class (rho 0: p = 1 <-> q in class
// 5; rho 2, 4: the q-class of p = 3 and of the rest differ), so with
// u = floor(p / 6) the offset is one subtraction, t = m + K - u, with
// K = (X - (p mod 6)) / 6 per (class, q-class).  The lockstep phase reads the
// first kLockSteps6 entries of each class sequence from shared memory,
// packed as
//     u (bits 0-14) | k (bits 15-28, index in the prime table) | q-class 5 (bit 31)
// (p < 2^17 and k < 2^14 hold for every halo <= 2^17); the few n left after
// it continue one at a time over the global prime table.
#pragma once
#include <cstdint>

#include "../gb_internal.h"
#include "gb/gb.h"
#include "search.cuh"

namespace gb {

constexpr uint32_t kE6UBits = 15;
constexpr uint32_t kLockSteps6 = 96;  // lockstep entries of each class sequence

// Per-CTA search context in shared memory: the class tables' lengths (fixed
// for the kernel) and the current chunk (written by one thread before the
// search).  The generic pointers serve the per-n tail.
struct Ctx6 {
  const uint32_t* Q1;
  const uint32_t* Q5;
  uint32_t* HIST;
  uint32_t len[3];   // lockstep entries of each class (<= kLockSteps6)
  uint32_t kend[3];  // prime index after each class's last lockstep entry
  // the chunk
  uint64_t A;         // first even n
  uint64_t base_idx;  // output index of n = A
  uint64_t unit;      // segment
  uint64_t n[3];      // n_rho: first n of each class
  uint32_t M[3];      // n of each class
  uint32_t K[3][2];   // K for q-class 1 and 5
  // the chunk's accounting (zeroed before the search)
  uint32_t fb, maxp;
  unsigned long long psum;
  uint32_t next_task;  // the chunk's next warp task
  uint32_t maxk;       // 1 + largest prime index in the chunk's histogram
};

// Shared-memory pointers of a CTA's search (known to be shared memory at
// the call site, so the compiler addresses them with 32-bit offsets).
struct Smem6 {
  const uint32_t* Q1;
  const uint32_t* Q5;
  uint32_t* HIST;
  const uint32_t* E0;
  const uint32_t* E2;
  const uint32_t* E4;
};

__device__ __forceinline__ uint32_t e6_u(uint32_t e) { return e & ((1u << kE6UBits) - 1); }
__device__ __forceinline__ uint32_t e6_k(uint32_t e) { return (e >> kE6UBits) & 0x3fffu; }
__device__ __forceinline__ uint32_t div6(uint32_t p) { return __umulhi(p, 715827883u); }
// p mod 6 of the entries of class ri whose q lies in class 5 (q5 = 1) or 1
__device__ __forceinline__ uint32_t e6_pmod(int ri, uint32_t q5) {
  return ri == 0 ? (q5 ? 1 : 5) : ri == 1 ? (q5 ? 3 : 1) : (q5 ? 5 : 3);
}

// Scalar finish of one n = n_rho + 6m (ri = rho / 2) after the lockstep
// entries of its class: the window primes from cx->kend[ri] on, filtered
// to the class.  A minimal p of prime index below kSmemHistBins goes to the
// shared histogram (the flush derives the chunk's figures from it) and 0 is
// returned; otherwise the minimal p (0 if none) in the low 32 bits and 1 in
// bit 32 when the n counts as a fallback.
template <bool MINP>
__device__ __noinline__ uint64_t tail_one6(const SearchParams& s, const Ctx6* cx, int ri,
                                           uint32_t m) {
  const uint64_t n = cx->n[ri] + 6ull * m;
  const uint64_t half = n >> 1;
  const uint64_t idx = cx->base_idx + ((n - cx->A) >> 1);
  const uint32_t K1 = cx->K[ri][0], K5 = cx->K[ri][1];
  bool past_half = false;
  for (uint32_t k = cx->kend[ri]; k < s.nsearch; ++k) {
    const uint32_t p = s.primes[k];
    if (p > half) {
      past_half = true;
      break;
    }
    const bool p1 = p - 6 * div6(p) == 1;  // p >= 5 here
    if ((ri == 1 && !p1) || (ri == 2 && p1)) continue;  // q = n - p divisible by 3
    const bool q5 = ri == 0 ? p1 : ri == 2;
    const uint32_t bit = (q5 ? K5 : K1) - div6(p) + m;
    const uint32_t w = (q5 ? cx->Q5 : cx->Q1)[bit >> 5];
    if ((w >> (bit & 31)) & 1u) {
      if (MINP) s.minp[idx] = p;
      if (k < kSmemHistBins) {  // accounted from the histogram at the flush
        atomicAdd(&cx->HIST[k], 1u);
        return 0;
      }
      const uint32_t bin = k < GB_HIST_BINS - 1 ? k : GB_HIST_BINS - 1;
      if (s.hist) atomicAdd(&s.hist[bin], 1ull);
      if (s.unit_hist) atomicAdd(&s.unit_hist[cx->unit * GB_HIST_BINS + bin], 1ull);
      return (uint64_t)p | ((uint64_t)(k >= s.kfb) << 32);
    }
  }
  // every window prime p <= n/2 tried: the Phase-2 queue or a failure
  const uint64_t lim = half < s.p_lim ? half : s.p_lim;
  if (past_half || s.nsearch >= s.nprimes || s.primes[s.nsearch] > lim) {
    atomicAdd(&s.ctr[kCtrFailures], 1ull);
    atomicMin(&s.ctr[kCtrFirstFail], (unsigned long long)n);
    if (s.unit_failures) atomicAdd(&s.unit_failures[cx->unit], 1u);
    if (s.vbits) atomicAnd(&s.vbits[idx >> 5], ~(1u << (idx & 31)));
    return 1ull << 32;
  }
  const unsigned long long slot = atomicAdd(&s.ctr[kCtrQueue], 1ull);
  if (slot < s.queue_cap) {
    s.queue[slot].n = n;
    s.queue[slot].idx = idx;
    s.queue[slot].unit = cx->unit;
  } else {
    s.ctr[kCtrQueueOvf] = 1ull;
  }
  return 0;
}

// Window words of one class bitset for the WT U words of a lane, reloaded
// only when the key (the word offset, with the class in bit 31) changes.
template <int WT>
struct Cache6 {
  uint32_t lo[WT], hi[WT];
  uint32_t key = 0xffffffffu;
  __device__ __forceinline__ void at(const uint32_t* __restrict__ Q, uint32_t wo, uint32_t k,
                                     uint32_t wbase) {
    if (k == key) return;
    if (k + 1 == key) {
#pragma unroll
      for (int i = 0; i < WT; ++i) {
        hi[i] = lo[i];
        lo[i] = Q[wo + wbase + 32 * i];
      }
    } else {
#pragma unroll
      for (int i = 0; i < WT; ++i) {
        lo[i] = Q[wo + wbase + 32 * i];
        hi[i] = Q[wo + wbase + 32 * i + 1];
      }
    }
    key = k;
  }
};

// One lockstep step: the U words of a lane against one prime p.  No mask
// for p > n/2 is needed (unlike the odd-only search): a partition n = p + q
// with q < p would have been found at the smaller prime q, which is in the
// same class sequence, and every q < 5 reads a cleared bit.
template <bool MINP, int WT>
__device__ __forceinline__ uint32_t step6(const SearchParams& s, uint32_t (&U)[WT],
                                          const uint32_t (&lo)[WT], const uint32_t (&hi)[WT],
                                          uint32_t sh, uint32_t p, uint32_t wbase,
                                          uint64_t ibase) {  // p: MINP only
  uint32_t cnt = 0;
#pragma unroll
  for (int i = 0; i < WT; ++i) {
    uint32_t h = U[i] & __funnelshift_r(lo[i], hi[i], sh);
    U[i] ^= h;
    cnt += __popc(h);
    if (MINP) {
      if (h) {
        const uint64_t m0 = 32ull * (wbase + 32 * i);
        while (h) {
          const int b = __ffs(h) - 1;
          h &= h - 1;
          s.minp[ibase + 3 * (m0 + b)] = p;
        }
      }
    }
  }
  return cnt;
}

// One warp task: class ri (rho = 2 ri), words [task*kTaskWords, +kTaskWords)
// of that class; lane l owns words task*kTaskWords + l + 32i.  Lockstep over
// the class sequence with one window-word cache keyed by (offset, class).
template <bool MINP>
__device__ __forceinline__ void search_task6(const SearchParams& s, const Smem6& sm,
                                             const Ctx6* cx, int ri, uint32_t task,
                                             LaneAcc& acc) {
  const int lane = threadIdx.x & 31;
  const uint32_t M = cx->M[ri];
  const uint32_t nuw = (M + 31) >> 5;
  const uint32_t wbase = task * kTaskWords + lane;
  const uint64_t n0 = cx->n[ri];
  uint32_t U[kWT];
#pragma unroll
  for (int i = 0; i < kWT; ++i) {
    const uint32_t w = wbase + 32 * i;
    uint32_t mk = 0;
    if (w < nuw) {
      const uint32_t rem = M - 32 * w;
      mk = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1);
    }
    U[i] = mk;
  }
  // n = 4 (p = 2) and n = 6 (p = 3, q = 3): the classes hold no q = 2, 3
  if (task == 0 && lane == 0 && (U[0] & 1u) && ((ri == 2 && n0 == 4) || (ri == 0 && n0 == 6))) {
    U[0] &= ~1u;
    atomicAdd(&sm.HIST[ri == 2 ? 0 : 1], 1u);
    if (MINP) s.minp[cx->base_idx + ((n0 - cx->A) >> 1)] = ri == 2 ? 2 : 3;
  }
  // (selected, not indexed: a run-time index would put sm on the stack)
  const uint32_t* __restrict__ E = ri == 0 ? sm.E0 : ri == 1 ? sm.E2 : sm.E4;
  const uint32_t steps = cx->len[ri];
  const uint32_t K1 = cx->K[ri][0], K5 = cx->K[ri][1];
  const uint64_t ibase = cx->base_idx + ((n0 - cx->A) >> 1);
  Cache6<kWT> ca;
  for (uint32_t pos = 0; pos < steps; ++pos) {
    if ((pos & 7) == 0) {
      uint32_t any = 0;
#pragma unroll
      for (int i = 0; i < kWT; ++i) any |= U[i];
      if (!__any_sync(0xffffffffu, any)) break;
    }
    const uint32_t e = E[pos];
    const uint32_t q5 = e >> 31;
    const uint32_t off = (q5 ? K5 : K1) - e6_u(e);
    const uint32_t wo = off >> 5;
    ca.at(q5 ? sm.Q5 : sm.Q1, wo, wo | (q5 << 31), wbase);
    const uint32_t p = MINP ? 6 * e6_u(e) + e6_pmod(ri, q5) : 0;
    uint32_t cnt = step6<MINP, kWT>(s, U, ca.lo, ca.hi, off & 31, p, wbase, ibase);
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if (lane == 0 && cnt) atomicAdd(&sm.HIST[e6_k(e)], cnt);
  }
  // the n left after the lockstep entries, one at a time
#pragma unroll
  for (int i = 0; i < kWT; ++i) {
    uint32_t u = U[i];
    while (u) {
      const int b = __ffs(u) - 1;
      u &= u - 1;
      const uint64_t r = tail_one6<MINP>(s, cx, ri, 32 * (wbase + 32 * i) + b);
      const uint32_t p = (uint32_t)r;
      acc.fb += (uint32_t)(r >> 32);
      if (p > acc.maxp) acc.maxp = p;
      acc.psum += p;
    }
  }
}

// Whole-chunk search by the CTA plus the flush of its accounting (same
// contract as search_chunk in search.cuh).  sm.HIST, cx's fb, maxp and psum
// and cx->next_task must be zero before the call.  Warps take tasks from a
// shared counter, classes 2 and 4 (the longer sequences) first.  Ends with
// __syncthreads().
template <bool MINP, int NT>
__device__ __forceinline__ void search_chunk6(const SearchParams& s, const Smem6& sm, Ctx6* cx) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const uint32_t t0 = (((cx->M[0] + 31) >> 5) + kTaskWords - 1) / kTaskWords;
  const uint32_t t2 = (((cx->M[1] + 31) >> 5) + kTaskWords - 1) / kTaskWords;
  const uint32_t t4 = (((cx->M[2] + 31) >> 5) + kTaskWords - 1) / kTaskWords;
  LaneAcc acc{0, 0, 0};
  for (;;) {
    uint32_t task = 0;
    if (lane == 0) task = atomicAdd(&cx->next_task, 1u);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= t0 + t2 + t4) break;
    if (task < t2) search_task6<MINP>(s, sm, cx, 1, task, acc);
    else if (task < t2 + t4) search_task6<MINP>(s, sm, cx, 2, task - t2, acc);
    else search_task6<MINP>(s, sm, cx, 0, task - t2 - t4, acc);
  }
  // the chunk's figures: tails beyond the shared histogram (acc), plus
  // fallbacks, largest and summed minimal p read off the histogram
  __syncthreads();
  const uint64_t unit = cx->unit;
  uint32_t fbh = acc.fb, maxk = 0;
  unsigned long long ps = acc.psum;
  for (uint32_t k = tid; k < kSmemHistBins; k += NT) {
    const uint32_t v = sm.HIST[k];
    if (v) {
      if (s.hist) atomicAdd(&s.hist[k], (unsigned long long)v);
      if (s.unit_hist) atomicAdd(&s.unit_hist[unit * GB_HIST_BINS + k], (unsigned long long)v);
      if (k >= s.kfb) fbh += v;
      if (s.unit_psum) ps += (unsigned long long)v * s.primes[k];
      maxk = k + 1;
    }
  }
  fbh = __reduce_add_sync(0xffffffffu, fbh);
  maxk = __reduce_max_sync(0xffffffffu, maxk);
  if (lane == 0) {
    if (fbh) atomicAdd(&cx->fb, fbh);
    if (maxk) atomicMax(&cx->maxk, maxk);
  }
  if (acc.maxp) atomicMax(&cx->maxp, acc.maxp);
  if (ps) atomicAdd(&cx->psum, ps);
  __syncthreads();
  if (tid == 0) {
    const uint32_t hp = cx->maxk ? s.primes[cx->maxk - 1] : 0;
    const uint32_t maxp = hp > cx->maxp ? hp : cx->maxp;
    if (cx->fb) {
      atomicAdd(&s.ctr[kCtrFallbacks], (unsigned long long)cx->fb);
      if (s.unit_fallbacks) atomicAdd(&s.unit_fallbacks[unit], cx->fb);
    }
    if (maxp) {
      atomicMax(&s.ctr[kCtrMaxP], (unsigned long long)maxp);
      if (s.unit_maxp) atomicMax(&s.unit_maxp[unit], (unsigned long long)maxp);
    }
    if (cx->psum && s.unit_psum) atomicAdd(&s.unit_psum[unit], cx->psum);
  }
  __syncthreads();
}

// Fills the CTA's lockstep tables (kLockSteps6 entries each at most) from
// primes[2 .. nsearch):
//   E0: every p >= 5;  E2: 3, then p = 1 (mod 6);  E4: 3, then p = 5 (mod 6);
// and sets cx->len / cx->kend.  One warp; ends with __syncthreads().
__device__ __forceinline__ void load_tables6(const SearchParams& s, Ctx6* cx, uint32_t* E0,
                                             uint32_t* E2, uint32_t* E4) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const uint32_t ns = s.nsearch;
    constexpr uint32_t L = kLockSteps6;
    uint32_t n0 = 0, n2 = 1, n4 = 1, k0end = 2, k2end = 2, k4end = 2;
    for (uint32_t kb = 2; kb < ns && (n0 < L || n2 < L || n4 < L); kb += 32) {
      const uint32_t k = kb + lane;
      const bool in = k < ns;
      const uint32_t p = in ? s.primes[k] : 0;
      const bool p1 = p - 6 * div6(p) == 1;
      const uint32_t e = div6(p) | (k << kE6UBits);
      const uint32_t lt = (1u << lane) - 1;
      // E0: class bit = q in class 5 = (p = 1 mod 6)
      if (in && k - 2 < L) E0[k - 2] = e | ((uint32_t)p1 << 31);
      const uint32_t b2 = __ballot_sync(0xffffffffu, in && p1);
      const uint32_t b4 = __ballot_sync(0xffffffffu, in && !p1);
      const uint32_t i2 = n2 + __popc(b2 & lt), i4 = n4 + __popc(b4 & lt);
      if (in && p1 && i2 < L) E2[i2] = e;                  // q in class 1
      if (in && !p1 && i4 < L) E4[i4] = e | 0x80000000u;  // q in class 5
      // prime index after the last stored entry of each table
      const uint32_t last2 = __reduce_max_sync(0xffffffffu, in && p1 && i2 < L ? k + 1 : 0u);
      const uint32_t last4 = __reduce_max_sync(0xffffffffu, in && !p1 && i4 < L ? k + 1 : 0u);
      const uint32_t last0 = __reduce_max_sync(0xffffffffu, in && k - 2 < L ? k + 1 : 0u);
      if (last2) k2end = last2;
      if (last4) k4end = last4;
      if (last0) k0end = last0;
      n0 = min(L, n0 + __popc(__ballot_sync(0xffffffffu, in)));
      n2 = min(L, n2 + __popc(b2));
      n4 = min(L, n4 + __popc(b4));
    }
    if (lane == 0) {
      E2[0] = (1u << kE6UBits) | (1u << 31);  // rho 2: p = 3 (u = 0), q in class 5
      E4[0] = 1u << kE6UBits;                 // rho 4: p = 3, q in class 1
      cx->len[0] = n0;
      cx->len[1] = n2;
      cx->len[2] = n4;
      cx->kend[0] = k0end;
      cx->kend[1] = k2end;
      cx->kend[2] = k4end;
    }
  }
  __syncthreads();
}

}  // namespace gb
