// search.cuh -- word-parallel minimal-p search over an odd-only q-window
// held in shared memory, used by the batched windows pipeline (windows.cu);
// the range kernel searches the mod-6 layout instead (search6.cuh), and
// includes this file for its shared histogram size.
//
// Replaces goldbach_phase1_kernel (src/goldbach.cu:288-311), which runs one
// thread per even n, gathers one scattered bit per (n, p), divides n by 2
// per candidate and records no p.  Layout used here: for a chunk of even n
// = A + 2j (j < cnt) the shared-memory window holds bit i <-> odd q =
// A - H + 1 + 2i, so for an odd prime p < H
//     q = n - p  is window bit  off(p) + j,   off(p) = (H - 1 - p) / 2.
// A word of U (the unverified mask of 32 consecutive n) is matched against
// the 32 q-bits of one p with one funnel shift; the first p that hits a
// bit is that n's minimal p.
#pragma once
#include <cstdint>

#include "../gb_internal.h"
#include "gb/gb.h"

namespace gb {

constexpr int kWT = 8;                // U words per lane per warp task
constexpr int kTaskWords = 32 * kWT;  // words per warp task (8192 even n)
constexpr int kSmemHistBins = 1024;   // per-CTA histogram bins in shared memory

struct Chunk {
  uint64_t A;         // first even n
  uint64_t base_idx;  // output index of n = A (min_p / verified bits)
  uint64_t unit;      // segment (range) or window (batched windows)
  uint32_t cnt;       // even n in the chunk
};

struct LaneAcc {
  uint32_t fb;    // n with minimal p > p_small, or none
  uint32_t maxp;  // largest minimal p
  uint64_t psum;  // sum of minimal p
};

__device__ __forceinline__ void record_found_k(const SearchParams& s, uint32_t* HIST, uint32_t k,
                                               uint32_t p, uint64_t unit, LaneAcc& acc) {
  if (k < kSmemHistBins) {
    atomicAdd(&HIST[k], 1u);
  } else {
    const uint32_t bin = k < GB_HIST_BINS - 1 ? k : GB_HIST_BINS - 1;
    if (s.hist) atomicAdd(&s.hist[bin], 1ull);
    if (s.unit_hist) atomicAdd(&s.unit_hist[unit * GB_HIST_BINS + bin], 1ull);
  }
  if (k >= s.kfb) acc.fb++;
  if (p > acc.maxp) acc.maxp = p;
  acc.psum += p;
}

// Finishes one n = A + 2j already tested against the primes of index < k:
// scalar scan over the remaining window primes, then the Phase-2 queue
// (minimal p >= H) or a failure (no p <= min(n/2, p_lim)).  Returns the
// minimal p found here (0 if none) in the low 32 bits and 1 in bit 32 when
// the n counts as a Phase-2 fallback.  Arguments are passed by value so
// that the caller's accumulators stay in registers.
template <bool MINP>
__device__ __noinline__ uint64_t tail_one(const SearchParams& s, const uint32_t* __restrict__ Q,
                                          const uint16_t* __restrict__ SOFF, uint32_t* HIST,
                                          uint32_t k, uint32_t j, uint64_t A, uint64_t base_idx,
                                          uint64_t unit) {
  const uint64_t n = A + 2ull * j;
  const uint64_t half = n >> 1;
  const uint64_t idx = base_idx + j;
  const uint32_t H1 = s.halo - 1;
  uint32_t kk = k;
  for (; kk < s.nsearch; ++kk) {
    const uint32_t off = SOFF[kk];
    const uint32_t p = H1 - 2 * off;
    if (p > half) break;
    const uint32_t bit = off + j;
    if ((Q[bit >> 5] >> (bit & 31)) & 1u) {
      if (kk < kSmemHistBins) {
        atomicAdd(&HIST[kk], 1u);
      } else {
        const uint32_t bin = kk < GB_HIST_BINS - 1 ? kk : GB_HIST_BINS - 1;
        if (s.hist) atomicAdd(&s.hist[bin], 1ull);
        if (s.unit_hist) atomicAdd(&s.unit_hist[unit * GB_HIST_BINS + bin], 1ull);
      }
      if (MINP) s.minp[idx] = p;
      return (uint64_t)p | ((uint64_t)(kk >= s.kfb) << 32);
    }
  }
  const uint64_t lim = half < s.p_lim ? half : s.p_lim;
  if (kk < s.nsearch || kk >= s.nprimes || s.primes[kk] > lim) {
    atomicAdd(&s.ctr[kCtrFailures], 1ull);
    atomicMin(&s.ctr[kCtrFirstFail], (unsigned long long)n);
    if (s.unit_failures) atomicAdd(&s.unit_failures[unit], 1u);
    if (s.vbits) atomicAnd(&s.vbits[idx >> 5], ~(1u << (idx & 31)));
    return 1ull << 32;
  }
  const unsigned long long slot = atomicAdd(&s.ctr[kCtrQueue], 1ull);
  if (slot < s.queue_cap) {
    s.queue[slot].n = n;
    s.queue[slot].idx = idx;
    s.queue[slot].unit = unit;
  } else {
    s.ctr[kCtrQueueOvf] = 1ull;
  }
  return 0;  // the Phase-2 kernel accounts for it
}

// One warp task: words [task*256, task*256+256) of the chunk; lane l owns
// words task*256 + l + 32i.  Lockstep over the prime index k (p uniform
// across the warp, shift and window words uniform and bank-conflict free);
// the two window words of each U word are cached in registers and reloaded
// only when off >> 5 changes.  SMALLN: the chunk starts below 2H, so p <= n/2
// is enforced per bit.
template <bool MINP, bool SMALLN>
__device__ __forceinline__ void search_task(const SearchParams& s, const uint32_t* __restrict__ Q,
                                            const uint16_t* __restrict__ SOFF, uint32_t* HIST,
                                            uint32_t task, const Chunk& c, LaneAcc& acc) {
  const int lane = threadIdx.x & 31;
  const uint32_t nuw = (c.cnt + 31) >> 5;
  const uint32_t wbase = task * kTaskWords + lane;
  const uint32_t H1 = s.halo - 1;
  uint32_t U[kWT], lo[kWT], hi[kWT];
#pragma unroll
  for (int i = 0; i < kWT; ++i) {
    const uint32_t w = wbase + 32 * i;
    uint32_t m = 0;
    if (w < nuw) {
      const uint32_t rem = c.cnt - 32 * w;
      m = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1);
    }
    U[i] = m;
    lo[i] = hi[i] = 0;
  }
  // n = 4 is the only even n whose minimal p is 2 (n - 2 is even otherwise).
  if (c.A == 4 && task == 0 && lane == 0 && (U[0] & 1u)) {
    U[0] &= ~1u;
    record_found_k(s, HIST, 0, 2, c.unit, acc);
    if (MINP) s.minp[c.base_idx] = 2;
  }
  uint32_t cwo = 0xffffffffu;
  uint32_t k = 1;
  const uint32_t klock = s.klock;
  for (; k < klock; ++k) {
    if ((k & 7) == 1) {
      uint32_t any = 0;
#pragma unroll
      for (int i = 0; i < kWT; ++i) any |= U[i];
      if (!__any_sync(0xffffffffu, any)) break;
    }
    const uint32_t off = SOFF[k];
    const uint32_t wo = off >> 5, sh = off & 31;
    if (wo != cwo) {
      if (wo + 1 == cwo) {
#pragma unroll
        for (int i = 0; i < kWT; ++i) {
          hi[i] = lo[i];
          lo[i] = Q[wo + wbase + 32 * i];
        }
      } else {
#pragma unroll
        for (int i = 0; i < kWT; ++i) {
          lo[i] = Q[wo + wbase + 32 * i];
          hi[i] = Q[wo + wbase + 32 * i + 1];
        }
      }
      cwo = wo;
    }
    const uint32_t p = H1 - 2 * off;
    uint32_t thr = 0;
    if (SMALLN) {
      const uint64_t halfA = c.A >> 1;
      thr = p > halfA ? (uint32_t)(p - halfA) : 0u;  // bits j < thr have n < 2p
    }
    uint32_t cnt = 0;
#pragma unroll
    for (int i = 0; i < kWT; ++i) {
      uint32_t h = U[i] & __funnelshift_r(lo[i], hi[i], sh);
      if (SMALLN) {
        const uint32_t j0 = 32 * (wbase + 32 * i);
        const uint32_t vm =
            thr <= j0 ? 0xffffffffu : (thr - j0 >= 32 ? 0u : (0xffffffffu << (thr - j0)));
        h &= vm;
      }
      U[i] ^= h;
      cnt += __popc(h);
      if (MINP) {
        if (h) {
          const uint64_t ib = c.base_idx + 32ull * (wbase + 32 * i);
          while (h) {
            const int b = __ffs(h) - 1;
            h &= h - 1;
            s.minp[ib + b] = p;
          }
        }
      }
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if (lane == 0 && cnt) {
      atomicAdd(&HIST[k], cnt);
      if (k >= s.kfb) acc.fb += cnt;
      if (p > acc.maxp) acc.maxp = p;
      acc.psum += (uint64_t)cnt * p;
    }
  }
  // Tail: the n left after the lockstep primes, one at a time.  (Unrolled:
  // a runtime index into U would move the whole array to local memory.)
#pragma unroll
  for (int i = 0; i < kWT; ++i) {
    uint32_t u = U[i];
    while (u) {
      const int b = __ffs(u) - 1;
      u &= u - 1;
      const uint64_t r =
          tail_one<MINP>(s, Q, SOFF, HIST, k, 32 * (wbase + 32 * i) + b, c.A, c.base_idx, c.unit);
      const uint32_t p = (uint32_t)r;
      acc.fb += (uint32_t)(r >> 32);
      if (p > acc.maxp) acc.maxp = p;
      acc.psum += p;
    }
  }
}

// Search of a whole chunk by the CTA, followed by the flush of its
// shared-memory accounting.  Q must hold the chunk's q-window; HIST must be
// zero and s_acc (fb, maxp, psum) zeroed before the call.  Ends with a
// __syncthreads().
template <bool MINP, int NT>
__device__ __forceinline__ void search_chunk(const SearchParams& s, const uint32_t* Q,
                                             const uint16_t* SOFF, uint32_t* HIST,
                                             const Chunk& c, uint32_t* s_fb, uint32_t* s_maxp,
                                             unsigned long long* s_psum) {
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x;
  LaneAcc acc{0, 0, 0};
  const uint32_t nuw = (c.cnt + 31) >> 5;
  const uint32_t ntasks = (nuw + kTaskWords - 1) / kTaskWords;
  const bool smalln = c.A < 2ull * s.halo;
  for (uint32_t task = tid >> 5; task < ntasks; task += NW) {
    if (smalln) search_task<MINP, true>(s, Q, SOFF, HIST, task, c, acc);
    else search_task<MINP, false>(s, Q, SOFF, HIST, task, c, acc);
  }
  if (acc.fb) atomicAdd(s_fb, acc.fb);
  if (acc.maxp) atomicMax(s_maxp, acc.maxp);
  if (acc.psum) atomicAdd(s_psum, (unsigned long long)acc.psum);
  __syncthreads();
  if (s.hist || s.unit_hist) {
    for (uint32_t k = tid; k < kSmemHistBins; k += NT) {
      const uint32_t v = HIST[k];
      if (v) {
        if (s.hist) atomicAdd(&s.hist[k], (unsigned long long)v);
        if (s.unit_hist) atomicAdd(&s.unit_hist[c.unit * GB_HIST_BINS + k], (unsigned long long)v);
      }
    }
  }
  if (tid == 0) {
    if (*s_fb) {
      atomicAdd(&s.ctr[kCtrFallbacks], (unsigned long long)*s_fb);
      if (s.unit_fallbacks) atomicAdd(&s.unit_fallbacks[c.unit], *s_fb);
    }
    if (*s_maxp) {
      atomicMax(&s.ctr[kCtrMaxP], (unsigned long long)*s_maxp);
      if (s.unit_maxp) atomicMax(&s.unit_maxp[c.unit], (unsigned long long)*s_maxp);
    }
    if (*s_psum && s.unit_psum) atomicAdd(&s.unit_psum[c.unit], *s_psum);
  }
  __syncthreads();
}

// Window search offsets: SOFF[k] = (H - 1 - primes[k]) / 2 for 0 < k < nsearch.
template <int NT>
__device__ __forceinline__ void load_search_offsets(const SearchParams& s, uint16_t* SOFF) {
  for (uint32_t k = threadIdx.x; k < s.nsearch; k += NT)
    SOFF[k] = k ? (uint16_t)((s.halo - 1 - s.primes[k]) >> 1) : (uint16_t)0;
}

}  // namespace gb
