// search6.cuh -- word-parallel minimal-p search on the mod-6 layout.
//
// Same job as goldbach_phase1_kernel (src/goldbach.cu:288-311): the first
// prime p, ascending, with n - p prime.  The even n of
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
#include <type_traits>

#include "../gb_device.cuh"
#include "../gb_internal.h"
#include "gb/gb.h"

namespace gb {

constexpr int kSmemHistBins = 1024;  // per-CTA minimal-p histogram bins in shared memory

constexpr uint32_t kE6UBits = 15;
constexpr uint32_t kLockSteps6 = 256;  // table stride of each class sequence
// entries used: at most 255, so that an entry position fits a byte below the
// per-n output's "not from the lockstep" marker 0xFF (and the prime index
// stays below 1024, the shared histogram)
constexpr uint32_t kLockEntries6 = kLockSteps6 - 1;

// The lockstep runs in levels: level 0 takes every word of the chunk through
// the entries [0, 32); each later level takes the words still holding an
// unresolved n (a per-class survivor list written by the level before it,
// densely packed) through its own span, and the last level runs to the end
// of the table.  A word costs the steps of the task it sits in (a task ends
// when all its words are resolved), so re-packing the survivors keeps the
// slow words together: near 1e12 about 45%, 17% and 3.7% of the words are
// still alive after 28, 40 and 56 entries, and four levels took about 0.76
// of the word-steps of a single split at 40 entries (1.50 against 1.55 ms
// for 2^30 even n near 1e12; 3, 5 and 7 levels measured 1.51, 1.50 and
// 1.56 ms).  Level starts with 8 words per lane, on [4, 1e12]: (32, 44, 60)
// 557.6 ms; (28, 40, 56) 562.7; (36, 48, 64) 560.7; (32, 48, 64) 559.8;
// (24, 36, 52) 568.7; (40, 52, 68) 568.4; (20, 32, 48) 582.7.
constexpr int kLevels6 = 4;
__host__ __device__ constexpr uint32_t level6_start(int l) {
  return l == 0 ? 0u : l == 1 ? 32u : l == 2 ? 44u : 60u;
}
// the paired steps load two entries at an even position with one 8-byte load
static_assert(level6_start(1) % 2 == 0 && level6_start(2) % 2 == 0 && level6_start(3) % 2 == 0,
              "level starts must be even");
constexpr int kWT6 = 8;                      // U words per lane per warp task (6: 587.7,
                                             // 7: 601.0, 8: 562.5, 9: 570.0, 10: 585.1,
                                             // 12: 656.4 ms on [4, 1e12]; with the
                                             // paired levels and the faster sieve,
                                             // 7: 449.7, 8: 436.9, 9: 437.9 ms)
constexpr uint32_t kTaskWords6 = 32 * kWT6;  // words per warp task

// Per-CTA search context (static shared memory): the class tables' lengths
// (fixed for the kernel) and the current chunk (written by one thread
// before the sieve).
struct Ctx6 {
  uint32_t nbw;      // words of each class bitset
  uint32_t len[3];   // lockstep entries of each class (<= kLockSteps6)
  uint32_t kend[3];  // prime index after each class's last lockstep entry
  // the chunk
  uint64_t A;         // first even n
  uint64_t base_idx;  // output index of n = A
  uint64_t unit;      // segment (range) or caller's window index (windows)
  uint32_t cnt;       // even n in the chunk
  uint64_t n[3];      // n_rho: first n of each class
  uint32_t M[3];      // n of each class
  uint32_t K[3][2];   // K for q-class 1 and 5
  // the chunk's accounting (zeroed before the sieve)
  uint32_t fb, maxp;        // from the per-n tails (the histogram gives the rest)
  unsigned long long psum;  // likewise
  uint32_t next_task[kLevels6];   // the chunk's next warp task of each level
  uint32_t scnt[kLevels6][3];     // survivor words pushed by each level, per class
  uint32_t maxk;            // 1 + largest prime index in the chunk's histogram
  // the CTA's survivor lists (fixed for the kernel): set b, class ri at
  // surv + (3b + ri) surv_cap; level l writes set l & 1
  uint2* surv;
  uint32_t surv_cap;
};



__shared__ Ctx6 g_cx6;
// dynamic shared memory of range6_kernel:
//   class wheel patterns | Q1 | Q5 (nbw words each) | HIST | E0 | E2 | E4
extern __shared__ uint32_t g_smem6[];

__device__ __forceinline__ uint2* surv6_list(int b, int ri) {
  return g_cx6.surv + (size_t)(3 * b + ri) * g_cx6.surv_cap;
}
__device__ __forceinline__ uint32_t level6_end(int ri, int l) {
  const uint32_t len = g_cx6.len[ri];
  return l + 1 < kLevels6 ? min(len, level6_start(l + 1)) : len;
}

__device__ __forceinline__ uint32_t* smem6_pat() { return g_smem6; }
__device__ __forceinline__ uint32_t* smem6_q(uint32_t cls5) {
  return g_smem6 + kWheel6Words + (cls5 ? g_cx6.nbw : 0u);
}
__device__ __forceinline__ uint32_t* smem6_hist() { return g_smem6 + kWheel6Words + 2 * g_cx6.nbw; }
__device__ __forceinline__ uint32_t* smem6_etab(int ri) {
  return smem6_hist() + kSmemHistBins + ri * kLockSteps6;
}
// per-n output: the entry position of each n of the chunk resolved in the
// lockstep (0xFF: resolved elsewhere, its minimal p written directly)
__device__ __forceinline__ uint8_t* smem6_eidx() {
  return reinterpret_cast<uint8_t*>(smem6_etab(0) + 3 * kLockSteps6);
}
__host__ __device__ constexpr size_t range6_smem_words(uint32_t nbw, uint32_t eidx_bytes = 0) {
  return kWheel6Words + 2 * (size_t)nbw + kSmemHistBins + 3 * kLockSteps6 + (eidx_bytes + 3) / 4;
}

__device__ __forceinline__ uint32_t e6_u(uint32_t e) { return e & ((1u << kE6UBits) - 1); }
__device__ __forceinline__ uint32_t e6_k(uint32_t e) { return (e >> kE6UBits) & 0x3fffu; }
__device__ __forceinline__ uint32_t div6(uint32_t p) { return __umulhi(p, 715827883u); }
// p mod 6 of the entries of class ri whose q lies in class 5 (q5 = 1) or 1
__device__ __forceinline__ uint32_t e6_pmod(int ri, uint32_t q5) {
  return ri == 0 ? (q5 ? 1 : 5) : ri == 1 ? (q5 ? 3 : 1) : (q5 ? 5 : 3);
}

// Scalar finish of one n = n_rho + 6m (ri = rho / 2) after the lockstep
// entries of its class: the window primes from kend[ri] on, filtered to the
// class.  A minimal p of prime index below kSmemHistBins goes to the shared
// histogram (the flush derives the chunk's figures from it); larger ones,
// Phase-2 queueing and failures are accounted here.
template <bool MINP>
__device__ __noinline__ void tail_one6(const SearchParams& s, int ri, uint32_t m) {
  const Ctx6& cx = g_cx6;
  const uint64_t n = cx.n[ri] + 6ull * m;
  const uint64_t half = n >> 1;
  const uint64_t idx = cx.base_idx + ((n - cx.A) >> 1);
  const uint32_t K1 = cx.K[ri][0], K5 = cx.K[ri][1];
  bool past_half = false;
  for (uint32_t k = cx.kend[ri]; k < s.nsearch; ++k) {
    const uint32_t p = s.primes[k];
    if (p > half) {
      past_half = true;
      break;
    }
    const bool p1 = p - 6 * div6(p) == 1;  // p >= 5 here
    if ((ri == 1 && !p1) || (ri == 2 && p1)) continue;  // q = n - p divisible by 3
    const uint32_t q5 = ri == 0 ? p1 : ri == 2;
    const uint32_t bit = (q5 ? K5 : K1) - div6(p) + m;
    const uint32_t w = smem6_q(q5)[bit >> 5];
    if ((w >> (bit & 31)) & 1u) {
      if (MINP) s.minp[idx] = p;
      if (k < kSmemHistBins) {
        atomicAdd(&smem6_hist()[k], 1u);
        return;
      }
      const uint32_t bin = k < GB_HIST_BINS - 1 ? k : GB_HIST_BINS - 1;
      if (s.hist) atomicAdd(&s.hist[bin], 1ull);
      if (s.unit_hist) atomicAdd(&s.unit_hist[cx.unit * GB_HIST_BINS + bin], 1ull);
      if (k >= s.kfb) atomicAdd(&g_cx6.fb, 1u);
      atomicMax(&g_cx6.maxp, p);
      atomicAdd(&g_cx6.psum, (unsigned long long)p);
      return;
    }
  }
  // every window prime p <= n/2 tried: the Phase-2 queue or a failure
  const uint64_t lim = half < s.p_lim ? half : s.p_lim;
  if (past_half || s.nsearch >= s.nprimes || s.primes[s.nsearch] > lim) {
    atomicAdd(&s.ctr[kCtrFailures], 1ull);
    atomicMin(&s.ctr[kCtrFirstFail], (unsigned long long)n);
    if (s.unit_failures) atomicAdd(&s.unit_failures[cx.unit], 1u);
    if (s.vbits) atomicAnd(&s.vbits[idx >> 5], ~(1u << (idx & 31)));
    atomicAdd(&g_cx6.fb, 1u);  // a failure counts as a fallback
    return;
  }
  const unsigned long long slot = atomicAdd(&s.ctr[kCtrQueue], 1ull);
  if (slot < s.queue_cap) {
    s.queue[slot].n = n;
    s.queue[slot].idx = idx;
    s.queue[slot].unit = cx.unit;
  } else {
    s.ctr[kCtrQueueOvf] = 1ull;
  }
}

// Word indices of a lane's U words: strided from a base word (level 0) or
// listed (later levels).
struct WordsStrided {
  uint32_t base;
  __device__ __forceinline__ uint32_t operator[](int i) const { return base + 32 * i; }
};
template <int WT>
struct WordsListed {
  uint32_t w[WT];
  __device__ __forceinline__ uint32_t operator[](int i) const { return w[i]; }
};

// Window words of one class bitset for the WT U words of a lane (word
// indices W), reloaded only when the key (the word offset, with the class
// in bit 31) changes.
template <int WT>
struct Cache6 {
  uint32_t lo[WT], hi[WT];
  uint32_t key = 0xffffffffu;
  template <typename Words>
  __device__ __forceinline__ void at(const uint32_t* __restrict__ Q, uint32_t wo, uint32_t k,
                                     const Words& W) {
    if (k == key) return;
    if (k + 1 == key) {
#pragma unroll
      for (int i = 0; i < WT; ++i) {
        hi[i] = lo[i];
        lo[i] = Q[wo + W[i]];
      }
    } else {
#pragma unroll
      for (int i = 0; i < WT; ++i) {
        lo[i] = Q[wo + W[i]];
        hi[i] = Q[wo + W[i] + 1];
      }
    }
    key = k;
  }
};

// One lockstep step: the U words of a lane against one prime p.  No mask
// for p > n/2 is needed: a partition n = p + q
// with q < p would have been found at the smaller prime q, which is in the
// same class sequence, and every q < 5 reads a cleared bit.
// With per-n output (MINP) the entry position pos of every n the step
// resolves goes to the chunk's byte array at the n's index in the chunk
// (jbase + 3 m for bit m of the class); the chunk writes the minimal p out
// in n order at its end (search_chunk6).
template <bool MINP, int WT, typename Words>
__device__ __forceinline__ uint32_t step6(uint32_t (&U)[WT], const uint32_t (&lo)[WT],
                                          const uint32_t (&hi)[WT], uint32_t sh, uint32_t pos,
                                          const Words& W, uint32_t jbase) {  // pos, jbase: MINP only
  uint32_t cnt = 0;
  uint8_t* X = smem6_eidx();
#pragma unroll
  for (int i = 0; i < WT; ++i) {
    uint32_t h = U[i] & __funnelshift_r(lo[i], hi[i], sh);
    U[i] ^= h;
    cnt += __popc(h);
    if (MINP) {
      if (h) {
        const uint32_t m0 = 32 * W[i];
        while (h) {
          const int b = __ffs(h) - 1;
          h &= h - 1;
          X[jbase + 3 * (m0 + b)] = (uint8_t)pos;
        }
      }
    }
  }
  return cnt;
}

// One warp task of class ri (rho = 2 ri) at level L, through the entries
// [level6_start(L), level6_end(ri, L)).  Level 0 (LISTED false): words
// [task*kTaskWords6, +kTaskWords6) of the class, lane l owning words
// task*kTaskWords6 + l + 32i; later levels: the entries [task*kTaskWords6,
// +kTaskWords6) of the class's survivor list of level L - 1.  Every level
// but the last appends the words still unresolved to the class's list of
// level L (at most one entry per word, so it cannot overflow); the last
// level writes their bits back in place.  Lockstep over the class
// sequence with one window-word cache keyed by (offset, class).  Not
// inlined: the task gets the whole register file of the thread (the chunk
// loop around it keeps nothing live across the call), and it calls nothing.
template <bool MINP, bool LISTED>
__device__ __noinline__ void search_task6(const SearchParams& s, int ri, uint32_t task, int L) {
  const Ctx6& cx = g_cx6;
  const int lane = threadIdx.x & 31;
  const uint64_t n0 = cx.n[ri];
  uint32_t U[kWT6];
  typename std::conditional<LISTED, WordsListed<kWT6>, WordsStrided>::type W;
  if constexpr (!LISTED) {
    const uint32_t M = cx.M[ri];
    const uint32_t nuw = (M + 31) >> 5;
    W.base = task * kTaskWords6 + lane;
#pragma unroll
    for (int i = 0; i < kWT6; ++i) {
      const uint32_t w = W[i];
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
      atomicAdd(&smem6_hist()[ri == 2 ? 0 : 1], 1u);
      if (MINP) s.minp[cx.base_idx + ((n0 - cx.A) >> 1)] = ri == 2 ? 2 : 3;
    }
  } else {
    const uint2* in = surv6_list((L - 1) & 1, ri);
    const uint32_t cnt_in = cx.scnt[L - 1][ri];
#pragma unroll
    for (int i = 0; i < kWT6; ++i) {
      const uint32_t j = task * kTaskWords6 + lane + 32 * i;
      const uint2 v = j < cnt_in ? in[j] : make_uint2(0u, 0u);
      W.w[i] = v.x;
      U[i] = v.y;
    }
  }
  const uint32_t* __restrict__ E = smem6_etab(ri);
  const uint32_t* __restrict__ Q1 = smem6_q(0);
  const uint32_t* __restrict__ Q5 = smem6_q(1);
  uint32_t* HIST = smem6_hist();
  const uint32_t K1 = cx.K[ri][0], K5 = cx.K[ri][1];
  const uint32_t jbase = (uint32_t)((n0 - cx.A) >> 1);  // index of n0 in the chunk
  Cache6<kWT6> ca;
  // without per-n output the step clears bits with one operation per word
  // and counts the lane's unresolved n: resolved = live before - live after
  uint32_t live = 0;
  if (!MINP) {
#pragma unroll
    for (int i = 0; i < kWT6; ++i) live += __popc(U[i]);
  }
  const uint32_t pos0 = level6_start(L), pend = level6_end(ri, L);
  if constexpr (!MINP) {
    // Without per-n output every level steps in pairs (its span starts at
    // an even entry: 0, 32, 44 or 60): the two steps' counts, at most
    // kWT6 * 32 * 32 = 8192 each, share one warp reduction packed in the
    // halves of a word, and the early-exit vote comes every fourth pair.
    // Each step clears the q-prime bits of the lane's words and counts the
    // lane's unresolved n: resolved = live before - live after.
    auto step = [&](uint32_t e) -> uint32_t {
      const uint32_t q5 = e >> 31;
      const uint32_t off = (q5 ? K5 : K1) - e6_u(e);
      const uint32_t wo = off >> 5;
      ca.at(q5 ? Q5 : Q1, wo, wo | (q5 << 31), W);
      const uint32_t sh = off & 31;
      uint32_t now = 0;
#pragma unroll
      for (int i = 0; i < kWT6; ++i) {
        U[i] &= ~__funnelshift_r(ca.lo[i], ca.hi[i], sh);
        now += __popc(U[i]);
      }
      const uint32_t c = live - now;
      live = now;
      return c;
    };
    uint32_t pos = pos0;
    bool done = false;
#pragma unroll 1
    for (; pos + 1 < pend; pos += 2) {
      if (((pos - pos0) & 7) == 0) {
        uint32_t any = 0;
#pragma unroll
        for (int i = 0; i < kWT6; ++i) any |= U[i];
        if (!__any_sync(0xffffffffu, any)) {
          done = true;
          break;
        }
      }
      const uint2 ee = *reinterpret_cast<const uint2*>(E + pos);
      const uint32_t c0 = step(ee.x);
      const uint32_t c1 = step(ee.y);
      const uint32_t v = __reduce_add_sync(0xffffffffu, c0 | (c1 << 16));
      if (lane == 0) {
        if (v & 0xffffu) atomicAdd(&HIST[e6_k(ee.x)], v & 0xffffu);
        if (v >> 16) atomicAdd(&HIST[e6_k(ee.y)], v >> 16);
      }
    }
    if (!done && pos < pend) {  // an odd last entry
      const uint32_t e = E[pos];
      const uint32_t v = __reduce_add_sync(0xffffffffu, step(e));
      if (lane == 0 && v) atomicAdd(&HIST[e6_k(e)], v);
    }
  } else {  // per-n output: one step at a time, each recording its entry position
    uint32_t held = 0, kheld = 0;  // a step's count waiting for the next step's
    bool pending = false;          // (warp-uniform)
#pragma unroll 1
    for (uint32_t pos = pos0; pos < pend; ++pos) {
      if (((pos - pos0) & 7) == 0) {
        uint32_t any = 0;
#pragma unroll
        for (int i = 0; i < kWT6; ++i) any |= U[i];
        if (!__any_sync(0xffffffffu, any)) break;
      }
      const uint32_t e = E[pos];
      const uint32_t q5 = e >> 31;
      const uint32_t off = (q5 ? K5 : K1) - e6_u(e);
      const uint32_t wo = off >> 5;
      ca.at(q5 ? Q5 : Q1, wo, wo | (q5 << 31), W);
      const uint32_t cnt = step6<MINP, kWT6>(U, ca.lo, ca.hi, off & 31, pos, W, jbase);
      // two steps' counts (at most kWT6 * 32 * 32 = 8192 each) share one warp
      // reduction, packed in the two halves of a word
      if (pending) {
        const uint32_t v = __reduce_add_sync(0xffffffffu, held | (cnt << 16));
        if (lane == 0) {
          if (v & 0xffffu) atomicAdd(&HIST[kheld], v & 0xffffu);
          if (v >> 16) atomicAdd(&HIST[e6_k(e)], v >> 16);
        }
        pending = false;
      } else {
        held = cnt;
        kheld = e6_k(e);
        pending = true;
      }
    }
    if (pending) {
      const uint32_t v = __reduce_add_sync(0xffffffffu, held);
      if (lane == 0 && v) atomicAdd(&HIST[kheld], v);
    }
  }
  if (L + 1 < kLevels6) {
    uint2* out = surv6_list(L & 1, ri);
    uint32_t* out_cnt = &g_cx6.scnt[L][ri];
    const uint32_t lt = (1u << lane) - 1;
#pragma unroll
    for (int i = 0; i < kWT6; ++i) {
      const uint32_t alive = __ballot_sync(0xffffffffu, U[i] != 0);
      if (alive) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(out_cnt, (uint32_t)__popc(alive));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (U[i]) out[base + __popc(alive & lt)] = make_uint2(W[i], U[i]);
      }
    }
  } else {
    uint2* in = surv6_list((L - 1) & 1, ri);
    const uint32_t cnt_in = cx.scnt[L - 1][ri];
#pragma unroll
    for (int i = 0; i < kWT6; ++i) {
      const uint32_t j = task * kTaskWords6 + lane + 32 * i;
      if (j < cnt_in) in[j].y = U[i];
    }
  }
}

// Whole-chunk search by the CTA plus the flush of its accounting into the
// call's counters and the chunk's unit.  The histogram, g_cx6's fb,
// maxp, psum, maxk, scnt and next_task must be zero before the call, and
// g_cx6's survivor lists set (surv_cap >= words of a class).  Warps take
// each level's tasks from a shared counter, classes 2 and 4 first.  Ends
// with __syncthreads().  (Two task call sites, the level a run-time
// argument: one call site per level made ptxas spill in every task.)
template <bool MINP, int NT>
__device__ __forceinline__ void search_chunk6(const SearchParams& s) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
#pragma unroll 1
  for (int l = 0; l < kLevels6; ++l) {
    uint32_t b0, b2, b4;
    if (l == 0) {  // every word of the chunk
      b0 = (((g_cx6.M[0] + 31) >> 5) + kTaskWords6 - 1) / kTaskWords6;
      b2 = (((g_cx6.M[1] + 31) >> 5) + kTaskWords6 - 1) / kTaskWords6;
      b4 = (((g_cx6.M[2] + 31) >> 5) + kTaskWords6 - 1) / kTaskWords6;
    } else {  // the survivor lists of the level before
      b0 = (g_cx6.scnt[l - 1][0] + kTaskWords6 - 1) / kTaskWords6;
      b2 = (g_cx6.scnt[l - 1][1] + kTaskWords6 - 1) / kTaskWords6;
      b4 = (g_cx6.scnt[l - 1][2] + kTaskWords6 - 1) / kTaskWords6;
    }
    for (;;) {
      uint32_t task = 0;
      if (lane == 0) task = atomicAdd(&g_cx6.next_task[l], 1u);
      task = __shfl_sync(0xffffffffu, task, 0);
      if (task >= b0 + b2 + b4) break;
      const int ri = task < b2 ? 1 : task < b2 + b4 ? 2 : 0;
      const uint32_t t = ri == 1 ? task : ri == 2 ? task - b2 : task - b2 - b4;
      if (l == 0) search_task6<MINP, false>(s, ri, t, 0);
      else search_task6<MINP, true>(s, ri, t, l);
    }
    __syncthreads();
  }
  // the n still unresolved after every lockstep entry, one per thread
  for (int ri = 0; ri < 3; ++ri) {
    const uint2* L = surv6_list((kLevels6 - 2) & 1, ri);
    const uint32_t cnt = g_cx6.scnt[kLevels6 - 2][ri];
    for (uint32_t j = tid; j < cnt; j += NT) {
      const uint2 v = L[j];
      uint32_t u = v.y;
      while (u) {
        const int b = __ffs(u) - 1;
        u &= u - 1;
        tail_one6<MINP>(s, ri, 32 * v.x + b);
      }
    }
  }
  // the chunk's figures: the tails' (in g_cx6) plus fallbacks, largest and
  // summed minimal p read off the histogram
  __syncthreads();
  if (MINP) {  // the lockstep's minimal p of every n, written out in n order
    const uint8_t* X = smem6_eidx();
    const uint32_t cnt = g_cx6.cnt;
    const uint32_t amod = (uint32_t)(g_cx6.A % 6);
    uint32_t* out = s.minp + g_cx6.base_idx;
    for (uint32_t j = tid; j < cnt; j += NT) {
      const uint32_t e = X[j];
      if (e != 0xFFu) {
        const int ri = (int)(((amod + 2 * (j % 3)) % 6) >> 1);  // (A + 2j) mod 6 = 2 ri
        const uint32_t en = smem6_etab(ri)[e];
        out[j] = 6 * e6_u(en) + e6_pmod(ri, en >> 31);
      }
    }
  }
  const uint32_t* HIST = smem6_hist();
  const uint64_t unit = g_cx6.unit;
  uint32_t fbh = 0, maxk = 0;
  unsigned long long ps = 0;
  for (uint32_t k = tid; k < kSmemHistBins; k += NT) {
    const uint32_t v = HIST[k];
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
    if (fbh) atomicAdd(&g_cx6.fb, fbh);
    if (maxk) atomicMax(&g_cx6.maxk, maxk);
  }
  if (ps) atomicAdd(&g_cx6.psum, ps);
  __syncthreads();
  if (tid == 0) {
    const uint32_t hp = g_cx6.maxk ? s.primes[g_cx6.maxk - 1] : 0;
    const uint32_t maxp = hp > g_cx6.maxp ? hp : g_cx6.maxp;
    if (g_cx6.fb) {
      atomicAdd(&s.ctr[kCtrFallbacks], (unsigned long long)g_cx6.fb);
      if (s.unit_fallbacks) atomicAdd(&s.unit_fallbacks[unit], g_cx6.fb);
    }
    if (maxp) {
      atomicMax(&s.ctr[kCtrMaxP], (unsigned long long)maxp);
      if (s.unit_maxp) atomicMax(&s.unit_maxp[unit], (unsigned long long)maxp);
    }
    if (g_cx6.psum && s.unit_psum) atomicAdd(&s.unit_psum[unit], g_cx6.psum);
  }
  __syncthreads();
}

// Fills the CTA's lockstep tables (kLockSteps6 entries each at most) from
// primes[2 .. nsearch):
//   E0: every p >= 5;  E2: 3, then p = 1 (mod 6);  E4: 3, then p = 5 (mod 6);
// and sets g_cx6.len / kend.  g_cx6.nbw must be set.  One warp; ends with
// __syncthreads().
__device__ __forceinline__ void load_tables6(const SearchParams& s) {
  if (threadIdx.x < 32) {
    uint32_t* E0 = smem6_etab(0);
    uint32_t* E2 = smem6_etab(1);
    uint32_t* E4 = smem6_etab(2);
    const int lane = threadIdx.x;
    const uint32_t ns = s.nsearch;
    constexpr uint32_t L = kLockEntries6;
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
      g_cx6.len[0] = n0;
      g_cx6.len[1] = n2;
      g_cx6.len[2] = n4;
      g_cx6.kend[0] = k0end;
      g_cx6.kend[1] = k2end;
      g_cx6.kend[2] = k4end;
    }
  }
  __syncthreads();
}

}  // namespace gb
