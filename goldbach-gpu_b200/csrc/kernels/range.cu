// range.cu -- fused segment sieve + minimal-p partition search (sm_100a),
// and the device Phase 2.
//
// One persistent launch replaces the reference's per-segment sequence
// (src/goldbach.cu:420-485): tiled_sieve_segment_kernel (:198-259) writing
// a segment bitset to HBM, goldbach_phase1_kernel (:288-311), the
// count_unverified_kernel (:184-195) with a global atomic per n, a D2H copy
// and a stream sync per segment, then the host Phase 2 (:362-373).
//
// Each CTA takes work items (chunks of NE consecutive even n) from a global
// counter.  For a chunk it sieves the q-window in the mod-6 layout (the two
// class bitsets of the odd q not divisible by 3, sieve6.cuh) into shared
// memory and searches it there (search6.cuh): the bitset never touches
// HBM.  n whose minimal p is beyond the window go to a device queue that
// fallback_kernel serves.
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_device.cuh"
#include "../gb_internal.h"
#include "gb/gb.h"
#include "search6.cuh"
#include "sieve6.cuh"

namespace gb {

// ---------------------------------------------------------------------------
// The fused kernel: the q-window is the two class bitsets Q1 / Q5 (no
// multiple of 3 stored), and the n of a chunk are searched by class n mod 6.

// Block shapes of range6_kernel: NT threads per CTA, launch-bounded to
// 1024 / NT CTAs per SM so that every shape gets 64 registers a thread.  The
// default is 512 x 2 (two 2^20-n chunks of 101 KB in an SM's shared memory);
// 256 x 4 fits chunks of 2^19 n or fewer, 1024 x 1 one chunk per SM.  The
// autotuner picks among them per range class.
constexpr int kRange6DefaultThreads = 512;

// floor((A - H - 1) / 6) for A possibly below H
__device__ __forceinline__ int64_t window_g0(uint64_t A, uint32_t H) {
  if (A >= (uint64_t)H + 1) return (int64_t)((A - H - 1) / 6);
  return -(int64_t)(((uint64_t)H + 1 - A + 5) / 6);
}

// last window w with off[w] <= item (off: nwin + 1 ascending prefix sums)
__device__ __forceinline__ uint32_t find_item_window(const uint64_t* off, uint32_t nwin, uint64_t item) {
  uint32_t lo = 0, hi = nwin;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

// WIN: windows mode (a.win set) -- a template parameter so that the range
// instantiation carries none of its state through the inlined sieve.
template <bool MINP, int NT, bool WIN>
__global__ void __launch_bounds__(NT, 1024 / NT) range6_kernel(const __grid_constant__ RangeArgs a) {
  const SearchParams& s = a.s;
  __shared__ unsigned long long s_item;
  // windows mode: the item's window and chunk, decoded by thread 0
  __shared__ uint64_t s_wA, s_wbase, s_wunit, s_wlbase;
  __shared__ int64_t s_wg0;
  __shared__ uint32_t s_wcnt, s_wlwords;
  const int tid = threadIdx.x;
  Ctx6& cx = g_cx6;
  uint32_t* pat6 = smem6_pat();
  for (uint32_t i = tid; i < kWheel6Words; i += NT) pat6[i] = a.wheel6[i];
  if (tid == 0) {
    cx.nbw = a.nbw;
    cx.surv = a.surv + (size_t)blockIdx.x * 6 * a.surv_cap;
    cx.surv_cap = a.surv_cap;
  }
  __syncthreads();
  load_tables6(s);
  uint32_t* Q1 = smem6_q(0);
  uint32_t* Q5 = smem6_q(1);
  uint32_t* HIST = smem6_hist();

  for (;;) {
    if (tid == 0) {
      s_item = atomicAdd(&s.ctr[kCtrWork], 1ull);
      if (WIN && s_item < a.total_items) {
        const uint32_t w = find_item_window(a.chunk_off, a.nwin, s_item);
        const WinDesc6 d = a.win[w];
        const uint64_t j0 = (s_item - a.chunk_off[w]) * a.chunk_evens;
        s_wA = d.start + 2 * j0;
        s_wcnt = (uint32_t)(d.count - j0 < a.chunk_evens ? d.count - j0 : a.chunk_evens);
        s_wbase = d.out_off + j0;
        s_wunit = d.orig;
        s_wg0 = d.g0;
        s_wlbase = d.lbase;
        s_wlwords = d.lwords;
      }
      cx.fb = 0;
      cx.maxp = 0;
      cx.psum = 0;
      for (int l = 0; l < kLevels6; ++l) {
        cx.next_task[l] = 0;
        cx.scnt[l][0] = cx.scnt[l][1] = cx.scnt[l][2] = 0;
      }
      cx.maxk = 0;
    }
    for (uint32_t i = tid; i < kSmemHistBins; i += NT) HIST[i] = 0;
    if (MINP) {  // no n resolved yet
      uint32_t* X = reinterpret_cast<uint32_t*>(smem6_eidx());
      for (uint32_t i = tid; i < a.chunk_evens / 4; i += NT) X[i] = 0xffffffffu;
    }
    __syncthreads();
    const unsigned long long item = s_item;
    if (item >= a.total_items) break;
    uint64_t A, base_idx, unit;
    uint32_t cnt;
    if (WIN) {
      A = s_wA;
      cnt = s_wcnt;
      base_idx = s_wbase;
      unit = s_wunit;
    } else {
      const uint64_t ls = item / a.chunks_per_seg;
      const uint64_t ci = item - ls * a.chunks_per_seg;
      const uint64_t seg = a.shard_index + ls * a.shard_count;
      const uint64_t seg_first = seg * a.seg_size;
      const uint64_t seg_rem = a.total_count - seg_first;
      const uint64_t seg_cnt = seg_rem < a.seg_size ? seg_rem : a.seg_size;
      const uint64_t j0 = ci * a.chunk_evens;
      if (j0 >= seg_cnt) {
        __syncthreads();
        continue;
      }
      A = a.start + 2 * (seg_first + j0);
      cnt = (uint32_t)(seg_cnt - j0 < a.chunk_evens ? seg_cnt - j0 : a.chunk_evens);
      base_idx = seg_first + j0;
      unit = seg;
    }
    const int64_t G0 = window_g0(A, s.halo);
    if (tid == 0) {
      cx.A = A;
      cx.base_idx = base_idx;
      cx.unit = unit;
      cx.cnt = cnt;
      const uint64_t last = A + 2ull * (cnt - 1);
      const uint32_t amod = (uint32_t)(A % 6);
      // A - 6 G0 is in [H + 1, H + 7), so every X fits 32 bits
      const uint32_t a6 = (uint32_t)((int64_t)A - 6 * G0);
#pragma unroll
      for (int ri = 0; ri < 3; ++ri) {
        const uint32_t d = (uint32_t)((2 * ri - (int)amod + 6) % 6);
        cx.n[ri] = A + d;  // (may pass 2^64 only for a class with no n: M = 0)
        cx.M[ri] = last - A >= d ? (uint32_t)((last - A - d) / 6 + 1) : 0u;
        // K = (X - (p mod 6)) / 6 with X = n_rho - c - 6 G0 (exact)
        cx.K[ri][0] = (a6 + d - 1 - e6_pmod(ri, 0)) / 6;
        cx.K[ri][1] = (a6 + d - 5 - e6_pmod(ri, 1)) / 6;
      }
    }
    const uint32_t nbits = s.halo / 6 + cnt / 3 + 96;
    // words the search can read for a real n (a word past them only meets
    // an empty unverified mask): a short chunk sieves no more than these
    const uint32_t nwords = min(a.nbw, (nbits + 31) / 32 + 2);
    const uint32_t* L1 = nullptr;
    const uint32_t* L5 = nullptr;
    uint32_t lsh = 0;
    if (WIN) {  // the window's large-prime mask from this chunk's base on
      const uint64_t d = (uint64_t)(G0 - s_wg0);
      L1 = a.lmask + s_wlbase + (d >> 5);
      L5 = L1 + s_wlwords;
      lsh = (uint32_t)(d & 31);
    }
    // q <= n - 3: the chunk's last n bounds the sieve (A + 2 cnt could pass 2^64)
    sieve_window6<NT>(Q1, Q5, nwords, nbits, G0, A + 2ull * (cnt - 1), pat6, s.primes,
                                 a.magic, a.a15, a.nsieve, a.kcoop, L1, L5, lsh);
    search_chunk6<MINP, NT>(s);
  }
}

// ---------------------------------------------------------------------------
// Device Phase 2 (replaces cpu_optimized_check, src/goldbach.cu:362-373, run
// on the host for every unverified n).  One warp per queued n; lanes take 32
// consecutive candidate primes beyond the window, test q = n - p with the
// deterministic Montgomery Miller-Rabin, and the lowest passing lane is the
// minimal p.
constexpr int kFallbackThreads = 256;

__global__ void __launch_bounds__(kFallbackThreads) fallback_kernel(const __grid_constant__ SearchParams s) {
  const int lane = threadIdx.x & 31;
  const unsigned long long queued = s.ctr[kCtrQueue];
  const uint64_t entries = queued < s.queue_cap ? queued : s.queue_cap;
  const uint64_t gw = (uint64_t)blockIdx.x * (kFallbackThreads / 32) + (threadIdx.x >> 5);
  const uint64_t nw = (uint64_t)gridDim.x * (kFallbackThreads / 32);
  for (uint64_t e = gw; e < entries; e += nw) {
    const QEntry q = s.queue[e];
    const uint64_t n = q.n;
    const uint64_t half = n >> 1;
    const uint64_t lim = half < s.p_lim ? half : s.p_lim;
    uint32_t found = 0;
    uint64_t kf = 0;
    for (uint64_t k = s.nsearch;; k += 32) {
      const uint64_t kk = k + lane;
      const uint32_t p = kk < s.nprimes ? s.primes[kk] : 0xffffffffu;
      const bool valid = kk < s.nprimes && p <= lim;
      const bool ok = valid && is_prime_u64(n - p);
      const uint32_t b = __ballot_sync(0xffffffffu, ok);
      if (b) {
        const int l = __ffs(b) - 1;
        found = __shfl_sync(0xffffffffu, p, l);
        kf = k + l;
        break;
      }
      if (__ballot_sync(0xffffffffu, valid) != 0xffffffffu) break;
    }
    if (lane == 0) {
      const bool fb = (found == 0) || (found > s.p_small);
      if (fb) {
        atomicAdd(&s.ctr[kCtrFallbacks], 1ull);
        if (s.unit_fallbacks) atomicAdd(&s.unit_fallbacks[q.unit], 1u);
      }
      if (found) {
        const uint32_t bin = kf < GB_HIST_BINS - 1 ? (uint32_t)kf : GB_HIST_BINS - 1;
        if (s.hist) atomicAdd(&s.hist[bin], 1ull);
        if (s.unit_hist) atomicAdd(&s.unit_hist[q.unit * GB_HIST_BINS + bin], 1ull);
        atomicMax(&s.ctr[kCtrMaxP], (unsigned long long)found);
        if (s.unit_maxp) atomicMax(&s.unit_maxp[q.unit], (unsigned long long)found);
        if (s.unit_psum) atomicAdd(&s.unit_psum[q.unit], (unsigned long long)found);
        if (s.minp) s.minp[q.idx] = found;
      } else {
        atomicAdd(&s.ctr[kCtrFailures], 1ull);
        atomicMin(&s.ctr[kCtrFirstFail], (unsigned long long)n);
        if (s.unit_failures) atomicAdd(&s.unit_failures[q.unit], 1u);
        if (s.vbits) atomicAnd(&s.vbits[q.idx >> 5], ~(1u << (q.idx & 31)));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Words of each class bitset: the largest q-window word offset a search
// step reads (H/6 + 96 bits), plus the U words of a class rounded up to
// whole warp tasks (the last task reads past the chunk's words), plus the
// second word of each funnel shift and a little slack.
uint32_t range6_words(uint32_t halo, uint32_t chunk_evens) {
  const uint32_t off_words = (halo / 6 + 96) / 32 + 1;
  const uint32_t class_words = (chunk_evens / 3 + 2 + 31) / 32;
  const uint32_t tasks = (class_words + kTaskWords6 - 1) / kTaskWords6;
  return off_words + tasks * kTaskWords6 + 4;
}

size_t range_smem_bytes(const RangeArgs& a) {
  return range6_smem_words(a.nbw, a.s.minp ? a.chunk_evens : 0) * sizeof(uint32_t);
}

template <typename K>
static int occupancy(K kernel, size_t smem, int threads) {
  int nb = 0;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem);
  return nb;
}

// The instantiation for a's block shape (threads 256, 512 or 1024) and
// outputs, handed to f(kernel, threads).
template <typename F>
static cudaError_t with_range_kernel(const RangeArgs& a, F f) {
  const uint32_t nt = a.threads ? a.threads : kRange6DefaultThreads;
  const int v = (a.s.minp != nullptr ? 1 : 0) + (a.win != nullptr ? 2 : 0);
#define GB_RANGE_SHAPE(T)                                 \
  case T:                                                 \
    switch (v) {                                          \
      case 0: return f(range6_kernel<false, T, false>, T); \
      case 1: return f(range6_kernel<true, T, false>, T);  \
      case 2: return f(range6_kernel<false, T, true>, T);  \
      default: return f(range6_kernel<true, T, true>, T);  \
    }
  switch (nt) {
    GB_RANGE_SHAPE(256)
    GB_RANGE_SHAPE(512)
    GB_RANGE_SHAPE(1024)
    default: return cudaErrorInvalidValue;
  }
#undef GB_RANGE_SHAPE
}

int range_max_blocks_per_sm(const RangeArgs& a) {
  const size_t smem = range_smem_bytes(a);
  int nb = 0;
  with_range_kernel(a, [&](auto kernel, int threads) {
    nb = occupancy(kernel, smem, threads);
    return cudaSuccess;
  });
  return nb;
}

template <typename K>
static cudaError_t launch_one(K kernel, const RangeArgs& a, int grid, size_t smem, cudaStream_t st,
                              int threads) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kernel<<<grid, threads, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_range(const RangeArgs& a, int grid, cudaStream_t st) {
  const size_t smem = range_smem_bytes(a);
  return with_range_kernel(a, [&](auto kernel, int threads) {
    return launch_one(kernel, a, grid, smem, st, threads);
  });
}

cudaError_t launch_fallback(const SearchParams& s, int grid, cudaStream_t st) {
  fallback_kernel<<<grid, kFallbackThreads, 0, st>>>(s);
  return cudaGetLastError();
}

}  // namespace gb
