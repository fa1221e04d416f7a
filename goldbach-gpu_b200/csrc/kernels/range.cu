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
// counter.  For chunk [A, A+2NE) it sieves the odd q-window [A-H+1,
// A+2NE+64) into shared memory (sieve_window.cuh) and searches it there
// (search.cuh): the bitset never touches HBM.  n whose minimal p is >= H
// (none below 1e12 for H >= 2^12) go to a device queue that fallback_kernel
// serves.
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_device.cuh"
#include "../gb_internal.h"
#include "gb/gb.h"
#include "search.cuh"
#include "sieve_window.cuh"

namespace gb {

constexpr int kRangeThreads = 512;

template <bool MINP>
__global__ void __launch_bounds__(kRangeThreads, 2) range_kernel(const __grid_constant__ RangeArgs a) {
  extern __shared__ uint32_t smem[];
  uint32_t* pat = smem;
  uint32_t* Q = pat + kWheelWords;
  uint32_t* HIST = Q + a.nbw;
  uint16_t* SOFF = reinterpret_cast<uint16_t*>(HIST + kSmemHistBins);
  __shared__ unsigned long long s_item, s_psum;
  __shared__ uint32_t s_fb, s_maxp;
  const int tid = threadIdx.x;
  const SearchParams& s = a.s;

  for (uint32_t i = tid; i < kWheelWords; i += kRangeThreads) pat[i] = a.wheel[i];
  load_search_offsets<kRangeThreads>(s, SOFF);

  for (;;) {
    if (tid == 0) {
      s_item = atomicAdd(&s.ctr[kCtrWork], 1ull);
      s_fb = 0;
      s_maxp = 0;
      s_psum = 0;
    }
    for (uint32_t i = tid; i < kSmemHistBins; i += kRangeThreads) HIST[i] = 0;
    __syncthreads();
    const unsigned long long item = s_item;
    if (item >= a.total_items) break;
    const uint64_t ls = item / a.chunks_per_seg;
    const uint64_t ci = item - ls * a.chunks_per_seg;
    const uint64_t seg = a.shard_index + ls * a.shard_count;
    const uint64_t seg_first = seg * a.seg_size;
    const uint64_t seg_rem = a.total_count - seg_first;
    const uint64_t seg_cnt = seg_rem < a.seg_size ? seg_rem : a.seg_size;
    const uint64_t j0 = ci * a.chunk_evens;
    if (j0 >= seg_cnt) {  // past the end of a short last segment
      __syncthreads();
      continue;
    }
    Chunk c;
    c.base_idx = seg_first + j0;
    c.A = a.start + 2 * c.base_idx;
    c.unit = seg;
    c.cnt = (uint32_t)(seg_cnt - j0 < a.chunk_evens ? seg_cnt - j0 : a.chunk_evens);

    // window bit i <-> odd index g0 + i, g0 = (A - H) / 2 (negative near 0)
    const int64_t g0 = (int64_t)(c.A >> 1) - (int64_t)(s.halo >> 1);
    const uint32_t nbits = s.halo / 2 + c.cnt + 32;
    const uint64_t q_top = c.A + 2ull * c.cnt;
    sieve_window<kRangeThreads>(Q, a.nbw, nbits, g0, q_top, pat, s.primes, a.magic, a.nsieve,
                                a.kcoop);
    search_chunk<MINP, kRangeThreads>(s, Q, SOFF, HIST, c, &s_fb, &s_maxp, &s_psum);
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
size_t range_smem_bytes(const RangeArgs& a) {
  return (size_t)(kWheelWords + a.nbw + kSmemHistBins) * sizeof(uint32_t) +
         (size_t)((a.s.nsearch + 1) & ~1u) * sizeof(uint16_t);
}

template <bool MINP>
static int occupancy(size_t smem) {
  int nb = 0;
  cudaFuncSetAttribute(range_kernel<MINP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, range_kernel<MINP>, kRangeThreads, smem);
  return nb;
}

int range_max_blocks_per_sm(const RangeArgs& a) {
  const size_t smem = range_smem_bytes(a);
  return a.s.minp ? occupancy<true>(smem) : occupancy<false>(smem);
}

cudaError_t launch_range(const RangeArgs& a, int grid, cudaStream_t st) {
  const size_t smem = range_smem_bytes(a);
  if (a.s.minp) {
    cudaError_t e = cudaFuncSetAttribute(range_kernel<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    range_kernel<true><<<grid, kRangeThreads, smem, st>>>(a);
  } else {
    cudaError_t e = cudaFuncSetAttribute(range_kernel<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    range_kernel<false><<<grid, kRangeThreads, smem, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_fallback(const SearchParams& s, int grid, cudaStream_t st) {
  fallback_kernel<<<grid, kFallbackThreads, 0, st>>>(s);
  return cudaGetLastError();
}

}  // namespace gb
