// windows.cu -- batched verification of many independent windows of even n.
//
// The reference verifies one contiguous range at a time with a host loop of
// launches per segment (src/goldbach.cu:420-485).  Windows far out (starts
// up to 1e18) need sieving primes up to 1e9, where recomputing every prime's
// first multiple per CTA chunk (as the fused range kernel does for primes up
// to 1e6) would cost ~5e7 divisions per chunk.  The batch is therefore
// staged through HBM:
//   A. tile sieve: every window's odd q-bitset [start-H+1, end] is sieved
//      tile by tile in shared memory with the wheel and the primes < 2^17,
//      and stored with coalesced 128-bit stores;
//   B. large primes: one thread per prime p in [2^17, sqrt(max q)] walks the
//      windows (sorted by their top q, so only those with p^2 <= top are
//      visited), computes the first multiple from a double-precision
//      quotient estimate (one remainder per window: the stage's whole cost)
//      and clears its multiples with global atomicAnd (at most a few per
//      window);
//   C. search: every chunk of NE even n loads its q-window from HBM into
//      shared memory and runs the same word-parallel search as the range
//      kernel (search.cuh);
//   D. the device Phase 2 (range.cu fallback_kernel) for minimal p >= H.
// In the persistent mode each stage is ONE launch over the whole batch, its
// CTAs pulling items from a device work counter.  In the plain mode the same
// four stages run window by window (the per-window launch pipeline), for
// comparison.
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_device.cuh"
#include "../gb_internal.h"
#include "gb/gb.h"
#include "search.cuh"
#include "sieve_window.cuh"

namespace gb {

constexpr int kWinThreads = 512;

__device__ __forceinline__ uint32_t find_window(const uint64_t* off, uint32_t nwin, uint64_t item) {
  uint32_t lo = 0, hi = nwin;  // last w with off[w] <= item
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per-window sieving bound: nsieve = #primes <= isqrt(q_top) (binary search
// in the resident table), so the host never looks these up one by one.
__global__ void win_nsieve_kernel(WinDesc* win, uint32_t nwin, const uint32_t* primes,
                                  uint64_t nprimes) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwin) return;
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
  win[w].nsieve = (uint32_t)(lo > kWheelPrimeCount + 1 ? lo : kWheelPrimeCount + 1);
}

cudaError_t launch_win_nsieve(WinDesc* win, uint32_t nwin, const uint32_t* primes, uint64_t nprimes,
                              cudaStream_t s) {
  if (!nwin) return cudaSuccess;
  win_nsieve_kernel<<<(nwin + 255) / 256, 256, 0, s>>>(win, nwin, primes, nprimes);
  return cudaGetLastError();
}

// A. tile sieve ---------------------------------------------------------------
__global__ void __launch_bounds__(kWinThreads) win_tile_kernel(const __grid_constant__ WindowsArgs a,
                                                               uint32_t w_only) {
  extern __shared__ uint32_t smem[];
  uint32_t* pat = smem;
  uint32_t* Q = smem + kWheelWords;
  __shared__ unsigned long long s_item;
  for (uint32_t i = threadIdx.x; i < kWheelWords; i += kWinThreads) pat[i] = a.wheel[i];
  const uint64_t lo_item = w_only < a.nwin ? a.tile_off[w_only] : 0;
  const uint64_t hi_item = w_only < a.nwin ? a.tile_off[w_only + 1] : a.total_tiles;
  for (;;) {
    if (threadIdx.x == 0) s_item = lo_item + atomicAdd(&a.s.ctr[kCtrWork], 1ull);
    __syncthreads();
    const uint64_t item = s_item;
    if (item >= hi_item) break;
    const uint32_t w = w_only < a.nwin ? w_only : find_window(a.tile_off, a.nwin, item);
    const WinDesc d = a.win[w];
    const uint64_t t = item - a.tile_off[w];
    const uint64_t b0 = t * a.tile_bits;
    const uint32_t nb = (uint32_t)(d.wbits - b0 < a.tile_bits ? d.wbits - b0 : a.tile_bits);
    const uint32_t nw = nb / 32;  // wbits and tile_bits are multiples of 32
    const int64_t g0 = (int64_t)(d.start >> 1) - (int64_t)(a.s.halo >> 1) + (int64_t)b0;
    // the tile's top q, or the window's when that is lower (compared in odd
    // index space: the tile's top may pass 2^64 for windows ending near it)
    const uint64_t gt = (uint64_t)(g0 + nb - 1);
    const uint64_t q_top = gt >= (d.q_top >> 1) ? d.q_top : 2 * gt + 1;
    const uint32_t ns = d.nsieve < a.nsmall ? d.nsieve : a.nsmall;
    sieve_window<kWinThreads>(Q, nw, nb, g0, q_top, pat, a.s.primes, a.magic, ns, a.kcoop);
    // 128-bit coalesced stores: wbase, b0 / 32 and nw are multiples of 4 words
    uint4* out = reinterpret_cast<uint4*>(a.bits + d.wbase + b0 / 32);
    for (uint32_t i = threadIdx.x; i < nw / 4; i += kWinThreads)
      out[i] = make_uint4(Q[4 * i], Q[4 * i + 1], Q[4 * i + 2], Q[4 * i + 3]);
    __syncthreads();
  }
}

// B. large primes -------------------------------------------------------------
__global__ void __launch_bounds__(256) win_large_kernel(const __grid_constant__ WindowsArgs a,
                                                        uint32_t w_only) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = a.nsmall + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < a.nlarge;
       k += stride) {
    const uint32_t p = a.s.primes[k];
    const double inv = 1.0 / (double)p;  // p >= 2^17: first_mark_f64 applies
    const uint64_t pp = (uint64_t)p * p;
    const uint64_t gpp = (pp - 1) >> 1;
    uint32_t w0, w1;
    if (w_only < a.nwin) {
      w0 = w_only;
      w1 = w_only + 1;
      if (a.win[w0].q_top < pp) continue;
    } else {
      // first window whose top reaches p^2 (windows sorted by q_top)
      uint32_t lo = 0, hi = a.nwin;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.win[mid].q_top < pp) lo = mid + 1;
        else hi = mid;
      }
      w0 = lo;
      w1 = a.nwin;
    }
    // one 16-byte load per window; the descriptor only on a hit (p is at
    // least 2^17, the bitsets 2^13..2^25 bits: most windows get none)
#pragma unroll 8
    for (uint32_t w = w0; w < w1; ++w) {
      const longlong2 v = a.wg[w];
      const uint64_t f = first_mark_f64(v.x, p, inv, gpp);
      if (f < (uint64_t)v.y) {
        uint32_t* bw = a.bits + a.win[w].wbase;
        for (uint64_t i = f; i < (uint64_t)v.y; i += p) atomicAnd(&bw[i >> 5], ~(1u << (i & 31)));
      }
    }
  }
}

// C. search -------------------------------------------------------------------
template <bool MINP>
__global__ void __launch_bounds__(kWinThreads, 2) win_search_kernel(const __grid_constant__ WindowsArgs a,
                                                                    uint32_t w_only) {
  extern __shared__ uint32_t smem[];
  uint32_t* Q = smem;
  uint32_t* HIST = Q + a.nbw;
  uint16_t* SOFF = reinterpret_cast<uint16_t*>(HIST + kSmemHistBins);
  __shared__ unsigned long long s_item, s_psum;
  __shared__ uint32_t s_fb, s_maxp;
  const SearchParams& s = a.s;
  load_search_offsets<kWinThreads>(s, SOFF);
  const uint64_t lo_item = w_only < a.nwin ? a.chunk_off[w_only] : 0;
  const uint64_t hi_item = w_only < a.nwin ? a.chunk_off[w_only + 1] : a.total_chunks;
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = lo_item + atomicAdd(&s.ctr[kCtrWork2], 1ull);
      s_fb = 0;
      s_maxp = 0;
      s_psum = 0;
    }
    for (uint32_t i = threadIdx.x; i < kSmemHistBins; i += kWinThreads) HIST[i] = 0;
    __syncthreads();
    const uint64_t item = s_item;
    if (item >= hi_item) break;
    const uint32_t w = w_only < a.nwin ? w_only : find_window(a.chunk_off, a.nwin, item);
    const WinDesc d = a.win[w];
    const uint64_t ci = item - a.chunk_off[w];
    const uint64_t j0 = ci * a.chunk_evens;
    Chunk c;
    c.cnt = (uint32_t)(d.count - j0 < a.chunk_evens ? d.count - j0 : a.chunk_evens);
    c.A = d.start + 2 * j0;
    c.base_idx = d.out_off + j0;
    c.unit = d.orig;  // caller's window index
    // chunk window = bits [j0, j0 + H/2 + cnt + 64) of the window bitset
    const uint32_t nwq = (s.halo / 2 + c.cnt + 64) / 32;
    const uint4* src = reinterpret_cast<const uint4*>(a.bits + d.wbase + j0 / 32);
    uint4* dst = reinterpret_cast<uint4*>(Q);
    const uint32_t n4 = (nwq + 3) / 4;
    for (uint32_t i = threadIdx.x; i < n4; i += kWinThreads) dst[i] = src[i];
    __syncthreads();
    search_chunk<MINP, kWinThreads>(s, Q, SOFF, HIST, c, &s_fb, &s_maxp, &s_psum);
  }
}

// D. narrow windows on the Miller-Rabin path: the n of each window, laid out
// window after window at off[i], for the single-n kernel -------------------
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

// ---------------------------------------------------------------------------
static size_t tile_smem(const WindowsArgs& a) {
  return (size_t)(kWheelWords + a.tile_bits / 32 + 2) * sizeof(uint32_t);
}
static size_t search_smem(const WindowsArgs& a) {
  return (size_t)(a.nbw + kSmemHistBins) * sizeof(uint32_t) +
         (size_t)((a.s.nsearch + 1) & ~1u) * sizeof(uint16_t);
}

cudaError_t launch_window_stages(const WindowsArgs& a, uint32_t w_only, int grid_tile,
                                 int grid_large, int grid_search, cudaStream_t st, int* launches) {
  cudaError_t e;
  const size_t ts = tile_smem(a), ss = search_smem(a);
  e = cudaFuncSetAttribute(win_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ts);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(win_search_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)ss);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(win_search_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)ss);
  if (e != cudaSuccess) return e;
  // the stages' work counters restart at 0
  if ((e = cudaMemsetAsync(&a.s.ctr[kCtrWork], 0, 8, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(&a.s.ctr[kCtrWork2], 0, 8, st)) != cudaSuccess) return e;
  win_tile_kernel<<<grid_tile, kWinThreads, ts, st>>>(a, w_only);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  ++*launches;
  if (a.nlarge > a.nsmall && grid_large > 0) {
    win_large_kernel<<<grid_large, 256, 0, st>>>(a, w_only);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ++*launches;
  }
  if (a.s.minp) win_search_kernel<true><<<grid_search, kWinThreads, ss, st>>>(a, w_only);
  else win_search_kernel<false><<<grid_search, kWinThreads, ss, st>>>(a, w_only);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  ++*launches;
  return cudaSuccess;
}

}  // namespace gb
