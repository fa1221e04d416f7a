// counts.cu -- Goldbach partition counts c(n) on the GPU.
//
// c(n) = #{p <= n/2 : p and n - p prime}, the reference's goldbach_count
// (src/cpu_goldbach.cpp:29-36, a scalar scan over a byte table on the CPU;
// "partition counting c(n) at scale" is its open roadmap item,
// RESULTS.md:169).  Here it is a correlation of the odd-prime bitset B
// (bit i <-> 2i+1 prime) with itself: for even n >= 6 and m = n/2 - 1,
//     c(n) = sum_{i=0}^{floor(m/2)} B[i] * B[m - i]
// (p = 2i+1, q = 2(m-i)+1; n = 4 = 2+2 adds one).  A warp takes 32
// consecutive n (m0 .. m0+31) and a slice of the words of i; for word w the
// 32 bits B[m0 + d - 32w - b] (b = 0..31) of every d come from one 64-bit
// window of B read at m0 - 32w - 31, bit-reversed once, then funnel-shifted
// by d: 32 AND + popcount word operations per word of i, each testing 32
// (n, p) pairs.  Lanes accumulate 32 counters each, reduced across the warp
// by a transposing butterfly (lane d ends with the total of n = 2(m0+d+1)).
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_internal.h"

namespace gb {

constexpr int kCountThreads = 256;
constexpr int kCountWarps = kCountThreads / 32;

// B: the padded bitset (words B[-2], B[-1] are zero, B[0] holds i = 0..31).
__global__ void __launch_bounds__(kCountThreads) counts_kernel(const uint32_t* __restrict__ B,
                                                               uint64_t m_first, uint64_t count,
                                                               uint32_t splits, uint64_t wps,
                                                               unsigned long long* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint64_t task = (uint64_t)blockIdx.x * kCountWarps + (threadIdx.x >> 5);
  const uint64_t g = task / splits, sp = task % splits;
  if (g * 32 >= count) return;  // warp-uniform
  const uint64_t m0 = m_first + 32 * g;
  const uint64_t nw = (m0 + 31) / 2 / 32 + 1;  // words holding i <= floor((m0+31)/2)
  const uint64_t w_lo = sp * wps;
  if (w_lo >= nw) return;  // warp-uniform
  const uint64_t w_hi = w_lo + wps < nw ? w_lo + wps : nw;
  // words whose 32 i are all <= floor(m0/2), i.e. need no mask for any d
  const uint64_t full = m0 / 2 >= 31 ? (m0 / 2 - 31) / 32 + 1 : 0;
  uint32_t acc[32];
#pragma unroll
  for (int d = 0; d < 32; ++d) acc[d] = 0;
  for (uint64_t w = w_lo + lane; w < w_hi; w += 32) {
    uint32_t bw = B[w];
    if (!bw) continue;
    // 64 bits of B from position a = m0 - 32w - 31 (>= -47 > -64: the padding)
    const int64_t a = (int64_t)m0 - 32 * (int64_t)w - 31;
    const int64_t aw = a >> 5;  // floor
    const uint32_t sh = (uint32_t)a & 31u;
    const uint32_t x0 = B[aw], x1 = B[aw + 1], x2 = B[aw + 2];
    const uint32_t rl = __brev(__funnelshift_r(x1, x2, sh));
    const uint32_t rh = __brev(__funnelshift_r(x0, x1, sh));
    if (w < full) {
#pragma unroll
      for (int d = 0; d < 32; ++d) acc[d] += __popc(bw & __funnelshift_rc(rl, rh, 32 - d));
    } else {  // the last word(s): only i <= floor((m0+d)/2) count
#pragma unroll
      for (int d = 0; d < 32; ++d) {
        const int64_t lim = (int64_t)((m0 + d) / 2) - 32 * (int64_t)w;
        const uint32_t mk = lim < 0 ? 0u : lim >= 31 ? 0xffffffffu : (2u << lim) - 1u;
        acc[d] += __popc(bw & mk & __funnelshift_rc(rl, rh, 32 - d));
      }
    }
  }
  // transposing butterfly: after the step of width k a lane keeps the half of
  // its counters selected by its lane bit k and adds the partner's copy
#pragma unroll
  for (int k = 16; k >= 1; k >>= 1) {
    const bool up = lane & k;
#pragma unroll
    for (int j = 0; j < k; ++j) {
      const uint32_t keep = up ? acc[j + k] : acc[j];
      const uint32_t give = up ? acc[j] : acc[j + k];
      acc[j] = keep + __shfl_xor_sync(0xffffffffu, give, k);
    }
  }
  const uint64_t j = g * 32 + lane;
  uint64_t v = acc[0];
  if (sp == 0 && m0 + lane == 1) v += 1;  // n = 4 = 2 + 2
  if (j < count && v) atomicAdd(&out[j], (unsigned long long)v);
}

cudaError_t launch_counts(const uint32_t* B, uint64_t m_first, uint64_t count, uint32_t splits,
                          uint64_t wps, unsigned long long* out, cudaStream_t s) {
  const uint64_t tasks = (count + 31) / 32 * splits;
  const uint64_t blocks = (tasks + kCountWarps - 1) / kCountWarps;
  if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
  counts_kernel<<<(unsigned)blocks, kCountThreads, 0, s>>>(B, m_first, count, splits, wps, out);
  return cudaGetLastError();
}

}  // namespace gb
