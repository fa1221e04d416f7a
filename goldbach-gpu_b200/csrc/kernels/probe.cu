// probe.cu -- peak-throughput probes for the roofline of the integer
// kernels: 32-bit ALU operations (funnel shift, three-input logic, add),
// shared-memory atomicAnd, and 64-bit Montgomery products (the unit of the
// Miller-Rabin work), each with independent work per thread so that issue
// throughput, not latency, is what gets measured.
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_device.cuh"
#include "../gb_internal.h"

namespace gb {

// 8 independent chains per thread, one 32-bit ALU op per chain per step.
__global__ void __launch_bounds__(256) probe_alu_kernel(uint32_t* sink, int iters) {
  uint32_t a = threadIdx.x, b = blockIdx.x, c = a ^ 0x9e3779b9u, d = b * 7u;
  uint32_t e = a + 3u, f = b ^ a, g = a * 3u, h = b + 11u;
  const uint32_t k = threadIdx.x | 1u;
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
    a = __funnelshift_r(a, k, i);
    b = (b ^ k) & (c | 5u);
    c = c + k;
    d = __funnelshift_r(d, k, 3);
    e = (e & k) ^ 0x55u;
    f = f + 0x1234567u;
    g = (g | k) ^ h;
    h = h + k;
  }
  const uint32_t x = a ^ b ^ c ^ d ^ e ^ f ^ g ^ h;
  if (x == 0x7fffffffu) sink[0] = x;  // keeps the chains alive
}

// Conflict-free shared-memory atomicAnd: lane l of a warp hits bank
// (37 l + step) mod 32, a permutation of the banks.
__global__ void __launch_bounds__(256) probe_atom_kernel(uint32_t* sink, int iters) {
  __shared__ uint32_t s[8192];
  for (int i = threadIdx.x; i < 8192; i += 256) s[i] = 0xffffffffu;
  __syncthreads();
  uint32_t idx = threadIdx.x * 37u;
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
    idx = (idx + 977u) & 8191u;
    atomicAnd(&s[idx], ~(1u << (i & 31)));
  }
  __syncthreads();
  if (s[threadIdx.x] == 0x12345u) sink[0] = s[threadIdx.x];
}

// 4 independent chains of mont_mul32 per thread (the product the single-n
// and Phase-2 kernels use), modulus an odd 64-bit number per thread.
__global__ void __launch_bounds__(256) probe_mont_kernel(uint32_t* sink, int iters) {
  const uint64_t n = 0xfffffffffffffc5ull - 2ull * (blockIdx.x * 256u + threadIdx.x);  // odd
  const Mont M = mont_init(n);
  const uint32_t ni = (uint32_t)M.ninv;
  uint64_t a = M.one, b = n >> 1, c = n / 3, d = n / 5;
#pragma unroll 2
  for (int i = 0; i < iters; ++i) {
    a = mont_mul32(a, b, n, ni);
    b = mont_mul32(b, c, n, ni);
    c = mont_mul32(c, d, n, ni);
    d = mont_mul32(d, a, n, ni);
  }
  if ((a ^ b ^ c ^ d) == 0x7fffffffull) sink[0] = 1;  // keeps the chains alive
}

cudaError_t run_probe(int kind, int sm_count, double* ops_per_s, cudaStream_t st) {
  uint32_t* sink = nullptr;
  cudaError_t e = cudaMalloc(&sink, 4);
  if (e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int grid = sm_count * 8, block = 256;
  const int iters = kind == 2 ? 1 << 11 : 1 << 14;
  const double per_thread = kind == 0 ? 8.0 * iters : kind == 2 ? 4.0 * iters : (double)iters;
  // a warm-up run, then the best of five (the peak: a run slowed by
  // anything else on the GPU or a clock ramp does not count)
  float best = 0;
  for (int rep = 0; rep < 6 && e == cudaSuccess; ++rep) {
    cudaEventRecord(e0, st);
    if (kind == 0) probe_alu_kernel<<<grid, block, 0, st>>>(sink, iters);
    else if (kind == 1) probe_atom_kernel<<<grid, block, 0, st>>>(sink, iters);
    else probe_mont_kernel<<<grid, block, 0, st>>>(sink, iters);
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && rep > 0 && (best == 0 || ms < best)) best = ms;
  }
  if (e == cudaSuccess) *ops_per_s = per_thread * grid * block / (best / 1e3);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  return e;
}

}  // namespace gb
