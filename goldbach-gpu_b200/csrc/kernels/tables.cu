// tables.cu -- device construction of the resident prime tables.
//
// Replaces the host-side table builders of the reference:
//   build_prime_bitset   src/prime_bitset.cpp:21-97 (OpenMP, racy)
//   small/gpu prime lists src/goldbach.cu:661-673
//   generate_cpu_primes  src/goldbach.cu:318-331
// The tables are built on the GPU by the same window sieve the range kernel
// uses, then compacted into an ascending uint32 list with a Barrett
// reciprocal per prime.
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_internal.h"
#include "sieve_window.cuh"

namespace gb {

// ---------------------------------------------------------------------------
// Wheel patterns: word W of the table belongs to group x; bit b of its
// local word w is 1 iff the odd number 2g+1, g = (32w+b) mod period, has no
// factor among the group's primes (2g+1 == 0 mod p  <=>  g mod p == (p-1)/2).
__device__ __forceinline__ uint32_t wheel_group_prime(int x, int j) {
  switch (x) {
    case 0: return j == 0 ? 3 : j == 1 ? 5 : j == 2 ? 7 : j == 3 ? 11 : j == 4 ? 13 : 0;
    case 1: return j == 0 ? 17 : j == 1 ? 19 : j == 2 ? 23 : 0;
    case 2: return j == 0 ? 29 : j == 1 ? 31 : 0;
    case 3: return j == 0 ? 37 : j == 1 ? 41 : 0;
    case 4: return j == 0 ? 43 : j == 1 ? 47 : 0;
    case 5: return j == 0 ? 53 : j == 1 ? 59 : 0;
    default: return j == 0 ? 61 : j == 1 ? 67 : 0;
  }
}

__global__ void wheel_init_kernel(uint32_t* wheel) {
  const uint32_t W = blockIdx.x * blockDim.x + threadIdx.x;
  if (W >= kWheelWords) return;
  int x = 0;
  while (x + 1 < kWheelGroups && W >= wheel_offset(x + 1)) ++x;
  const uint32_t P = wheel_period(x);
  const uint32_t w = W - wheel_offset(x);
  uint32_t v = 0;
  for (int b = 0; b < 32; ++b) {
    const uint32_t g = (32u * w + b) % P;
    bool keep = true;
    for (int j = 0; j < 5; ++j) {
      const uint32_t p = wheel_group_prime(x, j);
      if (p && g % p == (p - 1) / 2) keep = false;
    }
    if (keep) v |= 1u << b;
  }
  wheel[W] = v;
}

// Mod-6 patterns: word W of class c's table, group x: bit b = 1 iff
// 6g + c has no factor in the group, g = (32w + b) mod period.
__device__ __forceinline__ uint32_t wheel6_group_prime(int x, int j) {
  return x == 0 ? (j == 0 ? 5 : j == 1 ? 7 : j == 2 ? 11 : j == 3 ? 13 : 0) : wheel_group_prime(x, j);
}

__global__ void wheel6_init_kernel(uint32_t* wheel6) {
  const uint32_t W = blockIdx.x * blockDim.x + threadIdx.x;
  if (W >= kWheel6Words) return;
  const int cls5 = W >= kWheel6ClassWords;
  const uint32_t wc = W - (cls5 ? kWheel6ClassWords : 0);
  int x = 0;
  while (x + 1 < kWheel6Groups && wc >= wheel6_group_offset(x + 1)) ++x;
  const uint32_t P = wheel6_period(x);
  const uint32_t w = wc - wheel6_group_offset(x);
  const uint32_t c = cls5 ? 5 : 1;
  uint32_t v = 0;
  for (int b = 0; b < 32; ++b) {
    const uint32_t g = (32u * w + b) % P;
    bool keep = true;
    for (int j = 0; j < 5; ++j) {
      const uint32_t p = wheel6_group_prime(x, j);
      if (p && (6ull * g + c) % p == 0) keep = false;
    }
    if (keep) v |= 1u << b;
  }
  wheel6[W] = v;
}

cudaError_t launch_wheel_init(uint32_t* wheel, uint32_t* wheel6, cudaStream_t s) {
  wheel_init_kernel<<<(kWheelWords + 255) / 256, 256, 0, s>>>(wheel);
  wheel6_init_kernel<<<(kWheel6Words + 255) / 256, 256, 0, s>>>(wheel6);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Bitset sieve: CTA t sieves bits [t*tile, min(nbits, (t+1)*tile)) of the
// odd-only window starting at q_lo and stores them with coalesced stores.
constexpr int kSieveThreads = 512;

__global__ void __launch_bounds__(kSieveThreads) sieve_bits_kernel(SieveArgs a) {
  extern __shared__ uint32_t smem[];
  uint32_t* pat = smem;
  uint32_t* Q = smem + kWheelWords;
  for (uint32_t i = threadIdx.x; i < kWheelWords; i += kSieveThreads) pat[i] = a.wheel[i];
  __syncthreads();
  const uint64_t t = blockIdx.x;
  const uint64_t b0 = t * a.tile_bits;
  const uint64_t rem = a.nbits - b0;
  const uint32_t nb = rem < a.tile_bits ? (uint32_t)rem : a.tile_bits;
  const uint32_t nw = (nb + 31) / 32;
  const int64_t g0 = (int64_t)((a.q_lo - 1) / 2 + b0);
  uint64_t q_top = a.q_lo + 2 * (b0 + nb - 1);
  if (q_top < a.q_lo) q_top = ~0ull;  // wrapped past 2^64
  sieve_window<kSieveThreads>(Q, nw, nb, g0, q_top, pat, a.primes, a.magic, a.nsieve, a.kcoop);
  uint32_t* out = a.out + b0 / 32;
  for (uint32_t i = threadIdx.x; i < nw; i += kSieveThreads) {
    uint32_t v = Q[i];
    if (i == nw - 1 && (nb & 31)) v &= (1u << (nb & 31)) - 1;
    out[i] = v;
  }
}

cudaError_t launch_sieve_bits(const SieveArgs& a, cudaStream_t s) {
  if (a.nbits == 0) return cudaSuccess;
  const size_t smem = (kWheelWords + a.tile_bits / 32 + 2) * sizeof(uint32_t);
  cudaError_t e = cudaFuncSetAttribute(sieve_bits_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const uint64_t tiles = (a.nbits + a.tile_bits - 1) / a.tile_bits;
  sieve_bits_kernel<<<(unsigned)tiles, kSieveThreads, smem, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Compaction of an odd-only bitset into an ascending prime list.
constexpr int kCompactWords = 1024;  // words per block (one per thread)

size_t compact_scratch_blocks(uint64_t nbits) {
  const uint64_t words = (nbits + 31) / 32;
  return (size_t)((words + kCompactWords - 1) / kCompactWords);
}

__global__ void __launch_bounds__(kCompactWords) compact_count_kernel(const uint32_t* bits,
                                                                     uint64_t nwords,
                                                                     uint32_t* blocks) {
  const uint64_t w = (uint64_t)blockIdx.x * kCompactWords + threadIdx.x;
  uint32_t c = w < nwords ? __popc(bits[w]) : 0;
  c = __reduce_add_sync(0xffffffffu, c);
  __shared__ uint32_t ws[kCompactWords / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = ws[threadIdx.x];
    v = __reduce_add_sync(0xffffffffu, v);
    if (threadIdx.x == 0) blocks[blockIdx.x] = v;
  }
}

// Exclusive scan of the per-block counts by one block, in place; the grand
// total plus `prefix` goes to *total.
__global__ void __launch_bounds__(1024) compact_scan_kernel(uint32_t* blocks, uint32_t n,
                                                            uint64_t prefix,
                                                            unsigned long long* total) {
  __shared__ unsigned long long carry;
  __shared__ uint32_t wsum[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < n; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < n ? blocks[i] : 0;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t s = wsum[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, s, d);
        if (lane >= d) s += y;
      }
      wsum[lane] = s;  // inclusive
    }
    __syncthreads();
    const uint32_t wpre = warp ? wsum[warp - 1] : 0;
    const unsigned long long c = carry;
    if (i < n) blocks[i] = (uint32_t)(c + wpre + x - v);
    __syncthreads();
    if (threadIdx.x == 1023) carry = c + wpre + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = prefix + carry;
}

__global__ void __launch_bounds__(kCompactWords) compact_write_kernel(
    const uint32_t* bits, uint64_t nwords, uint64_t q_lo, const uint32_t* blocks,
    uint32_t* primes, uint64_t* magic, uint2* a15, uint64_t prefix, uint64_t cap) {
  const uint64_t w = (uint64_t)blockIdx.x * kCompactWords + threadIdx.x;
  uint32_t v = w < nwords ? bits[w] : 0;
  const uint32_t c = __popc(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  __shared__ uint32_t wsum[32];
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = wsum[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, d);
      if (lane >= d) s += y;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  uint64_t pos = prefix + blocks[blockIdx.x] + (warp ? wsum[warp - 1] : 0) + (x - c);
  while (v) {
    const int b = __ffs(v) - 1;
    v &= v - 1;
    const uint64_t q = q_lo + 2 * (32 * w + b);
    if (pos < cap) {
      primes[pos] = (uint32_t)q;
      magic[pos] = ~0ull / q;
      // class offsets of the mod-6 sieve: a1 = -1/6, a5 = -5/6 (mod q)
      uint2 a = make_uint2(0, 0);
      if (q >= 5) {
        const uint64_t inv6 = (q % 6 == 1) ? (5 * q + 1) / 6 : (q + 1) / 6;
        const uint64_t a1 = q - inv6;
        a = make_uint2((uint32_t)a1, (uint32_t)((5 * a1) % q));
      }
      a15[pos] = a;
    }
    ++pos;
  }
}

__global__ void put_two_kernel(uint32_t* primes, uint64_t* magic, uint2* a15) {
  primes[0] = 2;
  magic[0] = ~0ull / 2;
  a15[0] = make_uint2(0, 0);
}

cudaError_t launch_compact_primes(const uint32_t* bits, uint64_t nbits, uint64_t q_lo,
                                  uint32_t* primes, uint64_t* magic, uint2* a15, uint64_t prefix,
                                  uint64_t cap, unsigned long long* d_total,
                                  uint32_t* scratch_blocks, uint32_t nblocks_cap,
                                  cudaStream_t s) {
  const uint64_t nwords = (nbits + 31) / 32;
  const uint32_t nblocks = (uint32_t)compact_scratch_blocks(nbits);
  if (nblocks > nblocks_cap) return cudaErrorInvalidValue;
  if (prefix == 1) put_two_kernel<<<1, 1, 0, s>>>(primes, magic, a15);
  if (nblocks == 0) return cudaGetLastError();
  compact_count_kernel<<<nblocks, kCompactWords, 0, s>>>(bits, nwords, scratch_blocks);
  compact_scan_kernel<<<1, 1024, 0, s>>>(scratch_blocks, nblocks, prefix, d_total);
  compact_write_kernel<<<nblocks, kCompactWords, 0, s>>>(bits, nwords, q_lo, scratch_blocks,
                                                         primes, magic, a15, prefix, cap);
  return cudaGetLastError();
}

}  // namespace gb
