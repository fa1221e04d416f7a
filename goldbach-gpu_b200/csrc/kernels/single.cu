// single.cu -- batched single-n minimal partitions and batched primality.
//
// Replaces goldbach_single_kernel + check_single (src/single_check.cu:
// 95-282).  The reference sieves p in chunks of 1e8 on the CPU, copies them
// to the GPU, runs one thread per p with a 128-bit-remainder Miller-Rabin
// and keeps whichever thread finishes first, so its p is not the minimal
// one.  Here one warp serves one query n from a device work counter (query
// cost is uneven):
//   1. lanes take 32 consecutive primes p from the resident table and drop
//      those with q = n - p divisible by a prime r <= 61, using
//      q == 0 (mod r)  <=>  n mod r == p mod r  (n mod r computed once);
//   2. survivors are gathered in order until 32 are pending, then each lane
//      runs the base-2 strong test on one of them (Montgomery, 64-bit);
//   3. the lowest lane that passed gets the other six bases of the
//      deterministic set, one base per lane; if all pass, its p is the
//      minimal p (every smaller candidate was rejected above).
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_device.cuh"
#include "../gb_internal.h"

namespace gb {

constexpr int kSingleThreads = 256;
constexpr int kSingleWarps = kSingleThreads / 32;
constexpr uint64_t kSmallN = 1ull << 21;  // below this, q may be tiny: plain path

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Lane-parallel ascending scan with the full primality test per lane.
__device__ uint32_t minp_plain(const SingleArgs& a, uint64_t n) {
  const int lane = threadIdx.x & 31;
  const uint64_t half = n >> 1;
  const uint64_t lim = half < a.p_lim ? half : a.p_lim;
  for (uint64_t k = 1;; k += 32) {
    const uint64_t kk = k + lane;
    const uint32_t p = kk < a.nprimes ? a.primes[kk] : 0xffffffffu;
    const bool valid = kk < a.nprimes && p <= lim;
    const bool ok = valid && is_prime_u64(n - p);
    const uint32_t b = __ballot_sync(0xffffffffu, ok);
    if (b) return __shfl_sync(0xffffffffu, p, __ffs(b) - 1);
    if (__ballot_sync(0xffffffffu, valid) != 0xffffffffu) return 0;
  }
}

#define GB_SMALL_PRIMES(X) \
  X(3) X(5) X(7) X(11) X(13) X(17) X(19) X(23) X(29) X(31) X(37) X(41) X(43) X(47) X(53) X(59) X(61)

__device__ uint32_t minp_big(const SingleArgs& a, uint64_t n, uint32_t* buf) {
  const int lane = threadIdx.x & 31;
  const uint64_t half = n >> 1;
  const uint64_t lim = half < a.p_lim ? half : a.p_lim;
#define GB_NMOD(r) const uint32_t nm##r = (uint32_t)(n % r##u);
  GB_SMALL_PRIMES(GB_NMOD)
#undef GB_NMOD
  uint64_t k = 1;
  uint32_t nsurv = 0;
  bool exhausted = false;
  for (;;) {
    while (nsurv < 32 && !exhausted) {
      const uint64_t kk = k + lane;
      const uint32_t p = kk < a.nprimes ? a.primes[kk] : 0xffffffffu;
      const bool valid = kk < a.nprimes && p <= lim;
      bool pass = valid;
#define GB_SIEVE(r) pass = pass && (p % r##u != nm##r);
      GB_SMALL_PRIMES(GB_SIEVE)
#undef GB_SIEVE
      const uint32_t b = __ballot_sync(0xffffffffu, pass);
      if (pass) buf[nsurv + __popc(b & lanemask_lt())] = (uint32_t)kk;
      nsurv += __popc(b);
      if (__ballot_sync(0xffffffffu, valid) != 0xffffffffu) exhausted = true;
      k += 32;
    }
    __syncwarp();
    if (nsurv == 0) return 0;
    const uint32_t take = nsurv < 32 ? nsurv : 32;
    bool ok2 = false;
    uint64_t q = 0;
    uint32_t pk = 0;
    if (lane < (int)take) {
      pk = a.primes[buf[lane]];
      q = n - pk;
      uint64_t d = q - 1;
      const int s = __ffsll((long long)d) - 1;
      d >>= s;
      const Mont M = mont_init(q);
      ok2 = sprp2(M, d, s);
    }
    uint32_t b = __ballot_sync(0xffffffffu, ok2);
    while (b) {
      const int l = __ffs(b) - 1;
      const uint64_t qc = __shfl_sync(0xffffffffu, q, l);
      const uint32_t pc = __shfl_sync(0xffffffffu, pk, l);
      bool ok = true;
      if (lane < 6) {
        uint64_t d = qc - 1;
        const int s = __ffsll((long long)d) - 1;
        d >>= s;
        const Mont M = mont_init(qc);
        ok = sprp_base_k(M, mont_r2(M), lane + 1, d, s);
      }
      if (__all_sync(0xffffffffu, ok)) return pc;
      b &= b - 1;
    }
    // none of the first `take` survivors is prime: drop them
    __syncwarp();
    uint32_t keep = 0;
    if (lane + take < nsurv) keep = buf[lane + take];
    __syncwarp();
    if (lane + take < nsurv) buf[lane] = keep;
    __syncwarp();
    nsurv -= take;
  }
}

__global__ void __launch_bounds__(kSingleThreads) single_kernel(SingleArgs a) {
  __shared__ uint32_t sbuf[kSingleWarps][64];
  const int lane = threadIdx.x & 31;
  uint32_t* buf = sbuf[threadIdx.x >> 5];
  for (;;) {
    unsigned long long qi = 0;
    if (lane == 0) qi = atomicAdd(&a.ctr[0], 1ull);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if (qi >= a.count) break;
    const uint64_t n = a.n[qi];
    uint32_t p = 0;
    if (n >= 4 && !(n & 1)) {
      if (n == 4) p = 2;
      else if (n < kSmallN) p = minp_plain(a, n);
      else p = minp_big(a, n, buf);
    }
    if (lane == 0) {
      a.p_out[qi] = p;
      a.q_out[qi] = p ? n - p : 0;
      if (p) {
        atomicAdd(&a.ctr[1], 1ull);
        atomicMax(&a.ctr[2], (unsigned long long)p);
      }
    }
  }
}

cudaError_t launch_single(const SingleArgs& a, int grid, cudaStream_t s) {
  single_kernel<<<grid, kSingleThreads, 0, s>>>(a);
  return cudaGetLastError();
}

// Per-request totals of a single-lane batch: request r owns the n of
// [off[r], off[r+1]); agg[4r..4r+3] = verified, failures, max p, sum of p.
__global__ void segment_reduce_kernel(const uint64_t* p, const uint64_t* off, uint32_t nreq,
                                      unsigned long long* agg) {
  const uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= nreq) return;
  unsigned long long v = 0, f = 0, mx = 0, sum = 0;
  for (uint64_t i = off[r] + lane; i < off[r + 1]; i += 32) {
    const uint64_t x = p[i];
    if (x) {
      ++v;
      sum += x;
      if (x > mx) mx = x;
    } else {
      ++f;
    }
  }
  for (int o = 16; o; o >>= 1) {
    v += __shfl_down_sync(0xffffffffu, v, o);
    f += __shfl_down_sync(0xffffffffu, f, o);
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    const unsigned long long m2 = __shfl_down_sync(0xffffffffu, mx, o);
    if (m2 > mx) mx = m2;
  }
  if (lane == 0) {
    agg[4 * r] = v;
    agg[4 * r + 1] = f;
    agg[4 * r + 2] = mx;
    agg[4 * r + 3] = sum;
  }
}

cudaError_t launch_segment_reduce(const uint64_t* p, const uint64_t* off, uint32_t nreq,
                                  unsigned long long* agg, cudaStream_t s) {
  if (!nreq) return cudaSuccess;
  segment_reduce_kernel<<<(nreq + 7) / 8, 256, 0, s>>>(p, off, nreq, agg);
  return cudaGetLastError();
}

__global__ void is_prime_kernel(const uint64_t* n, uint64_t count, uint8_t* out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = is_prime_u64(n[i]) ? 1 : 0;
}

cudaError_t launch_is_prime(const uint64_t* n, uint64_t count, uint8_t* out, cudaStream_t s) {
  if (!count) return cudaSuccess;
  uint64_t blocks = (count + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  is_prime_kernel<<<(unsigned)blocks, 256, 0, s>>>(n, count, out);
  return cudaGetLastError();
}

}  // namespace gb
