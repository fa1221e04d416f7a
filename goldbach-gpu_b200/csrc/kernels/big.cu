// big.cu -- Goldbach partitions of even n beyond 2^64 (multi-precision).
//
// Replaces big_check (src/big_check.cpp:35-144), which scans the primes up
// to 1e7 in OpenMP batches of 1000 and keeps the first q = n - p that GMP's
// mpz_probab_prime_p(q, 25) accepts -- a valid partition, not guaranteed
// the minimal one.  Here the candidates p (ascending, from the resident
// prime table) are tested in launches of kBigBatch:
//   1. big_filter_kernel: one thread per candidate drops q = n - p when a
//      prime r < kBigTrialBound divides it, from n mod r (computed on the
//      host once per n) and p mod r, and appends the survivors' indices;
//   2. big_mr_kernel<N>: one thread per survivor runs strong probable-prime
//      tests to the 12 prime bases 2, 3, ..., 37 -- the base set of the
//      reference's Miller-Rabin (src/goldbach.cu:333-360) -- on N 32-bit
//      limbs, stopping at the first failing base, and lowers the batch's
//      best candidate index when every base passes.
// The smallest passing index is the minimal p: every smaller candidate was
// tested and failed.  The test is deterministic for q < 3.3e24 (the 12
// prime bases admit no strong pseudoprime below that) and a probable-prime
// test beyond, like the reference's.
//
// The Montgomery product is the coarsely integrated operand-scanning form
// (CIOS) on 32-bit limbs with 64-bit accumulators, R = 2^(32 N), N a power
// of two from 4 to 128 (n up to 4096 bits; the limbs above n's own are
// zero).  Operands live in the thread's local memory for the wide sizes.
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_internal.h"

namespace gb {

constexpr int kBigThreads = 128;

// The 12 prime bases of the strong tests.
__device__ __constant__ const uint32_t kBigBases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};

__global__ void __launch_bounds__(256) big_filter_kernel(const __grid_constant__ BigArgs a, uint32_t k0,
                                                         uint32_t kcount) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kcount) return;
  const uint32_t k = k0 + i;
  const uint32_t p = a.primes[k];
  bool keep = p <= a.p_lim;
  for (uint32_t j = 0; keep && j < a.ntrial; ++j)
    if (p % a.trial[j] == a.nmod[j]) keep = false;  // r divides q = n - p (q far above r)
  if (keep) {
    const uint32_t slot = atomicAdd(a.nsurv, 1u);
    a.surv[slot] = i;
  }
}

// r = x * y * R^-1 mod q (x, y < q; q odd; R = 2^(32 N)); r may be x or y
// (it is written after the last read of both).  The inner loops unroll in
// full for the register-resident sizes only.
template <int N>
__device__ void big_mont_mul(uint32_t* r, const uint32_t* x, const uint32_t* y, const uint32_t* q,
                             uint32_t qinv) {
  constexpr int U = N <= 16 ? N : 4;
  uint32_t t[N + 2];
#pragma unroll
  for (int j = 0; j < N + 2; ++j) t[j] = 0;
  for (int i = 0; i < N; ++i) {
    const uint32_t yi = y[i];
    uint64_t c = 0;
#pragma unroll U
    for (int j = 0; j < N; ++j) {
      const uint64_t v = (uint64_t)x[j] * yi + t[j] + c;
      t[j] = (uint32_t)v;
      c = v >> 32;
    }
    uint64_t v = (uint64_t)t[N] + c;
    t[N] = (uint32_t)v;
    t[N + 1] = (uint32_t)(v >> 32);
    const uint32_t m = t[0] * qinv;
    v = (uint64_t)m * q[0] + t[0];
    c = v >> 32;
#pragma unroll U
    for (int j = 1; j < N; ++j) {
      v = (uint64_t)m * q[j] + t[j] + c;
      t[j - 1] = (uint32_t)v;
      c = v >> 32;
    }
    v = (uint64_t)t[N] + c;
    t[N - 1] = (uint32_t)v;
    t[N] = t[N + 1] + (uint32_t)(v >> 32);
  }
  // t < 2q: subtract q once if t >= q
  bool ge = t[N] != 0;
  if (!ge) {
    ge = true;  // equal counts as >=
    for (int j = N - 1; j >= 0; --j)
      if (t[j] != q[j]) {
        ge = t[j] > q[j];
        break;
      }
  }
  if (ge) {
    uint64_t b = 0;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const uint64_t v = (uint64_t)t[j] - q[j] - b;
      r[j] = (uint32_t)v;
      b = (v >> 32) & 1;
    }
  } else {
#pragma unroll
    for (int j = 0; j < N; ++j) r[j] = t[j];
  }
}

// x = 2x mod q (x < q).
template <int N>
__device__ void big_dbl_mod(uint32_t* x, const uint32_t* q) {
  uint32_t top = 0;
  for (int j = 0; j < N; ++j) {
    const uint32_t nt = x[j] >> 31;
    x[j] = (x[j] << 1) | top;
    top = nt;
  }
  bool ge = top != 0;
  if (!ge) {
    ge = true;
    for (int j = N - 1; j >= 0; --j)
      if (x[j] != q[j]) {
        ge = x[j] > q[j];
        break;
      }
  }
  if (ge) {
    uint64_t b = 0;
    for (int j = 0; j < N; ++j) {
      const uint64_t v = (uint64_t)x[j] - q[j] - b;
      x[j] = (uint32_t)v;
      b = (v >> 32) & 1;
    }
  }
}

template <int N>
__device__ bool big_eq(const uint32_t* x, const uint32_t* y) {
  for (int j = 0; j < N; ++j)
    if (x[j] != y[j]) return false;
  return true;
}

// Strong probable-prime test of odd q > 2^64 to every base of kBigBases.
template <int N>
__device__ bool big_is_probable_prime(const uint32_t* q) {
  uint32_t qinv = q[0];  // -q^-1 mod 2^32 by Newton steps
  for (int i = 0; i < 4; ++i) qinv *= 2u - q[0] * qinv;
  qinv = 0u - qinv;
  // one = R mod q, r2 = R^2 mod q, by doublings of 1
  uint32_t one[N], r2[N], mone[N], d[N], base[N], x[N];
  for (int j = 0; j < N; ++j) one[j] = 0;
  one[0] = 1;
  for (int i = 0; i < 32 * N; ++i) big_dbl_mod<N>(one, q);
  for (int j = 0; j < N; ++j) r2[j] = one[j];
  for (int i = 0; i < 32 * N; ++i) big_dbl_mod<N>(r2, q);
  {  // mone = q - one (that is -1 in Montgomery form)
    uint64_t b = 0;
    for (int j = 0; j < N; ++j) {
      const uint64_t v = (uint64_t)q[j] - one[j] - b;
      mone[j] = (uint32_t)v;
      b = (v >> 32) & 1;
    }
  }
  // q - 1 = d 2^s
  int s = 0;
  {
    int lw = 0;
    while (lw < N && (q[lw] & ~(lw == 0 ? 1u : 0u)) == 0) ++lw;  // q - 1 has its lowest set bit here
    const uint32_t low = lw == 0 ? (q[0] & ~1u) : q[lw];
    s = 32 * lw + __ffs(low) - 1;
    for (int j = 0; j < N; ++j) d[j] = q[j];
    d[0] &= ~1u;  // q - 1 (q odd)
    const int ws = s >> 5, bs = s & 31;
    for (int j = 0; j < N; ++j) {
      const uint32_t lo = j + ws < N ? d[j + ws] : 0;
      const uint32_t hi = j + ws + 1 < N ? d[j + ws + 1] : 0;
      d[j] = bs ? (lo >> bs) | (hi << (32 - bs)) : lo;
    }
  }
  int top = N - 1;
  while (top > 0 && d[top] == 0) --top;
  const int nbits = 32 * top + 32 - __clz(d[top]);
  for (int bi = 0; bi < 12; ++bi) {
    uint32_t a[N];
    for (int j = 0; j < N; ++j) a[j] = 0;
    a[0] = kBigBases[bi];
    big_mont_mul<N>(base, a, r2, q, qinv);  // base in Montgomery form
    for (int j = 0; j < N; ++j) x[j] = base[j];
    for (int b = nbits - 2; b >= 0; --b) {
      big_mont_mul<N>(x, x, x, q, qinv);
      if ((d[b >> 5] >> (b & 31)) & 1u) big_mont_mul<N>(x, x, base, q, qinv);
    }
    if (big_eq<N>(x, one) || big_eq<N>(x, mone)) continue;
    bool ok = false;
    for (int i = 1; i < s && !ok; ++i) {
      big_mont_mul<N>(x, x, x, q, qinv);
      if (big_eq<N>(x, mone)) ok = true;
      else if (big_eq<N>(x, one)) break;
    }
    if (!ok) return false;
  }
  return true;
}

template <int N>
__global__ void __launch_bounds__(kBigThreads) big_mr_kernel(const __grid_constant__ BigArgs a, uint32_t k0) {
  const uint32_t nsurv = *a.nsurv;
  for (uint32_t t = blockIdx.x * kBigThreads + threadIdx.x; t < nsurv; t += gridDim.x * kBigThreads) {
    const uint32_t i = a.surv[t];
    if (i >= *a.best) continue;  // a smaller candidate already passed
    const uint32_t p = a.primes[k0 + i];
    uint32_t q[N];
    uint64_t b = p;
    for (int j = 0; j < N; ++j) {  // q = n - p
      const uint64_t v = (uint64_t)a.n[j] - (uint32_t)b - (b >> 32);
      q[j] = (uint32_t)v;
      b = ((v >> 32) & 1) << 32;
    }
    atomicAdd(a.mr_tests, 1ull);
    if (big_is_probable_prime<N>(q)) atomicMin(a.best, i);
  }
}

cudaError_t launch_big_filter(const BigArgs& a, uint32_t k0, uint32_t kcount, cudaStream_t s) {
  big_filter_kernel<<<(kcount + 255) / 256, 256, 0, s>>>(a, k0, kcount);
  return cudaGetLastError();
}

cudaError_t launch_big_mr(const BigArgs& a, uint32_t k0, int grid, cudaStream_t s) {
  switch (a.limbs) {
    case 4: big_mr_kernel<4><<<grid, kBigThreads, 0, s>>>(a, k0); break;
    case 8: big_mr_kernel<8><<<grid, kBigThreads, 0, s>>>(a, k0); break;
    case 16: big_mr_kernel<16><<<grid, kBigThreads, 0, s>>>(a, k0); break;
    case 32: big_mr_kernel<32><<<grid, kBigThreads, 0, s>>>(a, k0); break;
    case 64: big_mr_kernel<64><<<grid, kBigThreads, 0, s>>>(a, k0); break;
    case 128: big_mr_kernel<128><<<grid, kBigThreads, 0, s>>>(a, k0); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace gb
