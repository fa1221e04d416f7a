// big.cu -- Goldbach partitions of even n beyond 2^64 (multi-precision).
//
// Replaces big_check (src/big_check.cpp:35-144), which scans the primes up
// to 1e7 in OpenMP batches of 1000 and keeps the first q = n - p that GMP's
// mpz_probab_prime_p(q, 25) accepts -- a valid partition, not guaranteed
// the minimal one.  Here the candidates p (ascending, from the resident
// prime table) are tested in batches (host/gb_big.cpp):
//   1. big_filter_kernel: one thread per candidate drops q = n - p when a
//      trial prime r divides it, from n mod r (computed on the host once per
//      n) and p mod r, and appends the survivors' indices;
//   2. big_base2_kernel<N>: one thread per survivor runs the strong
//      probable-prime test to base 2 and lists the passers (almost all of
//      them primes);
//   3. big_bases_kernel<N>: one thread per (passer, base) runs the 11 other
//      bases 3, 5, ..., 37 -- with base 2 the base set of the reference's
//      Miller-Rabin (src/goldbach.cu:333-360) -- in parallel, so a prime q
//      costs two exponentiations of latency, not twelve.
// The smallest passer no base rejects is the minimal p: every smaller
// candidate was tested and failed.  The test is deterministic for
// q < 3.3e24 (the 12 prime bases admit no strong pseudoprime below that) and
// a probable-prime test beyond, like the reference's.
//
// The Montgomery product is the coarsely integrated operand-scanning form
// (CIOS) on 32-bit limbs with 64-bit accumulators, R = 2^(32 nl) for n of
// nl limbs; the arrays are sized by the template width N (a power of two
// from 4 to 128, n up to 4096 bits) and the loops run over nl.  Operands
// live in the thread's local memory for the wide sizes.
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
                             uint32_t qinv, int nl) {
  constexpr int U = N <= 16 ? N : 4;
  uint32_t t[N + 2];
#pragma unroll
  for (int j = 0; j < N + 2; ++j) t[j] = 0;
  for (int i = 0; i < nl; ++i) {
    const uint32_t yi = y[i];
    uint64_t c = 0;
#pragma unroll U
    for (int j = 0; j < nl; ++j) {
      const uint64_t v = (uint64_t)x[j] * yi + t[j] + c;
      t[j] = (uint32_t)v;
      c = v >> 32;
    }
    uint64_t v = (uint64_t)t[nl] + c;
    t[nl] = (uint32_t)v;
    t[nl + 1] = (uint32_t)(v >> 32);
    const uint32_t m = t[0] * qinv;
    v = (uint64_t)m * q[0] + t[0];
    c = v >> 32;
#pragma unroll U
    for (int j = 1; j < nl; ++j) {
      v = (uint64_t)m * q[j] + t[j] + c;
      t[j - 1] = (uint32_t)v;
      c = v >> 32;
    }
    v = (uint64_t)t[nl] + c;
    t[nl - 1] = (uint32_t)v;
    t[nl] = t[nl + 1] + (uint32_t)(v >> 32);
  }
  // t < 2q: subtract q once if t >= q
  bool ge = t[nl] != 0;
  if (!ge) {
    ge = true;  // equal counts as >=
    for (int j = nl - 1; j >= 0; --j)
      if (t[j] != q[j]) {
        ge = t[j] > q[j];
        break;
      }
  }
  if (ge) {
    uint64_t b = 0;
    for (int j = 0; j < nl; ++j) {
      const uint64_t v = (uint64_t)t[j] - q[j] - b;
      r[j] = (uint32_t)v;
      b = (v >> 32) & 1;
    }
  } else {
    for (int j = 0; j < nl; ++j) r[j] = t[j];
  }
}

// x = 2x mod q (x < q).
template <int N>
__device__ void big_dbl_mod(uint32_t* x, const uint32_t* q, int nl) {
  uint32_t top = 0;
  for (int j = 0; j < nl; ++j) {
    const uint32_t nt = x[j] >> 31;
    x[j] = (x[j] << 1) | top;
    top = nt;
  }
  bool ge = top != 0;
  if (!ge) {
    ge = true;
    for (int j = nl - 1; j >= 0; --j)
      if (x[j] != q[j]) {
        ge = x[j] > q[j];
        break;
      }
  }
  if (ge) {
    uint64_t b = 0;
    for (int j = 0; j < nl; ++j) {
      const uint64_t v = (uint64_t)x[j] - q[j] - b;
      x[j] = (uint32_t)v;
      b = (v >> 32) & 1;
    }
  }
}

__device__ __forceinline__ bool big_eq(const uint32_t* x, const uint32_t* y, int nl) {
  for (int j = 0; j < nl; ++j)
    if (x[j] != y[j]) return false;
  return true;
}

// Strong probable-prime test of odd q (> 2^64, nl limbs) to base kBigBases[bi].
template <int N>
__device__ bool big_sprp(const uint32_t* q, int nl, int bi) {
  uint32_t qinv = q[0];  // -q^-1 mod 2^32 by Newton steps
  for (int i = 0; i < 4; ++i) qinv *= 2u - q[0] * qinv;
  qinv = 0u - qinv;
  // one = R mod q, r2 = R^2 mod q (R = 2^(32 nl)), by doublings of 1
  uint32_t one[N], r2[N], mone[N], d[N], base[N], x[N];
  for (int j = 0; j < nl; ++j) one[j] = 0;
  one[0] = 1;
  for (int i = 0; i < 32 * nl; ++i) big_dbl_mod<N>(one, q, nl);
  for (int j = 0; j < nl; ++j) r2[j] = one[j];
  for (int i = 0; i < 32 * nl; ++i) big_dbl_mod<N>(r2, q, nl);
  {  // mone = q - one (that is -1 in Montgomery form)
    uint64_t b = 0;
    for (int j = 0; j < nl; ++j) {
      const uint64_t v = (uint64_t)q[j] - one[j] - b;
      mone[j] = (uint32_t)v;
      b = (v >> 32) & 1;
    }
  }
  // q - 1 = d 2^s
  int s = 0;
  {
    int lw = 0;
    while (lw < nl && (q[lw] & ~(lw == 0 ? 1u : 0u)) == 0) ++lw;  // q - 1 has its lowest set bit here
    const uint32_t low = lw == 0 ? (q[0] & ~1u) : q[lw];
    s = 32 * lw + __ffs(low) - 1;
    for (int j = 0; j < nl; ++j) d[j] = q[j];
    d[0] &= ~1u;  // q - 1 (q odd)
    const int ws = s >> 5, bs = s & 31;
    for (int j = 0; j < nl; ++j) {
      const uint32_t lo = j + ws < nl ? d[j + ws] : 0;
      const uint32_t hi = j + ws + 1 < nl ? d[j + ws + 1] : 0;
      d[j] = bs ? (lo >> bs) | (hi << (32 - bs)) : lo;
    }
  }
  int top = nl - 1;
  while (top > 0 && d[top] == 0) --top;
  const int nbits = 32 * top + 32 - __clz(d[top]);
  uint32_t a[N];
  for (int j = 0; j < nl; ++j) a[j] = 0;
  a[0] = kBigBases[bi];
  big_mont_mul<N>(base, a, r2, q, qinv, nl);  // the base in Montgomery form
  for (int j = 0; j < nl; ++j) x[j] = base[j];
  for (int b = nbits - 2; b >= 0; --b) {
    big_mont_mul<N>(x, x, x, q, qinv, nl);
    if ((d[b >> 5] >> (b & 31)) & 1u) big_mont_mul<N>(x, x, base, q, qinv, nl);
  }
  if (big_eq(x, one, nl) || big_eq(x, mone, nl)) return true;
  for (int i = 1; i < s; ++i) {
    big_mont_mul<N>(x, x, x, q, qinv, nl);
    if (big_eq(x, mone, nl)) return true;
    if (big_eq(x, one, nl)) return false;
  }
  return false;
}

// q = n - p on nl limbs.
template <int N>
__device__ __forceinline__ void big_q(const BigArgs& a, uint32_t p, uint32_t* q) {
  uint32_t borrow = 0;
  for (int j = 0; j < (int)a.nl; ++j) {
    const uint64_t v = (uint64_t)a.n[j] - (j == 0 ? p : 0u) - borrow;
    q[j] = (uint32_t)v;
    borrow = (uint32_t)(v >> 32) & 1u;
  }
}

// Phase 0: base 2 on every survivor; the candidates that pass it join the
// passers list (each with a slot of 11 later verdicts).
template <int N>
__global__ void __launch_bounds__(kBigThreads) big_base2_kernel(const __grid_constant__ BigArgs a, uint32_t k0) {
  const uint32_t nsurv = *a.nsurv;
  for (uint32_t t = blockIdx.x * kBigThreads + threadIdx.x; t < nsurv; t += gridDim.x * kBigThreads) {
    const uint32_t i = a.surv[t];
    uint32_t q[N];
    big_q<N>(a, a.primes[k0 + i], q);
    atomicAdd(a.mr_tests, 1ull);
    if (big_sprp<N>(q, (int)a.nl, 0)) {
      const uint32_t slot = atomicAdd(a.npass, 1u);
      a.pass[slot] = i;
      a.fail[slot] = 0;
    }
  }
}

// Phase 1: the 11 other bases, one thread per (passer, base); a failing
// base marks its passer.
template <int N>
__global__ void __launch_bounds__(kBigThreads) big_bases_kernel(const __grid_constant__ BigArgs a, uint32_t k0) {
  const uint32_t work = *a.npass * 11u;
  for (uint32_t t = blockIdx.x * kBigThreads + threadIdx.x; t < work; t += gridDim.x * kBigThreads) {
    const uint32_t slot = t / 11u, bi = 1 + t % 11u;
    uint32_t q[N];
    big_q<N>(a, a.primes[k0 + a.pass[slot]], q);
    if (!big_sprp<N>(q, (int)a.nl, (int)bi)) atomicOr(&a.fail[slot], 1u);
  }
}

cudaError_t launch_big_filter(const BigArgs& a, uint32_t k0, uint32_t kcount, cudaStream_t s) {
  big_filter_kernel<<<(kcount + 255) / 256, 256, 0, s>>>(a, k0, kcount);
  return cudaGetLastError();
}

cudaError_t launch_big_mr(const BigArgs& a, uint32_t k0, int phase, int grid, cudaStream_t s) {
#define GB_BIG_CASE(W)                                                        \
  case W:                                                                     \
    if (phase == 0) big_base2_kernel<W><<<grid, kBigThreads, 0, s>>>(a, k0);  \
    else big_bases_kernel<W><<<grid, kBigThreads, 0, s>>>(a, k0);             \
    break;
  switch (a.limbs) {
    GB_BIG_CASE(4)
    GB_BIG_CASE(8)
    GB_BIG_CASE(16)
    GB_BIG_CASE(32)
    GB_BIG_CASE(64)
    GB_BIG_CASE(128)
    default: return cudaErrorInvalidValue;
  }
#undef GB_BIG_CASE
  return cudaGetLastError();
}

}  // namespace gb
