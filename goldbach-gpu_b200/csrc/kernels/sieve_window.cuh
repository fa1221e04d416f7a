// sieve_window.cuh -- odd-only window sieve in shared memory (sm_100a).
//
// Replaces the reference's tiled_sieve_segment_kernel (src/goldbach.cu:
// 198-259).  Differences that matter for speed and correctness:
//   * primes 3..67 are not marked one multiple at a time: seven periodic
//     wheel patterns (gb_device.cuh) are ANDed into every word;
//   * the first multiple of each sieving prime comes from a Barrett
//     reduction (one 64-bit mulhi) instead of a 64-bit division;
//   * primes with many multiples in the window are marked by a whole warp
//     (lane l takes multiples l, l+32, ...), the rest by one thread each;
//   * every clear is an atomicAnd on shared memory.  The reference's
//     `sh_tile[w] &= ~mask` (src/goldbach.cu:250) is a plain read-modify-
//     write that loses clears when two threads hit one word.
#pragma once
#include "../gb_device.cuh"

namespace gb {

// Index (within the window) of the first odd multiple of p that is >= p^2
// and inside the window; the window starts at odd q0 = 2*g0 + 1.  Returns a
// value >= limit when there is none below `limit`.
__device__ __forceinline__ uint64_t first_mark(int64_t g0, uint32_t p, uint64_t magic) {
  const uint64_t pp = (uint64_t)p * p;
  const uint64_t gpp = (pp - 1) >> 1;  // odd index of p^2
  if (g0 < 0 || (uint64_t)g0 <= gpp) return gpp - (uint64_t)g0;  // start at p^2
  const uint64_t q0 = 2 * (uint64_t)g0 + 1;
  uint32_t r = mod_p(q0, p, magic);
  uint64_t delta = r ? p - r : 0;  // q0 + delta: first multiple >= q0 (64-bit: + p below
                                   // may pass 2^32 for the primes near 2^32 of q near 2^64)
  if (!(delta & 1)) {              // q0 odd: the multiple is odd iff delta even
  } else {
    delta += p;
  }
  return delta >> 1;
}

// first_mark with the remainder from a double-precision quotient estimate
// (inv = 1/p correctly rounded; p >= 2^13) and gpp = (p^2 - 1) / 2 given.
__device__ __forceinline__ uint64_t first_mark_f64(int64_t g0, uint32_t p, double inv,
                                                   uint64_t gpp) {
  if (g0 < 0 || (uint64_t)g0 <= gpp) return gpp - (uint64_t)g0;  // start at p^2
  const uint64_t q0 = 2 * (uint64_t)g0 + 1;
  const uint32_t r = mod_p_f64(q0, p, inv);
  uint64_t delta = r ? p - r : 0;  // q0 + delta: the first multiple >= q0
  if (delta & 1) delta += p;       // q0 is odd: the multiple is odd iff delta is even
  return delta >> 1;
}

// Sieves bits [0, nbits) of the window into Q (nwords words are written;
// nwords*32 >= nbits).  Bit i <-> q = 2*(g0 + i) + 1; set iff q is prime,
// exact for every q <= q_top (q_top <= 2*(g0+nbits)-1).  `pat` is the
// wheel pattern table in shared memory.  primes[kWheelPrimeCount+1 ..
// nsieve) are the marking primes (71, 73, ...); those below kcoop are
// marked warp-cooperatively.  Ends with __syncthreads().
template <int NT>
__device__ void sieve_window(uint32_t* __restrict__ Q, uint32_t nwords, uint32_t nbits,
                             int64_t g0, uint64_t q_top, const uint32_t* __restrict__ pat,
                             const uint32_t* __restrict__ primes,
                             const uint64_t* __restrict__ magic, uint32_t nsieve,
                             uint32_t kcoop) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  constexpr int NW = NT / 32;

  // 1. wheel fill: word t covers odd indices g0 + 32t .. +31.
  {
    uint32_t r[kWheelGroups];
    const int64_t g = g0 + 32 * (int64_t)tid;
#pragma unroll
    for (int x = 0; x < kWheelGroups; ++x) {
      const int64_t P = wheel_period(x);
      int64_t m = g % P;
      if (m < 0) m += P;
      r[x] = (uint32_t)m;
    }
    for (uint32_t t = tid; t < nwords; t += NT) {
      uint32_t w = 0xffffffffu;
#pragma unroll
      for (int x = 0; x < kWheelGroups; ++x) {
        const uint32_t P = wheel_period(x);
        const uint32_t step = (uint32_t)((32ull * NT) % P);
        const uint32_t rr = r[x];
        const uint32_t* pp = pat + wheel_offset(x) + (rr >> 5);
        w &= __funnelshift_r(pp[0], pp[1], rr & 31);
        uint32_t nr = rr + step;
        r[x] = nr >= P ? nr - P : nr;
      }
      Q[t] = w;
    }
  }
  __syncthreads();

  // 2. the first window: no odd number below 3 is prime, and the wheel
  //    primes themselves were cleared by their own patterns.
  if (g0 < 34) {
    const int64_t hi = 34 - g0 < (int64_t)nbits ? 34 - g0 : (int64_t)nbits;
    for (int64_t i = tid; i < hi; i += NT) {
      const int64_t gi = g0 + i;
      const int64_t q = 2 * gi + 1;
      bool prime = false;
      if (q >= 3 && q <= kWheelMaxPrime) {
        prime = true;
        for (int d = 3; d * d <= q; d += 2)
          if (q % d == 0) prime = false;
      }
      const uint32_t bit = 1u << (i & 31);
      if (prime) atomicOr(&Q[i >> 5], bit);
      else atomicAnd(&Q[i >> 5], ~bit);
    }
    __syncthreads();
  }

  // 3. warp-cooperative marking of primes with many multiples.
  const uint32_t kfirst = kWheelPrimeCount + 1;
  const uint32_t kc = kcoop < nsieve ? kcoop : nsieve;
  for (uint32_t k = kfirst + warp; k < kc; k += NW) {
    const uint32_t p = __ldg(primes + k);
    if ((uint64_t)p * p > q_top) break;
    const uint64_t f = first_mark(g0, p, __ldg(magic + k));
    if (f >= nbits) continue;
    const uint32_t stride = 32 * p;
    for (uint32_t i = (uint32_t)f + lane * p; i < nbits; i += stride)
      atomicAnd(&Q[i >> 5], ~(1u << (i & 31)));
  }
  // 4. one thread per prime for the rest.  (Loading four primes per step
  //    to overlap their table loads measured slower: 5.4 vs 4.2 ms for 2^30
  //    n near 1e12.)
  for (uint32_t k = (kc > kfirst ? kc : kfirst) + tid; k < nsieve; k += NT) {
    const uint32_t p = __ldg(primes + k);
    if ((uint64_t)p * p > q_top) break;
    const uint64_t f = first_mark(g0, p, __ldg(magic + k));
    for (uint64_t i = f; i < nbits; i += p) atomicAnd(&Q[i >> 5], ~(1u << (i & 31)));
  }
  __syncthreads();
}

}  // namespace gb
