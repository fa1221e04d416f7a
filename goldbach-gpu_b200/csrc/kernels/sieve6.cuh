// sieve6.cuh -- mod-6 window sieve in shared memory (sm_100a).
//
// Same job as sieve_window.cuh (and as the reference's
// tiled_sieve_segment_kernel, src/goldbach.cu:198-259), on a layout that
// never stores a multiple of 3: the window's odd q not divisible by 3 are
// split into two class bitsets,
//     Q1: bit t <-> q = 6(G0+t) + 1,      Q5: bit t <-> q = 6(G0+t) + 5,
// which together hold 1/3 of the numbers (the odd-only layout holds 1/2).
// Each prime p >= 5 has one multiple in every 6p numbers per class, so in
// both bitsets its multiples are p bits apart: the sieve marks 2/3 of the
// bits it would mark odd-only.  The first multiple in a window costs one
// reduction r = G0 mod p for both classes (a double-precision quotient
// estimate where the window allows it, else Barrett), using the per-prime
// class offsets a1 = -1/6 and a5 = -5/6 (mod p) kept with the prime table:
//     6(G0+t) + c == 0 (mod p)  <=>  t == a_c - r (mod p).
#pragma once
#include "../gb_device.cuh"

namespace gb {

// First t >= 0 of class c (offset a_c, r = G0 mod p) whose q is >= p^2.
__device__ __forceinline__ uint64_t first_mark6(int64_t G0, uint32_t p, uint32_t ac, uint32_t r,
                                               uint32_t c) {
  uint64_t t = ac >= r ? ac - r : ac + p - r;
  // q(t) = 6(G0 + t) + c is below p^2 only in windows that start below p^2;
  // compared in G (q itself may not fit an int64 near 2^64)
  const uint64_t pp = (uint64_t)p * p;
  const int64_t gmin = (int64_t)((pp - c + 5) / 6);  // first G with 6G + c >= p^2
  if (G0 + (int64_t)t < gmin) {
    const int64_t tmin = gmin - G0;
    t += (uint64_t)p * (((uint64_t)(tmin - (int64_t)t) + p - 1) / p);
  }
  return t;
}

// First marks of p in both classes as 32-bit offsets, lim (>= every
// in-window offset) when there is none below it.  The p^2 clamp of
// first_mark6 is needed only when the window starts below p^2 + 4 (6 G0 is
// compared, not computed per class).
__device__ __forceinline__ void first_marks6(int64_t G0, uint32_t p, uint2 ac, uint32_t r,
                                             uint32_t lim, uint32_t& t1, uint32_t& t5) {
  const uint64_t pp = (uint64_t)p * p;
  if (G0 < 0 || 6 * (uint64_t)G0 < pp + 4) {
    const uint64_t f1 = first_mark6(G0, p, ac.x, r, 1);
    const uint64_t f5 = first_mark6(G0, p, ac.y, r, 5);
    t1 = f1 < lim ? (uint32_t)f1 : lim;
    t5 = f5 < lim ? (uint32_t)f5 : lim;
  } else {
    const uint32_t a = ac.x >= r ? ac.x - r : ac.x + p - r;  // < p
    const uint32_t b = ac.y >= r ? ac.y - r : ac.y + p - r;
    t1 = a < lim ? a : lim;
    t5 = b < lim ? b : lim;
  }
}

// r = G0 mod p for a signed window base.
__device__ __forceinline__ uint32_t base_mod(int64_t G0, uint32_t p, uint64_t magic) {
  if (G0 >= 0) return mod_p((uint64_t)G0, p, magic);
  const uint32_t m = mod_p((uint64_t)(-G0), p, magic);
  return m ? p - m : 0;
}

// floor(sqrt(x)), at most 2^32 - 1.
__device__ __forceinline__ uint32_t isqrt64(uint64_t x) {
  uint64_t r = (uint64_t)sqrt((double)x);
  if (r > 0xffffffffull) r = 0xffffffffull;
  while (r * r > x) --r;
  while (r < 0xffffffffull && (r + 1) * (r + 1) <= x) ++r;
  return (uint32_t)r;
}

// r = G0 mod p from a double-precision quotient estimate, for 0 <= G0 <
// 2^53 and p < 2^31; gs = G0 / 2^64 (exact), gl = G0 mod 2^32.  With
// magic = floor((2^64 - 1) / p), G0 magic / 2^64 is within 2 G0 / 2^64 of
// G0 / p, and rounding magic to a double adds G0 / p * 2^-53 at most, so the
// estimate is within 1/4 of G0 / p; adding 1.5 * 2^52 rounds it to
// floor(G0 / p) or one more, held in the double's low bits.  G0 - p q then
// lies in (-p, p), and 32-bit arithmetic finishes it.
__device__ __forceinline__ uint32_t near_mod(double gs, uint32_t gl, uint32_t p, uint64_t magic) {
  const double est = fma(gs, __ull2double_rn(magic), 6755399441055744.0);  // + 1.5 * 2^52
  const uint32_t r = gl - (uint32_t)__double_as_longlong(est) * p;
  return min(r, r + p);
}

// First marks of both classes, for a window that starts at or above
// p^2 + 4 (first_marks6's short path, unclamped): both < p.
__device__ __forceinline__ void near_marks6(uint32_t p, uint2 ac, uint32_t r, uint32_t& t1, uint32_t& t5) {
  t1 = ac.x >= r ? ac.x - r : ac.x + p - r;
  t5 = ac.y >= r ? ac.y - r : ac.y + p - r;
}

// First marks t1, t5 of p in the window (>= nbits: none below it).  fastr:
// the window allows near_mod (p < 2^31 for every p used); near: p <= the
// window's psafe, so both offsets are below p.  With both, each offset is
// a - r wrapped into [0, p) by one unsigned min (a - r + p < 2^32).
__device__ __forceinline__ void window_marks6(bool fastr, bool near, double gs, uint32_t gl, int64_t G0,
                                              uint32_t p, uint64_t mg, uint2 ac, uint32_t nbits,
                                              uint32_t& t1, uint32_t& t5) {
  if (fastr && near) {
    const uint32_t r = near_mod(gs, gl, p, mg);
    t1 = ac.x - r;
    t1 = min(t1, t1 + p);
    t5 = ac.y - r;
    t5 = min(t5, t5 + p);
    return;
  }
  const uint32_t r = fastr ? near_mod(gs, gl, p, mg) : base_mod(G0, p, mg);
  if (near) near_marks6(p, ac, r, t1, t5);
  else first_marks6(G0, p, ac, r, nbits, t1, t5);
}

// Sieves bits [0, nbits) of both class bitsets (nwords words each written).
// Exact for every q <= q_top.  pat6: the class wheel patterns (shared
// memory).  primes[kWheelPrimeCount+1 .. nsieve) are the marking primes
// (71, 73, ...), those below kcoop marked warp-cooperatively.  With a mask
// (L1 non-null), word t of each class is also ANDed with the 32 mask bits
// from bit lsh of word t of L1 / L5 (the multiples of the primes beyond
// nsieve, cleared by the windows' large-prime pass); the mask must hold
// nwords + 1 words from there.  Ends with __syncthreads().
template <int NT>
__device__ void sieve_window6(uint32_t* __restrict__ Q1, uint32_t* __restrict__ Q5,
                              uint32_t nwords, uint32_t nbits, int64_t G0, uint64_t q_top,
                              const uint32_t* __restrict__ pat6,
                              const uint32_t* __restrict__ primes,
                              const uint64_t* __restrict__ magic, const uint2* __restrict__ a15,
                              uint32_t nsieve, uint32_t kcoop,
                              const uint32_t* __restrict__ L1 = nullptr,
                              const uint32_t* __restrict__ L5 = nullptr, uint32_t lsh = 0) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  constexpr int NW = NT / 32;

  // 1. wheel fill of both classes: each thread builds words t and t + 1
  //    (G0 + 32t .. +63) per step, from three pattern words per group.
#pragma unroll
  for (int cls5 = 0; cls5 < 2; ++cls5) {
    uint32_t* Q = cls5 ? Q5 : Q1;
    uint32_t r[kWheel6Groups];
    const int64_t g = G0 + 64 * (int64_t)tid;
#pragma unroll
    for (int x = 0; x < kWheel6Groups; ++x) {
      const int64_t P = wheel6_period(x);
      int64_t m = g % P;
      if (m < 0) m += P;
      r[x] = (uint32_t)m;
    }
    for (uint32_t t = 2 * tid; t < nwords; t += 2 * NT) {
      uint32_t w0 = 0xffffffffu, w1 = 0xffffffffu;
#pragma unroll
      for (int x = 0; x < kWheel6Groups; ++x) {
        const uint32_t P = wheel6_period(x);
        const uint32_t step = (uint32_t)((64ull * NT) % P);
        const uint32_t rr = r[x];
        // bits [rr, rr + 64) of the pattern, which is stored to P + 64
        const uint32_t* pp = pat6 + wheel6_offset(cls5, x) + (rr >> 5);
        const uint32_t a = pp[0], b = pp[1], c = pp[2];
        w0 &= __funnelshift_r(a, b, rr & 31);
        w1 &= __funnelshift_r(b, c, rr & 31);
        const uint32_t nr = rr + step;
        r[x] = min(nr, nr - P);  // nr - P wraps above nr when nr < P
      }
      const bool two = t + 1 < nwords;
      if (L1) {  // the mask holds nwords + 1 words: word t + 2 only when t + 1 is in
        const uint32_t* L = cls5 ? L5 : L1;
        const uint32_t l1 = __ldg(L + t + 1);
        w0 &= __funnelshift_r(__ldg(L + t), l1, lsh);
        if (two) w1 &= __funnelshift_r(l1, __ldg(L + t + 2), lsh);
      }
      Q[t] = w0;
      if (two) Q[t + 1] = w1;
    }
  }
  __syncthreads();

  // 2. the first window: q < 5 (1 and below) is not prime, and the primes
  //    5..67 were cleared by their own patterns (q = 6G + c < 72 <=> G < 12).
  if (G0 < 12) {
    const int64_t hi = 12 - G0 < (int64_t)nbits ? 12 - G0 : (int64_t)nbits;
    for (int64_t i = tid; i < 2 * hi; i += NT) {
      const int cls5 = (int)(i >= hi);
      const int64_t t = cls5 ? i - hi : i;
      const int64_t q = 6 * (G0 + t) + (cls5 ? 5 : 1);
      bool prime = q >= 5;
      for (int d = 5; prime && d * d <= q; d += 2)
        if (q % d == 0) prime = false;
      uint32_t* Q = cls5 ? Q5 : Q1;
      const uint32_t bit = 1u << (t & 31);
      if (prime) atomicOr(&Q[t >> 5], bit);
      else atomicAnd(&Q[t >> 5], ~bit);
    }
    __syncthreads();
  }

  // 3. primes with many multiples: one warp per prime, both classes
  //    (stride 32p stays far below 2^32: these primes are < nbits / 64).
  const uint32_t kfirst = kWheelPrimeCount + 1;
  const uint32_t kc = kcoop < nsieve ? kcoop : nsieve;
  // the window's prime bounds, in 32 bits: p <= plim <=> p^2 <= q_top, and
  // p <= psafe <=> the window starts at or above p^2 + 4 (the short path
  // of the first marks)
  const uint32_t plim = isqrt64(q_top);
  const uint32_t psafe = G0 >= 1 ? isqrt64(6 * (uint64_t)G0 - 4) : 0u;
  // r = G0 mod p by the quotient estimate where the window allows it
  // (every prime used is <= plim)
  const bool fastr = G0 >= 0 && G0 < (1ll << 53) && plim < 0x80000000u;
  const double gs = (double)G0 * 0x1p-64;
  const uint32_t gl = (uint32_t)G0;
  {  // the next prime's table entries are loaded one iteration ahead
    uint32_t k = kfirst + warp;
    uint32_t pn = 0;
    uint64_t mn = 0;
    uint2 an = make_uint2(0, 0);
    if (k < kc) { pn = __ldg(primes + k); mn = __ldg(magic + k); an = __ldg(a15 + k); }
    for (; k < kc; k += NW) {
      const uint32_t p = pn;
      const uint64_t mg = mn;
      const uint2 ac = an;
      if (k + NW < kc) { pn = __ldg(primes + k + NW); mn = __ldg(magic + k + NW); an = __ldg(a15 + k + NW); }
      if (p > plim) break;
      uint32_t t1, t5;
      window_marks6(fastr, p <= psafe, gs, gl, G0, p, mg, ac, nbits, t1, t5);
      const uint32_t stride = 32 * p;
#pragma unroll 16
      for (uint32_t i = t1 + lane * p; i < nbits; i += stride)
        atomicAnd(&Q1[i >> 5], ~(1u << (i & 31)));
#pragma unroll 16
      for (uint32_t i = t5 + lane * p; i < nbits; i += stride)
        atomicAnd(&Q5[i >> 5], ~(1u << (i & 31)));
    }
  }
  // 4. one thread per prime for the rest, both classes in one loop; primes
  //    >= nbits (possibly near 2^32) take a loop-free body.
  {  // the next prime's table entries are loaded one iteration ahead
    uint32_t k = (kc > kfirst ? kc : kfirst) + tid;
    uint32_t pn = 0;
    uint64_t mn = 0;
    uint2 an = make_uint2(0, 0);
    if (k < nsieve) { pn = __ldg(primes + k); mn = __ldg(magic + k); an = __ldg(a15 + k); }
    for (; k < nsieve; k += NT) {
      const uint32_t p = pn;
      const uint64_t mg = mn;
      const uint2 ac = an;
      if (k + NT < nsieve) { pn = __ldg(primes + k + NT); mn = __ldg(magic + k + NT); an = __ldg(a15 + k + NT); }
      if (p > plim) break;
      uint32_t j1, j5;  // offsets >= nbits mean no mark
      window_marks6(fastr, p <= psafe, gs, gl, G0, p, mg, ac, nbits, j1, j5);
      if (p >= nbits) {  // at most one multiple per class: no loop (no divergent exits)
        if (j1 < nbits) atomicAnd(&Q1[j1 >> 5], ~(1u << (j1 & 31)));
        if (j5 < nbits) atomicAnd(&Q5[j5 >> 5], ~(1u << (j5 & 31)));
        continue;
      }
      // p < nbits here: j + p stays below 2 nbits < 2^32
      while (j1 < nbits || j5 < nbits) {  // two marks per class per pass
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (j1 < nbits) {
            atomicAnd(&Q1[j1 >> 5], ~(1u << (j1 & 31)));
            j1 += p;
          }
          if (j5 < nbits) {
            atomicAnd(&Q5[j5 >> 5], ~(1u << (j5 & 31)));
            j5 += p;
          }
        }
      }
    }
  }
  __syncthreads();
}

}  // namespace gb
