// gb_device.cuh -- device arithmetic shared by the sm_100a kernels.
//
//  * mod_p: x mod p for 64-bit x and a 32-bit prime p by a precomputed
//    Barrett reciprocal; replaces the per-thread 64-bit division of the
//    reference's tiled sieve (src/goldbach.cu:229).
//  * 64-bit Montgomery Miller-Rabin with the deterministic 7-base set;
//    replaces the (__uint128_t)a*b % m mulmod of src/goldbach.cu:119-158
//    and src/single_check.cu:30-88, which compiles to a software 128-bit
//    remainder on the GPU.
//  * the wheel: odd-only bit patterns of the primes 3..67, tiled over a
//    window instead of marking those primes one multiple at a time.
#pragma once
#include <cstdint>

#ifndef GB_HOST_ONLY
#define GB_HD __host__ __device__ __forceinline__
#else
#define GB_HD inline
#endif

namespace gb {

// ---------------------------------------------------------------------------
// Odd-only index convention (include/prime_bitset.hpp:7-8, generalised):
// a window starting at odd q0 holds bit i <-> q0 + 2i.  A global odd index
// g <-> q = 2g + 1 is used to tile the wheel patterns.

// Wheel groups: products of small odd primes whose composite pattern has a
// period small enough for shared memory.  Primes 3..67 are removed by the
// patterns; marking starts at 71.
constexpr int kWheelGroups = 7;
constexpr int kWheelMaxPrime = 67;
constexpr int kFirstMarkedPrime = 71;
// number of odd primes <= 67 (3,5,...,67): the index of 71 in an odd-prime list
constexpr int kWheelPrimeCount = 18;

struct WheelGroup {
  uint32_t period;   // product of the group's primes (in odd-index units)
  uint32_t offset;   // first word of the group's pattern in the pattern table
  uint32_t nprimes;
  uint32_t primes[5];
};

// Pattern storage: each group stores bits [0, period + 64) of its periodic
// pattern (bit b = 1 iff 2g+1 has no factor in the group for g = b mod period),
// rounded up to whole words plus one spare word for the funnel shift.
GB_HD constexpr uint32_t wheel_words(uint32_t period) { return (period + 64 + 31) / 32 + 1; }

constexpr uint32_t kP0 = 3 * 5 * 7 * 11 * 13;  // 15015
constexpr uint32_t kP1 = 17 * 19 * 23;         // 7429
constexpr uint32_t kP2 = 29 * 31;              // 899
constexpr uint32_t kP3 = 37 * 41;              // 1517
constexpr uint32_t kP4 = 43 * 47;              // 2021
constexpr uint32_t kP5 = 53 * 59;              // 3127
constexpr uint32_t kP6 = 61 * 67;              // 4087
constexpr uint32_t kO0 = 0;
constexpr uint32_t kO1 = kO0 + wheel_words(kP0);
constexpr uint32_t kO2 = kO1 + wheel_words(kP1);
constexpr uint32_t kO3 = kO2 + wheel_words(kP2);
constexpr uint32_t kO4 = kO3 + wheel_words(kP3);
constexpr uint32_t kO5 = kO4 + wheel_words(kP4);
constexpr uint32_t kO6 = kO5 + wheel_words(kP5);
constexpr uint32_t kWheelWords = kO6 + wheel_words(kP6);

#ifndef GB_HOST_ONLY
__device__ __constant__ const WheelGroup kWheel[kWheelGroups] = {
    {kP0, kO0, 5, {3, 5, 7, 11, 13}}, {kP1, kO1, 3, {17, 19, 23, 0, 0}},
    {kP2, kO2, 2, {29, 31, 0, 0, 0}}, {kP3, kO3, 2, {37, 41, 0, 0, 0}},
    {kP4, kO4, 2, {43, 47, 0, 0, 0}}, {kP5, kO5, 2, {53, 59, 0, 0, 0}},
    {kP6, kO6, 2, {61, 67, 0, 0, 0}}};
#endif
GB_HD constexpr uint32_t wheel_period(int x) {
  return x == 0 ? kP0 : x == 1 ? kP1 : x == 2 ? kP2 : x == 3 ? kP3 : x == 4 ? kP4 : x == 5 ? kP5 : kP6;
}
GB_HD constexpr uint32_t wheel_offset(int x) {
  return x == 0 ? kO0 : x == 1 ? kO1 : x == 2 ? kO2 : x == 3 ? kO3 : x == 4 ? kO4 : x == 5 ? kO5 : kO6;
}

// ---------------------------------------------------------------------------
// Mod-6 layout.  Odd q not divisible by 3 are 6G+1 or 6G+5; the two class
// bitsets hold bit t <-> q = 6(G0+t)+c, c in {1, 5}.  The wheel for the
// primes 5..67 becomes one periodic pattern per (class, group) indexed by
// G mod period: bit x = 1 iff 6x+c has no factor in the group.
constexpr int kWheel6Groups = 7;
constexpr uint32_t kQ0 = 5 * 7 * 11 * 13;  // 5005
GB_HD constexpr uint32_t wheel6_period(int x) {
  return x == 0 ? kQ0 : x == 1 ? kP1 : x == 2 ? kP2 : x == 3 ? kP3 : x == 4 ? kP4 : x == 5 ? kP5 : kP6;
}
GB_HD constexpr uint32_t wheel6_group_offset(int x) {
  uint32_t o = 0;
  for (int i = 0; i < x; ++i) o += wheel_words(wheel6_period(i));
  return o;
}
constexpr uint32_t kWheel6ClassWords = wheel6_group_offset(kWheel6Groups);
constexpr uint32_t kWheel6Words = 2 * kWheel6ClassWords;  // class 1 groups, then class 5
GB_HD constexpr uint32_t wheel6_offset(int cls5, int x) {
  return (cls5 ? kWheel6ClassWords : 0) + wheel6_group_offset(x);
}

// ---------------------------------------------------------------------------
// Barrett: magic = floor((2^64-1)/p).  For every x < 2^64 the estimate
// floor(x*magic/2^64) is floor(x/p) or one less, so one correction suffices.
#ifndef GB_HOST_ONLY
__device__ __forceinline__ uint32_t mod_p(uint64_t x, uint32_t p, uint64_t magic) {
  uint64_t qt = __umul64hi(x, magic);
  uint64_t r = x - qt * (uint64_t)p;
  return (uint32_t)(r >= p ? r - p : r);
}

// The same remainder from a double-precision quotient estimate, inv the
// correctly rounded 1/p.  The conversion of x, inv and the product each
// carry a relative error of at most 2^-53, so the estimate is within
// 3 * 2^-53 * x/p < 1 of x / p whenever x / p < 2^51 (every x < 2^64 for
// p >= 2^13), its truncation is floor(x / p) - 1, + 0 or + 1, and one signed
// correction of the 64-bit remainder x - q p (in (-p, 2p)) finishes it.
__device__ __forceinline__ uint32_t mod_p_f64(uint64_t x, uint32_t p, double inv) {
  const uint64_t q = (uint64_t)(__ull2double_rn(x) * inv);
  int64_t r = (int64_t)(x - q * (uint64_t)p);
  if (r < 0) r += p;
  else if (r >= (int64_t)p) r -= p;
  return (uint32_t)r;
}

// ---------------------------------------------------------------------------
// Montgomery arithmetic modulo an odd 64-bit n, R = 2^64.
struct Mont {
  uint64_t n;     // modulus (odd)
  uint64_t ninv;  // -n^{-1} mod 2^64
  uint64_t one;   // R mod n (1 in Montgomery form)
};

__device__ __forceinline__ uint64_t mont_neg_inv(uint64_t n) {
  uint64_t x = n;          // n*n == 1 (mod 8): 3 correct bits
  x *= 2 - n * x;          // 6
  x *= 2 - n * x;          // 12
  x *= 2 - n * x;          // 24
  x *= 2 - n * x;          // 48
  x *= 2 - n * x;          // 96 >= 64
  return 0 - x;
}

__device__ __forceinline__ Mont mont_init(uint64_t n) {
  Mont m;
  m.n = n;
  m.ninv = mont_neg_inv(n);
  // 2^64 mod n: for n > 2^63 it is 2^64 - n, otherwise (2^64 - n) mod n.
  uint64_t t = 0 - n;
  m.one = (n >> 63) ? t : t % n;
  return m;
}

// a*b*R^{-1} mod n for a, b < n.  The 128-bit sum T + m*n is formed from
// high halves; the low halves cancel to 0 or 2^64 (carry = lo != 0).
__device__ __forceinline__ uint64_t mont_mul(uint64_t a, uint64_t b, const Mont& M) {
  uint64_t lo = a * b;
  uint64_t hi = __umul64hi(a, b);
  uint64_t m = lo * M.ninv;
  uint64_t mh = __umul64hi(m, M.n);
  uint64_t t = hi + mh;
  bool c = t < hi;
  uint64_t r = t + (lo != 0);
  c |= r < t;
  if (c || r >= M.n) r -= M.n;
  return r;
}

// The same product on 32-bit limbs with explicit carry chains (operand
// scanning: the 128-bit a*b, then one reduction step per limb with
// m = t_i * (-n^-1 mod 2^32), then one conditional subtraction picked by
// the borrow mask).  ninv0 is the low word of Mont::ninv.
__device__ __forceinline__ uint64_t mont_mul32(uint64_t a, uint64_t b, uint64_t n, uint32_t ninv0) {
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  const uint32_t n0 = (uint32_t)n, n1 = (uint32_t)(n >> 32);
  uint32_t r0, r1;
  asm("{\n\t"
      ".reg .u32 t0, t1, t2, t3, t4, m, s0, s1, bw;\n\t"
      "mul.lo.u32 t0, %2, %4;\n\t"
      "mul.hi.u32 t1, %2, %4;\n\t"
      "mad.lo.cc.u32 t1, %3, %4, t1;\n\t"
      "madc.hi.u32 t2, %3, %4, 0;\n\t"
      "mad.lo.cc.u32 t1, %2, %5, t1;\n\t"
      "madc.hi.cc.u32 t2, %2, %5, t2;\n\t"
      "addc.u32 t3, 0, 0;\n\t"
      "mad.lo.cc.u32 t2, %3, %5, t2;\n\t"
      "madc.hi.u32 t3, %3, %5, t3;\n\t"
      "mul.lo.u32 m, t0, %8;\n\t"
      "mad.lo.cc.u32 t0, m, %6, t0;\n\t"
      "madc.hi.cc.u32 t1, m, %6, t1;\n\t"
      "addc.cc.u32 t2, t2, 0;\n\t"
      "addc.cc.u32 t3, t3, 0;\n\t"
      "addc.u32 t4, 0, 0;\n\t"
      "mad.lo.cc.u32 t1, m, %7, t1;\n\t"
      "madc.hi.cc.u32 t2, m, %7, t2;\n\t"
      "addc.cc.u32 t3, t3, 0;\n\t"
      "addc.u32 t4, t4, 0;\n\t"
      "mul.lo.u32 m, t1, %8;\n\t"
      "mad.lo.cc.u32 t1, m, %6, t1;\n\t"
      "madc.hi.cc.u32 t2, m, %6, t2;\n\t"
      "addc.cc.u32 t3, t3, 0;\n\t"
      "addc.u32 t4, t4, 0;\n\t"
      "mad.lo.cc.u32 t2, m, %7, t2;\n\t"
      "madc.hi.cc.u32 t3, m, %7, t3;\n\t"
      "addc.u32 t4, t4, 0;\n\t"
      "sub.cc.u32 s0, t2, %6;\n\t"
      "subc.cc.u32 s1, t3, %7;\n\t"
      "subc.u32 bw, t4, 0;\n\t"
      "lop3.b32 %0, t2, s0, bw, 0xE4;\n\t"
      "lop3.b32 %1, t3, s1, bw, 0xE4;\n\t"
      "}"
      : "=r"(r0), "=r"(r1)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1), "r"(n0), "r"(n1), "r"(ninv0));
  return ((uint64_t)r1 << 32) | r0;
}

__device__ __forceinline__ uint64_t mod_dbl(uint64_t a, uint64_t n) {
  uint64_t s = a + a;
  if (s < a || s >= n) s -= n;
  return s;
}

// Strong probable prime test to base 2 (n odd > 2, n-1 = d*2^s).  In
// Montgomery form, multiplying by the base 2 is a modular doubling.
__device__ __forceinline__ bool sprp2(const Mont& M, uint64_t d, int s) {
  uint64_t x = mod_dbl(M.one, M.n);  // 2 in Montgomery form
  int top = 63 - __clzll(d);
  for (int b = top - 1; b >= 0; --b) {
    x = mont_mul(x, x, M);
    if ((d >> b) & 1) x = mod_dbl(x, M.n);
  }
  const uint64_t mone = M.n - M.one;
  if (x == M.one || x == mone) return true;
  for (int i = 1; i < s; ++i) {
    x = mont_mul(x, x, M);
    if (x == mone) return true;
    if (x == M.one) return false;
  }
  return false;
}

// Strong probable prime test to a base given in Montgomery form.
__device__ __forceinline__ bool sprp_m(const Mont& M, uint64_t am, uint64_t d, int s) {
  uint64_t x = am;
  int top = 63 - __clzll(d);
  for (int b = top - 1; b >= 0; --b) {
    x = mont_mul(x, x, M);
    if ((d >> b) & 1) x = mont_mul(x, am, M);
  }
  const uint64_t mone = M.n - M.one;
  if (x == M.one || x == mone) return true;
  for (int i = 1; i < s; ++i) {
    x = mont_mul(x, x, M);
    if (x == mone) return true;
    if (x == M.one) return false;
  }
  return false;
}

// R^2 mod n from R mod n by 64 modular doublings.
__device__ __forceinline__ uint64_t mont_r2(const Mont& M) {
  uint64_t r = M.one;
#pragma unroll 8
  for (int i = 0; i < 64; ++i) r = mod_dbl(r, M.n);
  return r;
}

__device__ __constant__ const uint64_t kMR7Bases[7] = {2ULL,      325ULL,     9375ULL,
                                                       28178ULL,  450775ULL,  9780504ULL,
                                                       1795265022ULL};

// base k (1..6) of the 7-base set applied to odd n > 2^31 (so that the base
// is already reduced and non-zero mod n) or any odd n (reduced here).
__device__ __forceinline__ bool sprp_base_k(const Mont& M, uint64_t r2, int k, uint64_t d, int s) {
  uint64_t a = kMR7Bases[k];
  if (a >= M.n) a %= M.n;
  if (a == 0) return true;
  return sprp_m(M, mont_mul(a, r2, M), d, s);
}

// Deterministic primality for every 64-bit n: trial division by the primes
// <= 31, then strong tests to the 7 bases.  Composites below 37^2 have a
// factor <= 31, so the bases only see n >= 1369, where no base is 0 mod a
// composite n.
__device__ __forceinline__ bool is_prime_u64(uint64_t n) {
  if (n < 2) return false;
  if (!(n & 1)) return n == 2;
  const uint32_t sp[10] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31};
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    if (n == sp[i]) return true;
    if (n % sp[i] == 0) return false;
  }
  if (n < 1369) return true;
  uint64_t d = n - 1;
  int s = __ffsll((long long)d) - 1;
  d >>= s;
  Mont M = mont_init(n);
  if (!sprp2(M, d, s)) return false;
  uint64_t r2 = mont_r2(M);
#pragma unroll 1
  for (int k = 1; k < 7; ++k)
    if (!sprp_base_k(M, r2, k, d, s)) return false;
  return true;
}
#endif  // GB_HOST_ONLY

}  // namespace gb
