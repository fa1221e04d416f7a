// single.cu -- batched single-n minimal partitions and batched primality.
//
// Replaces goldbach_single_kernel + check_single (src/single_check.cu:
// 95-282).  The reference sieves p in chunks of 1e8 on the CPU, copies them
// to the GPU, runs one thread per p with a 128-bit-remainder Miller-Rabin
// and keeps whichever thread finishes first, so its p is not the minimal
// one.  Here every lane of a warp owns one query n (taken from a device work
// counter as it frees up) and walks the candidate primes p = 3, 5, 7, ...
// in order until q = n - p is prime:
//   1. candidates come in batches of 32 consecutive primes, filtered by the
//      whole warp for the query that needs them (lane i tests the i-th
//      prime): q is dropped when a prime r <= 61 divides it, tested on
//      x = q mod M for three products M of those primes (x = n mod M - p
//      mod M, n mod M computed once per query) by exact-division checks;
//   2. each lane runs one strong probable-prime test per round on its own
//      next survivor: base 2 first, then, for a base-2 pass, the six other
//      bases of the deterministic set one per round, so a query takes about
//      12 rounds (about 5.7 base-2 tests for n near 2^63) and every lane
//      does useful work in every round;
//   3. a round's exponentiation is uniform across the warp: a fixed 2-bit
//      window (squaring twice, then one product with 1, a, a^2 or a^3 picked
//      by the two exponent bits) over the warp's longest exponent, so lanes
//      with different q and bases never diverge.
// Queries n < 2^21 (where q may be a prime <= 61) take a warp-cooperative
// scan with the full test per candidate instead.  Small batches, where
// latency rather than throughput sets the time, take single_warp_kernel
// (one warp per query).
#include <cuda_runtime.h>

#include <cstdint>

#include "../gb_device.cuh"
#include "../gb_internal.h"

namespace gb {

constexpr int kSingleThreads = 256;
constexpr uint64_t kSmallN = 1ull << 21;  // below this, q may be tiny: plain path
constexpr uint32_t kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Lane-parallel ascending scan with the full primality test per lane (the
// whole warp serves one n).
__device__ uint32_t minp_plain(const SingleArgs& a, uint64_t n, uint64_t lim) {
  const int lane = threadIdx.x & 31;
  for (uint64_t k = 1;; k += 32) {
    const uint64_t kk = k + lane;
    const uint32_t p = kk < a.nprimes ? a.primes[kk] : 0xffffffffu;
    const bool valid = kk < a.nprimes && p <= lim;
    const bool ok = valid && is_prime_u64(n - p);
    const uint32_t b = __ballot_sync(kFull, ok);
    if (b) return __shfl_sync(kFull, p, __ffs(b) - 1);
    if (__ballot_sync(kFull, valid) != kFull) return 0;
  }
}

// Exact division by an odd r on 32-bit x: x * r^-1 (mod 2^32) lands in
// [0, (2^32-1)/r] exactly for the multiples of r.
__host__ __device__ constexpr uint32_t inv32(uint32_t r) {
  uint32_t x = r;  // r*r == 1 (mod 8)
  for (int i = 0; i < 4; ++i) x *= 2u - r * x;
  return x;
}
template <uint32_t R>
__device__ __forceinline__ bool divides(uint32_t x) {
  constexpr uint32_t kInv = inv32(R), kLim = 0xffffffffu / R;
  static_assert(R * kInv == 1u, "inverse");
  return x * kInv <= kLim;
}

constexpr uint32_t kM1 = 3u * 5 * 7 * 11 * 13 * 17 * 19 * 23;  // 111546435
constexpr uint32_t kM2 = 29u * 31 * 37 * 41 * 43;              // 58642669
constexpr uint32_t kM3 = 47u * 53 * 59 * 61;                   // 8965109

// q = n - p has no prime factor <= 61, from n mod M1, M2, M3.
__device__ __forceinline__ bool no_small_factor(uint32_t nm1, uint32_t nm2, uint32_t nm3,
                                                uint32_t p) {
  uint32_t x = nm1 + kM1 - p % kM1;
  x = x >= kM1 ? x - kM1 : x;
  bool f = divides<3>(x) | divides<5>(x) | divides<7>(x) | divides<11>(x) | divides<13>(x) |
           divides<17>(x) | divides<19>(x) | divides<23>(x);
  uint32_t y = nm2 + kM2 - p % kM2;
  y = y >= kM2 ? y - kM2 : y;
  f |= divides<29>(y) | divides<31>(y) | divides<37>(y) | divides<41>(y) | divides<43>(y);
  uint32_t z = nm3 + kM3 - p % kM3;
  z = z >= kM3 ? z - kM3 : z;
  f |= divides<47>(z) | divides<53>(z) | divides<59>(z) | divides<61>(z);
  return !f;
}

// Montgomery context for mont_mul32: the modulus, -n^-1 mod 2^32 and R mod n.
struct Mont32 {
  uint64_t n;
  uint64_t one;
  uint32_t ni;
};

// R mod n without a 64-bit division: 2^(k+1) - n for the top bit k of n,
// then doubled up to 2^64 (no doubling for n >= 2^63).
__device__ __forceinline__ Mont32 mont32_init(uint64_t n) {
  Mont32 M;
  M.n = n;
  M.ni = 0u - inv32((uint32_t)n);
  const int k = 63 - __clzll(n);
  uint64_t x = k == 63 ? 0 - n : (2ull << k) - n;
  for (int j = k + 1; j < 64; ++j) x = mod_dbl(x, n);
  M.one = x;
  return M;
}

// Strong probable-prime test of every lane's odd modulus M.n = d 2^s + 1 to
// its base a1 (Montgomery form), the loop lengths set by the warp's longest
// exponent and largest s (lanes with act false only run along).
__device__ __forceinline__ bool sprp_warp(const Mont32& M, uint64_t a1, uint64_t d, int s, bool act) {
  const uint32_t ni = M.ni;
  const uint64_t a2 = mont_mul32(a1, a1, M.n, ni);
  const uint64_t a3 = mont_mul32(a2, a1, M.n, ni);
  const int top = 63 - __clzll(d);  // d >= 1
  const int T = (int)__reduce_max_sync(kFull, act ? (uint32_t)top : 0u) | 1;  // odd
  // bit pairs (i+1, i) from i = T-1 down to 0; the first pair starts x
  uint32_t b = (uint32_t)(d >> (T - 1)) & 3u;
  uint64_t x = b == 0 ? M.one : b == 1 ? a1 : b == 2 ? a2 : a3;
  for (int i = T - 3; i >= 0; i -= 2) {
    x = mont_mul32(x, x, M.n, ni);
    x = mont_mul32(x, x, M.n, ni);
    b = (uint32_t)(d >> i) & 3u;
    x = mont_mul32(x, b == 0 ? M.one : b == 1 ? a1 : b == 2 ? a2 : a3, M.n, ni);
  }
  const uint64_t mone = M.n - M.one;
  bool ok = x == M.one || x == mone;
  bool done = ok;
  const int S = (int)__reduce_max_sync(kFull, act ? (uint32_t)s : 0u);
  for (int i = 1; i < S; ++i) {
    x = mont_mul32(x, x, M.n, ni);
    if (!done && i < s) {
      if (x == mone) ok = done = true;
      else if (x == M.one) done = true;
    }
  }
  return ok;
}

__global__ void __launch_bounds__(kSingleThreads) single_kernel(SingleArgs a) {
  const int lane = threadIdx.x & 31;
  // the lane's query
  bool have = false, drained = false;
  uint64_t qi = 0, n = 0;
  uint32_t lim = 0, nm1 = 0, nm2 = 0, nm3 = 0;
  uint32_t kb = 1;      // prime index of the next candidate batch
  uint32_t cmask = 0;   // the current batch's survivors not yet tested
  uint32_t cbase = 0;   // prime index of the current batch's bit 0
  bool last = false;    // the current batch reached the end of the candidates
  int stage = 0;        // 0: next candidate, base 2; k = 1..6: base k of the set
  uint32_t p = 0;       // the candidate under test
  bool ready = false;   // p taken for this round (stage 0)
  Mont32 M{3, 1, 1};
  uint64_t d = 1, r2 = 0;
  int s = 1;
  uint32_t found = 0, maxp = 0;
  auto finish = [&](uint32_t pf) {
    a.p_out[qi] = pf;
    a.q_out[qi] = pf ? n - pf : 0;
    if (pf) {
      ++found;
      maxp = pf > maxp ? pf : maxp;
    }
    have = false;
  };
  for (;;) {
    // every lane gets a query with a candidate ready, or the queue is empty
    for (;;) {
      const uint32_t need = __ballot_sync(kFull, !have && !drained);
      if (need) {
        unsigned long long base = 0;
        if (lane == __ffs(need) - 1) base = atomicAdd(&a.ctr[0], (unsigned long long)__popc(need));
        base = __shfl_sync(kFull, base, __ffs(need) - 1);
        if (!have && !drained) {
          qi = base + __popc(need & lanemask_lt());
          if (qi >= a.count) {
            drained = true;
          } else {
            n = a.n[qi];
            have = true;
            stage = 0;
            kb = 1;
            cmask = 0;
            last = false;
            const uint64_t half = n >> 1;
            lim = (uint32_t)(half < a.p_lim ? half : a.p_lim);
            nm1 = (uint32_t)(n % kM1);
            nm2 = (uint32_t)(n % kM2);
            nm3 = (uint32_t)(n % kM3);
            if (n < 4 || (n & 1)) finish(0);
            else if (n == 4) finish(2);
          }
        }
      }
      // candidate batches for the lanes that ran out, one query at a time
      for (;;) {
        const uint32_t m = __ballot_sync(kFull, have && stage == 0 && !ready && cmask == 0 && !last);
        if (!m) break;
        const int j = __ffs(m) - 1;
        const uint64_t nj = __shfl_sync(kFull, n, j);
        const uint32_t limj = __shfl_sync(kFull, lim, j);
        if (nj < kSmallN) {
          const uint32_t pj = minp_plain(a, nj, limj);
          if (lane == j) finish(pj);
          continue;
        }
        const uint32_t kj = __shfl_sync(kFull, kb, j);
        const uint32_t m1 = __shfl_sync(kFull, nm1, j);
        const uint32_t m2 = __shfl_sync(kFull, nm2, j);
        const uint32_t m3 = __shfl_sync(kFull, nm3, j);
        const uint64_t k = (uint64_t)kj + lane;
        const uint32_t pk = k < a.nprimes ? a.primes[k] : 0xffffffffu;
        const bool valid = k < a.nprimes && pk <= limj;
        const uint32_t pass = __ballot_sync(kFull, valid && no_small_factor(m1, m2, m3, pk));
        const uint32_t vb = __ballot_sync(kFull, valid);
        if (lane == j) {
          cmask = pass;
          cbase = kj;
          kb = kj + 32;
          last = vb != kFull;
        }
      }
      // set up this round's test
      if (have && stage == 0 && !ready) {
        if (cmask == 0) {
          finish(0);  // every prime p <= min(n/2, p_lim) tried
        } else {
          const int bit = __ffs(cmask) - 1;
          cmask &= cmask - 1;
          p = a.primes[cbase + bit];
          ready = true;
        }
      }
      if (!__ballot_sync(kFull, !have && !drained)) break;
    }
    if (!__any_sync(kFull, have)) break;
    // one strong test per lane: base 2 of a new candidate, or base `stage`
    uint64_t am = 0;
    bool skip = false;
    if (have) {
      if (stage == 0) {
        const uint64_t q = n - p;
        d = q - 1;
        s = __ffsll((long long)d) - 1;
        d >>= s;
        M = mont32_init(q);
        am = mod_dbl(M.one, M.n);  // 2
      } else {
        uint64_t b = kMR7Bases[stage];
        if (b >= M.n) b %= M.n;
        skip = b == 0;
        am = mont_mul32(b, r2, M.n, M.ni);
      }
    }
    const bool ok = sprp_warp(M, am, d, s, have) || skip;
    ready = false;
    if (have) {
      if (!ok) {
        stage = 0;  // composite (a base-2 pseudoprime when stage > 0)
      } else if (stage == 0) {
        // R^2 mod q = 2^64 in Montgomery form: 2 squared six times
        uint64_t t = mod_dbl(M.one, M.n);
#pragma unroll
        for (int i = 0; i < 6; ++i) t = mont_mul32(t, t, M.n, M.ni);
        r2 = t;
        stage = 1;
      } else if (++stage == 7) {
        finish(p);
      }
    }
  }
  // the warp's counts, one atomic each
  found = __reduce_add_sync(kFull, found);
  maxp = __reduce_max_sync(kFull, maxp);
  if (lane == 0) {
    if (found) atomicAdd(&a.ctr[1], (unsigned long long)found);
    if (maxp) atomicMax(&a.ctr[2], (unsigned long long)maxp);
  }
}

// Latency path for small batches: one warp per query.  Survivors of the
// small-prime filter are gathered in order (shared memory) until 32 are
// pending; each lane runs the base-2 test on one of them, and the lowest
// lane that passed gets the six other bases, one base per lane.  A lone
// query then costs about two strong-test latencies instead of the dozen
// the lane-per-query kernel spends on it one after another.
__device__ uint32_t minp_warp(const SingleArgs& a, uint64_t n, uint32_t* buf) {
  const int lane = threadIdx.x & 31;
  const uint64_t half = n >> 1;
  const uint32_t lim = (uint32_t)(half < a.p_lim ? half : a.p_lim);
  const uint32_t nm1 = (uint32_t)(n % kM1), nm2 = (uint32_t)(n % kM2), nm3 = (uint32_t)(n % kM3);
  uint64_t k = 1;
  uint32_t nsurv = 0;
  bool exhausted = false;
  for (;;) {
    while (nsurv < 32 && !exhausted) {
      const uint64_t kk = k + lane;
      const uint32_t p = kk < a.nprimes ? a.primes[kk] : 0xffffffffu;
      const bool valid = kk < a.nprimes && p <= lim;
      const bool pass = valid && no_small_factor(nm1, nm2, nm3, p);
      const uint32_t b = __ballot_sync(kFull, pass);
      if (pass) buf[nsurv + __popc(b & lanemask_lt())] = (uint32_t)kk;
      nsurv += __popc(b);
      if (__ballot_sync(kFull, valid) != kFull) exhausted = true;
      k += 32;
    }
    __syncwarp();
    if (nsurv == 0) return 0;
    const uint32_t take = nsurv < 32 ? nsurv : 32;
    const bool act = lane < (int)take;
    uint32_t pk = 0;
    uint64_t q = 3;
    if (act) {
      pk = a.primes[buf[lane]];
      q = n - pk;
    }
    uint64_t d = q - 1;
    int s = __ffsll((long long)d) - 1;
    d >>= s;
    Mont32 M = mont32_init(q);
    const bool ok2 = sprp_warp(M, mod_dbl(M.one, M.n), d, s, act) && act;
    uint32_t b = __ballot_sync(kFull, ok2);
    while (b) {
      const int l = __ffs(b) - 1;
      const uint64_t qc = __shfl_sync(kFull, q, l);
      const uint32_t pc = __shfl_sync(kFull, pk, l);
      uint64_t dc = qc - 1;
      const int sc = __ffsll((long long)dc) - 1;
      dc >>= sc;
      const Mont32 Mc = mont32_init(qc);
      uint64_t r2 = mod_dbl(Mc.one, Mc.n);
#pragma unroll
      for (int i = 0; i < 6; ++i) r2 = mont_mul32(r2, r2, Mc.n, Mc.ni);
      uint64_t base = kMR7Bases[lane < 6 ? lane + 1 : 1];
      if (base >= qc) base %= qc;
      const bool test = lane < 6 && base != 0;
      const bool ok = sprp_warp(Mc, mont_mul32(base, r2, Mc.n, Mc.ni), dc, sc, test) || !test;
      if (__all_sync(kFull, ok)) return pc;
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

__global__ void __launch_bounds__(kSingleThreads) single_warp_kernel(SingleArgs a) {
  __shared__ uint32_t sbuf[kSingleThreads / 32][64];
  const int lane = threadIdx.x & 31;
  uint32_t* buf = sbuf[threadIdx.x >> 5];
  uint32_t found = 0, maxp = 0;
  for (;;) {
    unsigned long long qi = 0;
    if (lane == 0) qi = atomicAdd(&a.ctr[0], 1ull);
    qi = __shfl_sync(kFull, qi, 0);
    if (qi >= a.count) break;
    const uint64_t n = a.n[qi];
    uint32_t p = 0;
    if (n >= 4 && !(n & 1)) {
      const uint64_t half = n >> 1;
      if (n == 4) p = 2;
      else if (n < kSmallN) p = minp_plain(a, n, half < a.p_lim ? half : a.p_lim);
      else p = minp_warp(a, n, buf);
    }
    if (lane == 0) {
      a.p_out[qi] = p;
      a.q_out[qi] = p ? n - p : 0;
      if (p) {
        ++found;
        maxp = p > maxp ? p : maxp;
      }
    }
  }
  if (lane == 0) {
    if (found) atomicAdd(&a.ctr[1], (unsigned long long)found);
    if (maxp) atomicMax(&a.ctr[2], (unsigned long long)maxp);
  }
}

// Batches below kLaneBatchMin queries take the warp-per-query kernel: they
// fit the GPU's resident warps at once, so the per-query latency (about
// two strong tests there, a dozen per lane in single_kernel) sets the time.
cudaError_t launch_single(const SingleArgs& a, int grid, cudaStream_t s) {
  if (a.count < kLaneBatchMin) single_warp_kernel<<<grid, kSingleThreads, 0, s>>>(a);
  else single_kernel<<<grid, kSingleThreads, 0, s>>>(a);
  return cudaGetLastError();
}

void single_kernel_node(const SingleArgs& a, int grid, void** argv, cudaKernelNodeParams* kp) {
  argv[0] = (void*)&a;
  *kp = cudaKernelNodeParams{};
  kp->func = a.count < kLaneBatchMin ? (void*)single_warp_kernel : (void*)single_kernel;
  kp->gridDim = dim3((unsigned)grid);
  kp->blockDim = dim3(kSingleThreads);
  kp->kernelParams = argv;
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

void segment_reduce_node(const SegReduceArgs& r, void** argv, cudaKernelNodeParams* kp) {
  argv[0] = (void*)&r.p;
  argv[1] = (void*)&r.off;
  argv[2] = (void*)&r.nreq;
  argv[3] = (void*)&r.agg;
  *kp = cudaKernelNodeParams{};
  kp->func = (void*)segment_reduce_kernel;
  kp->gridDim = dim3((r.nreq + 7) / 8);
  kp->blockDim = dim3(256);
  kp->kernelParams = argv;
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
