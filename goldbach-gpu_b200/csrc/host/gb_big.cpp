// gb_big.cpp -- C-ABI entry point for even n beyond 2^64 (big_check).
//
// The reference's big_check (src/big_check.cpp:35-144) sieves the primes up
// to 1e7 on the host and runs GMP's mpz_probab_prime_p(n - p, 25) on OpenMP
// threads in batches of 1000 primes, keeping the first success.  Here the
// candidates come from the resident prime table in batches of kBigBatch:
// the filter kernel drops q = n - p with a factor below kBigTrialBound (from
// n mod r, computed here once), the base-2 kernel tests the survivors, the
// bases kernel runs the other 11 bases on the base-2 passers in parallel
// (kernels/big.cu), and the smallest passer no base rejects, in the first
// batch that has one, is the minimal p.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gb_ctx.h"

namespace gb {

constexpr uint32_t kBigBatch = 8192;          // candidates per launch pair
constexpr uint32_t kBigTrialBound = 4096;     // trial primes below this

gb_status big_impl(gb_ctx* c, Workspace& w, const uint32_t* n_limbs, uint32_t nlimbs,
                   uint64_t p_limit, uint64_t* p_out, uint32_t* q_limbs, gb_big_result* res) {
  if (!n_limbs || !p_out || nlimbs == 0) return fail(w, GB_EINVAL, "null argument");
  uint32_t m = nlimbs;
  while (m > 0 && n_limbs[m - 1] == 0) --m;
  if (m > GB_BIG_MAX_LIMBS) return fail(w, GB_EINVAL, "n has more than GB_BIG_MAX_LIMBS limbs");
  if (m == 0 || (n_limbs[0] & 1) || (m == 1 && n_limbs[0] < 4))
    return fail(w, GB_EINVAL, "n must be even and >= 4");
  if (!p_limit) p_limit = GB_PHASE2_LIMIT_DEFAULT;
  if (p_limit > 0xfffffffbull) return fail(w, GB_EINVAL, "p_limit above 2^32");
  gb_big_result r{};
  if (q_limbs) std::memset(q_limbs, 0, nlimbs * 4);
  if (m <= 2) {  // below 2^64: the deterministic single-n path
    const uint64_t n = m == 1 ? n_limbs[0] : ((uint64_t)n_limbs[1] << 32 | n_limbs[0]);
    uint64_t p = 0, q = 0;
    gb_single_opts so{};
    so.p_limit = p_limit;
    gb_single_result sr{};
    gb_status st = single_impl(c, w, nullptr, &n, 1, &p, &q, &so, &sr);
    if (st != GB_OK) return st;
    *p_out = p;
    if (q_limbs && p) {
      q_limbs[0] = (uint32_t)q;
      if (nlimbs > 1) q_limbs[1] = (uint32_t)(q >> 32);
    }
    r.candidates = 1;
    r.device_ms = sr.device_ms;
    if (res) *res = r;
    return GB_OK;
  }
  uint32_t N = 4;
  while (N < m) N <<= 1;
  gb_status st = ensure_primes(c, w, std::max<uint64_t>(p_limit, kBigTrialBound));
  if (st != GB_OK) return st;
  uint64_t np = 0;
  if ((st = count_le(c, w, p_limit, &np)) != GB_OK) return st;
  // trial primes 3 .. kBigTrialBound and n mod each (from the top limb down)
  std::vector<uint32_t> trial, nmod;
  for (uint32_t p : c->h_primes) {
    if (p < 3) continue;
    if (p >= kBigTrialBound) break;
    uint64_t rem = 0;
    for (uint32_t i = m; i-- > 0;) rem = ((rem << 32) | n_limbs[i]) % p;
    trial.push_back(p);
    nmod.push_back((uint32_t)rem);
  }
  std::vector<uint32_t> npad(N, 0);
  std::copy(n_limbs, n_limbs + m, npad.begin());
  Temps tmp(c, nullptr);
  void *d_n, *d_trial, *d_nmod, *d_surv, *d_pass, *d_small;
  if ((st = ws_buffer(c, w, tmp, 0, N * 4, &d_n)) != GB_OK ||
      (st = ws_buffer(c, w, tmp, 1, trial.size() * 4, &d_trial)) != GB_OK ||
      (st = ws_buffer(c, w, tmp, 2, nmod.size() * 4, &d_nmod)) != GB_OK ||
      (st = ws_buffer(c, w, tmp, 3, kBigBatch * 4, &d_surv)) != GB_OK ||
      (st = ws_buffer(c, w, tmp, 4, kBigBatch * 8, &d_pass)) != GB_OK ||
      (st = ws_buffer(c, w, tmp, 5, 64, &d_small)) != GB_OK)
    return st;
  BigArgs a{};
  a.n = (const uint32_t*)d_n;
  a.limbs = N;
  a.nl = m;
  a.primes = c->d_primes;
  a.p_lim = p_limit;
  a.trial = (const uint32_t*)d_trial;
  a.nmod = (const uint32_t*)d_nmod;
  a.ntrial = (uint32_t)trial.size();
  a.surv = (uint32_t*)d_surv;
  a.pass = (uint32_t*)d_pass;
  a.fail = (uint32_t*)d_pass + kBigBatch;
  a.nsurv = (uint32_t*)d_small;
  a.npass = (uint32_t*)d_small + 1;
  a.mr_tests = (unsigned long long*)((char*)d_small + 8);
  cudaStream_t s = c->stream;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) {
    if (e == cudaSuccess && x != cudaSuccess) e = x;
  };
  chk(cudaMemcpyAsync(d_n, npad.data(), N * 4, cudaMemcpyHostToDevice, s));
  chk(cudaMemcpyAsync(d_trial, trial.data(), trial.size() * 4, cudaMemcpyHostToDevice, s));
  chk(cudaMemcpyAsync(d_nmod, nmod.data(), nmod.size() * 4, cudaMemcpyHostToDevice, s));
  chk(cudaMemsetAsync(a.mr_tests, 0, 8, s));
  chk(cudaEventRecord(w.ev0, s));
  uint32_t best = 0xffffffffu;
  uint64_t k0 = 1;  // p = 2 leaves q = n - 2 even
  uint32_t pk = 0;
  std::vector<uint32_t> pass(2 * kBigBatch);
  while (k0 < np && e == cudaSuccess) {
    const uint32_t kc = (uint32_t)std::min<uint64_t>(kBigBatch, np - k0);
    chk(cudaMemsetAsync(a.nsurv, 0, 8, s));  // survivors and passers
    chk(launch_big_filter(a, (uint32_t)k0, kc, s));
    chk(launch_big_mr(a, (uint32_t)k0, 0, c->sm_count * 4, s));
    chk(launch_big_mr(a, (uint32_t)k0, 1, c->sm_count * 4, s));
    uint32_t np_ = 0;
    chk(cudaMemcpyAsync(&np_, a.npass, 4, cudaMemcpyDeviceToHost, s));
    chk(cudaStreamSynchronize(s));
    r.candidates += kc;
    if (e == cudaSuccess && np_) {
      chk(cudaMemcpyAsync(pass.data(), a.pass, np_ * 4, cudaMemcpyDeviceToHost, s));
      chk(cudaMemcpyAsync(pass.data() + kBigBatch, a.fail, np_ * 4, cudaMemcpyDeviceToHost, s));
      chk(cudaStreamSynchronize(s));
      for (uint32_t j = 0; j < np_; ++j)
        if (!pass[kBigBatch + j] && pass[j] < best) best = pass[j];
    }
    if (best != 0xffffffffu) {
      chk(cudaMemcpy(&pk, c->d_primes + k0 + best, 4, cudaMemcpyDeviceToHost));
      break;
    }
    k0 += kc;
  }
  chk(cudaEventRecord(w.ev1, s));
  unsigned long long tests = 0;
  chk(cudaMemcpyAsync(&tests, a.mr_tests, 8, cudaMemcpyDeviceToHost, s));
  chk(cudaStreamSynchronize(s));
  if (e != cudaSuccess) return cuda_fail(w, e, "big n");
  float ms = 0;
  cudaEventElapsedTime(&ms, w.ev0, w.ev1);
  *p_out = best != 0xffffffffu ? pk : 0;
  if (q_limbs && *p_out) {  // q = n - p
    uint64_t borrow = *p_out;
    for (uint32_t i = 0; i < m; ++i) {
      const uint64_t v = (uint64_t)n_limbs[i] - (borrow & 0xffffffffu) - (borrow >> 32);
      q_limbs[i] = (uint32_t)v;
      borrow = ((v >> 32) & 1) << 32;
    }
  }
  r.mr_tests = tests;
  r.device_ms = ms;
  if (res) *res = r;
  return GB_OK;
}

}  // namespace gb
