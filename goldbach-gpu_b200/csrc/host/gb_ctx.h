// gb_ctx.h -- the context behind the C-ABI (internal).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../gb_internal.h"
#ifndef GB_HOST_ONLY
#define GB_HOST_ONLY
#endif
#include "../gb_device.cuh"
#include "gb/gb.h"

struct gb_server;  // serving loop (gb_serve.cpp)

struct gb_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_k0 = nullptr, ev_k1 = nullptr;
  uint64_t budget = 0;  // device bytes this context may hold
  uint64_t held = 0;
  std::map<void*, size_t> allocs;
  std::string err;
  std::mutex mu;  // serialises device work of this context

  // resident tables
  uint32_t* d_wheel = nullptr;
  uint32_t* d_primes = nullptr;  // all primes <= primes_limit, ascending, 2 first
  uint64_t* d_magic = nullptr;   // Barrett reciprocals, one per prime
  uint64_t nprimes = 0;
  uint64_t primes_limit = 0;
  std::vector<uint32_t> h_primes;  // host copy of the primes <= kHostPrimeLimit

  // work buffers
  unsigned long long* d_ctr = nullptr;   // kCtrCount (range) / 4 (single)
  unsigned long long* d_hist = nullptr;  // GB_HIST_BINS
  gb::QEntry* d_queue = nullptr;
  uint32_t queue_cap = 0;

  gb_server* server = nullptr;
};

namespace gb {

constexpr uint64_t kHostPrimeLimit = 1ull << 22;
// primes searched word-parallel (lockstep) before the per-n tail
constexpr uint64_t kLockPrimes = 128;

gb_status fail(gb_ctx* c, gb_status st, const std::string& msg);
gb_status cuda_fail(gb_ctx* c, cudaError_t e, const char* what);
gb_status dev_alloc(gb_ctx* c, void** p, size_t bytes);
void dev_free(gb_ctx* c, void* p);
gb_status ensure_primes(gb_ctx* c, uint64_t limit);
// number of primes <= x in the resident table (x <= primes_limit)
gb_status count_le(gb_ctx* c, uint64_t x, uint64_t* out);
uint64_t isqrt_u64(uint64_t n);

}  // namespace gb
