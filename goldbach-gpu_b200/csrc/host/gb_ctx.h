// gb_ctx.h -- the context behind the C-ABI (internal).
//
// A context owns one device's resident tables.  Device work runs through a
// Workspace (counters, histogram, Phase-2 queue, events, error text) and
// may take its temporary buffers from an Arena instead of cudaMalloc, so
// that several lanes (the serving loop's single-n and range lanes) can run
// concurrently on one context without allocating or freeing while the
// device is busy.
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

namespace gb {

// Bump allocator over a device region reserved once; reset per batch.
struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  size_t used = 0;
  void* take(size_t bytes) {
    const size_t off = (used + 255) & ~size_t(255);
    if (off + bytes > cap) return nullptr;
    used = off + bytes;
    return base + off;
  }
};

struct Workspace {
  unsigned long long* ctr = nullptr;   // kCtrCount
  unsigned long long* hist = nullptr;  // GB_HIST_BINS
  QEntry* queue = nullptr;
  uint32_t queue_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ek0 = nullptr, ek1 = nullptr, ek2 = nullptr;
  cudaGraphExec_t win_exec = nullptr;  // the windows batch's launches (updated per batch)
  void* scratch = nullptr;  // per-call kernel scratch, grown on demand
  size_t scratch_bytes = 0;
  // per-call device buffers of the public entry points (slot i grown on
  // demand and kept, up to kKeptBufferBytes; larger ones are per call)
  static constexpr int kBufSlots = 8;
  void* buf[kBufSlots] = {};
  size_t buf_bytes[kBufSlots] = {};
  // pinned staging for the counters and the histogram read back by each call
  unsigned long long* h_stage = nullptr;  // kCtrCount + GB_HIST_BINS
  std::string err;
};

}  // namespace gb

struct gb_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  uint64_t budget = 0;  // device bytes this context may hold
  uint64_t held = 0;
  std::map<void*, size_t> allocs;
  std::mutex alloc_mu;  // guards budget accounting (dev_alloc / dev_free)
  std::mutex mu;        // serialises the public entry points
  std::string err;

  // resident tables (read-only while any lane runs)
  uint32_t* d_wheel = nullptr;   // odd-only wheel patterns
  uint32_t* d_wheel6 = nullptr;  // mod-6 class wheel patterns
  uint32_t* d_primes = nullptr;  // all primes <= primes_limit, ascending, 2 first
  uint64_t* d_magic = nullptr;   // Barrett reciprocals, one per prime
  uint2* d_a15 = nullptr;        // mod-6 class offsets (-1/6, -5/6 mod p), one per prime
  uint64_t nprimes = 0;
  uint64_t primes_limit = 0;
  std::vector<uint32_t> h_primes;  // host copy of the primes <= kHostPrimeLimit
  std::vector<uint32_t> h_sample;  // primes[i * kSampleStride]: locates a count on the host

  gb::Workspace ws;  // the public entry points' workspace
  gb_server* server = nullptr;
  // gb_autotune_range's choices per range class (bit length of the limit,
  // p_small, phase2_limit) -> (chunk_evens, halo, block threads, even n/s)
  struct Tuned {
    uint32_t chunk, halo, threads;
    double rate;
  };
  std::map<std::vector<uint64_t>, Tuned> tuned;
  // gb_autotune_windows's choices per batch class (bit length of the
  // largest top, bit length of the window count)
  std::map<std::vector<uint64_t>, gb_windows_tune> tuned_windows;
};

namespace gb {

constexpr uint64_t kHostPrimeLimit = 1ull << 22;
constexpr uint64_t kSampleStride = 1024;
// primes searched word-parallel (lockstep) before the per-n tail

gb_status fail(Workspace& w, gb_status st, const std::string& msg);
gb_status cuda_fail(Workspace& w, cudaError_t e, const char* what);
gb_status dev_alloc(gb_ctx* c, void** p, size_t bytes, std::string* err = nullptr);
void dev_free(gb_ctx* c, void* p);
gb_status ws_init(gb_ctx* c, Workspace& w, uint32_t queue_cap);
void ws_free(gb_ctx* c, Workspace& w);
// The workspace's scratch buffer, grown to at least `bytes`.
gb_status ws_scratch(gb_ctx* c, Workspace& w, size_t bytes, void** p);
// Per-call device buffers kept between calls (no cudaMalloc / cudaFree per
// call for the usual sizes): slot `slot` of the workspace, grown to `bytes`;
// above kKeptBufferBytes the buffer comes from `t` and is freed with it.
constexpr size_t kKeptBufferBytes = 256ull << 20;
struct Temps;
gb_status ws_buffer(gb_ctx* c, Workspace& w, Temps& t, int slot, size_t bytes, void** p);
gb_status ensure_primes(gb_ctx* c, Workspace& w, uint64_t limit);
// number of primes <= x in the resident table (x <= primes_limit)
gb_status count_le(gb_ctx* c, Workspace& w, uint64_t x, uint64_t* out);
uint64_t isqrt_u64(uint64_t n);

// Temporary device buffers of one call: from the arena when there is one
// (never freed one by one), from dev_alloc otherwise (freed by release()).
struct Temps {
  gb_ctx* c;
  Arena* arena;
  std::vector<void*> owned;
  Temps(gb_ctx* c_, Arena* a) : c(c_), arena(a) {}
  ~Temps() { release(); }
  gb_status get(size_t bytes, void** p, Workspace& w);
  void release();
};

// The work behind the public entry points; callers hold no lock, but the
// tables must already cover the call (ensure_primes) when lanes run
// concurrently.
gb_status range_impl(gb_ctx* c, Workspace& w, Arena* arena, uint64_t start, uint64_t limit,
                     const gb_range_opts* opts, gb_range_result* res, const gb_range_out* out);
gb_status single_impl(gb_ctx* c, Workspace& w, Arena* arena, const uint64_t* n, size_t count,
                      uint64_t* p_out, uint64_t* q_out, const gb_single_opts* opts,
                      gb_single_result* res);
gb_status big_impl(gb_ctx* c, Workspace& w, const uint32_t* n_limbs, uint32_t nlimbs,
                   uint64_t p_limit, uint64_t* p_out, uint32_t* q_limbs, gb_big_result* res);
uint64_t windows_request_bytes(const gb_window& w, const gb_windows_opts& o);
gb_status autotune_windows_impl(gb_ctx* c, Workspace& w, const gb_window* win, size_t count,
                                const gb_windows_opts* base, gb_windows_opts* tuned,
                                gb_windows_tune* res);
gb_status windows_impl(gb_ctx* c, Workspace& w, Arena* arena, const gb_window* win, size_t count,
                       const gb_windows_opts* opts, gb_window_result* res, uint32_t* min_p_concat,
                       gb_windows_summary* sum);

}  // namespace gb
