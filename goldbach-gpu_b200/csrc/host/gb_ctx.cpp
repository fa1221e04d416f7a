// gb_ctx.cpp -- C-ABI entry points: context, tables, range verification,
// single-n batches and batched primality.
//
// The range call is the library form of run_gpu_worker (src/goldbach.cu:
// 378-500) plus the table derivation of main (src/goldbach.cu:637-673).
// The segment geometry (seg_end, q_low, q_high at :425-431) survives only as
// the reporting unit; the device work is split into fixed chunks that the
// persistent kernel schedules itself.
#include "gb_ctx.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

namespace gb {

gb_status fail(Workspace& w, gb_status st, const std::string& msg) {
  w.err = msg;
  return st;
}

gb_status cuda_fail(Workspace& w, cudaError_t e, const char* what) {
  return fail(w, e == cudaErrorMemoryAllocation ? GB_ENOMEM : GB_ECUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define GB_CU(call, what)                                 \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(w, e_, what); \
  } while (0)

gb_status dev_alloc(gb_ctx* c, void** p, size_t bytes, std::string* err) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  std::lock_guard<std::mutex> lk(c->alloc_mu);
  if (c->held + bytes > c->budget) {
    if (err) {
      char buf[256];
      snprintf(buf, sizeof buf,
               "insufficient VRAM: required %llu MB more, budget %llu MB, held %llu MB",
               (unsigned long long)(bytes >> 20), (unsigned long long)(c->budget >> 20),
               (unsigned long long)(c->held >> 20));
      *err = buf;
    }
    return GB_ENOMEM;
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    if (err) *err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return GB_ENOMEM;
  }
  c->held += bytes;
  c->allocs[*p] = bytes;
  return GB_OK;
}

void dev_free(gb_ctx* c, void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(c->alloc_mu);
  auto it = c->allocs.find(p);
  if (it != c->allocs.end()) {
    c->held -= it->second;
    c->allocs.erase(it);
  }
  cudaFree(p);
}

gb_status Temps::get(size_t bytes, void** p, Workspace& w) {
  if (arena) {
    *p = arena->take(bytes);
    return *p ? GB_OK : fail(w, GB_ENOMEM, "serving arena exhausted");
  }
  gb_status st = dev_alloc(c, p, bytes, &w.err);
  if (st == GB_OK) owned.push_back(*p);
  return st;
}

void Temps::release() {
  for (void* p : owned) dev_free(c, p);
  owned.clear();
}

gb_status ws_init(gb_ctx* c, Workspace& w, uint32_t queue_cap) {
  gb_status st;
  if ((st = dev_alloc(c, (void**)&w.ctr, kCtrCount * 8, &w.err)) != GB_OK ||
      (st = dev_alloc(c, (void**)&w.hist, GB_HIST_BINS * 8, &w.err)) != GB_OK ||
      (st = dev_alloc(c, (void**)&w.queue, (size_t)queue_cap * sizeof(QEntry), &w.err)) != GB_OK)
    return st;
  w.queue_cap = queue_cap;
  if (cudaMallocHost((void**)&w.h_stage, (kCtrCount + GB_HIST_BINS) * 8) != cudaSuccess)
    return fail(w, GB_ENOMEM, "pinned staging buffer");
  if (cudaEventCreate(&w.ev0) != cudaSuccess || cudaEventCreate(&w.ev1) != cudaSuccess ||
      cudaEventCreate(&w.ek0) != cudaSuccess || cudaEventCreate(&w.ek1) != cudaSuccess ||
      cudaEventCreate(&w.ek2) != cudaSuccess)
    return fail(w, GB_ECUDA, "cudaEventCreate");
  return GB_OK;
}

gb_status ws_scratch(gb_ctx* c, Workspace& w, size_t bytes, void** p) {
  if (bytes > w.scratch_bytes) {
    dev_free(c, w.scratch);
    w.scratch = nullptr;
    w.scratch_bytes = 0;
    gb_status st = dev_alloc(c, &w.scratch, bytes, &w.err);
    if (st != GB_OK) return st;
    w.scratch_bytes = bytes;
  }
  *p = w.scratch;
  return GB_OK;
}

gb_status ws_buffer(gb_ctx* c, Workspace& w, Temps& t, int slot, size_t bytes, void** p) {
  if (t.arena || bytes > kKeptBufferBytes || slot >= Workspace::kBufSlots) return t.get(bytes, p, w);
  if (bytes > w.buf_bytes[slot]) {
    dev_free(c, w.buf[slot]);
    w.buf[slot] = nullptr;
    w.buf_bytes[slot] = 0;
    const size_t grow = std::max<size_t>(bytes, 64 << 10);
    gb_status st = dev_alloc(c, &w.buf[slot], grow, &w.err);
    if (st != GB_OK) return st;
    w.buf_bytes[slot] = grow;
  }
  *p = w.buf[slot];
  return GB_OK;
}

void ws_free(gb_ctx* c, Workspace& w) {
  for (int i = 0; i < Workspace::kBufSlots; ++i) {
    dev_free(c, w.buf[i]);
    w.buf[i] = nullptr;
    w.buf_bytes[i] = 0;
  }
  if (w.h_stage) cudaFreeHost(w.h_stage);
  w.h_stage = nullptr;
  dev_free(c, w.ctr);
  dev_free(c, w.hist);
  dev_free(c, w.queue);
  dev_free(c, w.scratch);
  w.ctr = nullptr;
  w.hist = nullptr;
  w.queue = nullptr;
  w.scratch = nullptr;
  w.scratch_bytes = 0;
  if (w.win_exec) cudaGraphExecDestroy(w.win_exec);
  w.win_exec = nullptr;
  for (cudaEvent_t* e : {&w.ev0, &w.ev1, &w.ek0, &w.ek1, &w.ek2})
    if (*e) {
      cudaEventDestroy(*e);
      *e = nullptr;
    }
}

uint64_t isqrt_u64(uint64_t n) {  // exact floor(sqrt(n)), src/goldbach.cu:637-646
  uint64_t r = (uint64_t)std::sqrt((double)n);
  while (r > 0 && (r > 0xffffffffull || r * r > n)) --r;
  while (r < 0xffffffffull && (r + 1) * (r + 1) <= n) ++r;
  return r;
}

// Upper bound on pi(x) (Rosser-Schoenfeld: pi(x) < 1.25506 x / ln x, x > 1).
static uint64_t pi_upper(uint64_t x) {
  if (x < 100) return 26;
  return (uint64_t)(1.2551 * (double)x / std::log((double)x)) + 64;
}

gb_status count_le(gb_ctx* c, Workspace& w, uint64_t x, uint64_t* out) {
  if (x >= c->primes_limit && c->primes_limit) {
    *out = c->nprimes;
    return GB_OK;
  }
  if (x <= kHostPrimeLimit || c->nprimes == c->h_primes.size()) {
    *out = std::upper_bound(c->h_primes.begin(), c->h_primes.end(),
                            (uint32_t)std::min<uint64_t>(x, 0xffffffffu)) -
           c->h_primes.begin();
    return GB_OK;
  }
  // the host sample brackets x within one block of kSampleStride primes;
  // one copy of that block finishes the count
  const uint64_t b = std::upper_bound(c->h_sample.begin(), c->h_sample.end(),
                                      (uint32_t)std::min<uint64_t>(x, 0xffffffffu)) -
                     c->h_sample.begin();  // samples <= x
  if (b == 0) {
    *out = 0;
    return GB_OK;
  }
  const uint64_t lo = (b - 1) * kSampleStride;
  const uint64_t len = std::min<uint64_t>(kSampleStride, c->nprimes - lo);
  std::vector<uint32_t> blk(len);
  GB_CU(cudaMemcpy(blk.data(), c->d_primes + lo, len * 4, cudaMemcpyDeviceToHost), "count_le");
  *out = lo + (std::upper_bound(blk.begin(), blk.end(), (uint32_t)std::min<uint64_t>(x, 0xffffffffu)) -
               blk.begin());
  return GB_OK;
}

// Builds (or grows) the resident prime table to cover [2, limit] on the
// device: the wheel alone is exact below 71^2, and each further stage
// sieves [3, L^2] with the primes <= L of the previous one.
gb_status ensure_primes(gb_ctx* c, Workspace& w, uint64_t limit) {
  if (limit <= c->primes_limit) return GB_OK;
  if (limit > 0xffffffffull && limit <= 0x100000002ull) limit = 0xffffffffull;  // sqrt of n near 2^64
  if (limit <= c->primes_limit) return GB_OK;
  if (c->server)  // the serving lanes read the tables without a lock
    return fail(w, GB_EINVAL, "prime tables are frozen while serving: size them in gb_serve_start");
  uint64_t target = std::max<uint64_t>(limit, 1ull << 22);
  if (target > 0xffffffffull) return fail(w, GB_EINVAL, "prime table limit above 2^32");
  if (!(target & 1)) target++;  // odd top
  if (target > 0xffffffffull) target = 0xfffffffbull;
  const uint64_t cap = pi_upper(target);
  const uint64_t nbits_max = (target - 3) / 2 + 1;
  const size_t nblk = compact_scratch_blocks(nbits_max);
  uint32_t* primes = nullptr;
  uint64_t* magic = nullptr;
  uint2* a15 = nullptr;
  Temps t(c, nullptr);
  uint32_t *bits, *blocks;
  unsigned long long* total;
  gb_status st;
  if ((st = dev_alloc(c, (void**)&primes, cap * 4, &w.err)) != GB_OK) return st;
  if ((st = dev_alloc(c, (void**)&magic, cap * 8, &w.err)) != GB_OK ||
      (st = dev_alloc(c, (void**)&a15, cap * 8, &w.err)) != GB_OK ||
      (st = t.get(((nbits_max + 31) / 32 + 4) * 4, (void**)&bits, w)) != GB_OK ||
      (st = t.get((nblk + 1) * 4, (void**)&blocks, w)) != GB_OK ||
      (st = t.get(8, (void**)&total, w)) != GB_OK) {
    dev_free(c, primes);
    dev_free(c, magic);
    dev_free(c, a15);
    return st;
  }
  auto bail = [&](cudaError_t e, const char* what) {
    dev_free(c, primes);
    dev_free(c, magic);
    dev_free(c, a15);
    return cuda_fail(w, e, what);
  };
  uint64_t cur = 0, count = 0;
  std::vector<uint32_t> head;
  while (cur < target) {
    uint64_t next = cur == 0 ? std::min<uint64_t>(target, 5039)
                             : std::min<uint64_t>(target, (cur + 1) * (cur + 1) - 1);
    const uint64_t nbits = (next - 3) / 2 + 1;
    uint64_t nsieve = kWheelPrimeCount + 1, kcoop = kWheelPrimeCount + 1;
    const uint32_t tile = 1u << 18;
    if (cur) {
      const uint64_t r = isqrt_u64(next);
      nsieve = std::upper_bound(head.begin(), head.end(), (uint32_t)r) - head.begin();
      kcoop = std::upper_bound(head.begin(), head.end(), (uint32_t)(tile / 64)) - head.begin();
      kcoop = std::min(kcoop, nsieve);
    }
    SieveArgs a{};
    a.q_lo = 3;
    a.nbits = nbits;
    a.tile_bits = tile;
    a.primes = primes;
    a.magic = magic;
    a.nsieve = (uint32_t)nsieve;
    a.kcoop = (uint32_t)kcoop;
    a.wheel = c->d_wheel;
    a.out = bits;
    cudaError_t e = launch_sieve_bits(a, c->stream);
    if (e == cudaSuccess)
      e = launch_compact_primes(bits, nbits, 3, primes, magic, a15, 1, cap, total, blocks,
                                (uint32_t)(nblk + 1), c->stream);
    unsigned long long tot = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tot, total, 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return bail(e, "prime table build");
    count = tot;
    if (count > cap) return bail(cudaErrorInvalidValue, "prime table overflow");
    const uint64_t nh = std::min<uint64_t>(count, 8192);
    head.resize(nh);
    e = cudaMemcpy(head.data(), primes, nh * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bail(e, "prime table copy");
    cur = next;
  }
  t.release();
  dev_free(c, c->d_primes);
  dev_free(c, c->d_magic);
  dev_free(c, c->d_a15);
  c->d_primes = primes;
  c->d_magic = magic;
  c->d_a15 = a15;
  c->nprimes = count;
  c->primes_limit = target;
  const uint64_t nh = std::min<uint64_t>(count, pi_upper(kHostPrimeLimit));
  std::vector<uint32_t> h(nh);  // host copy of the small primes: parameter derivation only
  GB_CU(cudaMemcpy(h.data(), primes, nh * 4, cudaMemcpyDeviceToHost), "prime table copy");
  h.resize(std::upper_bound(h.begin(), h.end(), (uint32_t)kHostPrimeLimit) - h.begin());
  c->h_primes.swap(h);
  const uint64_t ns = (count + kSampleStride - 1) / kSampleStride;
  std::vector<uint32_t> smp(ns);
  GB_CU(cudaMemcpy2D(smp.data(), 4, primes, kSampleStride * 4, 4, ns, cudaMemcpyDeviceToHost),
        "prime table sample");
  c->h_sample.swap(smp);
  return GB_OK;
}

// ---------------------------------------------------------------------------
gb_status range_impl(gb_ctx* c, Workspace& w, Arena* arena, uint64_t start, uint64_t limit,
                     const gb_range_opts* opts, gb_range_result* res, const gb_range_out* out) {
  if (limit & 1) limit--;
  if (start < 4) start = 4;
  // an odd start rounds up; 2^64 - 1 has no even successor
  if (start == UINT64_MAX) return fail(w, GB_EINVAL, "START must be less than LIMIT");
  if (start & 1) start++;
  if (start > limit) return fail(w, GB_EINVAL, "START must be less than LIMIT");
  gb_range_opts o{};
  if (opts) o = *opts;
  if (!o.seg_size) o.seg_size = 10000000ull;
  if (!o.p_small) o.p_small = 1000000ull;
  if (!o.phase2_limit) o.phase2_limit = GB_PHASE2_LIMIT_DEFAULT;
  if (o.p_small > GB_P_SMALL_MAX)
    return fail(w, GB_EINVAL, "P_SMALL must be <= 4000000000 to prevent mathematical overflow.");
  if (o.phase2_limit > GB_P_SMALL_MAX) return fail(w, GB_EINVAL, "phase2_limit must be <= 4e9");
  const uint64_t count = (limit - start) / 2 + 1;
  const uint32_t H = o.halo ? o.halo : 32768u;
  if (H < 128 || H > (1u << 17) || (H & 63))
    return fail(w, GB_EINVAL, "halo must be a multiple of 64 in [128, 2^17]");
  uint32_t NE = o.chunk_evens;
  if (!NE) {
    // 2^20 n: two CTAs per SM (the two class bitsets hold 2^20 / 3 bits each)
    NE = 1u << 20;
    while (NE > 8192 && NE / 2 >= count) NE >>= 1;
  }
  if (NE < 8192 || NE > (1u << 20) || (NE & (NE - 1)))
    return fail(w, GB_EINVAL, "chunk_evens must be a power of two in [2^13, 2^20]");
  if (out && out->min_p && NE > kMinpChunk) NE = kMinpChunk;  // per-n output: smaller chunks
  if (o.block_threads && o.block_threads != 256 && o.block_threads != 512 && o.block_threads != 1024)
    return fail(w, GB_EINVAL, "block_threads must be 256, 512 or 1024");
  const uint32_t sc = o.shard_count ? o.shard_count : 1;
  if (o.shard_index >= sc) return fail(w, GB_EINVAL, "shard_index >= shard_count");
  const uint64_t nseg = (count + o.seg_size - 1) / o.seg_size;
  const uint64_t my_segs = nseg > o.shard_index ? (nseg - o.shard_index + sc - 1) / sc : 0;
  const uint64_t cps = (o.seg_size + NE - 1) / NE;
  const uint64_t p_lim = std::max(o.p_small, o.phase2_limit);
  const uint64_t root = isqrt_u64(limit);
  gb_status st = ensure_primes(c, w, std::max<uint64_t>({p_lim, (uint64_t)H, root + 2}));
  if (st != GB_OK) return st;

  RangeArgs a{};
  SearchParams& sp = a.s;
  a.start = start;
  a.total_count = count;
  a.seg_size = o.seg_size;
  a.shard_index = o.shard_index;
  a.shard_count = sc;
  a.chunks_per_seg = cps;
  a.total_items = my_segs * cps;
  a.chunk_evens = NE;
  a.threads = o.block_threads;
  // two class bitsets of H/6 + NE/3 bits (plus the over-read of the last
  // warp task); primes p <= H - 13 keep every q = n - p in the window
  a.nbw = range6_words(H, NE);
  const uint64_t search_top = std::min<uint64_t>(H - 13, p_lim);
  const uint64_t window_bits = H / 6 + NE / 3;
  uint64_t ns = 0, kf = 0, nsv = 0, kc = 0;
  if ((st = count_le(c, w, search_top, &ns)) != GB_OK ||
      (st = count_le(c, w, o.p_small, &kf)) != GB_OK ||
      (st = count_le(c, w, root, &nsv)) != GB_OK ||
      (st = count_le(c, w, window_bits / 64, &kc)) != GB_OK)
    return st;
  sp.halo = H;
  sp.nsearch = (uint32_t)ns;
  sp.kfb = (uint32_t)std::min<uint64_t>(kf, 0xffffffffu);
  sp.p_lim = p_lim;
  sp.p_small = o.p_small;
  sp.primes = c->d_primes;
  sp.nprimes = c->nprimes;
  sp.ctr = w.ctr;
  sp.hist = w.hist;
  sp.queue = w.queue;
  sp.queue_cap = w.queue_cap;
  a.magic = c->d_magic;
  a.nsieve = (uint32_t)std::max<uint64_t>(nsv, kWheelPrimeCount + 1);
  a.kcoop = (uint32_t)std::max<uint64_t>(kc, kWheelPrimeCount + 1);
  a.wheel6 = c->d_wheel6;
  a.a15 = c->d_a15;

  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : c->stream;
  gb_range_out od{};
  if (out) od = *out;
  Temps tmp(c, arena);
  int slot = 0;
  auto dev_out = [&](void* user, size_t bytes, void** dptr) -> gb_status {
    *dptr = nullptr;
    if (!user) return GB_OK;
    if (o.on_device) {
      *dptr = user;
      return GB_OK;
    }
    return ws_buffer(c, w, tmp, slot++, bytes, dptr);
  };
  const uint64_t vwords = (count + 31) / 32;
  void *d_vbits, *d_minp, *d_shist, *d_sfb, *d_sfail;
  if ((st = dev_out(od.verified_bits, vwords * 4, &d_vbits)) != GB_OK ||
      (st = dev_out(od.min_p, count * 4, &d_minp)) != GB_OK ||
      (st = dev_out(od.seg_hist, nseg * GB_HIST_BINS * 8, &d_shist)) != GB_OK ||
      (st = dev_out(od.seg_fallbacks, nseg * 4, &d_sfb)) != GB_OK ||
      (st = dev_out(od.seg_failures, nseg * 4, &d_sfail)) != GB_OK)
    return st;
  if (od.minp_hist && o.on_device) sp.hist = (unsigned long long*)od.minp_hist;
  sp.vbits = (uint32_t*)d_vbits;
  sp.minp = (uint32_t*)d_minp;
  sp.unit_hist = (unsigned long long*)d_shist;
  sp.unit_fallbacks = (uint32_t*)d_sfb;
  sp.unit_failures = (uint32_t*)d_sfail;

  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) {
    if (e == cudaSuccess && x != cudaSuccess) e = x;
  };
  uint32_t last_word = count & 31 ? (1u << (count & 31)) - 1 : 0xffffffffu;
  chk(cudaEventRecord(w.ev0, s));
  chk(cudaMemsetAsync(sp.ctr, 0, kCtrCount * 8, s));
  chk(cudaMemsetAsync(sp.ctr + kCtrFirstFail, 0xff, 8, s));
  chk(cudaMemsetAsync(sp.hist, 0, GB_HIST_BINS * 8, s));
  if (sp.vbits) {
    chk(cudaMemsetAsync(sp.vbits, 0xff, vwords * 4, s));
    // bits past the last n are zero (pageable source: staged at the call)
    if (count & 31) chk(cudaMemcpyAsync(sp.vbits + vwords - 1, &last_word, 4, cudaMemcpyHostToDevice, s));
  }
  if (sp.minp) chk(cudaMemsetAsync(sp.minp, 0, count * 4, s));
  if (sp.unit_hist) chk(cudaMemsetAsync(sp.unit_hist, 0, nseg * GB_HIST_BINS * 8, s));
  if (sp.unit_fallbacks) chk(cudaMemsetAsync(sp.unit_fallbacks, 0, nseg * 4, s));
  if (sp.unit_failures) chk(cudaMemsetAsync(sp.unit_failures, 0, nseg * 4, s));
  if (e != cudaSuccess) return cuda_fail(w, e, "range setup");
  int launches = 0;
  int bps = range_max_blocks_per_sm(a);
  if (bps < 1) bps = 1;
  uint64_t grid = (uint64_t)c->sm_count * bps;
  if (a.total_items < grid) grid = std::max<uint64_t>(1, a.total_items);
  if (a.total_items) {  // survivor lists of the levelled search
    a.surv_cap = a.nbw;
    void* p = nullptr;
    if ((st = ws_scratch(c, w, (size_t)grid * 6 * a.surv_cap * sizeof(uint2), &p)) != GB_OK) return st;
    a.surv = (uint2*)p;
  }
  if (a.total_items) {
    chk(cudaEventRecord(w.ek0, s));
    chk(launch_range(a, (int)grid, s));
    chk(cudaEventRecord(w.ek1, s));
    chk(launch_fallback(sp, c->sm_count * 4, s));
    launches += 2;
  }
  chk(cudaEventRecord(w.ev1, s));
  unsigned long long ctr[kCtrCount];
  unsigned long long* st_ctr = w.h_stage;  // pinned: the counters, then the histogram
  chk(cudaMemcpyAsync(st_ctr, sp.ctr, kCtrCount * 8, cudaMemcpyDeviceToHost, s));
  const bool hist_host = od.minp_hist && !o.on_device;
  if (hist_host)
    chk(cudaMemcpyAsync(st_ctr + kCtrCount, sp.hist, GB_HIST_BINS * 8, cudaMemcpyDeviceToHost, s));
  if (!o.on_device) {
    if (od.verified_bits) chk(cudaMemcpyAsync(od.verified_bits, sp.vbits, vwords * 4, cudaMemcpyDeviceToHost, s));
    if (od.min_p) chk(cudaMemcpyAsync(od.min_p, sp.minp, count * 4, cudaMemcpyDeviceToHost, s));
    if (od.seg_hist) chk(cudaMemcpyAsync(od.seg_hist, sp.unit_hist, nseg * GB_HIST_BINS * 8, cudaMemcpyDeviceToHost, s));
    if (od.seg_fallbacks) chk(cudaMemcpyAsync(od.seg_fallbacks, sp.unit_fallbacks, nseg * 4, cudaMemcpyDeviceToHost, s));
    if (od.seg_failures) chk(cudaMemcpyAsync(od.seg_failures, sp.unit_failures, nseg * 4, cudaMemcpyDeviceToHost, s));
  }
  chk(cudaStreamSynchronize(s));
  std::memcpy(ctr, st_ctr, sizeof ctr);
  if (hist_host && e == cudaSuccess) std::memcpy(od.minp_hist, st_ctr + kCtrCount, GB_HIST_BINS * 8);
  float ms = 0, kms = 0;
  if (e == cudaSuccess) {
    cudaEventElapsedTime(&ms, w.ev0, w.ev1);
    if (a.total_items) cudaEventElapsedTime(&kms, w.ek0, w.ek1);
  }
  if (e != cudaSuccess) return cuda_fail(w, e, "range verification");
  if (ctr[kCtrQueueOvf]) return fail(w, GB_EOVERFLOW, "Phase-2 queue overflow: raise the halo");
  if (res) {
    std::memset(res, 0, sizeof *res);
    uint64_t checked = 0;
    for (uint64_t sgi = o.shard_index; sgi < nseg; sgi += sc)
      checked += std::min<uint64_t>(o.seg_size, count - sgi * o.seg_size);
    res->checked = checked;
    res->failures = ctr[kCtrFailures];
    res->verified = checked - ctr[kCtrFailures];
    res->phase2_fallbacks = ctr[kCtrFallbacks];
    res->first_failure_n = ctr[kCtrFailures] ? ctr[kCtrFirstFail] : 0;
    res->max_minp = ctr[kCtrMaxP];
    res->num_segments = nseg;
    res->queued = std::min<uint64_t>(ctr[kCtrQueue], w.queue_cap);
    res->kernel_launches = launches;
    res->device_ms = ms;
    res->kernel_ms = kms;
  }
  return GB_OK;
}

// ---------------------------------------------------------------------------
gb_status single_impl(gb_ctx* c, Workspace& w, Arena* arena, const uint64_t* n, size_t count,
                      uint64_t* p_out, uint64_t* q_out, const gb_single_opts* opts,
                      gb_single_result* res) {
  if (count && (!n || !p_out || !q_out)) return fail(w, GB_EINVAL, "null buffer");
  gb_single_opts o{};
  if (opts) o = *opts;
  if (!o.p_limit) o.p_limit = GB_PHASE2_LIMIT_DEFAULT;
  if (o.p_limit > 0xfffffffbull) return fail(w, GB_EINVAL, "p_limit above 2^32");
  gb_status st = ensure_primes(c, w, o.p_limit);
  if (st != GB_OK) return st;
  uint64_t np = 0;
  if ((st = count_le(c, w, o.p_limit, &np)) != GB_OK) return st;
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : c->stream;
  const uint64_t* dn = n;
  uint64_t *dp = p_out, *dq = q_out;
  Temps tmp(c, arena);
  if (!o.on_device && count) {
    void* t;
    if ((st = ws_buffer(c, w, tmp, 0, count * 8 * 3, &t)) != GB_OK) return st;
    dn = (const uint64_t*)t;
    dp = (uint64_t*)t + count;
    dq = (uint64_t*)t + 2 * count;
  }
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) {
    if (e == cudaSuccess && x != cudaSuccess) e = x;
  };
  chk(cudaEventRecord(w.ev0, s));
  if (!o.on_device && count) chk(cudaMemcpyAsync((void*)dn, n, count * 8, cudaMemcpyHostToDevice, s));
  chk(cudaMemsetAsync(w.ctr, 0, 4 * 8, s));
  int launches = 0;
  if (count) {
    SingleArgs a{};
    a.n = dn;
    a.count = count;
    a.p_out = dp;
    a.q_out = dq;
    a.primes = c->d_primes;
    a.nprimes = np;
    a.p_lim = o.p_limit;
    a.ctr = w.ctr;
    uint64_t grid = (uint64_t)c->sm_count * 6;
    grid = std::min<uint64_t>(grid, (count + 7) / 8);
    chk(launch_single(a, (int)std::max<uint64_t>(grid, 1), s));
    ++launches;
  }
  if (!o.on_device && count) {
    chk(cudaMemcpyAsync(p_out, dp, count * 8, cudaMemcpyDeviceToHost, s));
    chk(cudaMemcpyAsync(q_out, dq, count * 8, cudaMemcpyDeviceToHost, s));
  }
  chk(cudaEventRecord(w.ev1, s));
  unsigned long long ctr[4] = {0, 0, 0, 0};
  chk(cudaMemcpyAsync(ctr, w.ctr, sizeof ctr, cudaMemcpyDeviceToHost, s));
  chk(cudaStreamSynchronize(s));
  float ms = 0;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, w.ev0, w.ev1);
  if (e != cudaSuccess) return cuda_fail(w, e, "single batch");
  if (res) {
    res->found = ctr[1];
    res->max_p = ctr[2];
    res->kernel_launches = launches;
    res->device_ms = ms;
  }
  return GB_OK;
}

}  // namespace gb

using namespace gb;

// ---------------------------------------------------------------------------
extern "C" {

const char* gb_strerror(gb_status st) {
  switch (st) {
    case GB_OK: return "ok";
    case GB_EINVAL: return "invalid argument";
    case GB_ENOMEM: return "insufficient device memory";
    case GB_ECUDA: return "CUDA error";
    case GB_ETIMEOUT: return "timed out";
    case GB_ECANCELED: return "cancelled";
    case GB_ENODEV: return "no CUDA device";
    case GB_EOVERFLOW: return "internal queue overflow";
    case GB_EAGAIN: return "not ready";
    case GB_EBUSY: return "busy: queued work at its bound";
    default: return "unknown error";
  }
}

const char* gb_last_error(const gb_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

gb_status gb_mem_info(const gb_ctx* ctx, uint64_t* held, uint64_t* budget) {
  if (!ctx) return GB_EINVAL;
  if (held) *held = ctx->held;
  if (budget) *budget = ctx->budget;
  return GB_OK;
}

int gb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

gb_status gb_device_info(int device, char* name, size_t name_len, uint64_t* total_mem) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    cudaGetLastError();
    return GB_ENODEV;
  }
  if (name && name_len) {
    std::strncpy(name, prop.name, name_len - 1);
    name[name_len - 1] = 0;
  }
  if (total_mem) *total_mem = prop.totalGlobalMem;
  return GB_OK;
}

uint64_t gb_estimate_device_bytes(const gb_config* cfg) {
  uint64_t want = GB_PHASE2_LIMIT_DEFAULT;
  if (cfg && cfg->cand_limit) want = cfg->cand_limit;
  if (cfg && cfg->max_n) want = std::max<uint64_t>(want, isqrt_u64(cfg->max_n) + 2);
  want = std::max<uint64_t>(want, 1ull << 22);
  const uint64_t np = pi_upper(want);
  // primes + reciprocals + class offsets, the build bitset and scan
  // blocks, wheels, counters, histogram, the Phase-2 queue, and the range
  // search's survivor lists (2 CTAs on up to 160 SMs, 2 sets of 3 lists of
  // up to 2^20/96 + 512 words)
  return np * 20 + want / 16 + (want / 65536 + 1) * 4 + (kWheelWords + kWheel6Words) * 4 +
         kCtrCount * 8 + GB_HIST_BINS * 8 + (1ull << 20) * sizeof(QEntry) +
         320ull * 6 * ((1u << 20) / 96 + 512) * 8;
}

gb_status gb_create(int device, const gb_config* cfg, gb_ctx** out) {
  if (!out) return GB_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return GB_ENODEV;
  }
  if (device < 0 || device >= ndev) return GB_EINVAL;
  gb_ctx* c = new (std::nothrow) gb_ctx();
  if (!c) return GB_ENOMEM;
  c->device = device;
  auto bail = [&](gb_status st) {
    gb_destroy(c);
    return st;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(GB_ECUDA);
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(GB_ECUDA);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  c->budget = (cfg && cfg->device_mem_budget) ? cfg->device_mem_budget : (uint64_t)fr;
  if (dev_alloc(c, (void**)&c->d_wheel, kWheelWords * 4) != GB_OK ||
      dev_alloc(c, (void**)&c->d_wheel6, kWheel6Words * 4) != GB_OK)
    return bail(GB_ENOMEM);
  if (launch_wheel_init(c->d_wheel, c->d_wheel6, c->stream) != cudaSuccess) return bail(GB_ECUDA);
  gb_status st = ws_init(c, c->ws, 1u << 20);
  if (st != GB_OK) return bail(st);
  uint64_t want = GB_PHASE2_LIMIT_DEFAULT;
  if (cfg && cfg->cand_limit) want = cfg->cand_limit;
  if (cfg && cfg->max_n) want = std::max<uint64_t>(want, isqrt_u64(cfg->max_n) + 2);
  if ((st = ensure_primes(c, c->ws, want)) != GB_OK) return bail(st);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(GB_ECUDA);
  *out = c;
  return GB_OK;
}

void gb_serve_shutdown(gb_ctx* ctx);  // gb_serve.cpp

void gb_destroy(gb_ctx* c) {
  if (!c) return;
  gb_serve_shutdown(c);
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  ws_free(c, c->ws);
  std::vector<void*> ptrs;
  for (auto& kv : c->allocs) ptrs.push_back(kv.first);
  for (void* p : ptrs) dev_free(c, p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

uint64_t gb_num_segments(uint64_t start, uint64_t limit, uint64_t seg_size) {
  if (limit & 1) limit--;
  if (start < 4) start = 4;
  if (start & 1) start++;
  if (start > limit || seg_size == 0) return 0;
  const uint64_t count = (limit - start) / 2 + 1;
  return (count + seg_size - 1) / seg_size;
}

#define GB_PUBLIC(ctx, call)                  \
  do {                                        \
    std::lock_guard<std::mutex> lk(ctx->mu);  \
    cudaSetDevice(ctx->device);               \
    ctx->ws.err.clear();                      \
    const gb_status st_ = (call);             \
    ctx->err = ctx->ws.err;                   \
    return st_;                               \
  } while (0)

gb_status gb_verify_range(gb_ctx* c, uint64_t start, uint64_t limit, const gb_range_opts* opts,
                          gb_range_result* res, const gb_range_out* out) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, range_impl(c, c->ws, nullptr, start, limit, opts, res, out));
}

gb_status gb_check_single_batch(gb_ctx* c, const uint64_t* n, size_t count, uint64_t* p_out,
                                uint64_t* q_out, const gb_single_opts* opts,
                                gb_single_result* res) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, single_impl(c, c->ws, nullptr, n, count, p_out, q_out, opts, res));
}

gb_status gb_verify_windows(gb_ctx* c, const gb_window* w, size_t count, const gb_windows_opts* opts,
                            gb_window_result* res, uint32_t* min_p_concat, gb_windows_summary* sum) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, windows_impl(c, c->ws, nullptr, w, count, opts, res, min_p_concat, sum));
}

static gb_status sieve_bitset_impl(gb_ctx* c, Workspace& w, uint64_t q_lo, uint64_t nbits,
                                   uint32_t* words, int on_device, void* stream) {
  if (!words || !(q_lo & 1)) return fail(w, GB_EINVAL, "q_lo must be odd");
  if (nbits == 0) return GB_OK;
  // the last bit's q, q_lo + 2 (nbits - 1), must not pass 2^64 - 1
  if (nbits - 1 > (UINT64_MAX - q_lo) / 2) return fail(w, GB_EINVAL, "window passes 2^64");
  const uint64_t top = q_lo + 2 * (nbits - 1);
  const uint64_t root = isqrt_u64(top);
  gb_status st = ensure_primes(c, w, root + 2);
  if (st != GB_OK) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  Temps tmp(c, nullptr);
  uint32_t* d = words;
  const uint64_t nwords = (nbits + 31) / 32;
  if (!on_device && (st = ws_buffer(c, w, tmp, 0, nwords * 4, (void**)&d)) != GB_OK) return st;
  const uint32_t tile = 1u << 18;
  uint64_t ns = 0, kc = 0;
  if ((st = count_le(c, w, root, &ns)) != GB_OK || (st = count_le(c, w, tile / 64, &kc)) != GB_OK)
    return st;
  SieveArgs a{};
  a.q_lo = q_lo;
  a.nbits = nbits;
  a.tile_bits = tile;
  a.primes = c->d_primes;
  a.magic = c->d_magic;
  a.nsieve = (uint32_t)std::max<uint64_t>(ns, kWheelPrimeCount + 1);
  a.kcoop = (uint32_t)std::max<uint64_t>(std::min(kc, ns), kWheelPrimeCount + 1);
  a.wheel = c->d_wheel;
  a.out = d;
  cudaError_t e = launch_sieve_bits(a, s);
  if (e == cudaSuccess && !on_device) e = cudaMemcpyAsync(words, d, nwords * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(w, e, "sieve bitset");
  return GB_OK;
}

gb_status gb_sieve_bitset(gb_ctx* c, uint64_t q_lo, uint64_t nbits, uint32_t* words, int on_device,
                          void* stream) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, sieve_bitset_impl(c, c->ws, q_lo, nbits, words, on_device, stream));
}

// Autotuner: candidates timed on a sample slice at the top of the range
// (where the sieving primes are largest, so the slice is the range's
// hardest), through range_impl with no per-n outputs.
static gb_status autotune_impl(gb_ctx* c, Workspace& w, uint64_t start, uint64_t limit,
                               const gb_range_opts* base, gb_range_opts* tuned,
                               gb_autotune_result* res) {
  if (!tuned) return fail(w, GB_EINVAL, "null tuned");
  gb_range_opts o{};
  if (base) o = *base;
  gb_autotune_result r{};
  if (limit & 1) limit--;
  if (start < 4) start = 4;
  if (start == UINT64_MAX) return fail(w, GB_EINVAL, "start must be <= limit");
  if (start & 1) start++;
  if (start > limit) return fail(w, GB_EINVAL, "start must be <= limit");
  const uint64_t count = (limit - start) / 2 + 1;
  const uint64_t p_small = o.p_small ? o.p_small : 1000000ull;
  const uint64_t phase2 = o.phase2_limit ? o.phase2_limit : GB_PHASE2_LIMIT_DEFAULT;
  uint64_t bits = 0;
  for (uint64_t x = limit; x; x >>= 1) ++bits;
  const std::vector<uint64_t> key{bits, p_small, phase2};
  *tuned = o;
  if (count < (1ull << 22)) {  // too short to be worth timing: the defaults
    if (res) *res = r;
    return GB_OK;
  }
  auto it = c->tuned.find(key);
  if (it != c->tuned.end()) {
    tuned->chunk_evens = it->second.chunk;
    tuned->halo = it->second.halo;
    tuned->block_threads = it->second.threads;
    r.chunk_evens = it->second.chunk;
    r.halo = it->second.halo;
    r.block_threads = it->second.threads;
    r.even_n_per_s = it->second.rate;
    r.cached = 1;
    if (res) *res = r;
    return GB_OK;
  }
  const uint64_t sample = std::min<uint64_t>(count, 1ull << 28);
  const uint64_t s0 = limit - 2 * (sample - 1);
  gb_range_opts t = o;
  t.on_device = 0;
  t.shard_index = 0;
  t.shard_count = 1;
  gb_range_result rr{};
  gb_status st = range_impl(c, w, nullptr, s0, limit, &t, &rr, nullptr);  // warm-up
  if (st != GB_OK) return st;
  double best = -1;
  for (uint32_t threads : {512u, 256u, 1024u})
    for (uint32_t chunk : {1u << 18, 1u << 19, 1u << 20})
      for (uint32_t halo : {1u << 14, 1u << 15, 1u << 16}) {
        t.chunk_evens = chunk;
        t.halo = halo;
        t.block_threads = threads;
        if ((st = range_impl(c, w, nullptr, s0, limit, &t, &rr, nullptr)) != GB_OK) return st;
        ++r.candidates;
        const double rate = rr.kernel_ms > 0 ? sample / (rr.kernel_ms / 1e3) : 0;
        if (rate > best) {
          best = rate;
          r.chunk_evens = chunk;
          r.halo = halo;
          r.block_threads = threads;
        }
      }
  r.even_n_per_s = best;
  r.sample_evens = sample;
  c->tuned[key] = gb_ctx::Tuned{r.chunk_evens, r.halo, r.block_threads, best};
  tuned->chunk_evens = r.chunk_evens;
  tuned->halo = r.halo;
  tuned->block_threads = r.block_threads;
  if (res) *res = r;
  return GB_OK;
}

gb_status gb_autotune_range(gb_ctx* c, uint64_t start, uint64_t limit, const gb_range_opts* base,
                            gb_range_opts* tuned, gb_autotune_result* res) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, autotune_impl(c, c->ws, start, limit, base, tuned, res));
}

gb_status gb_check_big(gb_ctx* c, const uint32_t* n_limbs, uint32_t nlimbs, uint64_t p_limit,
                       uint64_t* p_out, uint32_t* q_limbs, gb_big_result* res) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, big_impl(c, c->ws, n_limbs, nlimbs, p_limit, p_out, q_limbs, res));
}

gb_status gb_autotune_windows(gb_ctx* c, const gb_window* w, size_t count, const gb_windows_opts* base,
                              gb_windows_opts* tuned, gb_windows_tune* res) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, autotune_windows_impl(c, c->ws, w, count, base, tuned, res));
}

// Partition counts (kernels/counts.cu): the odd-prime bitset of [1, n_max]
// is sieved into a padded device buffer (two zero words in front, slack
// behind for the correlation's 64-bit windows), then one warp per 32
// consecutive n and slice of the bitset's words.
static gb_status counts_impl(gb_ctx* c, Workspace& w, uint64_t start, uint64_t count,
                             uint64_t* counts, const gb_count_opts* opts) {
  if (!count) return GB_OK;
  if (!counts) return fail(w, GB_EINVAL, "null counts");
  if (start < 4) start = 4;
  if (start & 1) start++;
  if (count > (GB_COUNTS_MAX_N - start) / 2 + 1 || start > GB_COUNTS_MAX_N)
    return fail(w, GB_EINVAL, "n above the partition-count limit (2^40)");
  gb_count_opts o{};
  if (opts) o = *opts;
  const uint64_t n_max = start + 2 * (count - 1);
  const uint64_t nbits = (n_max - 1) / 2 + 1;  // odd q = 1 .. n_max - 1
  const uint64_t nwords = (nbits + 31) / 32;
  gb_status st = ensure_primes(c, w, isqrt_u64(n_max) + 2);
  if (st != GB_OK) return st;
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : c->stream;
  Temps tmp(c, nullptr);
  uint32_t* buf = nullptr;
  unsigned long long* d_out = (unsigned long long*)counts;
  if ((st = ws_buffer(c, w, tmp, 0, (nwords + 8) * 4, (void**)&buf)) != GB_OK) return st;
  if (!o.on_device && (st = ws_buffer(c, w, tmp, 1, count * 8, (void**)&d_out)) != GB_OK) return st;
  const uint32_t tile = 1u << 18;
  const uint64_t root = isqrt_u64(n_max);
  uint64_t ns = 0, kc = 0;
  if ((st = count_le(c, w, root, &ns)) != GB_OK || (st = count_le(c, w, tile / 64, &kc)) != GB_OK)
    return st;
  SieveArgs a{};
  a.q_lo = 1;
  a.nbits = nbits;
  a.tile_bits = tile;
  a.primes = c->d_primes;
  a.magic = c->d_magic;
  a.nsieve = (uint32_t)std::max<uint64_t>(ns, kWheelPrimeCount + 1);
  a.kcoop = (uint32_t)std::max<uint64_t>(std::min(kc, ns), kWheelPrimeCount + 1);
  a.wheel = c->d_wheel;
  a.out = buf + 2;
  // Work split: enough warp tasks to fill the GPU, at most 2^22 words each.
  const uint64_t groups = (count + 31) / 32;
  const uint64_t wmax = n_max / 4 / 32 + 1;  // words of i for the largest n
  uint64_t splits = std::max<uint64_t>(1, ((uint64_t)c->sm_count * 64 + groups - 1) / groups);
  splits = std::max<uint64_t>(splits, (wmax + (1u << 22) - 1) >> 22);
  uint64_t wps = (wmax + splits - 1) / splits;
  wps = std::max<uint64_t>(32, (wps + 31) & ~31ull);
  splits = (wmax + wps - 1) / wps;
  cudaError_t e = cudaMemsetAsync(buf, 0, (nwords + 8) * 4, s);
  if (e == cudaSuccess) e = launch_sieve_bits(a, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, count * 8, s);
  if (e == cudaSuccess) e = cudaEventRecord(w.ek0, s);
  if (e == cudaSuccess) e = launch_counts(buf + 2, start / 2 - 1, count, (uint32_t)splits, wps, d_out, s);
  if (e == cudaSuccess) e = cudaEventRecord(w.ek1, s);
  if (e == cudaSuccess && !o.on_device) e = cudaMemcpyAsync(counts, d_out, count * 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(w, e, "partition counts");
  return GB_OK;
}

gb_status gb_goldbach_counts(gb_ctx* c, uint64_t start, uint64_t count, uint64_t* counts,
                             const gb_count_opts* opts) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, counts_impl(c, c->ws, start, count, counts, opts));
}

static gb_status primes_upto_impl(gb_ctx* c, Workspace& w, uint64_t limit, uint32_t* primes,
                                  uint64_t cap, uint64_t* count) {
  if (!count) return fail(w, GB_EINVAL, "null count");
  if (limit > 0xfffffffbull) return fail(w, GB_EINVAL, "limit above the 32-bit prime table");
  gb_status st = ensure_primes(c, w, std::max<uint64_t>(limit, 2));
  if (st != GB_OK) return st;
  uint64_t n = 0;
  if ((st = count_le(c, w, limit, &n)) != GB_OK) return st;
  *count = n;
  if (primes && cap) GB_CU(cudaMemcpy(primes, c->d_primes, std::min(n, cap) * 4, cudaMemcpyDeviceToHost), "primes copy");
  return GB_OK;
}

gb_status gb_primes_upto(gb_ctx* c, uint64_t limit, uint32_t* primes, uint64_t cap, uint64_t* count) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, primes_upto_impl(c, c->ws, limit, primes, cap, count));
}

static gb_status is_prime_impl(gb_ctx* c, Workspace& w, const uint64_t* n, size_t count,
                               uint8_t* out, int on_device, void* stream) {
  if (count && (!n || !out)) return fail(w, GB_EINVAL, "null buffer");
  if (!count) return GB_OK;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  const uint64_t* dn = n;
  uint8_t* dout = out;
  Temps tmp(c, nullptr);
  gb_status st;
  if (!on_device) {
    if ((st = ws_buffer(c, w, tmp, 0, count * 8, (void**)&dn)) != GB_OK ||
        (st = ws_buffer(c, w, tmp, 1, count, (void**)&dout)) != GB_OK)
      return st;
  }
  cudaError_t e = cudaSuccess;
  if (!on_device) e = cudaMemcpyAsync((void*)dn, n, count * 8, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_is_prime(dn, count, dout, s);
  if (e == cudaSuccess && !on_device) e = cudaMemcpyAsync(out, dout, count, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(w, e, "is_prime batch");
  return GB_OK;
}

gb_status gb_is_prime_batch(gb_ctx* c, const uint64_t* n, size_t count, uint8_t* out, int on_device,
                            void* stream) {
  if (!c) return GB_EINVAL;
  GB_PUBLIC(c, is_prime_impl(c, c->ws, n, count, out, on_device, stream));
}

}  // extern "C"

extern "C" gb_status gb_probe_peaks(gb_ctx* c, double* alu_ops_per_s, double* smem_atomics_per_s) {
  if (!c || !alu_ops_per_s || !smem_atomics_per_s) return GB_EINVAL;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (run_probe(0, c->sm_count, alu_ops_per_s, c->stream) != cudaSuccess ||
      run_probe(1, c->sm_count, smem_atomics_per_s, c->stream) != cudaSuccess)
    return GB_ECUDA;
  return GB_OK;
}

extern "C" gb_status gb_probe_mont_products(gb_ctx* c, double* per_s) {
  if (!c || !per_s) return GB_EINVAL;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  return run_probe(2, c->sm_count, per_s, c->stream) == cudaSuccess ? GB_OK : GB_ECUDA;
}
