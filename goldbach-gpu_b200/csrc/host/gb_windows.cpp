// gb_windows.cpp -- C-ABI entry point for batched windows.
//
// Many independent windows of consecutive even n (e.g. 4096 windows at
// offsets in [1e15, 1e18]) in one batch.  The reference has no batch mode:
// each window would be one `goldbach --start=A LIMIT` process with its own
// segment loop (src/goldbach.cu:420-485).  GB_WINDOWS_PERSISTENT runs the
// batch as one CUDA graph of three launches: the large-prime pass over
// every window's class masks (kernels/windows.cu), range6_kernel in windows
// mode over every (window, chunk) item from one device work counter, and the
// device Phase 2.
// GB_WINDOWS_PLAIN runs the same launches window by window (the per-window
// launch pipeline, kept for comparison).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "gb_ctx.h"

namespace gb {
// Primes up to this bound sieve each chunk's q-window in shared memory; the
// larger ones go through the large-prime pass (kernels/windows.cu), whose
// quotient estimate needs p > 2^17.
constexpr uint64_t kWinChunkSieveBound = 1ull << 20;
// CTAs per SM of the large-prime pass (grid-stride over the primes: a fine
// grid evens out primes that visit many windows and primes that visit few)
constexpr uint64_t kLargeBlocksPerSM = 64;
// Default break-even divisor of the Miller-Rabin split (see windows_impl).
constexpr double kMrBelowDivisor = 2600.0;

// floor((A - H - 1) / 6) for A possibly below H (range.cu window_g0)
static int64_t host_window_g0(uint64_t A, uint32_t H) {
  if (A >= (uint64_t)H + 1) return (int64_t)((A - H - 1) / 6);
  return -(int64_t)(((uint64_t)H + 1 - A + 5) / 6);
}

// The sieve pipeline over windows w[0..count).
static gb_status windows_sieve_impl(gb_ctx* c, Workspace& ws, Arena* arena, const gb_window* w,
                                    size_t count, const gb_windows_opts* opts, gb_window_result* res,
                                    uint32_t* min_p_concat, gb_windows_summary* sum) {
  if (count && !w) return fail(ws, GB_EINVAL, "null windows");
  gb_windows_opts o{};
  if (opts) o = *opts;
  if (o.mode != GB_WINDOWS_PERSISTENT && o.mode != GB_WINDOWS_PLAIN)
    return fail(ws, GB_EINVAL, "unknown windows mode");
  if (o.on_device) return fail(ws, GB_EINVAL, "windows: on_device outputs are not supported");
  if (sum) std::memset(sum, 0, sizeof *sum);
  if (count == 0) return GB_OK;
  if (count > 0xffffffffull) return fail(ws, GB_EINVAL, "too many windows");
  const uint32_t H = o.halo ? o.halo : 32768u;
  if (H < 128 || H > (1u << 17) || (H & 63)) return fail(ws, GB_EINVAL, "halo must be a multiple of 64 in [128, 2^17]");
  uint32_t NE = o.chunk_evens ? o.chunk_evens : (1u << 20);
  if (NE < 8192 || NE > (1u << 20) || (NE & (NE - 1)))
    return fail(ws, GB_EINVAL, "chunk_evens must be a power of two in [2^13, 2^20]");
  if (min_p_concat && NE > kMinpChunk) NE = kMinpChunk;  // per-n output: smaller chunks
  if (o.block_threads && o.block_threads != 256 && o.block_threads != 512 && o.block_threads != 1024)
    return fail(ws, GB_EINVAL, "block_threads must be 256, 512 or 1024");
  const uint64_t p_lim = o.phase2_limit ? o.phase2_limit : GB_PHASE2_LIMIT_DEFAULT;
  if (p_lim > GB_P_SMALL_MAX) return fail(ws, GB_EINVAL, "phase2_limit must be <= 4e9");
  const uint64_t large_per_sm = o.large_ctas_per_sm ? o.large_ctas_per_sm : kLargeBlocksPerSM;
  if (o.gpu_share_pct > 100) return fail(ws, GB_EINVAL, "gpu_share_pct must be <= 100");
  const uint64_t share = o.gpu_share_pct ? o.gpu_share_pct : 100;
  uint64_t total_n = 0, q_max = 0;
  for (size_t i = 0; i < count; ++i) {
    if (w[i].start < 4 || (w[i].start & 1) || w[i].count == 0)
      return fail(ws, GB_EINVAL, "window start must be even and >= 4, count >= 1");
    const uint64_t last = w[i].start + 2 * (w[i].count - 1);
    if (w[i].count > GB_WINDOW_MAX_COUNT) return fail(ws, GB_EINVAL, "window wider than GB_WINDOW_MAX_COUNT");
    if (last < w[i].start) return fail(ws, GB_EINVAL, "window passes 2^64");
    q_max = std::max(q_max, last);
    total_n += w[i].count;
  }
  const uint64_t root = isqrt_u64(q_max);
  gb_status st = ensure_primes(c, ws, std::max<uint64_t>({p_lim, (uint64_t)H, root + 2, kWinChunkSieveBound}));
  if (st != GB_OK) return st;
  const uint32_t nbw = range6_words(H, NE);
  // descriptors, sorted by top q so that a prime visits a suffix of them
  std::vector<uint32_t> order(count);
  std::iota(order.begin(), order.end(), 0u);
  std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
    return w[x].start + 2 * (w[x].count - 1) < w[y].start + 2 * (w[y].count - 1);
  });
  std::vector<uint64_t> out_off(count + 1, 0);
  for (size_t i = 0; i < count; ++i) out_off[i + 1] = out_off[i] + w[i].count;
  std::vector<WinDesc6> desc(count);
  std::vector<WinLarge> wl(count);
  std::vector<uint64_t> chunk_off(count + 1, 0), chunk_one(2 * count, 0);
  uint64_t lwords_total = 0;
  for (size_t r = 0; r < count; ++r) {
    const uint32_t i = order[r];
    WinDesc6& d = desc[r];
    d.start = w[i].start;
    d.count = w[i].count;
    d.out_off = out_off[i];
    d.q_top = d.start + 2 * (d.count - 1);
    d.g0 = host_window_g0(d.start, H);
    d.orig = i;
    const uint64_t chunks = (d.count + NE - 1) / NE;
    // a chunk reads nwords + 1 mask words from its own base on (nwords as in
    // range6_kernel: the words its search can read for a real n); the mask
    // ends there, so the large-prime pass marks no bit nobody reads
    auto reach = [&](uint64_t ci) {  // mask words chunk ci reads, from the window base
      const uint64_t cnt = std::min<uint64_t>(NE, d.count - ci * NE);
      const uint64_t nbits = H / 6 + cnt / 3 + 96;
      const uint64_t nwords = std::min<uint64_t>(nbw, (nbits + 31) / 32 + 2);
      const int64_t gc = host_window_g0(d.start + 2 * (uint64_t)NE * ci, H);
      return ((uint64_t)(gc - d.g0) >> 5) + nwords + 2;
    };
    // the last full chunk or the (possibly short) last one reaches furthest
    uint64_t lw = reach(chunks - 1);
    if (chunks >= 2) lw = std::max(lw, reach(chunks - 2));
    d.lwords = (uint32_t)((lw + 3) & ~3ull);
    d.lbase = lwords_total;
    lwords_total += 2ull * d.lwords;
    wl[r].gd = (double)d.g0;
    wl[r].gl = (uint32_t)(uint64_t)d.g0;
    wl[r].lbits = d.g0 >= (int64_t)(1ll << 30) ? d.lwords * 32 : 0xffffffffu;
    chunk_off[r + 1] = chunk_off[r] + chunks;
    chunk_one[2 * r + 1] = chunks;
  }
  uint64_t ns = 0, kf = 0, nsmall = 0, nlarge = 0, kc = 0;
  if ((st = count_le(c, ws, std::min<uint64_t>(H - 13, p_lim), &ns)) != GB_OK ||
      (st = count_le(c, ws, p_lim, &kf)) != GB_OK ||
      (st = count_le(c, ws, std::min<uint64_t>(kWinChunkSieveBound, root), &nsmall)) != GB_OK ||
      (st = count_le(c, ws, root, &nlarge)) != GB_OK ||
      (st = count_le(c, ws, (H / 6 + NE / 3) / 64, &kc)) != GB_OK)
    return st;

  Temps tmp(c, arena);
  void *d_desc, *d_wl, *d_coff, *d_cone, *d_lmask, *d_fail, *d_maxp, *d_psum, *d_minp = nullptr;
  if ((st = ws_buffer(c, ws, tmp, 0, count * sizeof(WinDesc6), &d_desc)) != GB_OK ||
      (st = ws_buffer(c, ws, tmp, 1, count * sizeof(WinLarge), &d_wl)) != GB_OK ||
      (st = ws_buffer(c, ws, tmp, 2, (count + 1) * 8, &d_coff)) != GB_OK ||
      (st = ws_buffer(c, ws, tmp, 3, 2 * count * 8, &d_cone)) != GB_OK ||
      (st = ws_buffer(c, ws, tmp, 4, lwords_total * 4, &d_lmask)) != GB_OK ||
      (st = ws_buffer(c, ws, tmp, 5, count * 4, &d_fail)) != GB_OK ||
      (st = ws_buffer(c, ws, tmp, 6, count * 8, &d_maxp)) != GB_OK ||
      (st = ws_buffer(c, ws, tmp, 7, count * 8, &d_psum)) != GB_OK ||
      (min_p_concat && (st = ws_buffer(c, ws, tmp, 8, total_n * 4, &d_minp)) != GB_OK))
    return st;

  RangeArgs a{};
  SearchParams& sp = a.s;
  sp.halo = H;
  sp.nsearch = (uint32_t)ns;
  sp.kfb = (uint32_t)std::min<uint64_t>(kf, 0xffffffffu);
  sp.p_lim = p_lim;
  sp.p_small = p_lim;
  sp.primes = c->d_primes;
  sp.nprimes = c->nprimes;
  sp.ctr = ws.ctr;
  sp.unit_failures = (uint32_t*)d_fail;
  sp.unit_maxp = (unsigned long long*)d_maxp;
  sp.unit_psum = (unsigned long long*)d_psum;
  sp.minp = (uint32_t*)d_minp;
  sp.queue = ws.queue;
  sp.queue_cap = ws.queue_cap;
  a.chunk_evens = NE;
  a.threads = o.block_threads;
  a.nbw = nbw;
  a.magic = c->d_magic;
  a.nsieve = (uint32_t)std::max<uint64_t>(nsmall, kWheelPrimeCount + 1);
  a.kcoop = (uint32_t)std::max<uint64_t>(std::min(kc, nsmall), kWheelPrimeCount + 1);
  a.wheel6 = c->d_wheel6;
  a.a15 = c->d_a15;
  a.win = (const WinDesc6*)d_desc;
  a.chunk_off = (const uint64_t*)d_coff;
  a.nwin = (uint32_t)count;
  a.lmask = (const uint32_t*)d_lmask;
  a.total_items = chunk_off[count];
  WinLargeArgs la{};
  la.win = (const WinDesc6*)d_desc;
  la.wl = (const WinLarge*)d_wl;
  la.w_lo = 0;
  la.w_hi = (uint32_t)count;
  la.primes = c->d_primes;
  la.magic = c->d_magic;
  la.a15 = c->d_a15;
  la.k0 = (uint32_t)std::max<uint64_t>(nsmall, kWheelPrimeCount + 1);
  la.k1 = (uint32_t)std::max<uint64_t>(nlarge, la.k0);
  la.lmask = (uint32_t*)d_lmask;

  const int sm = c->sm_count;
  int bps = range_max_blocks_per_sm(a);
  if (bps < 1) bps = 1;
  // CTAs the chunk kernel may keep resident: its share of the GPU
  const uint64_t grid_max = std::max<uint64_t>(1, (uint64_t)sm * bps * share / 100);
  a.surv_cap = nbw;
  {
    void* p = nullptr;
    if ((st = ws_scratch(c, ws, (size_t)grid_max * 6 * a.surv_cap * sizeof(uint2), &p)) != GB_OK) return st;
    a.surv = (uint2*)p;
  }
  const uint64_t np = la.k1 - la.k0;
  // the large-prime pass is not capped by the share: its CTAs are short
  // (a few primes each, grid-stride) and free their slots as they finish,
  // where higher-priority work takes them; a capped grid left it with too
  // few warps per SM to hide its loads
  const int gl = (int)std::max<uint64_t>(1, std::min<uint64_t>((np + 255) / 256, (uint64_t)sm * large_per_sm));

  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : c->stream;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) {
    if (e == cudaSuccess && x != cudaSuccess) e = x;
  };
  chk(cudaMemcpyAsync(d_desc, desc.data(), count * sizeof(WinDesc6), cudaMemcpyHostToDevice, s));
  chk(cudaMemcpyAsync(d_wl, wl.data(), count * sizeof(WinLarge), cudaMemcpyHostToDevice, s));
  chk(cudaMemcpyAsync(d_coff, chunk_off.data(), (count + 1) * 8, cudaMemcpyHostToDevice, s));
  chk(cudaMemcpyAsync(d_cone, chunk_one.data(), 2 * count * 8, cudaMemcpyHostToDevice, s));
  chk(cudaMemsetAsync(d_fail, 0, count * 4, s));
  chk(cudaMemsetAsync(d_maxp, 0, count * 8, s));
  chk(cudaMemsetAsync(d_psum, 0, count * 8, s));
  if (d_minp) chk(cudaMemsetAsync(d_minp, 0, total_n * 4, s));
  chk(cudaMemsetAsync(sp.ctr, 0, kCtrCount * 8, s));
  chk(cudaMemsetAsync(sp.ctr + kCtrFirstFail, 0xff, 8, s));
  chk(launch_win_pairs((const WinDesc6*)d_desc, (uint32_t)count, c->d_primes, c->nprimes, la.k0,
                       sp.ctr + kCtrWork2, s));
  chk(cudaStreamSynchronize(s));  // host vectors above are pageable and local
  int launches = 0;
  float large_ms = 0, search_ms = 0;
  chk(cudaEventRecord(ws.ev0, s));
  if (o.mode == GB_WINDOWS_PERSISTENT) {
    // The batch's launches as one CUDA graph: captured per call (the
    // arguments change), applied to the workspace's executable graph by an
    // in-place update -- the topology repeats from batch to batch, so the
    // graph is instantiated once and relaunched -- and launched as one unit.
    // A caller that is itself capturing the stream gets the launches inline.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    chk(cudaStreamIsCapturing(s, &cs));
    const bool graph = e == cudaSuccess && cs == cudaStreamCaptureStatusNone;
    auto mark = [&](cudaEvent_t ev) {  // timing events: nodes of the graph
      chk(graph ? cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal) : cudaEventRecord(ev, s));
    };
    if (graph) chk(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    chk(cudaMemsetAsync(d_lmask, 0xff, lwords_total * 4, s));
    mark(ws.ek0);
    if (la.k1 > la.k0) {
      chk(launch_win_large(la, gl, s));
      ++launches;
    }
    mark(ws.ek1);
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(grid_max, a.total_items));
    chk(launch_range(a, grid, s));
    mark(ws.ek2);
    chk(launch_fallback(sp, sm * 4, s));
    launches += 2;
    if (graph) {
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(s, &g);  // ends the capture in every case
      chk(ec);
      if (e == cudaSuccess) {
        cudaGraphExecUpdateResultInfo info{};
        if (!ws.win_exec || cudaGraphExecUpdate(ws.win_exec, g, &info) != cudaSuccess) {
          cudaGetLastError();  // another topology: instantiate anew
          if (ws.win_exec) cudaGraphExecDestroy(ws.win_exec);
          ws.win_exec = nullptr;
          chk(cudaGraphInstantiate(&ws.win_exec, g, 0));
        }
        if (e == cudaSuccess) chk(cudaGraphLaunch(ws.win_exec, s));
      }
      if (g) cudaGraphDestroy(g);
    }
  } else {
    for (uint32_t r = 0; r < count && e == cudaSuccess; ++r) {
      const WinDesc6& d = desc[r];
      chk(cudaMemsetAsync((uint32_t*)d_lmask + d.lbase, 0xff, 2ull * d.lwords * 4, s));
      chk(cudaMemsetAsync(sp.ctr + kCtrWork, 0, 8, s));
      chk(cudaMemsetAsync(sp.ctr + kCtrQueue, 0, 8, s));
      WinLargeArgs l1 = la;
      l1.w_lo = r;
      l1.w_hi = r + 1;
      if (l1.k1 > l1.k0 && d.q_top >= kWinChunkSieveBound * kWinChunkSieveBound) {
        chk(launch_win_large(l1, gl, s));
        ++launches;
      }
      RangeArgs a1 = a;
      a1.win = (const WinDesc6*)d_desc + r;
      a1.chunk_off = (const uint64_t*)d_cone + 2 * r;
      a1.nwin = 1;
      a1.total_items = chunk_one[2 * r + 1];
      chk(launch_range(a1, (int)std::min<uint64_t>(grid_max, a1.total_items), s));
      chk(launch_fallback(sp, std::max(1, sm / 4), s));
      launches += 2;
    }
  }
  chk(cudaEventRecord(ws.ev1, s));
  std::vector<uint32_t> fails(count);
  std::vector<uint64_t> maxp(count), psum(count);
  unsigned long long ctr[kCtrCount];
  chk(cudaMemcpyAsync(fails.data(), d_fail, count * 4, cudaMemcpyDeviceToHost, s));
  chk(cudaMemcpyAsync(maxp.data(), d_maxp, count * 8, cudaMemcpyDeviceToHost, s));
  chk(cudaMemcpyAsync(psum.data(), d_psum, count * 8, cudaMemcpyDeviceToHost, s));
  chk(cudaMemcpyAsync(ctr, sp.ctr, sizeof ctr, cudaMemcpyDeviceToHost, s));
  if (d_minp) chk(cudaMemcpyAsync(min_p_concat, d_minp, total_n * 4, cudaMemcpyDeviceToHost, s));
  chk(cudaStreamSynchronize(s));
  float ms = 0;
  if (e == cudaSuccess) {
    cudaEventElapsedTime(&ms, ws.ev0, ws.ev1);
    if (o.mode == GB_WINDOWS_PERSISTENT) {
      cudaEventElapsedTime(&large_ms, ws.ek0, ws.ek1);
      cudaEventElapsedTime(&search_ms, ws.ek1, ws.ek2);
    }
  }
  if (e != cudaSuccess) return cuda_fail(ws, e, "windows");
  if (ctr[kCtrQueueOvf]) return fail(ws, GB_EOVERFLOW, "Phase-2 queue overflow: raise the halo");
  if (res) {
    for (size_t i = 0; i < count; ++i) {
      res[i].failures = fails[i];
      res[i].verified = w[i].count - fails[i];
      res[i].max_minp = maxp[i];
      res[i].minp_sum = psum[i];
    }
  }
  if (sum) {
    sum->total_n = total_n;
    sum->failures = ctr[kCtrFailures];
    sum->kernel_launches = launches;
    sum->device_ms = ms;
    sum->sieved_windows = count;
    sum->large_pairs = ctr[kCtrWork2];
    sum->large_ms = large_ms;
    sum->search_ms = search_ms;
  }
  return GB_OK;
}


// Narrow windows on the Miller-Rabin path: every n of every window through
// the single-n kernel (minimal p over the resident table, q by the 7-base
// MR), then one per-window reduction.  Plain mode launches the single-n
// kernel window by window.
static gb_status windows_mr_impl(gb_ctx* c, Workspace& ws, Arena* arena, const gb_window* w,
                                 size_t count, const gb_windows_opts& o, uint64_t p_lim,
                                 gb_window_result* res, uint32_t* min_p_concat,
                                 gb_windows_summary* sum) {
  uint64_t total = 0;
  std::vector<uint64_t> off(count + 1, 0);
  for (size_t i = 0; i < count; ++i) off[i + 1] = off[i] + w[i].count;
  total = off[count];
  uint64_t np = 0;
  gb_status st = count_le(c, ws, p_lim, &np);
  if (st != GB_OK) return st;
  Temps tmp(c, arena);
  void *d_w, *d_off, *d_n, *d_p, *d_q, *d_agg;
  if ((st = tmp.get(count * sizeof(gb_window), &d_w, ws)) != GB_OK ||
      (st = tmp.get((count + 1) * 8, &d_off, ws)) != GB_OK ||
      (st = tmp.get(total * 8, &d_n, ws)) != GB_OK || (st = tmp.get(total * 8, &d_p, ws)) != GB_OK ||
      (st = tmp.get(total * 8, &d_q, ws)) != GB_OK || (st = tmp.get(count * 32, &d_agg, ws)) != GB_OK)
    return st;
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : c->stream;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) {
    if (e == cudaSuccess && x != cudaSuccess) e = x;
  };
  int launches = 0;
  chk(cudaEventRecord(ws.ev0, s));
  chk(cudaMemcpyAsync(d_w, w, count * sizeof(gb_window), cudaMemcpyHostToDevice, s));
  chk(cudaMemcpyAsync(d_off, off.data(), (count + 1) * 8, cudaMemcpyHostToDevice, s));
  chk(launch_win_expand((const gb_window*)d_w, (const uint64_t*)d_off, (uint32_t)count, (uint64_t*)d_n, s));
  ++launches;
  SingleArgs a{};
  a.primes = c->d_primes;
  a.nprimes = np;
  a.p_lim = p_lim;
  a.ctr = ws.ctr;
  const size_t parts = o.mode == GB_WINDOWS_PLAIN ? count : 1;
  for (size_t i = 0; i < parts && e == cudaSuccess; ++i) {
    const uint64_t b = parts == 1 ? 0 : off[i], n = parts == 1 ? total : w[i].count;
    a.n = (const uint64_t*)d_n + b;
    a.count = n;
    a.p_out = (uint64_t*)d_p + b;
    a.q_out = (uint64_t*)d_q + b;
    chk(cudaMemsetAsync(ws.ctr, 0, 4 * 8, s));
    const uint64_t share = o.gpu_share_pct ? o.gpu_share_pct : 100;
    const uint64_t gcap = std::max<uint64_t>(1, (uint64_t)c->sm_count * 6 * share / 100);
    const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>(gcap, (n + 7) / 8));
    chk(launch_single(a, (int)grid, s));
    ++launches;
  }
  chk(launch_segment_reduce((const uint64_t*)d_p, (const uint64_t*)d_off, (uint32_t)count,
                            (unsigned long long*)d_agg, s));
  ++launches;
  chk(cudaEventRecord(ws.ev1, s));
  std::vector<unsigned long long> agg(count * 4);
  std::vector<uint64_t> pv(min_p_concat ? total : 0);
  chk(cudaMemcpyAsync(agg.data(), d_agg, count * 32, cudaMemcpyDeviceToHost, s));
  if (min_p_concat) chk(cudaMemcpyAsync(pv.data(), d_p, total * 8, cudaMemcpyDeviceToHost, s));
  chk(cudaStreamSynchronize(s));
  if (e != cudaSuccess) return cuda_fail(ws, e, "windows (Miller-Rabin path)");
  float ms = 0;
  cudaEventElapsedTime(&ms, ws.ev0, ws.ev1);
  uint64_t fails = 0;
  for (size_t i = 0; i < count; ++i) {
    if (res) {
      res[i].verified = agg[4 * i];
      res[i].failures = agg[4 * i + 1];
      res[i].max_minp = agg[4 * i + 2];
      res[i].minp_sum = agg[4 * i + 3];
    }
    fails += agg[4 * i + 1];
  }
  for (uint64_t j = 0; j < pv.size(); ++j) min_p_concat[j] = (uint32_t)pv[j];
  if (sum) {
    sum->total_n = total;
    sum->failures = fails;
    sum->kernel_launches = launches;
    sum->device_ms = ms;
  }
  return GB_OK;
}

// Splits the batch, trading the sieve bound against Miller-Rabin: windows
// narrower than the sieve's break-even take the Miller-Rabin path (the
// sieve's large-prime pass costs about 1.5 ps of GPU time per sieving prime
// per window, the single-n path about 3 ns per n, so the break-even width
// is about pi(sqrt(top)) / 2000 even n; 2600 measured best on 4096 windows
// in [1e15, 1e18]).  Results do not depend on the split.
gb_status windows_impl(gb_ctx* c, Workspace& ws, Arena* arena, const gb_window* w, size_t count,
                       const gb_windows_opts* opts, gb_window_result* res, uint32_t* min_p_concat,
                       gb_windows_summary* sum) {
  gb_windows_opts o{};
  if (opts) o = *opts;
  if (!count || !w || o.on_device || o.mr_below == 1 ||
      (o.mode != GB_WINDOWS_PERSISTENT && o.mode != GB_WINDOWS_PLAIN))
    return windows_sieve_impl(c, ws, arena, w, count, opts, res, min_p_concat, sum);
  std::vector<char> narrow(count, 0);
  size_t nn = 0;
  for (size_t i = 0; i < count; ++i) {
    const uint64_t last = w[i].start + 2 * (w[i].count - 1);
    if (w[i].start < 4 || (w[i].start & 1) || w[i].count == 0 || last < w[i].start)
      return windows_sieve_impl(c, ws, arena, w, count, opts, res, min_p_concat, sum);  // reports it
    uint64_t lim = o.mr_below;
    if (!lim) {
      const double r = std::sqrt((double)last);
      const double div = o.mr_divisor ? (double)o.mr_divisor : kMrBelowDivisor;
      lim = r > 1e4 ? (uint64_t)(1.1 * r / std::log(r) / div) : 0;
    }
    narrow[i] = w[i].count < lim;
    nn += narrow[i];
  }
  if (nn == 0) return windows_sieve_impl(c, ws, arena, w, count, opts, res, min_p_concat, sum);
  const uint64_t p_lim = o.phase2_limit ? o.phase2_limit : GB_PHASE2_LIMIT_DEFAULT;
  if (p_lim > GB_P_SMALL_MAX) return fail(ws, GB_EINVAL, "phase2_limit must be <= 4e9");
  gb_status st = ensure_primes(c, ws, std::max<uint64_t>(p_lim, kWinChunkSieveBound));
  if (st != GB_OK) return st;
  // both parts in their own arrays, results put back in the caller's order
  std::vector<gb_window> wa, wb;
  std::vector<size_t> ia, ib;
  std::vector<uint64_t> out_off(count + 1, 0);
  for (size_t i = 0; i < count; ++i) {
    out_off[i + 1] = out_off[i] + w[i].count;
    (narrow[i] ? wa : wb).push_back(w[i]);
    (narrow[i] ? ia : ib).push_back(i);
  }
  std::vector<gb_window_result> ra(wa.size()), rb(wb.size());
  uint64_t na = 0, nb = 0;
  for (const gb_window& x : wa) na += x.count;
  for (const gb_window& x : wb) nb += x.count;
  std::vector<uint32_t> ma(min_p_concat ? na : 0), mb(min_p_concat ? nb : 0);
  gb_windows_summary sa{}, sb{};
  if ((st = windows_mr_impl(c, ws, arena, wa.data(), wa.size(), o, p_lim, ra.data(),
                            min_p_concat ? ma.data() : nullptr, &sa)) != GB_OK)
    return st;
  if (!wb.empty() && (st = windows_sieve_impl(c, ws, arena, wb.data(), wb.size(), &o, rb.data(),
                                              min_p_concat ? mb.data() : nullptr, &sb)) != GB_OK)
    return st;
  uint64_t pa = 0, pb = 0;
  for (size_t k = 0; k < ia.size(); ++k) {
    if (res) res[ia[k]] = ra[k];
    if (min_p_concat) std::memcpy(min_p_concat + out_off[ia[k]], ma.data() + pa, wa[k].count * 4);
    pa += wa[k].count;
  }
  for (size_t k = 0; k < ib.size(); ++k) {
    if (res) res[ib[k]] = rb[k];
    if (min_p_concat) std::memcpy(min_p_concat + out_off[ib[k]], mb.data() + pb, wb[k].count * 4);
    pb += wb[k].count;
  }
  if (sum) {
    sum->total_n = sa.total_n + sb.total_n;
    sum->failures = sa.failures + sb.failures;
    sum->kernel_launches = sa.kernel_launches + sb.kernel_launches;
    sum->device_ms = sa.device_ms + sb.device_ms;
    sum->sieved_windows = sb.sieved_windows;
    sum->large_pairs = sb.large_pairs;
    sum->large_ms = sb.large_ms;
    sum->search_ms = sb.search_ms;
  }
  return GB_OK;
}

// Upper bound of the device bytes one window takes from a caller's arena in
// windows_impl: its share of the sieve path's buffers (descriptor, record,
// offsets, results, class masks) or, when it is narrow enough for the
// Miller-Rabin path, of that path's (its n, p, q and a reduction record);
// arena alignment included.  Used by serving to admit batches by memory.
uint64_t windows_request_bytes(const gb_window& w, const gb_windows_opts& o) {
  const uint64_t H = o.halo ? o.halo : 32768u;
  const uint64_t last = w.start + 2 * (w.count - 1);
  uint64_t lim = o.mr_below;
  if (!lim) {
    const double r = std::sqrt((double)last);
    const double div = o.mr_divisor ? (double)o.mr_divisor : kMrBelowDivisor;
    lim = r > 1e4 ? (uint64_t)(1.1 * r / std::log(r) / div) : 0;
  }
  const uint64_t fixed = sizeof(WinDesc6) + sizeof(WinLarge) + 24 + 4 + 16 + 16 + 4 * 256;
  if (w.count < lim) return fixed + w.count * 24 + 64 + 4 * 256;
  const uint64_t lwords = (w.count / 3 + H / 6 + 96) / 32 + 16;
  return fixed + 2 * lwords * 4;
}

// Autotuner of the windows pipeline: the persistent mode on a sample of the
// batch (every k-th window, at most 512) for each candidate, after one
// warm-up call; the fastest device time wins.  Cached per batch class.
gb_status autotune_windows_impl(gb_ctx* c, Workspace& ws, const gb_window* w, size_t count,
                                const gb_windows_opts* base, gb_windows_opts* tuned,
                                gb_windows_tune* res) {
  if (!tuned || (count && !w)) return fail(ws, GB_EINVAL, "null argument");
  gb_windows_opts o{};
  if (base) o = *base;
  *tuned = o;
  gb_windows_tune r{};
  if (count == 0) {
    if (res) *res = r;
    return GB_OK;
  }
  uint64_t top = 0;
  for (size_t i = 0; i < count; ++i) top = std::max<uint64_t>(top, w[i].start + 2 * (w[i].count - 1));
  uint64_t tb = 0, cb = 0;
  for (uint64_t x = top; x; x >>= 1) ++tb;
  for (uint64_t x = count; x; x >>= 1) ++cb;
  const std::vector<uint64_t> key{tb, cb, o.phase2_limit};
  auto it = c->tuned_windows.find(key);
  if (it != c->tuned_windows.end()) {
    r = it->second;
    r.candidates = 0;
    r.cached = 1;
  } else {
    const size_t step = (count + 511) / 512;
    std::vector<gb_window> smp;
    for (size_t i = 0; i < count; i += step) smp.push_back(w[i]);
    std::vector<gb_window_result> wr(smp.size());
    gb_windows_opts t = o;
    t.mode = GB_WINDOWS_PERSISTENT;
    t.on_device = 0;
    gb_windows_summary sum{};
    gb_status st = windows_impl(c, ws, nullptr, smp.data(), smp.size(), &t, wr.data(), nullptr, &sum);
    if (st != GB_OK) return st;  // warm-up (tables)
    uint64_t n = 0;
    for (const gb_window& x : smp) n += x.count;
    double best = -1;
    for (uint32_t div : {2600u, 1300u, 5200u})
      for (uint32_t chunk : {1u << 20, 1u << 19})
        for (uint32_t large : {64u, 16u})
          for (uint32_t threads : {512u, 256u}) {
            t.mr_divisor = div;
            t.chunk_evens = chunk;
            t.large_ctas_per_sm = large;
            t.block_threads = threads;
            if ((st = windows_impl(c, ws, nullptr, smp.data(), smp.size(), &t, wr.data(), nullptr,
                                   &sum)) != GB_OK)
              return st;
            ++r.candidates;
            const double rate = sum.device_ms > 0 ? n / (sum.device_ms / 1e3) : 0;
            if (rate > best) {
              best = rate;
              r.mr_divisor = div;
              r.chunk_evens = chunk;
              r.large_ctas_per_sm = large;
              r.block_threads = threads;
            }
          }
    r.even_n_per_s = best;
    r.sample_windows = (uint32_t)smp.size();
    c->tuned_windows[key] = r;
  }
  tuned->mr_divisor = r.mr_divisor;
  tuned->chunk_evens = r.chunk_evens;
  tuned->large_ctas_per_sm = r.large_ctas_per_sm;
  tuned->block_threads = r.block_threads;
  if (res) *res = r;
  return GB_OK;
}

}  // namespace gb
