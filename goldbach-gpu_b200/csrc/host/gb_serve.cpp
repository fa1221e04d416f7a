// gb_serve.cpp -- serving loop: continuous batching of single-n and range
// requests over one context's resident tables.
//
// No counterpart in the reference, which answers one query per process
// (`single_check <n>` re-sieves 1e8 candidates on the CPU for every query,
// src/single_check.cu:186-198).  Here:
//   * lane 0 (single, high-priority stream): single n and short ranges,
//     expanded n by n, through the single-n kernel plus a per-request
//     reduction, from a small arena reserved at start;
//   * lanes 1 .. R (range): the longer ranges, from one shared queue,
//     through the windows pipeline, with device memory split on demand from
//     one pool: a lane forms its next batch from the waiting requests in
//     arrival order as far as the pool's free memory allows and returns the
//     memory when the batch completes; the kernels of a range batch fill
//     at most 7/8 of the GPU divided among the busy range lanes.
// Each lane is a host thread with its own CUDA stream and workspace, so the
// lanes' batches overlap on the GPU, and nothing is allocated while they run
// (the pool and the workspaces are reserved at start).  A request that would
// push its lanes' queued work past max_pending / max_pending_n is answered at
// once with GB_EBUSY.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <map>
#include <unordered_map>

#include "gb_ctx.h"
#include "latency_hist.h"

using namespace gb;

namespace {

struct Pending {
  uint64_t ticket;
  gb_request r;
};

struct Lane {
  Workspace ws;
  Arena arena;             // the single lane's fixed buffers
  void* arena_mem = nullptr;
  cudaStream_t stream = nullptr;
  std::thread th;
  std::atomic<uint64_t> batches{0};  // read by gb_serve_stats_get from other threads
  bool busy = false;       // a range lane with a batch on the GPU (under the server mutex)
};

// First-fit allocator over one device allocation (host-side bookkeeping,
// under the server mutex): the range lanes' batches take their memory from
// it and give it back when they complete.
struct Pool {
  char* base = nullptr;
  uint64_t cap = 0, used = 0, peak = 0;
  std::map<uint64_t, uint64_t> free_;  // offset -> bytes, coalesced
  void init(void* p, uint64_t bytes) {
    base = (char*)p;
    cap = bytes & ~255ull;
    free_.clear();
    if (cap) free_[0] = cap;
  }
  uint64_t largest() const {
    uint64_t m = 0;
    for (const auto& f : free_) m = std::max(m, f.second);
    return m;
  }
  bool alloc(uint64_t bytes, uint64_t* off) {
    bytes = (bytes + 255) & ~255ull;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *off = it->first;
      const uint64_t rest = it->second - bytes;
      free_.erase(it);
      if (rest) free_[*off + bytes] = rest;
      used += bytes;
      peak = std::max(peak, used);
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t bytes) {
    bytes = (bytes + 255) & ~255ull;
    used -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

constexpr uint32_t kSingleReqCap = 1u << 16;  // requests per single-lane batch
constexpr int kMaxRangeLanes = 8;
constexpr uint64_t kBatchSlack = 64 << 10;  // per-batch alignment of the pool block

}  // namespace

struct gb_server {
  gb_ctx* c = nullptr;
  gb_serve_opts o{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> q[2];  // 0: single lane, 1: the range lanes
  // requests queued per queue and the stop request, readable without the
  // mutex by a lane that polls (opts.spin_us)
  std::atomic<uint64_t> queued[2];
  std::atomic<bool> stopping{false};
  std::unordered_map<uint64_t, gb_response> done;
  uint64_t next_ticket = 1;
  bool stop = false;
  int nlanes = 0;            // 1 + range lanes
  Lane lane[1 + kMaxRangeLanes];
  Pool pool;                 // range lanes' device memory
  void* pool_mem = nullptr;
  uint64_t queued_n = 0;     // even n waiting in the range queue
  int busy_range = 0;        // range lanes with a batch on the GPU
  // single-lane pinned staging
  uint64_t *h_n = nullptr, *h_p = nullptr, *h_off = nullptr;
  unsigned long long* h_agg = nullptr;
  bool single_graph = false;  // the single lane runs its small batches as a graph
  // stats
  LatencyHist lat;  // completed requests' latencies since start or the last reset
  uint64_t submitted = 0, completed = 0, rejected = 0, busy = 0, t0 = 0;
};

namespace {

// Device bytes of a range request in a range-lane batch (its windows call).
uint64_t range_bytes(const gb_request& r) {
  gb_windows_opts o{};
  return windows_request_bytes(gb_window{r.a, r.count}, o);
}

// Records a batch's responses under one lock with one wake-up of the
// waiting callers (a lock and a notify_all per request would wake every
// gb_wait caller once per request of the batch).
void finish_batch(gb_server* S, const std::vector<Pending>& take, std::vector<gb_response>& resp,
                  uint64_t t_done) {
  std::lock_guard<std::mutex> lk(S->mu);
  for (size_t i = 0; i < take.size(); ++i) {
    const uint64_t arr = take[i].r.arrival_ns;
    resp[i].latency_us = t_done > arr ? (t_done - arr) / 1e3 : 0.0;
    S->done[take[i].ticket] = resp[i];
    S->completed++;
    if (resp[i].status == GB_OK) S->lat.add(resp[i].latency_us);
  }
  S->cv_done.notify_all();
}

// With opts.spin_us, a lane about to wait for work polls its queue for up to
// that long first (a blocked thread takes tens of microseconds to wake).
void poll_queue(gb_server* S, int ln) {
  if (!S->o.spin_us) return;
  const uint64_t end = now_ns() + 1000ull * S->o.spin_us;
  while (!S->queued[ln].load(std::memory_order_acquire) &&
         !S->stopping.load(std::memory_order_relaxed) && now_ns() < end)
    std::this_thread::yield();
}

// The single lane's batch pipeline (two uploads, the counter reset, the
// single-n kernel, the per-request reduction, two downloads) as one CUDA
// graph, built once with the lane's fixed buffers; each batch updates the
// copy sizes and the two kernels' arguments and launches it.  Only batches
// of fewer than kLaneBatchMin n use it (the kernel node is the
// warp-per-query kernel).
struct SingleGraph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  cudaGraphNode_t up_n = nullptr, up_off = nullptr, reset = nullptr, ks = nullptr,
                  kr = nullptr, down_p = nullptr, down_agg = nullptr;
  ~SingleGraph() {
    if (x) cudaGraphExecDestroy(x);
    if (g) cudaGraphDestroy(g);
  }
};

struct SingleBufs {
  uint64_t *d_n, *d_p, *d_q, *d_off;
  unsigned long long* d_agg;
};

bool build_single_graph(gb_server* S, const SingleBufs& B, const SingleArgs& a0,
                        SingleGraph* G) {
  Lane& L = S->lane[0];
  if (cudaGraphCreate(&G->g, 0) != cudaSuccess) return false;
  // a chain: each node depends on the one before
  bool ok = cudaGraphAddMemcpyNode1D(&G->up_n, G->g, nullptr, 0, B.d_n, S->h_n, 8,
                                     cudaMemcpyHostToDevice) == cudaSuccess;
  cudaGraphNode_t prev = G->up_n;
  ok = ok && cudaGraphAddMemcpyNode1D(&G->up_off, G->g, &prev, 1, B.d_off, S->h_off, 16,
                                      cudaMemcpyHostToDevice) == cudaSuccess;
  prev = G->up_off;
  cudaMemsetParams ms{};
  ms.dst = L.ws.ctr;
  ms.value = 0;
  ms.elementSize = 4;
  ms.width = 8;  // 4 counters of 8 bytes
  ms.height = 1;
  ok = ok && cudaGraphAddMemsetNode(&G->reset, G->g, &prev, 1, &ms) == cudaSuccess;
  prev = G->reset;
  void* argv[4];
  cudaKernelNodeParams kp;
  single_kernel_node(a0, 1, argv, &kp);
  ok = ok && cudaGraphAddKernelNode(&G->ks, G->g, &prev, 1, &kp) == cudaSuccess;
  prev = G->ks;
  const SegReduceArgs r0{B.d_p, B.d_off, 1, B.d_agg};
  segment_reduce_node(r0, argv, &kp);
  ok = ok && cudaGraphAddKernelNode(&G->kr, G->g, &prev, 1, &kp) == cudaSuccess;
  prev = G->kr;
  ok = ok && cudaGraphAddMemcpyNode1D(&G->down_p, G->g, &prev, 1, S->h_p, B.d_p, 8,
                                      cudaMemcpyDeviceToHost) == cudaSuccess;
  prev = G->down_p;
  ok = ok && cudaGraphAddMemcpyNode1D(&G->down_agg, G->g, &prev, 1, S->h_agg, B.d_agg, 32,
                                      cudaMemcpyDeviceToHost) == cudaSuccess;
  ok = ok && cudaGraphInstantiate(&G->x, G->g, 0) == cudaSuccess;
  if (!ok) cudaGetLastError();
  return ok;
}

// One batch through the graph: pos n, nreq requests, args a (count = pos).
cudaError_t run_single_graph(gb_server* S, const SingleBufs& B, const SingleArgs& a, int grid,
                             uint32_t nreq, SingleGraph* G) {
  Lane& L = S->lane[0];
  const uint64_t pos = a.count;
  cudaError_t e;
  if ((e = cudaGraphExecMemcpyNodeSetParams1D(G->x, G->up_n, B.d_n, S->h_n, pos * 8,
                                              cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaGraphExecMemcpyNodeSetParams1D(G->x, G->up_off, B.d_off, S->h_off,
                                              (nreq + 1) * 8ull, cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaGraphExecMemcpyNodeSetParams1D(G->x, G->down_p, S->h_p, B.d_p, pos * 8,
                                              cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaGraphExecMemcpyNodeSetParams1D(G->x, G->down_agg, S->h_agg, B.d_agg, nreq * 32ull,
                                              cudaMemcpyDeviceToHost)) != cudaSuccess)
    return e;
  void* argv[4];
  cudaKernelNodeParams kp;
  single_kernel_node(a, grid, argv, &kp);
  if ((e = cudaGraphExecKernelNodeSetParams(G->x, G->ks, &kp)) != cudaSuccess) return e;
  const SegReduceArgs r{B.d_p, B.d_off, nreq, B.d_agg};
  segment_reduce_node(r, argv, &kp);
  if ((e = cudaGraphExecKernelNodeSetParams(G->x, G->kr, &kp)) != cudaSuccess) return e;
  return cudaGraphLaunch(G->x, L.stream);
}

void single_lane(gb_server* S) {
  Lane& L = S->lane[0];
  gb_ctx* c = S->c;
  const uint32_t cap = S->o.max_single_batch;
  // fixed device layout in the lane arena
  uint64_t* d_n = (uint64_t*)L.arena.take((size_t)cap * 8);
  uint64_t* d_p = (uint64_t*)L.arena.take((size_t)cap * 8);
  uint64_t* d_q = (uint64_t*)L.arena.take((size_t)cap * 8);
  uint64_t* d_off = (uint64_t*)L.arena.take((size_t)(kSingleReqCap + 1) * 8);
  unsigned long long* d_agg = (unsigned long long*)L.arena.take((size_t)kSingleReqCap * 32);
  uint64_t np = 0;
  count_le(c, L.ws, GB_PHASE2_LIMIT_DEFAULT, &np);
  const SingleBufs B{d_n, d_p, d_q, d_off, d_agg};
  SingleArgs base{};
  base.n = d_n;
  base.count = 1;
  base.p_out = d_p;
  base.q_out = d_q;
  base.primes = c->d_primes;
  base.nprimes = np;
  base.p_lim = GB_PHASE2_LIMIT_DEFAULT;
  base.ctr = L.ws.ctr;
  SingleGraph G;
  const bool graph = !S->o.no_graph && build_single_graph(S, B, base, &G);
  S->single_graph = graph;
  std::vector<Pending> take;
  std::vector<gb_response> resps;
  for (;;) {
    take.clear();
    uint64_t total = 0;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      lk.unlock();
      poll_queue(S, 0);
      lk.lock();
      S->cv_work.wait(lk, [&] { return S->stop || !S->q[0].empty(); });
      if (S->q[0].empty()) break;  // stop requested and drained
      while (!S->q[0].empty() && take.size() < kSingleReqCap) {
        const Pending& f = S->q[0].front();
        const uint64_t w = f.r.kind == GB_REQ_SINGLE ? 1 : f.r.count;
        if (total + w > cap) break;
        take.push_back(f);
        total += w;
        S->q[0].pop_front();
        S->queued[0].fetch_sub(1, std::memory_order_relaxed);
      }
    }
    uint64_t pos = 0;
    for (size_t i = 0; i < take.size(); ++i) {
      S->h_off[i] = pos;
      const gb_request& r = take[i].r;
      if (r.kind == GB_REQ_SINGLE) S->h_n[pos++] = r.a;
      else
        for (uint64_t j = 0; j < r.count; ++j) S->h_n[pos++] = r.a + 2 * j;
    }
    S->h_off[take.size()] = pos;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) {
      if (e == cudaSuccess && x != cudaSuccess) e = x;
    };
    SingleArgs a = base;
    a.count = pos;
    const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)c->sm_count * 6, (pos + 7) / 8));
    if (graph && pos < kLaneBatchMin) {
      chk(run_single_graph(S, B, a, (int)grid, (uint32_t)take.size(), &G));
    } else {
      chk(cudaMemcpyAsync(d_n, S->h_n, pos * 8, cudaMemcpyHostToDevice, L.stream));
      chk(cudaMemcpyAsync(d_off, S->h_off, (take.size() + 1) * 8, cudaMemcpyHostToDevice, L.stream));
      chk(cudaMemsetAsync(L.ws.ctr, 0, 4 * 8, L.stream));
      chk(launch_single(a, (int)grid, L.stream));
      chk(launch_segment_reduce(d_p, d_off, (uint32_t)take.size(), d_agg, L.stream));
      chk(cudaMemcpyAsync(S->h_p, d_p, pos * 8, cudaMemcpyDeviceToHost, L.stream));
      chk(cudaMemcpyAsync(S->h_agg, d_agg, take.size() * 32, cudaMemcpyDeviceToHost, L.stream));
    }
    chk(cudaStreamSynchronize(L.stream));
    const uint64_t t_done = now_ns();
    const uint32_t batch = (uint32_t)L.batches++;
    resps.assign(take.size(), gb_response{});
    for (size_t i = 0; i < take.size(); ++i) {
      gb_response& resp = resps[i];
      resp.kind = take[i].r.kind;
      resp.lane = 0;
      resp.batch = batch;
      resp.status = e == cudaSuccess ? GB_OK : GB_ECUDA;
      if (e == cudaSuccess) {
        if (resp.kind == GB_REQ_SINGLE) {
          resp.p = S->h_p[S->h_off[i]];
          resp.q = resp.p ? take[i].r.a - resp.p : 0;
        }
        resp.verified = S->h_agg[4 * i];
        resp.failures = S->h_agg[4 * i + 1];
        resp.max_minp = S->h_agg[4 * i + 2];
        resp.minp_sum = S->h_agg[4 * i + 3];
      }
    }
    finish_batch(S, take, resps, t_done);
  }
}

// Range lane ln: batches from the shared range queue, memory from the pool.
void range_lane(gb_server* S, int ln) {
  Lane& L = S->lane[ln];
  gb_ctx* c = S->c;
  std::vector<Pending> take;
  std::vector<gb_window> win;
  std::vector<gb_window_result> res;
  std::vector<gb_response> resps;
  for (;;) {
    take.clear();
    uint64_t off = 0, bytes = 0;
    bool nomem = false;
    int sharing = 1;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      lk.unlock();
      poll_queue(S, 1);
      lk.lock();
      for (;;) {  // until the front request fits the pool (or stop)
        if (!S->q[1].empty()) {
          const uint64_t need = range_bytes(S->q[1].front().r) + kBatchSlack;
          if (need <= S->pool.largest()) break;
          if (S->busy_range == 0) {  // all memory free and still too big
            nomem = true;
            break;
          }
        } else if (S->stop) {
          break;
        }
        S->cv_work.wait(lk);
      }
      if (S->q[1].empty()) break;  // stop requested and drained
      if (nomem) {
        take.push_back(S->q[1].front());
        S->q[1].pop_front();
        S->queued[1].fetch_sub(1, std::memory_order_relaxed);
        S->queued_n -= take[0].r.count;
      } else {
        const uint64_t avail = S->pool.largest();
        bytes = kBatchSlack;
        while (!S->q[1].empty() && take.size() < S->o.max_range_batch) {
          const Pending& f = S->q[1].front();
          const uint64_t b = range_bytes(f.r);
          if (bytes + b > avail) break;
          take.push_back(f);
          bytes += b;
          S->queued_n -= f.r.count;
          S->q[1].pop_front();
          S->queued[1].fetch_sub(1, std::memory_order_relaxed);
        }
        S->pool.alloc(bytes, &off);  // bytes <= the largest free block
        L.busy = true;
        sharing = ++S->busy_range;
      }
    }
    const uint32_t batch = (uint32_t)L.batches++;
    gb_status st = GB_ENOMEM;
    res.assign(take.size(), gb_window_result{});
    if (!nomem) {
      win.resize(take.size());
      for (size_t i = 0; i < take.size(); ++i) win[i] = gb_window{take[i].r.a, take[i].r.count};
      gb_windows_opts o{};
      o.mode = GB_WINDOWS_PERSISTENT;
      o.stream = L.stream;
      o.gpu_share_pct = (uint32_t)std::max(1, 7 * 100 / 8 / sharing);
      Arena arena;
      arena.base = S->pool.base + off;
      arena.cap = bytes;
      gb_windows_summary sum{};
      st = windows_impl(c, L.ws, &arena, win.data(), win.size(), &o, res.data(), nullptr, &sum);
      {
        std::lock_guard<std::mutex> lk(S->mu);
        S->pool.release(off, bytes);
        L.busy = false;
        --S->busy_range;
      }
      S->cv_work.notify_all();  // memory freed: a waiting lane may fit its batch now
    }
    const uint64_t t_done = now_ns();
    resps.assign(take.size(), gb_response{});
    for (size_t i = 0; i < take.size(); ++i) {
      gb_response& resp = resps[i];
      resp.kind = GB_REQ_RANGE;
      resp.lane = (uint32_t)ln;
      resp.batch = batch;
      resp.status = st;
      if (st == GB_OK) {
        resp.verified = res[i].verified;
        resp.failures = res[i].failures;
        resp.max_minp = res[i].max_minp;
        resp.minp_sum = res[i].minp_sum;
      }
    }
    finish_batch(S, take, resps, t_done);
  }
}

void free_server(gb_server* S) {
  gb_ctx* c = S->c;
  for (Lane& L : S->lane) {
    if (L.stream) {
      cudaStreamSynchronize(L.stream);
      cudaStreamDestroy(L.stream);
    }
    ws_free(c, L.ws);
    dev_free(c, L.arena_mem);
  }
  dev_free(c, S->pool_mem);
  if (S->h_n) cudaFreeHost(S->h_n);
  if (S->h_p) cudaFreeHost(S->h_p);
  if (S->h_off) cudaFreeHost(S->h_off);
  if (S->h_agg) cudaFreeHost(S->h_agg);
  delete S;
}

}  // namespace

extern "C" {

uint64_t gb_now_ns(void) { return now_ns(); }

gb_status gb_serve_start(gb_ctx* c, const gb_serve_opts* opts) {
  if (!c) return GB_EINVAL;
  std::lock_guard<std::mutex> lk(c->mu);
  if (c->server) return GB_EINVAL;
  cudaSetDevice(c->device);
  gb_server* S = new gb_server();
  S->queued[0] = 0;
  S->queued[1] = 0;
  S->c = c;
  if (opts) S->o = *opts;
  if (!S->o.max_n) S->o.max_n = ~0ull;
  if (!S->o.max_single_batch) S->o.max_single_batch = 1u << 18;
  if (!S->o.max_range_batch) S->o.max_range_batch = 4096;
  if (!S->o.small_range) S->o.small_range = 1u << 15;
  if (S->o.small_range > S->o.max_single_batch) S->o.small_range = S->o.max_single_batch;
  if (!S->o.range_lanes) S->o.range_lanes = 2;
  if (!S->o.max_pending) S->o.max_pending = 1u << 16;
  if (!S->o.max_pending_n) S->o.max_pending_n = 1ull << 31;
  auto bail = [&](gb_status x) {
    c->err = c->ws.err;
    free_server(S);
    return x;
  };
  if (S->o.range_lanes > kMaxRangeLanes) {
    c->ws.err = "range_lanes must be <= 8";
    return bail(GB_EINVAL);
  }
  S->nlanes = 1 + (int)S->o.range_lanes;
  // resident tables for every n served: sieving primes to sqrt(max_n) and
  // the candidate primes; frozen while the lanes run
  gb_status st = ensure_primes(c, c->ws, std::max<uint64_t>(isqrt_u64(S->o.max_n) + 2,
                                                            GB_PHASE2_LIMIT_DEFAULT));
  if (st != GB_OK) return bail(st);
  const uint64_t cap = S->o.max_single_batch;
  const uint64_t single_bytes = cap * 24 + (kSingleReqCap + 1) * 8 + kSingleReqCap * 32 + 4096;
  int lo_prio = 0, hi_prio = 0;
  cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
  // survivor lists of the chunk kernel at its default shape on the full GPU
  const size_t surv_bytes = (size_t)c->sm_count * 2 * 6 * range6_words(32768, 1u << 20) * sizeof(uint2);
  for (int i = 0; i < S->nlanes; ++i) {
    Lane& L = S->lane[i];
    if ((st = ws_init(c, L.ws, 1u << 16)) != GB_OK) return bail(st);
    if (i == 0) {
      if ((st = dev_alloc(c, &L.arena_mem, single_bytes, &c->ws.err)) != GB_OK) return bail(st);
      L.arena.base = (char*)L.arena_mem;
      L.arena.cap = single_bytes;
    } else {
      void* p = nullptr;
      if ((st = ws_scratch(c, L.ws, surv_bytes, &p)) != GB_OK) return bail(st);
    }
    // the single lane's short batches go ahead of the range lanes' blocks
    if (cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking, i == 0 ? hi_prio : lo_prio) !=
        cudaSuccess)
      return bail(GB_ECUDA);
  }
  // the range lanes' pool: as asked, else half of what the device has free
  // now, within the context's budget
  uint64_t pool = S->o.pool_bytes ? S->o.pool_bytes : S->o.range_arena_bytes;
  if (!pool) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return bail(GB_ECUDA);
    pool = fr / 2;
    const uint64_t left = c->budget > c->held ? c->budget - c->held : 0;
    pool = std::min<uint64_t>(pool, left > (64ull << 20) ? left - (64ull << 20) : 0);
  }
  if (pool < (256ull << 10)) {
    c->ws.err = "no device memory left for the serving pool";
    return bail(GB_ENOMEM);
  }
  if ((st = dev_alloc(c, &S->pool_mem, pool, &c->ws.err)) != GB_OK) return bail(st);
  S->pool.init(S->pool_mem, pool);
  if (cudaHostAlloc((void**)&S->h_n, cap * 8, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void**)&S->h_p, cap * 8, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void**)&S->h_off, (kSingleReqCap + 1) * 8, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void**)&S->h_agg, kSingleReqCap * 32, cudaHostAllocDefault) != cudaSuccess)
    return bail(GB_ENOMEM);
  S->t0 = now_ns();
  c->server = S;
  S->lane[0].th = std::thread([S] {
    cudaSetDevice(S->c->device);
    single_lane(S);
  });
  for (int i = 1; i < S->nlanes; ++i)
    S->lane[i].th = std::thread([S, i] {
      cudaSetDevice(S->c->device);
      range_lane(S, i);
    });
  return GB_OK;
}

gb_status gb_submit(gb_ctx* c, const gb_request* reqs, size_t count, uint64_t* tickets) {
  if (!c || (count && (!reqs || !tickets))) return GB_EINVAL;
  gb_server* S = c->server;
  if (!S) return GB_EINVAL;
  const uint64_t t = now_ns();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) return GB_ECANCELED;
  for (size_t i = 0; i < count; ++i) {
    Pending p{S->next_ticket++, reqs[i]};
    if (!p.r.arrival_ns) p.r.arrival_ns = t;
    tickets[i] = p.ticket;
    S->submitted++;
    const gb_request& r = p.r;
    bool ok = r.a >= 4 && !(r.a & 1) && r.a <= S->o.max_n;
    if (r.kind == GB_REQ_RANGE) {
      const uint64_t last = r.a + 2 * (r.count - 1);
      ok = ok && r.count >= 1 && r.count <= GB_WINDOW_MAX_COUNT && last >= r.a && last <= S->o.max_n;
    } else if (r.kind != GB_REQ_SINGLE) {
      ok = false;
    }
    const int ln = (r.kind == GB_REQ_SINGLE || r.count <= S->o.small_range) ? 0 : 1;
    gb_status bad = ok ? GB_OK : GB_EINVAL;
    if (bad == GB_OK && ln == 1 && range_bytes(r) + kBatchSlack > S->pool.cap)
      bad = GB_ENOMEM;  // would never fit the range lanes' memory
    // backpressure: the queue of the request's lanes is at its bound (an
    // empty queue always takes the request)
    if (bad == GB_OK && ln == 0 && S->q[0].size() >= S->o.max_pending) bad = GB_EBUSY;
    if (bad == GB_OK && ln == 1 && !S->q[1].empty() && S->queued_n + r.count > S->o.max_pending_n)
      bad = GB_EBUSY;
    if (bad != GB_OK) {
      gb_response resp{};
      resp.status = bad;
      resp.kind = r.kind;
      S->done[p.ticket] = resp;
      S->completed++;
      S->rejected++;
      if (bad == GB_EBUSY) S->busy++;
      continue;
    }
    if (ln == 1) S->queued_n += r.count;
    S->q[ln].push_back(p);
    S->queued[ln].fetch_add(1, std::memory_order_release);
  }
  S->cv_work.notify_all();
  return GB_OK;
}

gb_status gb_poll(gb_ctx* c, uint64_t ticket, gb_response* out) {
  if (!c || !c->server || !out) return GB_EINVAL;
  gb_server* S = c->server;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->done.find(ticket);
  if (it == S->done.end()) return ticket && ticket < S->next_ticket ? GB_EAGAIN : GB_EINVAL;
  *out = it->second;
  S->done.erase(it);
  return GB_OK;
}

gb_status gb_wait(gb_ctx* c, uint64_t ticket, gb_response* out, uint64_t timeout_ms) {
  if (!c || !c->server || !out) return GB_EINVAL;
  gb_server* S = c->server;
  std::unique_lock<std::mutex> lk(S->mu);
  if (!ticket || ticket >= S->next_ticket) return GB_EINVAL;  // never issued
  // capped at 2^40 ms (about 35 years), so that UINT64_MAX ("no bound") fits
  // the clock arithmetic of the wait instead of wrapping to a negative time
  const uint64_t ms = std::min<uint64_t>(timeout_ms, 1ull << 40);
  const bool got = S->cv_done.wait_for(lk, std::chrono::milliseconds((int64_t)ms), [&] {
    return S->done.count(ticket) != 0;
  });
  if (!got) return GB_ETIMEOUT;
  *out = S->done[ticket];
  S->done.erase(ticket);
  return GB_OK;
}

gb_status gb_serve_stats_get(gb_ctx* c, gb_serve_stats* out, int reset) {
  if (!c || !c->server || !out) return GB_EINVAL;
  gb_server* S = c->server;
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(out, 0, sizeof *out);
  out->submitted = S->submitted;
  out->completed = S->completed;
  out->pending = S->q[0].size() + S->q[1].size();
  out->rejected = S->rejected;
  out->batches_single = S->lane[0].batches;
  for (int i = 1; i < S->nlanes; ++i) out->batches_range += S->lane[i].batches;
  out->busy = S->busy;
  out->pool_bytes = S->pool.cap;
  out->pool_peak_bytes = S->pool.peak;
  out->elapsed_s = (now_ns() - S->t0) / 1e9;
  if (S->lat.count()) {
    out->p50_us = S->lat.quantile(0.50);
    out->p99_us = S->lat.quantile(0.99);
    out->max_us = S->lat.max();
    out->mean_us = S->lat.mean();
    out->completed_per_s = S->lat.count() / std::max(out->elapsed_s, 1e-9);
  }
  if (reset) {
    S->lat.clear();
    S->t0 = now_ns();
  }
  return GB_OK;
}

gb_status gb_serve_stop(gb_ctx* c) {
  if (!c || !c->server) return GB_EINVAL;
  gb_server* S = c->server;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->stopping.store(true, std::memory_order_relaxed);
  }
  S->cv_work.notify_all();
  for (Lane& L : S->lane)
    if (L.th.joinable()) L.th.join();
  std::lock_guard<std::mutex> lk(c->mu);
  c->server = nullptr;
  free_server(S);
  return GB_OK;
}

void gb_serve_shutdown(gb_ctx* c) {
  if (c && c->server) gb_serve_stop(c);
}

}  // extern "C"
