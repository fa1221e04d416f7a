// gb_internal.h -- argument blocks and launch functions shared by the host
// side of the C-ABI (host/*.cpp) and the sm_100a kernels (kernels/*.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "gb/gb.h"

namespace gb {

// Global counters of a call (device array of unsigned long long).
enum Counter : int {
  kCtrWork = 0,       // next work item (dynamic scheduling)
  kCtrFallbacks = 1,  // n with minimal p > p_small (incl. failures)
  kCtrFailures = 2,   // n without a partition within the bound
  kCtrFirstFail = 3,  // smallest failing n (atomicMin; init ~0)
  kCtrMaxP = 4,       // largest minimal p (atomicMax)
  kCtrQueue = 5,      // entries pushed to the Phase-2 queue
  kCtrQueueOvf = 6,   // set when the queue overflowed
  kCtrWork2 = 7,      // second work counter (multi-stage pipelines)
  kCtrCount = 8
};

// Phase-2 queue entry: an even n whose minimal p is beyond the window halo.
struct QEntry {
  uint64_t n;
  uint64_t idx;   // output index (min_p / verified bits)
  uint64_t unit;  // segment or window
};

// Everything the minimal-p search and the Phase-2 kernel read or account.
struct SearchParams {
  uint32_t halo;     // H: window holds q >= A - H + 1; primes p < H searched there
  uint32_t nsearch;  // primes[1 .. nsearch) searched in the window (all p <= min(H-1, p_lim))
  uint32_t kfb;      // first k whose prime exceeds p_small
  uint64_t p_lim;    // candidate bound max(p_small, phase2_limit)
  uint64_t p_small;
  const uint32_t* primes;  // all primes ascending (2 first)
  uint64_t nprimes;
  unsigned long long* ctr;        // kCtrCount
  unsigned long long* hist;       // nullable: GB_HIST_BINS
  unsigned long long* unit_hist;  // nullable: units x GB_HIST_BINS
  uint32_t* unit_fallbacks;       // nullable
  uint32_t* unit_failures;        // nullable
  unsigned long long* unit_maxp;  // nullable
  unsigned long long* unit_psum;  // nullable: sum of minimal p per unit
  uint32_t* minp;                 // nullable: per n
  uint32_t* vbits;                // nullable: verified bits, prefilled with ones
  QEntry* queue;
  uint32_t queue_cap;
};

// Batched windows (mod-6 layout).  Window w covers the even n = start + 2j,
// j < count.  Its large-prime mask is two class bitsets, L1 then L5, of
// lwords words each at word lbase of the mask buffer: bit t of class c <->
// q = 6(g0 + t) + c, with g0 = floor((start - H - 1) / 6) the first chunk's
// window base.  A bit is cleared when q is a multiple of a sieving prime
// above the chunk sieve's bound (other than the prime itself).
struct WinDesc6 {
  uint64_t start;
  uint64_t count;
  uint64_t out_off;  // output index of its first n
  uint64_t q_top;    // largest n of the window (bounds the sieving primes)
  int64_t g0;        // window base of the mask
  uint64_t lbase;    // first word of L1 (L5 follows at lbase + lwords)
  uint32_t lwords;   // words of each class mask
  uint32_t orig;     // index of the window in the caller's order
};

// What the large-prime pass reads for every (prime, window) pair: the mask
// base g0 as a double (rounded) and its low 32 bits, and the bits of each
// class mask -- or ~0u for a window whose q may include a sieving prime
// itself (g0 < 2^30), which takes the exact path.
struct __align__(16) WinLarge {
  double gd;
  uint32_t gl;
  uint32_t lbits;
};

// With per-n output (SearchParams::minp) the chunks hold at most this many
// even n: a byte per n in shared memory keeps the entry position that
// resolved it until the chunk writes its minimal p out in n order.
constexpr uint32_t kMinpChunk = 1u << 16;

struct RangeArgs {
  SearchParams s;
  uint64_t start;          // first even n of the range
  uint64_t total_count;    // even n in the range
  uint64_t seg_size;       // even n per segment
  uint32_t shard_index, shard_count;
  uint64_t chunks_per_seg; // ceil(seg_size / chunk_evens)
  uint64_t total_items;    // (segments of this shard) * chunks_per_seg
  uint32_t chunk_evens;    // NE
  uint32_t threads;        // block size of range6_kernel: 256, 512 or 1024 (0: 512)
  uint32_t nbw;            // words of the q-window bitset (incl. padding)
  const uint64_t* magic;   // Barrett reciprocals, magic[k] for primes[k]
  uint32_t nsieve;         // primes[kWheelPrimeCount+1 .. nsieve) mark the window
  uint32_t kcoop;          // ... those below kcoop warp-cooperatively
  // class wheel patterns and per-prime class offsets of the mod-6 layout
  const uint32_t* wheel6;  // kWheel6Words
  const uint2* a15;
  uint2* surv;             // survivor lists: 6 per CTA of surv_cap entries each
  uint32_t surv_cap;       // >= words of one class bitset
  // windows mode (win != nullptr): the work items are the chunks of the
  // windows (chunk_off: nwin + 1 prefix sums), each window's outputs are
  // accounted to its caller index, and every chunk's q-window is ANDed with
  // the window's large-prime mask
  const WinDesc6* win;
  const uint64_t* chunk_off;
  uint32_t nwin;
  const uint32_t* lmask;
};

struct SieveArgs {
  uint64_t q_lo;           // odd
  uint64_t nbits;
  uint32_t tile_bits;      // bits per CTA tile (multiple of 32)
  const uint32_t* primes;
  const uint64_t* magic;
  uint32_t nsieve;         // primes[1..nsieve) usable for marking
  uint32_t kcoop;
  const uint32_t* wheel;
  uint32_t* out;           // ceil(nbits/32) words
};

// kernels/tables.cu
cudaError_t launch_wheel_init(uint32_t* wheel, uint32_t* wheel6, cudaStream_t s);
cudaError_t launch_sieve_bits(const SieveArgs& a, cudaStream_t s);
cudaError_t launch_counts(const uint32_t* B, uint64_t m_first, uint64_t count, uint32_t splits,
                          uint64_t wps, unsigned long long* out, cudaStream_t s);
// Appends the primes of `bits` (odd-only from q_lo) after `prefix` entries of
// `primes`; writes the new total into *d_total (device) and magic[] for them.
cudaError_t launch_compact_primes(const uint32_t* bits, uint64_t nbits, uint64_t q_lo,
                                  uint32_t* primes, uint64_t* magic, uint2* a15, uint64_t prefix,
                                  uint64_t cap, unsigned long long* d_total,
                                  uint32_t* scratch_blocks, uint32_t nblocks_cap,
                                  cudaStream_t s);
size_t compact_scratch_blocks(uint64_t nbits);

// kernels/range.cu
size_t range_smem_bytes(const RangeArgs& a);
uint32_t range6_words(uint32_t halo, uint32_t chunk_evens);
int range_max_blocks_per_sm(const RangeArgs& a);
cudaError_t launch_range(const RangeArgs& a, int grid, cudaStream_t s);
cudaError_t launch_fallback(const SearchParams& s, int grid, cudaStream_t st);

// kernels/windows.cu: the large-prime pass of the batched windows.  Primes
// primes[k0 .. k1) (each below 2^32) clear their multiples in the class masks
// of windows [w_lo, w_hi) of `win` / `wl` (sorted by q_top ascending); a
// prime visits only the windows with q_top >= p^2.
struct WinLargeArgs {
  const WinDesc6* win;
  const WinLarge* wl;
  uint32_t w_lo, w_hi;
  const uint32_t* primes;
  const uint64_t* magic;
  const uint2* a15;
  uint32_t k0, k1;
  uint32_t* lmask;
};
cudaError_t launch_win_large(const WinLargeArgs& a, int grid, cudaStream_t s);
// Adds the (prime, window) pairs the pass visits (primes from index k0 up to
// isqrt(q_top) of each window) to *pairs.
cudaError_t launch_win_pairs(const WinDesc6* win, uint32_t nwin, const uint32_t* primes, uint64_t nprimes,
                             uint32_t k0, unsigned long long* pairs, cudaStream_t s);

// kernels/big.cu: partitions of n beyond 2^64.  One batch of candidates
// primes[k0 .. k0 + kcount): the filter appends the indices (from k0) whose
// q = n - p no trial prime divides; phase 0 runs the base-2 strong test on
// them and lists the passers; phase 1 runs the 11 other bases, one thread
// per (passer, base), and marks the passers that fail one.
struct BigArgs {
  const uint32_t* n;        // n in `limbs` little-endian 32-bit limbs (zero-padded)
  uint32_t limbs;           // template width: 4, 8, 16, 32, 64 or 128
  uint32_t nl;              // n's own limbs (<= limbs): R = 2^(32 nl)
  const uint32_t* primes;
  uint64_t p_lim;           // candidates p <= p_lim
  const uint32_t* trial;    // trial primes r
  const uint32_t* nmod;     // n mod r
  uint32_t ntrial;
  uint32_t* surv;           // survivors (candidate index from k0)
  uint32_t* nsurv;
  uint32_t* pass;           // base-2 passers (candidate index from k0)
  uint32_t* fail;           // per passer: nonzero once a base fails
  uint32_t* npass;
  unsigned long long* mr_tests;
};
cudaError_t launch_big_filter(const BigArgs& a, uint32_t k0, uint32_t kcount, cudaStream_t s);
cudaError_t launch_big_mr(const BigArgs& a, uint32_t k0, int phase, int grid, cudaStream_t s);

// kernels/probe.cu: kind 0 = 32-bit ALU ops/s, 1 = shared-memory atomicAnd/s,
// 2 = 64-bit Montgomery products/s
cudaError_t run_probe(int kind, int sm_count, double* ops_per_s, cudaStream_t st);

// kernels/single.cu
struct SingleArgs {
  const uint64_t* n;
  uint64_t count;
  uint64_t* p_out;
  uint64_t* q_out;
  const uint32_t* primes;
  uint64_t nprimes;
  uint64_t p_lim;
  unsigned long long* ctr;  // [0] work, [1] found, [2] max p
};
// Batches below kLaneBatchMin queries take the warp-per-query kernel (latency),
// larger ones the lane-per-query kernel (throughput).
constexpr uint64_t kLaneBatchMin = 8192;
cudaError_t launch_single(const SingleArgs& a, int grid, cudaStream_t s);
// Arguments of segment_reduce_kernel, kept together for a graph's kernel node.
struct SegReduceArgs {
  const uint64_t* p;
  const uint64_t* off;
  uint32_t nreq;
  unsigned long long* agg;
};
// Kernel-node parameters of the launches launch_single / launch_segment_reduce
// would make (argv: caller storage for the argument pointers; a, r and argv
// must stay alive until the node is added or updated).
void single_kernel_node(const SingleArgs& a, int grid, void** argv, cudaKernelNodeParams* kp);
void segment_reduce_node(const SegReduceArgs& r, void** argv, cudaKernelNodeParams* kp);
cudaError_t launch_is_prime(const uint64_t* n, uint64_t count, uint8_t* out, cudaStream_t s);
cudaError_t launch_win_expand(const gb_window* w, const uint64_t* off, uint32_t nw, uint64_t* n,
                              cudaStream_t s);
cudaError_t launch_segment_reduce(const uint64_t* p, const uint64_t* off, uint32_t nreq,
                                  unsigned long long* agg, cudaStream_t s);

}  // namespace gb
