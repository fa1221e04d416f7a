/*
 * gb.h -- C-ABI of the B200 Goldbach verifier (libgoldbach_b200.so).
 *
 * The reference project (isaac-6/goldbach-gpu) exposes no library: its
 * boundary is the `goldbach` and `single_check` processes, and the seam below
 * them is run_gpu_worker() in src/goldbach.cu:378-500.  This header is the
 * library boundary those CLIs are rebuilt on; each entry point names the
 * reference code it replaces.
 *
 * Conventions
 *   - Plain C types only.  Every entry point returns a gb_status (0 = ok,
 *     negative = error); no C++ exception crosses this boundary.  This
 *     replaces the reference's CUDA_CHECK throw + g_system_error flag
 *     (src/goldbach.cu:105-114, 496-499).
 *   - Buffers are caller-owned.  Output pointers are HOST memory unless the
 *     call's options say `on_device`, in which case they are device
 *     pointers on the context's GPU.  The library owns all other device
 *     memory (resident prime tables and work buffers).
 *   - A context serves one thread at a time, except gb_submit / gb_poll /
 *     gb_serve_stats, which are thread-safe.
 *   - "minimal p" of an even n is the smallest prime p <= n/2 with n-p
 *     prime: the first hit of the ascending scan in
 *     src/cpu_goldbach.cpp:14-24.  0 means no such p within the bound.
 */
#ifndef GB_GB_H
#define GB_GB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int gb_status;
#define GB_OK 0
#define GB_EINVAL (-1)    /* bad argument */
#define GB_ENOMEM (-2)    /* device memory budget exceeded / allocation failed */
#define GB_ECUDA (-3)     /* CUDA runtime error */
#define GB_ETIMEOUT (-4)  /* a bounded device or host wait gave up */
#define GB_ECANCELED (-5) /* request cancelled / server stopped */
#define GB_ENODEV (-6)    /* no CUDA device */
#define GB_EOVERFLOW (-7) /* an internal queue would overflow */
#define GB_EAGAIN (-8)    /* serving: result not ready yet */
#define GB_EBUSY (-9)     /* serving: refused, the queued work is at its bound */

/* Minimal-p histogram: bin k counts n whose minimal p is the k-th prime
 * (2 -> bin 0, 3 -> 1, 5 -> 2, ...); minimal p of index >= GB_HIST_BINS-1
 * lands in the last bin.  Failures are counted separately. */
#define GB_HIST_BINS 4096

/* Phase-2 bound of the reference (PHASE2_SIEVE_LIMIT, src/goldbach.cu:316). */
#define GB_PHASE2_LIMIT_DEFAULT 100000000ULL
/* P_SMALL cap of the reference (MAX_P_SMALL, src/goldbach.cu:597). */
#define GB_P_SMALL_MAX 4000000000ULL

typedef struct gb_ctx gb_ctx;

typedef struct gb_config {
  /* Device memory the context may hold, in bytes (0 = what the device
   * reports free at creation).  Allocations beyond it fail with GB_ENOMEM,
   * like the VRAM guard of src/goldbach.cu:505-541. */
  uint64_t device_mem_budget;
  /* Prime tables are built lazily and grow on demand; these pre-size them. */
  uint64_t max_n;        /* sieving primes up to isqrt(max_n)+1 (0: grow) */
  uint64_t cand_limit;   /* candidate primes up to this bound (0: 1e8)    */
} gb_config;

/* Number of visible CUDA devices (0 if none or no driver). */
int gb_device_count(void);
/* Name and total memory of a device, as reported by
 * validate_hardware_and_limits (src/goldbach.cu:527-540). */
gb_status gb_device_info(int device, char* name, size_t name_len, uint64_t* total_mem);
/* Device bytes a context with this configuration holds once its tables are
 * built (the requirement the VRAM guard of src/goldbach.cu:505-541 checks). */
uint64_t gb_estimate_device_bytes(const gb_config* cfg);

/* Creates a context on `device` (src/goldbach.cu:388-417: stream, resident
 * tables).  cfg may be NULL. */
gb_status gb_create(int device, const gb_config* cfg, gb_ctx** out);
void gb_destroy(gb_ctx* ctx);
const char* gb_strerror(gb_status st);
/* Human-readable detail of the last error on this context ("" if none). */
const char* gb_last_error(const gb_ctx* ctx);
/* Device bytes the context holds now, and its budget. */
gb_status gb_mem_info(const gb_ctx* ctx, uint64_t* held, uint64_t* budget);

/* -------------------------------------------------------------------------
 * Range verification: every even n in [start, limit].
 * Replaces run_gpu_worker's segment loop (src/goldbach.cu:420-485): the
 * tiled sieve (:198-259), Phase 1 (:288-311), the unverified count
 * (:184-195) and the host Phase 2 (:362-373), all on the device.
 * ---------------------------------------------------------------------- */
typedef struct gb_range_opts {
  uint64_t seg_size;      /* even n per reported segment (SEG_SIZE; 0: 1e7) */
  uint64_t p_small;       /* Phase-1 bound P_SMALL (0: 1e6); the fallback
                             count is #{n : minimal p > p_small}           */
  uint64_t phase2_limit;  /* Phase-2 bound (0: 1e8); n with no p <=
                             max(p_small, phase2_limit) is a failure       */
  uint32_t chunk_evens;   /* even n per CTA window (0: auto; power of 2,
                             2^13..2^20; at most 2^16 when min_p is asked
                             for: each n's entry is kept in shared memory
                             until the chunk writes the minimal p out)     */
  uint32_t halo;          /* q-window halo in numbers (0: auto; multiple of
                             64, 128..2^17); primes p < halo are searched
                             in shared memory, larger ones on the Phase-2
                             path                                          */
  uint32_t shard_index;   /* process only segments s with                   */
  uint32_t shard_count;   /*   s % shard_count == shard_index (0/1: all)    */
  int on_device;          /* outputs below are device pointers              */
  void* stream;           /* cudaStream_t to launch on (NULL: ctx stream)   */
  uint32_t block_threads; /* threads per CTA of the sieve+search kernel:
                             256, 512 or 1024 (0: 512); the CTAs per SM
                             follow from the chunk's shared memory          */
} gb_range_opts;

typedef struct gb_range_result {
  uint64_t checked;          /* even n examined                            */
  uint64_t verified;         /* n with a minimal p within the bound        */
  uint64_t phase2_fallbacks; /* "Phase 2 fallbacks" of src/goldbach.cu:799 */
  uint64_t failures;         /* n with no partition within the bound       */
  uint64_t first_failure_n;  /* smallest failing n (0: none)               */
  uint64_t max_minp;         /* largest minimal p seen                     */
  uint64_t num_segments;     /* segments of seg_size even n in the range   */
  uint64_t queued;           /* n resolved on the Phase-2 device path      */
  uint64_t kernel_launches;  /* device kernels this call launched          */
  double device_ms;          /* device time of the call (CUDA events)      */
  double kernel_ms;          /* device time of the sieve+search kernel     */
} gb_range_result;

typedef struct gb_range_out {
  uint32_t* verified_bits;  /* ceil(count/32) words, bit j <-> start+2j      */
  uint32_t* min_p;          /* count entries: minimal p per n               */
  uint64_t* minp_hist;      /* GB_HIST_BINS                                 */
  uint32_t* seg_fallbacks;  /* num_segments: fallbacks per segment          */
  uint32_t* seg_failures;   /* num_segments: failures per segment           */
  uint64_t* seg_hist;       /* num_segments x GB_HIST_BINS                  */
} gb_range_out;

/* Number of segments [start, limit] splits into for a seg_size. */
uint64_t gb_num_segments(uint64_t start, uint64_t limit, uint64_t seg_size);

/* out may be NULL (summary only).  start/limit follow the reference's
 * normalisation (src/goldbach.cu:593-609): limit odd -> limit-1, start < 4
 * -> 4, start odd -> start+1; start must then be <= limit. */
gb_status gb_verify_range(gb_ctx* ctx, uint64_t start, uint64_t limit,
                          const gb_range_opts* opts, gb_range_result* res,
                          const gb_range_out* out);

/* -------------------------------------------------------------------------
 * Autotuner for gb_verify_range (no counterpart in the reference, whose
 * SEG_SIZE / P_SMALL the user picks by hand, src/goldbach.cu:560-609): times
 * gb_verify_range on the top min(2^28, count) even n of [start, limit] for
 * each candidate block shape (512 threads x 2 CTAs per SM, 256 x 4,
 * 1024 x 1), chunk_evens (2^18, 2^19, 2^20) and halo (2^14, 2^15, 2^16) the
 * shape's shared memory admits, after one warm-up call, and writes the
 * fastest into *tuned (a copy of *base with chunk_evens, halo and
 * block_threads set).  The choice is cached in the context
 * per range class (bit length of limit, p_small, phase2_limit): a later call
 * for the same class times nothing.  Ranges below 2^22 even n keep the
 * defaults.  Results of gb_verify_range do not depend on these knobs.
 * ---------------------------------------------------------------------- */
typedef struct gb_autotune_result {
  uint32_t chunk_evens;   /* chosen */
  uint32_t halo;          /* chosen */
  uint32_t block_threads; /* chosen */
  double even_n_per_s;    /* the chosen configuration's rate on the sample */
  uint32_t candidates;    /* configurations timed by this call (0: cached) */
  uint64_t sample_evens;  /* even n per timed call */
  int cached;             /* 1: the context had this range class */
} gb_autotune_result;
gb_status gb_autotune_range(gb_ctx* ctx, uint64_t start, uint64_t limit, const gb_range_opts* base,
                            gb_range_opts* tuned, gb_autotune_result* res);

/* -------------------------------------------------------------------------
 * Goldbach partition counts: counts[j] = c(n) for n = start + 2j, j < count,
 * where c(n) = #{p <= n/2 : p and n - p prime} (so c(4) = 1, c(6) = 1,
 * c(10) = 2).  Replaces goldbach_count (src/cpu_goldbach.cpp:29-36), the
 * reference's CPU-only scan behind its c(n) roadmap item (RESULTS.md:169).
 * start < 4 -> 4, odd start -> start + 1; n up to GB_COUNTS_MAX_N.  The
 * call holds the odd-prime bitset of [1, n_max] on the device (n_max / 16
 * bytes).  counts is host memory, or device memory with opts->on_device.
 * ---------------------------------------------------------------------- */
#define GB_COUNTS_MAX_N (1ull << 40)
typedef struct {
  int on_device;  /* counts is a device pointer */
  void* stream;   /* cudaStream_t; NULL: the context's stream */
} gb_count_opts;
gb_status gb_goldbach_counts(gb_ctx* ctx, uint64_t start, uint64_t count, uint64_t* counts,
                             const gb_count_opts* opts);

/* -------------------------------------------------------------------------
 * Odd-only prime bitset of a window (the GPU sieve on its own): bit i of
 * `words` <-> odd q_lo + 2*i is prime.  Replaces build_prime_bitset
 * (src/prime_bitset.cpp:21-97) and the tiled sieve's output layout
 * (src/goldbach.cu:198-259) with a race-free sm_100a sieve.  q_lo odd.
 * ---------------------------------------------------------------------- */
gb_status gb_sieve_bitset(gb_ctx* ctx, uint64_t q_lo, uint64_t nbits,
                          uint32_t* words, int on_device, void* stream);

/* Primes <= limit in ascending order (2 first), from the device prime
 * table.  *count receives the number of primes; `primes` (cap entries,
 * nullable) receives them.  Replaces generate_cpu_primes
 * (src/goldbach.cu:318-331). */
gb_status gb_primes_upto(gb_ctx* ctx, uint64_t limit, uint32_t* primes,
                         uint64_t cap, uint64_t* count);

/* Deterministic 64-bit primality (Montgomery Miller-Rabin, bases 2, 325,
 * 9375, 28178, 450775, 9780504, 1795265022) for a batch.  Replaces
 * gpu_is_prime_miller_rabin (src/goldbach.cu:144-158) and
 * is_prime_miller_rabin (src/single_check.cu:67-88). */
gb_status gb_is_prime_batch(gb_ctx* ctx, const uint64_t* n, size_t count,
                            uint8_t* out, int on_device, void* stream);

/* -------------------------------------------------------------------------
 * Batched single-n checks: for each even n >= 4 the minimal p and q = n-p.
 * Replaces check_single / goldbach_single_kernel (src/single_check.cu:
 * 95-282), which returns the first-finishing partition, with the minimal
 * one.  p = q = 0 for an n without a partition with p <= p_limit.
 * ---------------------------------------------------------------------- */
typedef struct gb_single_opts {
  uint64_t p_limit;  /* candidate bound (0: 1e8)                          */
  int on_device;     /* n / p_out / q_out are device pointers             */
  void* stream;
} gb_single_opts;

typedef struct gb_single_result {
  uint64_t found;           /* queries with a partition                   */
  uint64_t max_p;           /* largest minimal p                          */
  uint64_t kernel_launches;
  double device_ms;
} gb_single_result;

gb_status gb_check_single_batch(gb_ctx* ctx, const uint64_t* n, size_t count,
                                uint64_t* p_out, uint64_t* q_out,
                                const gb_single_opts* opts,
                                gb_single_result* res);

/* -------------------------------------------------------------------------
 * Batched single-n checks that allocate no device memory.
 *
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code running while a stream is captured into a CUDA graph, code living in
 * another framework's memory pool, or a real-time loop that must not touch
 * the allocator.  No context is needed and nothing is allocated: n, p_out
 * and q_out are device buffers on the current device (count entries each);
 * the kernel's counters and candidate primes live in a fixed file-scope
 * device array of about 26 KB that every GPU which loads this library holds
 * until the process exits.
 *   - p_limit bounds the candidate p (0: GB_NOALLOC_P_LIMIT, the largest
 *     prime below 2^16, which is the reach of the fixed table); a larger
 *     p_limit returns GB_EINVAL.  Results equal gb_check_single_batch with
 *     the same p_limit.
 *   - The first call in each CUDA context builds the table and
 *     synchronises `stream`: the first call on a device, and again the
 *     first call after cudaDeviceReset or from another context made
 *     current on the same device.  Make that call before any stream
 *     capture.
 *   - Later calls are asynchronous on `stream` (cudaStream_t, NULL: legacy
 *     default stream); the counters are cleared on every call.
 *   - All calls share the one array: calls that overlap on the GPU (two
 *     streams, two threads) race.  Serialise them.
 * ---------------------------------------------------------------------- */
#define GB_NOALLOC_P_LIMIT 65521ULL
gb_status gb_check_single_batch_noalloc(const uint64_t* n, size_t count, uint64_t* p_out,
                                        uint64_t* q_out, uint64_t p_limit, void* stream);

/* -------------------------------------------------------------------------
 * Even n beyond 2^64: the minimal prime p <= p_limit with n - p a probable
 * prime.  Replaces big_check (src/big_check.cpp:35-144), which keeps the
 * first q accepted by GMP's 25-round mpz_probab_prime_p that its OpenMP
 * threads find in batches of 1000 primes -- a valid partition, not
 * guaranteed minimal.  n is given as nlimbs little-endian 32-bit limbs (n
 * even, 4 <= n < 2^(32 GB_BIG_MAX_LIMBS)); q_limbs (nlimbs entries,
 * nullable) receives q = n - p.  q is accepted when no prime below 4096
 * divides it and it passes strong probable-prime tests to the 12 bases 2,
 * 3, ..., 37 (the reference's base set, src/goldbach.cu:333-360): a proof of
 * primality for q < 3.3e24, a probable-prime verdict beyond.  n below 2^64
 * take gb_check_single_batch (deterministic).  *p_out = 0: no p <= p_limit
 * (0: 1e8) gives a probable prime.
 * ---------------------------------------------------------------------- */
#define GB_BIG_MAX_LIMBS 128 /* n below 2^4096 (1233 decimal digits) */
typedef struct gb_big_result {
  uint64_t candidates;  /* candidate p examined (in whole batches)       */
  uint64_t mr_tests;    /* strong-test runs started (trial division passed) */
  double device_ms;
} gb_big_result;
gb_status gb_check_big(gb_ctx* ctx, const uint32_t* n_limbs, uint32_t nlimbs, uint64_t p_limit,
                       uint64_t* p_out, uint32_t* q_limbs, gb_big_result* res);

/* -------------------------------------------------------------------------
 * Batched windows: many independent ranges of consecutive even n.
 * ---------------------------------------------------------------------- */
typedef struct gb_window {
  uint64_t start; /* first even n (>= 4)                        */
  uint64_t count; /* number of even n (1 .. GB_WINDOW_MAX_COUNT) */
} gb_window;
#define GB_WINDOW_MAX_COUNT (1ull << 33) /* wider ranges: gb_verify_range */

#define GB_WINDOWS_PERSISTENT 0 /* one persistent launch, device work queue */
#define GB_WINDOWS_PLAIN 1      /* one pipeline of launches per window      */

typedef struct gb_windows_opts {
  int mode;               /* GB_WINDOWS_PERSISTENT or GB_WINDOWS_PLAIN      */
  uint32_t chunk_evens;   /* 0: autotuned                                   */
  uint32_t halo;          /* 0: auto                                        */
  uint64_t phase2_limit;  /* 0: 1e8                                         */
  int on_device;          /* windows / min_p / res are device pointers      */
  void* stream;
  uint64_t mr_below;      /* windows of fewer even n skip the sieve: their q
                             are tested by Miller-Rabin (the single-n
                             kernel).  0: automatic, where sieving would
                             cost more (about pi(sqrt(top)) / mr_divisor
                             n); 1: never                                  */
  uint32_t mr_divisor;    /* the automatic split's divisor (0: 2600)        */
  uint32_t large_ctas_per_sm; /* grid of the large-prime pass (0: 64)       */
  uint32_t block_threads; /* as gb_range_opts.block_threads (0: 512)        */
  uint32_t gpu_share_pct; /* the persistent kernels of the call (chunk
                             sieve + search, Miller-Rabin path) fill at most
                             this percentage of the GPU's resident CTA
                             slots (0: 100), leaving the rest to concurrent
                             work                                          */
} gb_windows_opts;

typedef struct gb_window_result {
  uint64_t verified;
  uint64_t failures;
  uint64_t max_minp;
  uint64_t minp_sum; /* sum of minimal p over the window (checksum)        */
} gb_window_result;

typedef struct gb_windows_summary {
  uint64_t total_n;
  uint64_t failures;
  uint64_t kernel_launches;
  double device_ms;
  uint64_t sieved_windows; /* windows on the sieve path (the rest: Miller-Rabin)  */
  uint64_t large_pairs;    /* (prime, window) pairs of the large-prime pass       */
  double large_ms;         /* device time of the large-prime pass (persistent)    */
  double search_ms;        /* device time of the chunk sieve + search (persistent) */
} gb_windows_summary;

/* min_p_concat (nullable) receives the minimal p of every n, window after
 * window (sum of counts entries). */
gb_status gb_verify_windows(gb_ctx* ctx, const gb_window* w, size_t count,
                            const gb_windows_opts* opts, gb_window_result* res,
                            uint32_t* min_p_concat, gb_windows_summary* sum);

/* Autotuner for gb_verify_windows (no counterpart in the reference): times
 * the persistent pipeline on a sample of the batch (every k-th window, at
 * most 512 windows) for each mr_divisor (1300, 2600, 5200), chunk_evens
 * (2^19, 2^20), large-prime grid (16, 64 CTAs per SM) and block shape
 * (512, 256 threads), after one warm-up call, and writes the fastest into
 * *tuned (a copy of *base with those four set).  The choice is cached in the
 * context per batch class (bit length of the largest top, bit length of the
 * window count); a later call for the same class times nothing.  Results of
 * gb_verify_windows do not depend on these knobs. */
typedef struct gb_windows_tune {
  uint32_t mr_divisor, chunk_evens, large_ctas_per_sm, block_threads; /* chosen */
  double even_n_per_s;    /* the choice's rate on the sample */
  uint32_t candidates;    /* configurations timed by this call (0: cached) */
  uint32_t sample_windows;
  int cached;
} gb_windows_tune;
gb_status gb_autotune_windows(gb_ctx* ctx, const gb_window* w, size_t count,
                              const gb_windows_opts* base, gb_windows_opts* tuned,
                              gb_windows_tune* res);

/* -------------------------------------------------------------------------
 * Serving: a request loop with continuous batching.
 *
 * The reference serves one query per process (`single_check <n>`, or a
 * `goldbach --start=A L` run).  Here requests are submitted from any thread
 * and complete independently.  Lanes run concurrently on their own streams
 * over the context's resident tables:
 *   - the single lane (lane 0, a high-priority stream) runs single n and
 *     short ranges (n by n) through the single-n kernel;
 *   - the range lanes (lanes 1 .. range_lanes) take the other ranges from
 *     one queue through the windows pipeline; a lane's kernels fill at most
 *     its share of the GPU (7/8 of it split among the busy range lanes), so
 *     the single lane always finds free SMs and a wide range never holds up
 *     the narrow ones behind it.
 * Device memory for the range batches is one pool reserved at start (from
 * the device's free memory); a range lane takes, when its previous batch
 * completes, every waiting request in arrival order as far as its batch
 * size and the pool's free memory allow, and gives the memory back when the
 * batch completes -- a request that does not fit yet waits in the queue.
 * Requests that arrive meanwhile join the next batches.  Backpressure: a
 * request that would bring the queued (not yet started) work of its lanes
 * above max_pending / max_pending_n completes at once with GB_EBUSY.  Each
 * result depends only on its own request.
 * ---------------------------------------------------------------------- */
#define GB_REQ_SINGLE 0 /* n = a (even, >= 4)                       */
#define GB_REQ_RANGE 1  /* every even n in [a, a + 2*(count-1)]      */

typedef struct gb_request {
  int kind;
  uint64_t a;
  uint64_t count;      /* GB_REQ_RANGE: even n in the range (>= 1)       */
  uint64_t arrival_ns; /* on gb_now_ns()'s clock; 0: at submission        */
} gb_request;

typedef struct gb_response {
  gb_status status;
  int kind;
  uint64_t p, q;      /* single: minimal partition (p = 0: none <= bound) */
  uint64_t verified;  /* range: n with a partition (single: 0 or 1)       */
  uint64_t failures;
  uint64_t max_minp;
  uint64_t minp_sum;  /* sum of minimal p over the request                */
  double latency_us;  /* arrival to completion                            */
  uint32_t lane;      /* 0: single lane, 1 .. range_lanes: a range lane   */
  uint32_t batch;     /* the lane batch that served it                    */
} gb_response;

typedef struct gb_serve_opts {
  uint64_t max_n;              /* largest n served (0: 2^64 - 1)               */
  uint32_t max_single_batch;   /* n per single-lane batch (0: 2^18)            */
  uint32_t max_range_batch;    /* requests per range-lane batch (0: 4096)      */
  uint64_t range_arena_bytes;  /* the range lanes' pool when pool_bytes is 0
                                  (0: see pool_bytes)                        */
  uint64_t small_range;        /* ranges of <= this many n run n by n (0: 2^15) */
  uint32_t no_graph;           /* 1: single-lane batches of < 8192 n as plain
                                  stream launches instead of one CUDA graph   */
  uint32_t spin_us;            /* a lane out of work polls its queue this long
                                  before it blocks (0: blocks at once; polling
                                  keeps a host core busy per lane)           */
  uint32_t range_lanes;        /* range lanes (0: 2)                           */
  uint64_t pool_bytes;         /* device memory pool of the range lanes (0:
                                  range_arena_bytes if set, else half of the
                                  free device memory at start, within the
                                  context's budget)                          */
  uint64_t max_pending;        /* queued single-lane requests (0: 2^16)        */
  uint64_t max_pending_n;      /* queued even n of the range lanes (0: 2^31)   */
} gb_serve_opts;

typedef struct gb_serve_stats {
  uint64_t submitted, completed, pending, rejected; /* rejected: invalid + busy */
  uint64_t batches_single, batches_range;
  /* latency of completed requests; p50 and p99 come from a fixed histogram
   * of 64 log buckets per octave (within 0.6% of the exact order statistic),
   * max and mean are exact */
  double p50_us, p99_us, max_us, mean_us;
  double elapsed_s;                       /* since start or last reset       */
  double completed_per_s;
  uint64_t busy;                          /* refused with GB_EBUSY           */
  uint64_t pool_bytes, pool_peak_bytes;   /* range pool: size, peak in use   */
} gb_serve_stats;

/* Measured peaks for the roofline of the integer kernels: 32-bit ALU
 * operations per second and conflict-free shared-memory atomicAnd per second
 * on this device (short probe kernels; no counterpart in the reference). */
gb_status gb_probe_peaks(gb_ctx* ctx, double* alu_ops_per_s, double* smem_atomics_per_s);
/* Measured peak of 64-bit Montgomery products per second (a*b*2^-64 mod n,
 * independent products on every thread): the unit of the Miller-Rabin work
 * in the single-n and Phase-2 kernels.  No counterpart in the reference. */
gb_status gb_probe_mont_products(gb_ctx* ctx, double* per_s);

/* Monotonic clock used for arrival times (nanoseconds). */
uint64_t gb_now_ns(void);
/* Starts the serving lanes on ctx (builds the tables for max_n first). */
gb_status gb_serve_start(gb_ctx* ctx, const gb_serve_opts* opts);
/* Queues count requests; tickets[i] identifies request i.  Thread-safe. */
gb_status gb_submit(gb_ctx* ctx, const gb_request* reqs, size_t count, uint64_t* tickets);
/* GB_OK and the response once done (the ticket is then released),
 * GB_EAGAIN while pending.  Thread-safe. */
gb_status gb_poll(gb_ctx* ctx, uint64_t ticket, gb_response* out);
/* Like gb_poll, waiting up to timeout_ms (GB_ETIMEOUT after that; capped at
 * 2^40 ms, so UINT64_MAX waits without a practical bound).  GB_EINVAL at
 * once for a ticket that was never issued. */
gb_status gb_wait(gb_ctx* ctx, uint64_t ticket, gb_response* out, uint64_t timeout_ms);
/* Latency percentiles and throughput; reset != 0 starts a new window. */
gb_status gb_serve_stats_get(gb_ctx* ctx, gb_serve_stats* out, int reset);
/* Drains the pending requests and stops the lanes. */
gb_status gb_serve_stop(gb_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* GB_GB_H */
