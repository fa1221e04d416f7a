// noalloc.cu -- batched single-n minimal partitions without any device
// allocation.
//
// Some callers cannot call cudaMalloc at all: code that runs while a CUDA
// stream is being captured into a graph, code inside another framework's
// memory pool that forbids stray allocations, or a real-time loop that must
// not touch the allocator after start-up.  gb_check_single_batch_noalloc
// serves them: the caller passes device buffers for the inputs and outputs,
// and everything else the kernel needs -- its work and result counters and
// its table of candidate primes -- lives in one file-scope array below, of a
// fixed size, that every GPU which loads this library holds until exit.
//
// The array's name seen from host code is a host-side stand-in, not a
// device address: passing it to a kernel would fault (or, where the GPU can
// reach host memory, silently use the wrong memory).  Its device address is
// looked up with cudaGetSymbolAddress, with the device current, and that
// address is what the kernels receive.  The table is built once per CUDA
// context (the array is per context: a reset or another context on the
// same device starts with it zeroed).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "../gb_internal.h"
#include "gb/gb.h"

namespace gb {

// Candidate primes: every prime below 2^16 (6542 of them, 2 first).
constexpr uint32_t kNoAllocTableCap = 6542;
constexpr uint32_t kNoAllocCounters = 4;  // work, found, max p, table size (as 64-bit words)
constexpr size_t kNoAllocBytes = kNoAllocCounters * 8 + kNoAllocTableCap * 4;

// The scratch: counters first, then the prime table.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// One CTA sieves the odd numbers below 2^16 in shared memory and writes the
// primes, ascending, after the counters.
__global__ void __launch_bounds__(1024) noalloc_table_kernel(unsigned char* scratch) {
  __shared__ uint32_t bits[1024];  // bit i <-> odd 2i + 1
  __shared__ uint32_t wsum[32];
  const int t = threadIdx.x;
  bits[t] = 0xffffffffu;
  __syncthreads();
  if (t == 0) bits[0] &= ~1u;  // 1 is not prime
  for (uint32_t d = 3 + 2 * t; d * d < 65536; d += 2048)
    for (uint32_t m = d * d; m < 65536; m += 2 * d) atomicAnd(&bits[m >> 6], ~(1u << ((m >> 1) & 31)));
  __syncthreads();
  const uint32_t v = bits[t];
  const uint32_t c = __popc(v);
  const int lane = t & 31, warp = t >> 5;
  uint32_t x = c;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(scratch);
  uint32_t* primes = reinterpret_cast<uint32_t*>(scratch + kNoAllocCounters * 8);
  uint32_t pos = 1 + (warp ? wsum[warp - 1] : 0) + (x - c);
  uint32_t w = v;
  while (w) {
    const int b = __ffs(w) - 1;
    w &= w - 1;
    if (pos < kNoAllocTableCap) primes[pos] = 2 * (32 * t + b) + 1;
    ++pos;
  }
  if (t == 0) {
    primes[0] = 2;
    ctr[3] = 1 + wsum[31];
  }
}

namespace {
// The scratch array exists once per CUDA context: a context created later
// on the same device (after cudaDeviceReset, or a context the caller made
// current through the driver API) loads the module afresh, with the array
// zeroed and possibly at another address.  Set-up is therefore cached per
// context, keyed by the driver's context ID, which is never reused within
// a process.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_entry_once;

struct ScratchSetup {
  unsigned long long ctx_id;  // driver context ID (device + 1 when IDs are unavailable)
  void* ptr;                  // device address of g_noalloc_scratch in that context
};
std::mutex g_setup_mu;
std::vector<ScratchSetup> g_setups;  // contexts whose table is built

// ID of the context current on this thread; the device number + 1 when the
// driver entry points cannot be had (then a reset is not detected).
unsigned long long current_context_key(int dev) {
  std::call_once(g_entry_once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_get_current && g_ctx_get_id && g_ctx_get_current(&ctx) == 0 && ctx &&
      g_ctx_get_id(ctx, &id) == 0)
    return id | (1ull << 63);  // kept apart from the device-number fallback
  return (unsigned long long)dev + 1;
}
}  // namespace

}  // namespace gb

using namespace gb;

extern "C" gb_status gb_check_single_batch_noalloc(const uint64_t* n, size_t count, uint64_t* p_out,
                                                   uint64_t* q_out, uint64_t p_limit,
                                                   void* stream) {
  if (count && (!n || !p_out || !q_out)) return GB_EINVAL;
  if (p_limit == 0) p_limit = GB_NOALLOC_P_LIMIT;
  if (p_limit > GB_NOALLOC_P_LIMIT) return GB_EINVAL;  // beyond the fixed prime table
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return GB_ENODEV;
  cudaStream_t s = (cudaStream_t)stream;
  void* ptr = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    // the symbol lookup also binds the runtime to the thread's context, so
    // the key read next names the context the kernels will run in
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return GB_ECUDA;
    const unsigned long long key = current_context_key(dev);
    bool ready = false;
    for (const ScratchSetup& e : g_setups)
      if (e.ctx_id == key && e.ptr == ptr) ready = true;
    if (!ready) {
      // first call in this context: build the table (synchronous)
      noalloc_table_kernel<<<1, 1024, 0, s>>>(static_cast<unsigned char*>(ptr));
      if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return GB_ECUDA;
      g_setups.push_back(ScratchSetup{key, ptr});
    }
  }
  if (!count) return GB_OK;
  unsigned long long* ctr = static_cast<unsigned long long*>(ptr);
  // counters start at zero on every call (the array keeps the last call's)
  if (cudaMemsetAsync(ctr, 0, 3 * sizeof(unsigned long long), s) != cudaSuccess) return GB_ECUDA;
  // the number of primes <= p_limit comes from the table itself
  SingleArgs a{};
  a.n = n;
  a.count = count;
  a.p_out = p_out;
  a.q_out = q_out;
  a.primes = reinterpret_cast<const uint32_t*>(static_cast<unsigned char*>(ptr) + kNoAllocCounters * 8);
  a.nprimes = kNoAllocTableCap;
  a.p_lim = p_limit;
  a.ctr = ctr;
  int sm = 148;
  cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
  uint64_t grid = (uint64_t)sm * 6;
  if (grid > (count + 7) / 8) grid = (count + 7) / 8;
  if (launch_single(a, (int)(grid ? grid : 1), s) != cudaSuccess) return GB_ECUDA;
  return GB_OK;
}
