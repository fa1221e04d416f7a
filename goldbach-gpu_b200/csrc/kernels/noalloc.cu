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
// obtained once per device with cudaGetSymbolAddress, with that device
// current, and that address is what the kernels receive.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

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
std::mutex g_setup_mu;
void* g_scratch_ptr[64];  // device address of g_noalloc_scratch per device
bool g_table_ready[64];
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
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return GB_ENODEV;
  cudaStream_t s = (cudaStream_t)stream;
  void* ptr = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return GB_ECUDA;
      g_scratch_ptr[dev] = ptr;
    }
    ptr = g_scratch_ptr[dev];
    if (!g_table_ready[dev]) {
      // first call on this device: build the table (synchronous)
      noalloc_table_kernel<<<1, 1024, 0, s>>>(static_cast<unsigned char*>(ptr));
      if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return GB_ECUDA;
      g_table_ready[dev] = true;
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
