// ref_phase2_shim.cu -- C entry points over the reference's static host
// helpers in src/goldbach.cu.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build_ref.sh compiles this file with the
// reference's src/ and include/ directories on the include path; the
// #include below pulls the unmodified reference translation unit in (its
// main() renamed), so its file-static functions can be reached:
//   cpu_miller_rabin     src/goldbach.cu:333-360 (12 prime bases)
//   cpu_optimized_check  src/goldbach.cu:362-373 (Phase 2)
//   generate_cpu_primes  src/goldbach.cu:318-331
#define main gbref_goldbach_main
#include "goldbach.cu"
#undef main

#include <mutex>

static std::once_flag g_once;
static std::vector<uint64_t> g_cpu_primes;

extern "C" {

int gbref_cpu_miller_rabin(uint64_t n) { return cpu_miller_rabin(n) ? 1 : 0; }

// Phase 2 of the reference with its own prime table (primes <= 1e8).
int gbref_cpu_optimized_check(uint64_t n) {
  std::call_once(g_once, [] { g_cpu_primes = generate_cpu_primes(PHASE2_SIEVE_LIMIT); });
  return cpu_optimized_check(n, g_cpu_primes) ? 1 : 0;
}

void gbref_cpu_miller_rabin_batch(const uint64_t* n, size_t count, uint8_t* out) {
  for (size_t i = 0; i < count; i++) out[i] = cpu_miller_rabin(n[i]) ? 1 : 0;
}

}  // extern "C"
