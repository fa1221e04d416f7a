// ref_shim.cpp -- C entry points over the reference's own CPU functions.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/build_ref.sh together with
// the reference sources src/segmented_sieve.cpp and src/cpu_goldbach.cpp
// (its main() renamed on the command line), straight from the read-only
// reference tree.  The resulting oracle/_ref/libgbref.so lets tests and the
// reference arm of bench.py call the reference's code unmodified:
//   simple_sieve / segmented_sieve   src/segmented_sieve.cpp:13-50
//   goldbach_verify / goldbach_count src/cpu_goldbach.cpp:14-36
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

// Defined in the reference sources linked into this library.
std::vector<uint64_t> simple_sieve(uint64_t limit);
std::vector<char> segmented_sieve(uint64_t low, uint64_t high);
bool goldbach_verify(uint64_t n, const std::vector<char>& is_prime);
uint64_t goldbach_count(uint64_t n, const std::vector<char>& is_prime);

extern "C" {

// Prime count of [low, high] from the reference segmented_sieve.
uint64_t gbref_count_primes(uint64_t low, uint64_t high) {
  std::vector<char> t = segmented_sieve(low, high);
  uint64_t c = 0;
  for (char x : t) c += x ? 1 : 0;
  return c;
}

// Byte table of [low, high] from the reference segmented_sieve.
void gbref_segmented_sieve(uint64_t low, uint64_t high, uint8_t* out) {
  std::vector<char> t = segmented_sieve(low, high);
  for (size_t i = 0; i < t.size(); i++) out[i] = t[i] ? 1 : 0;
}

// cpu_goldbach's own loop (src/cpu_goldbach.cpp:98-111) over [4, limit]:
// returns the number of even n for which goldbach_verify fails.
uint64_t gbref_verify_upto(uint64_t limit) {
  std::vector<char> t = segmented_sieve(0, limit);
  uint64_t fails = 0;
  for (uint64_t n = 4; n <= limit; n += 2)
    if (!goldbach_verify(n, t)) fails++;
  return fails;
}

// goldbach_count(n) for every even n in [4, limit] (out[(n-4)/2]).
void gbref_goldbach_counts(uint64_t limit, uint64_t* out) {
  std::vector<char> t = segmented_sieve(0, limit);
  for (uint64_t n = 4; n <= limit; n += 2) out[(n - 4) / 2] = goldbach_count(n, t);
}

// Reference CPU arm over windows far from 0, where cpu_goldbach's single
// [0, LIMIT] byte table cannot be built (1 TB at 1e12).  For each even n in
// [start, start + 2*(count-1)] it applies goldbach_verify's rule (scan every
// integer p = 2.. n/2 ascending, test is_prime[p] && is_prime[n-p]) with
// the byte tables produced by the reference segmented_sieve: one of [0, H]
// for p and one of [start-H, end] for q.  Returns the number of n left
// unverified with p <= H (0 on every range tested so far); min_p (nullable)
// receives the first p found.  Work is split over nthreads std::threads.
uint64_t gbref_window_verify(uint64_t start, uint64_t count, uint64_t H,
                             uint32_t* min_p, int nthreads) {
  if (count == 0) return 0;
  if (nthreads < 1) nthreads = 1;
  const uint64_t end = start + 2 * (count - 1);
  const std::vector<char> ptab = segmented_sieve(0, H);
  const uint64_t BLK = 1 << 16;
  const uint64_t nblk = (count + BLK - 1) / BLK;
  std::vector<uint64_t> unver(nthreads, 0);
  auto work = [&](int t) {
    for (uint64_t b = t; b < nblk; b += nthreads) {
      uint64_t j0 = b * BLK;
      uint64_t cnt = std::min<uint64_t>(BLK, count - j0);
      uint64_t A = start + 2 * j0, B = A + 2 * (cnt - 1);
      uint64_t lo = A > H + 2 ? A - H : 0;
      std::vector<char> q = segmented_sieve(lo, std::min(B, end));
      for (uint64_t j = 0; j < cnt; j++) {
        uint64_t n = A + 2 * j, found = 0;
        for (uint64_t p = 2; p <= n / 2 && p <= H; p++) {
          if (ptab[p] && q[n - p - lo]) {
            found = p;
            break;
          }
        }
        if (!found) unver[t]++;
        if (min_p) min_p[j0 + j] = (uint32_t)found;
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nthreads; t++) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  uint64_t s = 0;
  for (uint64_t u : unver) s += u;
  return s;
}

}  // extern "C"
