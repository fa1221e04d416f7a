// single_check_main.cpp -- the `single_check` CLI on top of gb.h.
//
// Drop-in for the reference's `single_check` (src/single_check.cu:284-319):
// same parsing, error strings and result lines ("n = p + q",
// "Goldbach holds. ✓").  The partition printed is the minimal one (smallest
// p), which is a valid partition as before.  The reference sieves candidate
// p on the CPU in chunks of 1e8; here the candidates come from the resident
// device prime table, so the "Sieve time (CPU)" line reports 0.
//
// Extension: more than one n may be given; each gets its own result block,
// and all are checked in one batched call.
#include <chrono>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "gb/gb.h"

int main(int argc, char** argv) {
  if (argc < 2 || std::string(argv[1]) == "-h" || std::string(argv[1]) == "--help") {
    std::cout << "GPU Single Number Goldbach Checker\n";
    std::cout << "Usage: " << argv[0] << " <N> [N ...]\n";
    std::cout << "Example: " << argv[0] << " 1000000000000\n";
    return 0;
  }
  std::vector<uint64_t> ns;
  for (int i = 1; i < argc; ++i) {
    uint64_t n;
    try {
      n = std::stoull(argv[i]);
    } catch (const std::out_of_range&) {
      std::cerr << "Error: Number is too large for 64-bit unsigned integer.\n";
      std::cerr << "Use 'big_check' for numbers > 1.84 x 10^19.\n";
      return 1;
    } catch (const std::exception&) {
      std::cerr << "Error: Invalid numeric argument.\n";
      return 1;
    }
    if (n < 4) {
      std::cerr << "Error: n must be >= 4.\n";
      return 1;
    }
    if (n % 2 != 0) {
      std::cerr << "Error: n must be an even integer.\n";
      return 1;
    }
    ns.push_back(n);
  }
  for (uint64_t n : ns) std::cout << "Checking Goldbach for n = " << n << "...\n";
  auto t0 = std::chrono::steady_clock::now();
  gb_ctx* ctx = nullptr;
  gb_status st = gb_create(0, nullptr, &ctx);
  if (st != GB_OK) {
    std::cerr << (st == GB_ENODEV ? "No CUDA devices found.\n" : "CUDA error: ") << (st == GB_ENODEV ? "" : gb_strerror(st))
              << (st == GB_ENODEV ? "" : "\n");
    return 1;
  }
  auto t1 = std::chrono::steady_clock::now();
  std::vector<uint64_t> p(ns.size()), q(ns.size());
  gb_single_result r{};
  st = gb_check_single_batch(ctx, ns.data(), ns.size(), p.data(), q.data(), nullptr, &r);
  auto t2 = std::chrono::steady_clock::now();
  if (st != GB_OK) {
    std::cerr << "CUDA error: " << gb_strerror(st) << " (" << gb_last_error(ctx) << ")\n";
    gb_destroy(ctx);
    return 1;
  }
  for (size_t i = 0; i < ns.size(); ++i) {
    std::cout << "Checking Goldbach for n = " << ns[i] << "\n\n";
    std::cout << "\n--- Result ---\n";
    if (p[i]) {
      std::cout << ns[i] << " = " << p[i] << " + " << q[i] << "\n";
      std::cout << "Goldbach holds. ✓\n";
    } else {
      std::cout << "NO PARTITION FOUND — counterexample!\n";
    }
  }
  const double table_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  const double total_ms = std::chrono::duration<double, std::milli>(t2 - t0).count();
  std::cout << "\n--- Timing ---\n";
  std::cout << "Sieve time (CPU) : 0 ms\n";
  std::cout << "Table build (GPU): " << table_ms << " ms\n";
  std::cout << "Kernel time (GPU): " << r.device_ms << " ms\n";
  std::cout << "Total            : " << total_ms << " ms\n";
  gb_destroy(ctx);
  return 0;
}
