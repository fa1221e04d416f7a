// big_check_main.cpp -- `big_check <N>`: a Goldbach partition of one even
// N of any size up to 4096 bits, on the GPU.
//
// Drop-in for the reference's big_check (src/big_check.cpp:35-174): the same
// argument rules, error strings and result lines ("<N>\n  = p + q",
// "Goldbach holds. ✓", "NO PARTITION FOUND -- counterexample!").  The p
// printed is the minimal one (the reference prints the first its threads
// find); q is accepted by a 12-base strong probable-prime test
// (gb_check_big), proven prime for q < 3.3e24.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "gb/gb.h"

namespace {

std::vector<uint32_t> parse_decimal(const std::string& s) {
  std::vector<uint32_t> v{0};
  for (char ch : s) {
    uint64_t carry = (uint64_t)(ch - '0');
    for (uint32_t& limb : v) {
      const uint64_t x = (uint64_t)limb * 10 + carry;
      limb = (uint32_t)x;
      carry = x >> 32;
    }
    if (carry) v.push_back((uint32_t)carry);
  }
  return v;
}

std::string to_decimal(std::vector<uint32_t> v) {
  while (v.size() > 1 && v.back() == 0) v.pop_back();
  std::vector<uint32_t> parts;  // base 1e9, least significant first
  while (!(v.size() == 1 && v[0] == 0)) {
    uint64_t rem = 0;
    for (size_t i = v.size(); i-- > 0;) {
      const uint64_t x = (rem << 32) | v[i];
      v[i] = (uint32_t)(x / 1000000000u);
      rem = x % 1000000000u;
    }
    parts.push_back((uint32_t)rem);
    while (v.size() > 1 && v.back() == 0) v.pop_back();
  }
  if (parts.empty()) return "0";
  std::string out = std::to_string(parts.back());
  for (size_t i = parts.size() - 1; i-- > 0;) {
    std::string p = std::to_string(parts[i]);
    out += std::string(9 - p.size(), '0') + p;
  }
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2 || std::string(argv[1]) == "-h" || std::string(argv[1]) == "--help") {
    std::cout << "Arbitrary Precision Goldbach Checker (GPU)\n";
    std::cout << "Usage:   " << argv[0] << " <N>\n";
    std::cout << "Example: " << argv[0] << " 1000000000000000000000000000000\n";
    return 0;
  }
  const std::string n_str = argv[1];
  for (char ch : n_str) {
    if (ch < '0' || ch > '9') {
      std::cerr << "Error: Input must be a positive integer.\n";
      return 1;
    }
  }
  const int last_digit = n_str.back() - '0';
  if (last_digit % 2 != 0) {
    std::cerr << "Error: Goldbach's conjecture applies to even integers >= 4.\n";
    std::cerr << "Input ends in '" << last_digit << "' (odd).\n";
    return 1;
  }
  if (n_str.size() <= 100) std::cout << "Checking Goldbach for n = " << n_str << "\n";
  else std::cout << "Checking Goldbach for n with " << n_str.size() << " digits\n";
  std::cout << "  (" << n_str.size() << " digits)\n\n";
  std::vector<uint32_t> n = parse_decimal(n_str);
  while (n.size() > 1 && n.back() == 0) n.pop_back();
  if ((n.size() == 1 && n[0] < 4)) {
    std::cerr << "Error: invalid number or not even / >= 4\n";
    return 1;
  }
  if (n.size() > GB_BIG_MAX_LIMBS) {
    std::cerr << "Error: n has more than " << 32 * GB_BIG_MAX_LIMBS << " bits.\n";
    return 1;
  }
  const auto t0 = std::chrono::steady_clock::now();
  gb_ctx* ctx = nullptr;
  gb_status st = gb_create(0, nullptr, &ctx);
  if (st != GB_OK) {
    std::cerr << "Error: " << gb_strerror(st) << "\n";
    return 1;
  }
  uint64_t p = 0;
  std::vector<uint32_t> q(n.size(), 0);
  gb_big_result r{};
  st = gb_check_big(ctx, n.data(), (uint32_t)n.size(), 0, &p, q.data(), &r);
  if (st != GB_OK) {
    std::cerr << "Error: " << gb_strerror(st) << " (" << gb_last_error(ctx) << ")\n";
    gb_destroy(ctx);
    return 1;
  }
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "\n--- Result ---\n";
  if (p > 0) {
    const std::string q_str = to_decimal(q);
    if (n_str.size() <= 100) {
      std::cout << n_str << "\n  = " << p << " + " << q_str << "\n";
    } else {
      std::cout << "n has " << n_str.size() << " digits\n";
      std::cout << "p = " << p << "\n";
      std::cout << "q has " << q_str.size() << " digits\n";
    }
    std::cout << "Goldbach holds. ✓\n";
  } else {
    std::cout << "NO PARTITION FOUND -- counterexample!\n";
  }
  std::cout << "\n--- Timing ---\n";
  std::cout << "Candidates   : " << r.candidates << " (" << r.mr_tests << " strong tests)\n";
  std::cout << "Total time   : " << ms / 1000.0 << " seconds\n";
  gb_destroy(ctx);
  return 0;
}
