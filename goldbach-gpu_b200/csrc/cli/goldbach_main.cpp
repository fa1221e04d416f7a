// goldbach_main.cpp -- the `goldbach` range verifier CLI on top of gb.h.
//
// Drop-in for the reference's `goldbach` (src/goldbach.cu:543-801): same
// argv grammar (positional <LIMIT> [SEG_SIZE] [P_SMALL] and --seg-size=,
// --p-small=, --batch-size=, --gpus=, --start=, --progress, --async,
// -h/--help), the same normalisation and error strings, the same summary
// lines and exit codes (0 ok; 1 failure, error or guard).  All device work
// goes through gb_verify_range; there is no CPU Phase 2.
//
// Additional flags: --chunk=N (even n per CTA window), --halo=N,
// --phase2-limit=N, --device-mem-mb=N (device memory budget, used by the
// VRAM guard), --json (one JSON summary line at the end), --journal=FILE
// (resumable runs, journal.h) with --journal-segments=K (segments per
// record) and --stop-after-batches=N (end the run after N new records, exit
// code 3: the way tests interrupt a run), --counts (print c(n), the number
// of Goldbach partitions, for every even n of [START, LIMIT] in the
// reference's `c(n) = k` form, src/cpu_goldbach.cpp:100-103), --autotune
// (pick chunk and halo with gb_autotune_range; --autotune-cache=FILE keeps
// the choice per range class across runs), --tile=N (the same as --chunk),
// --minp-out=FILE (the minimal p of every n, uint32 little-endian, in range
// order) and --bitmap-out=FILE (the verified bit of every n, bit j of byte
// j/8 for n = START + 2j); the output files are written from GPU 0 in order.
#include <atomic>
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "gb/gb.h"
#include "journal.h"

namespace {

using clk = std::chrono::steady_clock;

void print_usage(const char* prog) {
  std::cout << "Goldbach Multi-GPU Verifier\n\n"
            << "Usage:\n"
            << "  " << prog << " <LIMIT> [SEG_SIZE] [P_SMALL]\n"
            << "  " << prog << " <LIMIT> [--seg-size=N] [--p-small=N] [--gpus=N]\n\n"
            << "Required:\n"
            << "  LIMIT            Max even integer to check\n\n"
            << "Optional:\n"
            << "  --seg-size=N     Even integers per segment (default: 10,000,000)\n"
            << "  --p-small=N      GPU prime search bound (max: 4,000,000,000)\n"
            << "  --batch-size=N   Primes per GPU batch (default: 100000; accepted, unused)\n"
            << "  --gpus=N         Number of GPUs to use (default: 1)\n"
            << "  --start=N        Starting number for verification (default: 4)\n"
            << "  --progress       Show real-time progress updates\n"
            << "  --chunk=N        Even integers per CTA window (power of 2, default: auto)\n"
            << "  --halo=N         q-window halo in numbers (default: 32768)\n"
            << "  --phase2-limit=N Phase 2 prime bound (default: 100,000,000)\n"
            << "  --device-mem-mb=N Device memory budget per GPU in MB\n"
            << "  --json           Print a JSON summary line\n"
            << "  --journal=FILE   Record completed segments in FILE; rerun to resume\n"
            << "  --journal-segments=K  Segments per journal record (default: about 2^36 n)\n"
            << "  --stop-after-batches=N  Stop after N new journal records (exit code 3)\n"
            << "  --counts         Print c(n) = number of partitions for each even n\n"
            << "  --autotune       Pick chunk and halo for this range by timing a sample\n"
            << "  --autotune-cache=FILE  Reuse / record autotuned choices per range class\n"
            << "  --tile=N         Same as --chunk=N\n"
            << "  --minp-out=FILE  Write the minimal p of every n (uint32, in order)\n"
            << "  --bitmap-out=FILE Write the verified bit of every n (bit j <-> START+2j)\n"
            << "  -h, --help       Show this help message\n";
}

// Appends bit strings to a file whatever their alignment: bit j of the
// stream is bit j % 8 of byte j / 8.
struct BitWriter {
  FILE* f;
  uint32_t carry = 0;  // pending low bits of the next byte
  int ncarry = 0;
  bool put(const uint32_t* words, uint64_t nbits) {
    std::vector<uint8_t> out;
    out.reserve(nbits / 8 + 2);
    for (uint64_t i = 0; i < nbits; i += 8) {
      const uint64_t take = nbits - i < 8 ? nbits - i : 8;
      uint32_t b = (words[i >> 5] >> (i & 31)) & ((1u << take) - 1);
      carry |= b << ncarry;
      ncarry += (int)take;
      if (ncarry >= 8) {
        out.push_back((uint8_t)(carry & 0xff));
        carry >>= 8;
        ncarry -= 8;
      }
    }
    return std::fwrite(out.data(), 1, out.size(), f) == out.size();
  }
  bool finish() {
    if (!ncarry) return true;
    const uint8_t b = (uint8_t)carry;
    ncarry = 0;
    return std::fwrite(&b, 1, 1, f) == 1;
  }
};

struct Worker {
  gb_ctx* ctx = nullptr;
  gb_status st = GB_OK;
  std::string err;
  uint64_t checked = 0, fallbacks = 0, failures = 0, first_fail = 0, max_minp = 0, launches = 0;
  double device_ms = 0;
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    print_usage(argv[0]);
    return 0;
  }
  bool show_progress = false, json = false, counts_mode = false;
  uint64_t LIMIT = 0, SEG_SIZE = 10'000'000ULL, P_SMALL = 1'000'000ULL, START = 4;
  uint64_t chunk = 0, halo = 0, phase2 = 0, mem_mb = 0, batch = 100000, threads = 0;
  std::string journal_path, tune_cache, minp_path, bitmap_path;
  bool autotune = false;
  uint64_t journal_segs = 0, stop_after = 0;
  long requested_gpus = 1;
  std::vector<std::string> positional;
  try {
    for (int i = 1; i < argc; i++) {
      std::string arg = argv[i];
      if (arg == "-h" || arg == "--help") {
        print_usage(argv[0]);
        return 0;
      }
      if (arg == "--async") continue;
      if (arg == "--progress") { show_progress = true; continue; }
      if (arg == "--json") { json = true; continue; }
      if (arg == "--counts") { counts_mode = true; continue; }
      if (arg == "--autotune") { autotune = true; continue; }
      if (arg.rfind("--autotune-cache=", 0) == 0) { tune_cache = arg.substr(17); autotune = true; continue; }
      if (arg.rfind("--tile=", 0) == 0) { chunk = std::stoull(arg.substr(7)); continue; }
      if (arg.rfind("--minp-out=", 0) == 0) { minp_path = arg.substr(11); continue; }
      if (arg.rfind("--bitmap-out=", 0) == 0) { bitmap_path = arg.substr(13); continue; }
      if (arg.rfind("--batch-size=", 0) == 0) { batch = std::stoull(arg.substr(13)); continue; }
      if (arg.rfind("--gpus=", 0) == 0) { requested_gpus = std::stol(arg.substr(7)); continue; }
      if (arg.rfind("--seg-size=", 0) == 0) { SEG_SIZE = std::stoull(arg.substr(11)); continue; }
      if (arg.rfind("--p-small=", 0) == 0) { P_SMALL = std::stoull(arg.substr(10)); continue; }
      if (arg.rfind("--start=", 0) == 0) { START = std::stoull(arg.substr(8)); continue; }
      if (arg.rfind("--chunk=", 0) == 0) { chunk = std::stoull(arg.substr(8)); continue; }
      if (arg.rfind("--halo=", 0) == 0) { halo = std::stoull(arg.substr(7)); continue; }
      if (arg.rfind("--phase2-limit=", 0) == 0) { phase2 = std::stoull(arg.substr(15)); continue; }
      if (arg.rfind("--device-mem-mb=", 0) == 0) { mem_mb = std::stoull(arg.substr(16)); continue; }
      if (arg.rfind("--journal=", 0) == 0) { journal_path = arg.substr(10); continue; }
      if (arg.rfind("--journal-segments=", 0) == 0) { journal_segs = std::stoull(arg.substr(19)); continue; }
      if (arg.rfind("--stop-after-batches=", 0) == 0) { stop_after = std::stoull(arg.substr(21)); continue; }
      positional.push_back(arg);
    }
    if (positional.size() >= 1) LIMIT = std::stoull(positional[0]);
    if (positional.size() >= 2) SEG_SIZE = std::stoull(positional[1]);
    if (positional.size() >= 3) P_SMALL = std::stoull(positional[2]);
  } catch (...) {
    std::cerr << "Error: Invalid numeric argument.\n";
    return 1;
  }
  (void)batch;
  // src/goldbach.cu:593-622
  if (LIMIT < 4) { std::cerr << "Error: LIMIT must be >= 4.\n"; return 1; }
  if (LIMIT % 2 != 0) LIMIT--;
  if (SEG_SIZE == 0 || SEG_SIZE % 2 != 0) { std::cerr << "Error: SEG_SIZE must be even and > 0.\n"; return 1; }
  if (P_SMALL > GB_P_SMALL_MAX) {
    std::cerr << "Error: P_SMALL must be <= " << GB_P_SMALL_MAX << " to prevent mathematical overflow.\n";
    return 1;
  }
  if (P_SMALL > LIMIT) P_SMALL = LIMIT;
  if (START < 4) START = 4;
  if (START % 2 != 0) START++;
  if (START >= LIMIT) { std::cerr << "Error: START must be less than LIMIT.\n"; return 1; }
  if (P_SMALL < 1'000'000ULL) {
    std::cerr << "\n[!] WARNING: P_SMALL = " << P_SMALL << " is very small.\n"
              << "    This may cause excessive Phase 2 fallbacks.\n"
              << "    Recommended: P_SMALL >= 10^7 for numbers > 10^12\n"
              << "                 P_SMALL >= 10^8 for numbers > 10^18\n\n";
  }
  // exact isqrt (src/goldbach.cu:637-646) and the small table bound (:648-649)
  uint64_t sqrt_limit = 0;
  {
    uint64_t lo = 1, hi = LIMIT > (1ULL << 32) ? (1ULL << 32) : LIMIT;
    while (lo <= hi) {
      uint64_t mid = lo + (hi - lo) / 2;
      if (mid <= LIMIT / mid) { sqrt_limit = mid; lo = mid + 1; }
      else hi = mid - 1;
    }
  }
  uint64_t small_high = std::max<uint64_t>(sqrt_limit + 1, P_SMALL);
  if (small_high % 2 == 0) small_high++;
  const uint64_t p2 = phase2 ? phase2 : GB_PHASE2_LIMIT_DEFAULT;
  const uint64_t total = (LIMIT - START) / 2 + 1;
  const uint64_t nseg = (total + SEG_SIZE - 1) / SEG_SIZE;

  // Partition counts: c(n) for every even n of [START, LIMIT], on GPU 0.
  if (counts_mode) {
    if (gb_device_count() == 0) {
      std::cerr << "No CUDA devices found.\n";
      return 1;
    }
    gb_config ccfg{};
    ccfg.device_mem_budget = mem_mb << 20;
    gb_ctx* cctx = nullptr;
    gb_status st = gb_create(0, &ccfg, &cctx);
    if (st != GB_OK) {
      std::cerr << "[!] FATAL ERROR in GPU 0 Worker: " << gb_strerror(st) << "\n";
      return 1;
    }
    const uint64_t per = 1ull << 16;
    std::vector<uint64_t> c(per);
    auto tc = clk::now();
    for (uint64_t j = 0; j < total && st == GB_OK; j += per) {
      const uint64_t k = std::min(per, total - j);
      st = gb_goldbach_counts(cctx, START + 2 * j, k, c.data(), nullptr);
      for (uint64_t i = 0; st == GB_OK && i < k; ++i)
        std::printf("c(%" PRIu64 ") = %" PRIu64 "\n", START + 2 * (j + i), c[i]);
    }
    if (st != GB_OK) {
      std::cerr << "[!] FATAL ERROR in GPU 0 Worker: " << gb_strerror(st) << " (" << gb_last_error(cctx) << ")\n";
      gb_destroy(cctx);
      return 1;
    }
    gb_destroy(cctx);
    std::fflush(stdout);
    std::cout << "\n--- Summary ---\n";
    std::cout << "Even numbers counted : " << total << "\n";
    std::cout << "Total time           : " << std::chrono::duration<double, std::milli>(clk::now() - tc).count() << " ms\n";
    return 0;
  }

  const bool outputs = !minp_path.empty() || !bitmap_path.empty();
  if (outputs && !journal_path.empty()) {
    std::cerr << "Error: --minp-out / --bitmap-out cannot be combined with --journal.\n";
    return 1;
  }

  // The journal: what earlier runs of this command finished.
  gbj::Journal journal;
  Worker prior;  // journaled figures
  std::vector<std::pair<uint64_t, uint64_t>> pending;
  const bool journaling = !journal_path.empty();
  if (journaling) {
    std::string jerr;
    if (!journal.open(journal_path, gbj::Key{START, LIMIT, SEG_SIZE, P_SMALL, p2}, &jerr)) {
      std::cerr << "Error: " << jerr << "\n";
      return 1;
    }
    uint64_t done_segs = 0;
    for (const gbj::Record& r : journal.records()) {
      done_segs += r.hi - r.lo;
      prior.checked += r.checked;
      prior.fallbacks += r.fallbacks;
      prior.failures += r.failures;
      prior.max_minp = std::max(prior.max_minp, r.max_minp);
      if (r.first_fail && (!prior.first_fail || r.first_fail < prior.first_fail)) prior.first_fail = r.first_fail;
    }
    const uint64_t per = journal_segs ? journal_segs : std::max<uint64_t>(1, ((1ull << 36) + SEG_SIZE - 1) / SEG_SIZE);
    pending = gbj::pending_batches(journal.records(), nseg, per);
    if (!journal.records().empty())
      std::cout << "Resuming from journal " << journal_path << ": " << done_segs << " of " << nseg
                << " segments done, " << pending.size() << " batches to run\n";
    if (pending.empty() || prior.failures) {  // nothing left for the GPU
      if (prior.failures) {
        std::cout << "\n[!] Goldbach FAILED at n = " << prior.first_fail << "\n";
        return 1;
      }
      std::cout << "\n--- Verification Complete ---\n";
      std::cout << "All even numbers from " << START << " up to " << LIMIT << " satisfy Goldbach. ✓\n";
      std::cout << "Total computation time : 0 seconds\n";
      std::cout << "Phase 2 fallbacks      : " << prior.fallbacks << "\n";
      std::cout << "Max minimal p          : " << prior.max_minp << "\n";
      return 0;
    }
  }

  const int device_count = gb_device_count();
  if (device_count == 0) {
    std::cerr << "No CUDA devices found.\n";
    return 1;
  }
  if (requested_gpus > device_count) {
    std::cerr << "Requested " << requested_gpus << " GPUs, but only " << device_count
              << " available. Using " << device_count << ".\n";
  }
  int use_gpus = (requested_gpus <= 0 || requested_gpus > device_count) ? device_count : (int)requested_gpus;
  if (outputs && use_gpus > 1) {
    std::cout << "Per-n outputs are written in order from GPU 0: using 1 GPU.\n";
    use_gpus = 1;
  }

  // VRAM guard (src/goldbach.cu:505-541) against what a context will hold;
  // --device-mem-mb caps the available memory.
  gb_config cfg{};
  cfg.device_mem_budget = mem_mb << 20;
  cfg.max_n = LIMIT;
  cfg.cand_limit = std::max(P_SMALL, p2);
  const uint64_t required = gb_estimate_device_bytes(&cfg) + (50ull << 20);
  for (int g = 0; g < use_gpus; ++g) {
    char name[256] = {0};
    uint64_t total_mem = 0;
    gb_device_info(g, name, sizeof name, &total_mem);
    const uint64_t avail = mem_mb ? std::min<uint64_t>(mem_mb << 20, total_mem) : total_mem;
    if (required > avail) {
      std::cerr << "\n[!] ERROR: GPU " << g << " (" << name << ") has insufficient VRAM.\n";
      std::cerr << "    Required: " << required / (1024 * 1024) << " MB\n";
      std::cerr << "    Available: " << avail / (1024 * 1024) << " MB\n";
      std::cerr << "    Reduce SEG_SIZE or use a smaller LIMIT.\n";
      return 1;
    }
    std::cout << "[Hardware] GPU " << g << ": " << name << " (" << total_mem / (1024 * 1024)
              << " MB VRAM)\n";
  }
  // Contexts (one per GPU) build and keep the prime tables on the device.
  std::cout << "Building small primes bitset up to " << small_high << "...\n";
  auto t0 = clk::now();
  std::vector<Worker> w(use_gpus);
  for (int g = 0; g < use_gpus; ++g) {
    gb_status st = gb_create(g, &cfg, &w[g].ctx);
    if (st != GB_OK) {
      std::cerr << "[!] FATAL ERROR in GPU " << g << " Worker: " << gb_strerror(st) << "\n";
      std::cerr << "\n[!] Program aborted due to internal hardware/CUDA errors.\n";
      return 1;
    }
  }
  std::cout << "Pre-generating device primes up to " << std::max(P_SMALL, p2) << "...\n";
  if (autotune) {
    // one line per range class: "class BITS P_SMALL PHASE2 chunk C halo H
    // threads T" (a line without the threads field keeps the default shape)
    uint64_t bits = 0;
    for (uint64_t x = LIMIT; x; x >>= 1) ++bits;
    char key[128];
    std::snprintf(key, sizeof key, "class %" PRIu64 " %" PRIu64 " %" PRIu64, bits, P_SMALL, p2);
    bool found = false;
    if (!tune_cache.empty()) {
      std::ifstream in(tune_cache);
      std::string line;
      while (std::getline(in, line)) {
        unsigned long long c = 0, h = 0, t = 0;
        const size_t at = line.find(" chunk ");
        if (at != std::string::npos && line.substr(0, at) == key &&
            std::sscanf(line.c_str() + at, " chunk %llu halo %llu threads %llu", &c, &h, &t) >= 2) {
          chunk = c;
          halo = h;
          threads = t;
          found = true;
        }
      }
      if (found)
        std::cout << "[Autotune] chunk=" << chunk << " halo=" << halo << " threads=" << threads
                  << " (from " << tune_cache << ")\n";
    }
    if (!found) {
      gb_range_opts base{}, tuned{};
      base.seg_size = SEG_SIZE;
      base.p_small = P_SMALL;
      base.phase2_limit = p2;
      gb_autotune_result ar{};
      const gb_status st = gb_autotune_range(w[0].ctx, START, LIMIT, &base, &tuned, &ar);
      if (st != GB_OK) {
        std::cerr << "[!] FATAL ERROR in GPU 0 Worker: " << gb_strerror(st) << " (" << gb_last_error(w[0].ctx) << ")\n";
        return 1;
      }
      chunk = tuned.chunk_evens;
      halo = tuned.halo;
      threads = tuned.block_threads;
      if (ar.candidates)
        std::cout << "[Autotune] chunk=" << chunk << " halo=" << halo << " threads=" << threads
                  << " (" << std::scientific
                  << std::setprecision(3) << ar.even_n_per_s << " n/s on " << ar.sample_evens
                  << " n, " << ar.candidates << " candidates)\n" << std::defaultfloat << std::setprecision(6);
      else
        std::cout << "[Autotune] range too short to tune: defaults\n";
      if (!tune_cache.empty() && ar.candidates) {
        std::ofstream out(tune_cache, std::ios::app);
        out << key << " chunk " << chunk << " halo " << halo << " threads " << threads << "\n";
      }
    }
  }
  auto t1 = clk::now();
  std::cout << "Initialization completed in "
            << std::chrono::duration<double, std::milli>(t1 - t0).count() << " ms.\n\n";

  std::cout << "--- Launching Multi-GPU Verifier ---\n";
  std::cout << "Checking range : [" << START << ", " << LIMIT << "]\n";
  std::cout << "Total numbers  : " << total << "\n\n";
  std::cout << std::flush;

  // Work is handed out in batches of whole segments so that segment numbers
  // stay those of the full range; GPU g takes batches g, g+G, ...  Without
  // --progress each GPU makes a single call over all its segments.
  // With a journal the batches are the pending segment ranges, taken by
  // the GPUs in turn, each recorded when it completes.
  uint64_t segs_per_batch = nseg;
  if (show_progress) segs_per_batch = std::max<uint64_t>(1, (nseg + 63) / 64);
  if (outputs)  // host buffers of about 2^26 n per call
    segs_per_batch = std::min(segs_per_batch, std::max<uint64_t>(1, (1ull << 26) / SEG_SIZE));
  FILE* f_minp = minp_path.empty() ? nullptr : std::fopen(minp_path.c_str(), "wb");
  FILE* f_bits = bitmap_path.empty() ? nullptr : std::fopen(bitmap_path.c_str(), "wb");
  if ((!minp_path.empty() && !f_minp) || (!bitmap_path.empty() && !f_bits)) {
    std::cerr << "Error: cannot open an output file.\n";
    return 1;
  }
  BitWriter bitw{f_bits};
  std::vector<uint32_t> h_minp, h_bits;
  const uint64_t nbatch = journaling ? pending.size() : (nseg + segs_per_batch - 1) / segs_per_batch;
  std::atomic<uint64_t> processed{prior.checked};
  std::atomic<uint64_t> next_batch{0}, recorded{0};
  std::atomic<bool> stop{false}, interrupted{false};
  std::mutex journal_mu;
  auto t_main = clk::now();

  auto run = [&](int g) {
    Worker& W = w[g];
    const bool single_call = !show_progress && !journaling && !outputs;
    for (uint64_t b = journaling ? next_batch++ : (uint64_t)g; b < nbatch && !stop.load();
         b = journaling ? next_batch++ : b + use_gpus) {
      gb_range_opts o{};
      o.seg_size = SEG_SIZE;
      o.p_small = P_SMALL;
      o.phase2_limit = p2;
      o.chunk_evens = (uint32_t)chunk;
      o.halo = (uint32_t)halo;
      o.block_threads = (uint32_t)threads;
      uint64_t a = START, e = LIMIT;
      if (single_call) {
        o.shard_index = g;
        o.shard_count = use_gpus;
      } else if (journaling) {
        a = START + 2 * SEG_SIZE * pending[b].first;
        e = START + 2 * (std::min(total, SEG_SIZE * pending[b].second) - 1);
      } else {
        a = START + 2 * SEG_SIZE * segs_per_batch * b;
        const uint64_t last_idx = std::min(total, SEG_SIZE * segs_per_batch * (b + 1)) - 1;
        e = START + 2 * last_idx;
      }
      gb_range_result r{};
      gb_range_out ro{};
      const uint64_t bn = (e - a) / 2 + 1;
      if (f_minp) {
        h_minp.resize(bn);
        ro.min_p = h_minp.data();
      }
      if (f_bits) {
        h_bits.resize((bn + 31) / 32);
        ro.verified_bits = h_bits.data();
      }
      gb_status st = gb_verify_range(W.ctx, a, e, &o, &r, outputs ? &ro : nullptr);
      if (st == GB_OK && f_minp && std::fwrite(h_minp.data(), 4, bn, f_minp) != bn) st = GB_EINVAL;
      if (st == GB_OK && f_bits && !bitw.put(h_bits.data(), bn)) st = GB_EINVAL;
      if (st != GB_OK && W.err.empty() && outputs) W.err = "writing an output file failed";
      if (st != GB_OK) {
        W.st = st;
        W.err = gb_last_error(W.ctx);
        stop = true;
        return;
      }
      W.checked += r.checked;
      W.fallbacks += r.phase2_fallbacks;
      W.launches += r.kernel_launches;
      W.device_ms += r.device_ms;
      if (r.max_minp > W.max_minp) W.max_minp = r.max_minp;
      if (r.failures) {
        W.failures += r.failures;
        if (!W.first_fail || r.first_failure_n < W.first_fail) W.first_fail = r.first_failure_n;
        stop = true;
      }
      processed += r.checked;
      if (journaling) {
        std::lock_guard<std::mutex> lk(journal_mu);
        std::string jerr;
        gbj::Record rec{pending[b].first, pending[b].second, r.checked, r.phase2_fallbacks,
                        r.failures, r.failures ? r.first_failure_n : 0, r.max_minp};
        if (!journal.append(rec, &jerr)) {
          W.st = GB_EINVAL;
          W.err = jerr;
          stop = true;
          return;
        }
        if (stop_after && ++recorded >= stop_after && !stop.load()) {
          interrupted = true;
          stop = true;
        }
      }
      if (single_call) break;
    }
  };

  std::thread progress_thread;
  std::atomic<bool> progress_running{show_progress};
  if (show_progress) {
    progress_thread = std::thread([&]() {
      auto start_time = clk::now();
      auto print = [&]() {
        const uint64_t done = processed.load();
        const double el = std::chrono::duration<double>(clk::now() - start_time).count();
        const double pct = 100.0 * done / total;
        const uint64_t rate = el > 0 ? (uint64_t)(done / el) : 0;
        const uint64_t eta = rate ? (total - done) / rate : 0;
        std::cout << "\r[Progress] " << done << " / " << total << " (" << std::fixed
                  << std::setprecision(2) << pct << "%) "
                  << "| " << std::scientific << std::setprecision(2) << (double)rate
                  << " numbers/sec "
                  << "| ETA: " << eta << "s          " << std::flush;
        std::cout.unsetf(std::ios::floatfield);
        std::cout << std::setprecision(6);
      };
      // a line every 500 ms while running, and one when the work is done
      while (progress_running.load() && !stop.load() && processed.load() < total) {
        for (int i = 0; i < 50 && progress_running.load() && processed.load() < total; ++i)
          std::this_thread::sleep_for(std::chrono::milliseconds(10));
        print();
      }
      print();
      std::cout << "\r" << std::string(80, ' ') << "\r" << std::flush;
    });
  }
  std::vector<std::thread> workers;
  for (int g = 0; g < use_gpus; ++g) workers.emplace_back(run, g);
  for (auto& t : workers) t.join();
  const double total_ms = std::chrono::duration<double, std::milli>(clk::now() - t_main).count();
  if (show_progress) {
    progress_running = false;
    if (progress_thread.joinable()) progress_thread.join();
  }

  Worker sum = prior;
  bool sys_err = false;
  for (int g = 0; g < use_gpus; ++g) {
    if (w[g].st != GB_OK) {
      sys_err = true;
      std::cout << "[!] FATAL ERROR in GPU " << g << " Worker: " << gb_strerror(w[g].st)
                << (w[g].err.empty() ? "" : " (" + w[g].err + ")") << "\n";
    }
    sum.checked += w[g].checked;
    sum.fallbacks += w[g].fallbacks;
    sum.failures += w[g].failures;
    sum.launches += w[g].launches;
    sum.device_ms = std::max(sum.device_ms, w[g].device_ms);
    sum.max_minp = std::max(sum.max_minp, w[g].max_minp);
    if (w[g].first_fail && (!sum.first_fail || w[g].first_fail < sum.first_fail)) sum.first_fail = w[g].first_fail;
  }
  if (f_minp) std::fclose(f_minp);
  if (f_bits) {
    if (!bitw.finish()) sys_err = true;
    std::fclose(f_bits);
  }
  for (auto& x : w) gb_destroy(x.ctx);
  if (sys_err) {
    std::cerr << "\n[!] Program aborted due to internal hardware/CUDA errors.\n";
    return 1;
  }
  if (interrupted.load() && !sum.failures && processed.load() < total) {
    std::cout << "\nStopped after " << recorded.load() << " journal records ("
              << processed.load() << " of " << total << " numbers); rerun the same command to resume.\n";
    return 3;
  }
  if (json) {
    std::printf("{\"start\": %" PRIu64 ", \"limit\": %" PRIu64 ", \"checked\": %" PRIu64
                ", \"phase2_fallbacks\": %" PRIu64 ", \"failures\": %" PRIu64
                ", \"first_failure\": %" PRIu64 ", \"max_minp\": %" PRIu64
                ", \"wall_ms\": %.3f, \"device_ms\": %.3f, \"kernel_launches\": %" PRIu64 "}\n",
                START, LIMIT, sum.checked, sum.fallbacks, sum.failures, sum.first_fail,
                sum.max_minp, total_ms, sum.device_ms, sum.launches);
    std::fflush(stdout);
  }
  if (sum.failures) {
    std::cout << "\n[!] Goldbach FAILED at n = " << sum.first_fail << "\n";
    return 1;
  }
  std::cout << "\n--- Verification Complete ---\n";
  std::cout << "All even numbers from " << START << " up to " << LIMIT << " satisfy Goldbach. ✓\n";
  std::cout << "Total computation time : " << (total_ms / 1000.0) << " seconds\n";
  std::cout << "Phase 2 fallbacks      : " << sum.fallbacks << "\n";
  std::cout << "Max minimal p          : " << sum.max_minp << "\n";
  return 0;
}
