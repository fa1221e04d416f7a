// latency_hist.h -- fixed-size, log-bucketed latency histogram for the
// serving statistics: constant memory however long a server runs, and
// percentiles in a time that does not grow with the number of requests
// (a sorted copy of every latency would grow without bound and be sorted
// under the server's mutex).
//
// 64 buckets per octave from 2^-10 to 2^30 microseconds; a quantile is the
// geometric middle of the bucket holding the order statistic, clamped to
// the exact minimum and maximum, so it lies within 2^(1/128) - 1 = 0.55%
// of the exact value for every latency in that span; the lowest and the
// highest rank are the exact minimum and maximum.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace gb {

class LatencyHist {
 public:
  static constexpr int kPerOctave = 64;
  static constexpr int kMinLog2 = -10;
  static constexpr int kMaxLog2 = 30;
  static constexpr int kBuckets = (kMaxLog2 - kMinLog2) * kPerOctave;

  void add(double us) {
    if (!(us >= 0)) us = 0;  // NaN and negative values count as 0
    min_ = n_ ? std::min(min_, us) : us;
    max_ = n_ ? std::max(max_, us) : us;
    ++n_;
    sum_ += us;
    ++count_[index(us)];
  }

  void clear() {
    std::fill(count_.begin(), count_.end(), 0);
    n_ = 0;
    sum_ = min_ = max_ = 0;
  }

  uint64_t count() const { return n_; }
  double mean() const { return n_ ? sum_ / n_ : 0.0; }
  double max() const { return max_; }

  // The value of rank round(f (n - 1)) in ascending order (0-based).
  double quantile(double f) const {
    if (!n_) return 0.0;
    f = std::min(std::max(f, 0.0), 1.0);
    const uint64_t rank = (uint64_t)(f * (double)(n_ - 1) + 0.5);
    if (rank == 0) return min_;  // the ends are kept exactly
    if (rank >= n_ - 1) return max_;
    uint64_t c = 0;
    for (int b = 0; b < kBuckets; ++b) {
      c += count_[b];
      if (c > rank) return std::min(std::max(middle(b), min_), max_);
    }
    return max_;
  }

 private:
  static int index(double us) {
    if (us <= 0) return 0;
    const double i = std::floor((std::log2(us) - kMinLog2) * kPerOctave);
    return (int)std::min(std::max(i, 0.0), (double)(kBuckets - 1));
  }
  static double middle(int b) { return std::exp2(kMinLog2 + (b + 0.5) / kPerOctave); }

  std::vector<uint64_t> count_ = std::vector<uint64_t>(kBuckets, 0);
  uint64_t n_ = 0;
  double sum_ = 0, min_ = 0, max_ = 0;
};

}  // namespace gb
