"""The serving statistics' latency histogram (goldbach-gpu_b200/csrc/host/
latency_hist.h), compiled on the host with g++ and checked against exact
order statistics: every quantile within 0.55% of the sorted value of the
same rank, exact count, mean, minimum and maximum, and a reset that starts
a new window."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HOST = os.path.join(ROOT, "goldbach-gpu_b200", "csrc", "host")

_HARNESS = r"""
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>
#include "latency_hist.h"

static int fails = 0;
static void check(bool ok, const char* what, double a, double b) {
  if (!ok && fails++ < 20) std::printf("FAIL %s: %.9g vs %.9g\n", what, a, b);
}

// rank round(f (n - 1)) of the ascending order, as the server reports it
static double exact(std::vector<double> v, double f) {
  std::sort(v.begin(), v.end());
  return v[(size_t)(f * (double)(v.size() - 1) + 0.5)];
}

static void compare(const std::vector<double>& v, const char* label) {
  gb::LatencyHist h;
  double sum = 0;
  for (double x : v) { h.add(x); sum += x; }
  check(h.count() == v.size(), label, (double)h.count(), (double)v.size());
  check(std::fabs(h.mean() - sum / v.size()) <= 1e-9 * (sum / v.size()) + 1e-12, label, h.mean(), sum / v.size());
  check(h.max() == *std::max_element(v.begin(), v.end()), label, h.max(), 0);
  const double fs[] = {0.0, 0.01, 0.25, 0.5, 0.9, 0.99, 0.999, 1.0};
  for (double f : fs) {
    const double e = exact(v, f), q = h.quantile(f);
    check(std::fabs(q - e) <= 0.0055 * e, label, q, e);
  }
}

int main() {
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  std::vector<double> v;
  for (int i = 0; i < 200000; ++i) v.push_back(std::exp2(-1.0 + 21.0 * u(rng)));  // 0.5 us .. 1 s
  compare(v, "log-uniform");
  v.clear();
  for (int i = 0; i < 100000; ++i) v.push_back(60.0 + 5.0 * u(rng) + (u(rng) < 0.01 ? 5000.0 * u(rng) : 0.0));
  compare(v, "tail");
  compare(std::vector<double>{137.25}, "single");
  compare(std::vector<double>{3.0, 3.0, 3.0, 4.0}, "ties");
  compare(std::vector<double>{1e-9, 5.0, 4e10}, "beyond the bucket span");  // clamped buckets, exact ends
  gb::LatencyHist h;
  h.add(10.0); h.add(20.0);
  h.clear();
  check(h.count() == 0 && h.quantile(0.5) == 0.0 && h.max() == 0.0, "clear", (double)h.count(), 0);
  h.add(7.5);
  check(h.quantile(0.99) == 7.5 && h.mean() == 7.5, "after clear", h.quantile(0.99), 7.5);
  std::printf(fails ? "failed\n" : "ok\n");
  return fails ? 1 : 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_latency_histogram_quantiles(tmp_path):
    src = tmp_path / "hist_test.cpp"
    exe = tmp_path / "hist_test"
    src.write_text(_HARNESS)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", HOST, "-o", str(exe), str(src)],
                   check=True, capture_output=True, text=True, timeout=120)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:]
