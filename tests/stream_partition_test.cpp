// Properties of the streamed CG's CTA range splits (csrc/stream_partition.h),
// on seeded random item weights; prints "ok" or the first failure.
#include <cstdio>
#include <random>
#include <vector>

#include "stream_partition.h"

using hoefem::split_two_phase;
using hoefem::split_weighted;

// a range fits while the sum of c over its items stays within cap
struct CapFit {
  const std::vector<int>* c;
  int cap = 0, cur = 0;
  void start(int i) { cur = (*c)[i]; }
  bool add(int i) {
    cur += (*c)[i];
    return cur <= cap;
  }
};

// off[0..G] from 0 to n, non-decreasing; `full`: no empty range when n >= G
static bool valid(const std::vector<int>& off, int n, int G, bool full) {
  if ((int)off.size() != G + 1 || off[0] != 0 || off[G] != n) return false;
  for (int g = 0; g < G; ++g)
    if (off[g] > off[g + 1] || (full && n >= G && off[g] == off[g + 1])) return false;
  return true;
}

static double cost(const std::vector<int>& off, const std::vector<double>& a, const std::vector<double>& b) {
  double ma = 0.0, mb = 0.0;
  for (size_t g = 0; g + 1 < off.size(); ++g) {
    double x = 0.0, y = 0.0;
    for (int i = off[g]; i < off[g + 1]; ++i) {
      x += a[i];
      y += b[i];
    }
    ma = ma > x ? ma : x;
    mb = mb > y ? mb : y;
  }
  return ma + mb;
}

int main() {
  std::mt19937 rng(7);
  for (int trial = 0; trial < 400; ++trial) {
    const int n = 1 + rng() % 6000, G = 1 + rng() % 200;
    std::vector<double> a(n), b(n);
    std::vector<long long> w(n);
    std::vector<int> c(n);
    for (int i = 0; i < n; ++i) {
      a[i] = 1000 + rng() % 13000;
      b[i] = (rng() % 3 == 0) ? 0.0 : (double)(rng() % 20000);
      w[i] = (long long)(a[i] + b[i]);
      c[i] = 1 + rng() % 100;
    }
    std::vector<int> ow;
    split_weighted(w, G, ow);
    if (!valid(ow, n, G, false)) {
      std::printf("weighted split invalid: trial %d n %d G %d\n", trial, n, G);
      return 1;
    }
    hoefem::NoRangeFit none;
    std::vector<int> o1;
    if (split_two_phase(a, b, G, o1, none)) {
      if (!valid(o1, n, G, true)) {
        std::printf("two-phase split invalid: trial %d n %d G %d\n", trial, n, G);
        return 1;
      }
      // never much worse than equal summed weights (the cap grid is 1.5% of the mean)
      const double mean = [&] {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += a[i];
        return s / G;
      }();
      if (cost(o1, a, b) > cost(ow, a, b) + 0.02 * mean + 1e-9) {
        std::printf("two-phase cost %.0f above weighted %.0f: trial %d\n", cost(o1, a, b), cost(ow, a, b), trial);
        return 1;
      }
      std::vector<int> o1b;
      split_two_phase(a, b, G, o1b, none);
      if (o1b != o1) {
        std::printf("not deterministic: trial %d\n", trial);
        return 1;
      }
    }
    // with a per-range bound: every range keeps it whenever the cut could
    CapFit fit{&c, 0, 0};
    long long csum = 0;
    for (int x : c) csum += x;
    fit.cap = (int)(1.5 * (double)csum / G) + 100;
    std::vector<int> o2;
    if (split_two_phase(a, b, G, o2, fit)) {
      if (!valid(o2, n, G, true)) {
        std::printf("bounded split invalid: trial %d n %d G %d\n", trial, n, G);
        return 1;
      }
      int over = 0;
      for (int g = 0; g < G; ++g) {
        long long s = 0;
        for (int i = o2[g]; i < o2[g + 1]; ++i) s += c[i];
        over += s > fit.cap;
      }
      // the bound binds unless even relaxed caps could not meet it
      CapFit probe{&c, fit.cap, 0};
      int need = 1;
      probe.start(0);
      for (int i = 1; i < n; ++i)
        if (!probe.add(i)) {
          ++need;
          probe.start(i);
        }
      if (over && need <= G / 2) {
        std::printf("range over the bound although %d ranges suffice: trial %d\n", need, trial);
        return 1;
      }
    }
  }
  std::printf("ok\n");
  return 0;
}
