// Host-side splits of the streamed CG's work items (runs of node rows, in
// node order) into contiguous CTA ranges.  Plain C++ (no CUDA), so that the
// CPU tests compile it on its own.
#pragma once

#include <algorithm>
#include <vector>

namespace hoefem {

// G contiguous ranges of about equal weight: off[0..G], off[0] = 0,
// off[G] = w.size(); range g is items [off[g], off[g + 1]).
inline void split_weighted(const std::vector<long long>& w, int G, std::vector<int>& off) {
  long long total = 0;
  for (long long x : w) total += x;
  off.assign(G + 1, 0);
  long long cum = 0;
  int g = 1;
  for (size_t i = 0; i < w.size(); ++i) {
    cum += w[i];
    while (g < G && cum * (long long)G >= total * (long long)g) off[g++] = (int)(i + 1);
  }
  while (g <= G) off[g++] = (int)w.size();
}

// No constraint on a range beyond its two sums.
struct NoRangeFit {
  void start(int) {}
  bool add(int) { return true; }
};

// Ranges for work in two phases that each end at a grid barrier: item i
// costs a[i] in the first phase and b[i] in the second, so an iteration costs
// about max_g A_g + max_g B_g.  For caps T1 on A from 1.0 to 1.6 times the
// mean, the smallest cap T2 on B for which the greedy cut (each range
// extended while both sums stay within the caps; it needs the fewest ranges
// of any cut under these caps) fits in G ranges is found by bisection, and
// the pair with the smallest T1 + T2 is kept.  Then the cut also keeps every
// range within `fit` (start(i) opens a range at item i, add(i) extends it if
// the item fits), with both caps relaxed by 1% steps until the cut fits in G
// ranges (without `fit` if none does).  If the cut uses fewer than G ranges,
// the heaviest ranges are halved (a part of a range fits wherever the range
// does).  Returns false (off untouched) if no cap pair fits, for the caller's
// fallback.
template <class Fit>
bool split_two_phase(const std::vector<double>& a, const std::vector<double>& b, int G, std::vector<int>& off,
                     Fit& fit) {
  const size_t n = a.size();
  if (n == 0 || G <= 1) return false;
  double sa = 0.0, sb = 0.0, ma = 0.0, mb = 0.0;
  for (size_t i = 0; i < n; ++i) {
    sa += a[i];
    sb += b[i];
    ma = std::max(ma, a[i]);
    mb = std::max(mb, b[i]);
  }
  // the greedy cut under caps (T1, T2), with or without `fit`; stops counting
  // past G ranges unless the cut itself is wanted
  auto cut = [&](double T1, double T2, bool seg, std::vector<int>* out) {
    int g = 1;
    double x = 0.0, y = 0.0;
    if (out) out->assign(1, 0);
    if (seg) fit.start(0);
    for (size_t i = 0; i < n; ++i) {
      if (i > 0 && (x + a[i] > T1 || y + b[i] > T2 || (seg && !fit.add((int)i)))) {
        if (++g > G && !out) return g;
        if (out) out->push_back((int)i);
        if (seg) fit.start((int)i);
        x = y = 0.0;
      }
      x += a[i];
      y += b[i];
    }
    if (out) out->push_back((int)n);
    return g;
  };
  const double mA = sa / G, mB = sb / G;
  double best = -1.0, bT1 = 0.0, bT2 = 0.0;
  for (int k = 0; k <= 40; ++k) {
    const double T1 = std::max(ma, mA * (1.0 + 0.015 * k));
    double lo = std::max(mb, mB), hi = 4.0 * lo + sb / 16.0;
    if (cut(T1, hi, false, nullptr) > G) continue;
    for (int it = 0; it < 30; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (cut(T1, mid, false, nullptr) > G) lo = mid;
      else hi = mid;
    }
    if (best < 0.0 || T1 + hi < best) {
      best = T1 + hi;
      bT1 = T1;
      bT2 = hi;
    }
  }
  if (best < 0.0) return false;
  bool seg = false;
  for (int k = 0; k <= 30; ++k) {
    const double f = 1.0 + 0.01 * k;
    if (cut(bT1 * f, bT2 * f, true, nullptr) <= G) {
      bT1 *= f;
      bT2 *= f;
      seg = true;
      break;
    }
  }
  cut(bT1, bT2, seg, &off);
  while ((int)off.size() - 1 < G) {
    int r = -1;
    double worst = -1.0;
    for (size_t q = 0; q + 1 < off.size(); ++q) {
      if (off[q + 1] - off[q] < 2) continue;
      double x = 0.0, y = 0.0;
      for (int i = off[q]; i < off[q + 1]; ++i) {
        x += a[i];
        y += b[i];
      }
      const double wq = std::max(x / bT1, y / bT2);
      if (wq > worst) {
        worst = wq;
        r = (int)q;
      }
    }
    if (r < 0) break;
    double tot = 0.0;
    for (int i = off[r]; i < off[r + 1]; ++i) tot += a[i] / bT1 + b[i] / bT2;
    double c = 0.0;
    int at = off[r] + 1;
    for (int i = off[r]; i < off[r + 1] - 1; ++i) {
      c += a[i] / bT1 + b[i] / bT2;
      at = i + 1;
      if (c >= 0.5 * tot) break;
    }
    off.insert(off.begin() + r + 1, at);
  }
  while ((int)off.size() < G + 1) off.push_back((int)n);
  return true;
}

}  // namespace hoefem
