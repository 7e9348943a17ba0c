// PREPCUB (prepcub.f:54-109) run finding and the row tasks of the warp
// forward projections, for PJ 3Q / PJ 3F: host only and free of CUDA so a
// CPU test can compile it.
//
// The reference tests every voxel of an x line, t3*t3 + yy <= r in REAL,
// and makes the voxels that pass one run.  With t3 = i - LDPX that value
// only grows with |t3| (m*m is exact below 2^24 and rounding is monotone),
// so the voxels that pass are the interval |i - LDPX| <= m of the largest m
// that passes: found here from the square root and settled by the same float
// test, O(1) per line instead of O(nsam).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <vector>

namespace spi {

// emit(first x, last x, y index, z index) for every line that holds a run,
// 1-based, in PREPCUB's order (z outer, y inner)
template <class Emit>
inline void prepcub_lines(int nsam, int nrow, int nslice, float ri, int ldpx, int ldpy, int ldpz, Emit emit) {
  const float r = ri * ri;
  auto pass = [&](int m, float yy) {
    const float t3 = (float)m;
    return t3 * t3 + yy <= r;
  };
  const int mmax = std::max(ldpx - 1, nsam - ldpx);   // largest |t3| on the line
  for (int i1 = 1; i1 <= nslice; ++i1) {
    const float t = (float)(i1 - ldpz);
    const float xx = t * t;
    for (int i2 = 1; i2 <= nrow; ++i2) {
      const float t2 = (float)(i2 - ldpy);
      const float yy = t2 * t2 + xx;
      int m = (int)std::sqrt(std::max(0.0, (double)r - (double)yy));
      m = std::min(m, mmax);
      while (m < mmax && pass(m + 1, yy)) ++m;
      while (m >= 0 && !pass(m, yy)) --m;
      if (m < 0) continue;
      const int a = std::max(1, ldpx - m), b = std::min(nsam, ldpx + m);
      if (a <= b) emit(a, b, i2, i1);
    }
  }
}

// Row tasks of the warp forward projections (PJ 3Q's wpro_warp_kernel, PJ
// 3F's wpro_fbs_warp_kernel): the runs of every row y, in order of |z| (ties
// keep PREPCUB's order: -z first) or, with z_order, of z, cut into tasks of
// at most 32 runs of one row.  A task is {first run in rowruns, runs, x1, x2},
// x1..x2 the union of its runs' x ranges.  Run has i1, i2 (x range), y, z.
template <class Run>
inline void row_tasks(const std::vector<Run>& runs, bool z_order, std::vector<Run>& rowruns,
                      std::vector<std::array<int, 4>>& tasks) {
  std::vector<int> order(runs.size());
  for (size_t i = 0; i < runs.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
    const Run &a = runs[p], &b = runs[q];
    if (a.y != b.y) return a.y < b.y;
    return z_order ? a.z < b.z : std::abs(a.z) < std::abs(b.z);
  });
  rowruns.clear();
  tasks.clear();
  for (int i : order) rowruns.push_back(runs[i]);
  for (size_t i = 0; i < rowruns.size();) {
    size_t e = i + 1;
    while (e < rowruns.size() && e - i < 32 && rowruns[e].y == rowruns[i].y) ++e;
    int x1 = rowruns[i].i1, x2 = rowruns[i].i2;
    for (size_t q = i; q < e; ++q) {
      x1 = std::min(x1, rowruns[q].i1);
      x2 = std::max(x2, rowruns[q].i2);
    }
    tasks.push_back({(int)i, (int)(e - i), x1, x2});
    i = e;
  }
}

}  // namespace spi
