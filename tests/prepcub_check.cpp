// Compares spider_b200/csrc/pj_runs.h (PREPCUB run finding by interval) with
// a voxel-by-voxel restatement of PREPCUB (prepcub.f:54-109): every voxel of
// every x line tested with t3*t3 + yy <= r in REAL, the first that passes
// opening the run and every later one that passes extending it.  Then checks
// the row tasks built from those runs, in both orders: the reordered runs
// are a permutation of the runs, grouped by row in the requested order, and
// the tasks tile them with at most 32 runs of one row each and the union of
// their x ranges.  Prints the number of cases and mismatches; exit status 1
// on any mismatch.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <tuple>
#include <vector>

#include "../spider_b200/csrc/pj_runs.h"

struct Run { int i1, i2, y, z; };

static void by_voxel(int nsam, int nrow, int nslice, float ri, int ldpx, int ldpy, int ldpz, std::vector<Run>& out) {
  const float r = ri * ri;
  for (int i1 = 1; i1 <= nslice; ++i1) {
    const float t = (float)(i1 - ldpz);
    const float xx = t * t;
    for (int i2 = 1; i2 <= nrow; ++i2) {
      const float t2 = (float)(i2 - ldpy);
      const float yy = t2 * t2 + xx;
      bool first = true;
      for (int i3 = 1; i3 <= nsam; ++i3) {
        const float t3 = (float)(i3 - ldpx);
        const float rc = t3 * t3 + yy;
        if (first) {
          if (rc > r) continue;
          first = false;
          out.push_back(Run{i3, i3, i2, i1});
        } else if (rc <= r) {
          out.back().i2 = i3;
        }
      }
    }
  }
}

static bool tasks_ok(const std::vector<Run>& runs, bool z_order) {
  std::vector<Run> rr;
  std::vector<std::array<int, 4>> tasks;
  spi::row_tasks(runs, z_order, rr, tasks);
  if (rr.size() != runs.size()) return false;
  auto key = [](const Run& r) { return std::make_tuple(r.y, r.z, r.i1, r.i2); };
  std::vector<std::tuple<int, int, int, int>> a, b;
  for (const Run& r : runs) a.push_back(key(r));
  for (const Run& r : rr) b.push_back(key(r));
  std::sort(a.begin(), a.end());
  std::sort(b.begin(), b.end());
  if (a != b) return false;
  for (size_t i = 1; i < rr.size(); ++i) {
    if (rr[i].y < rr[i - 1].y) return false;
    if (rr[i].y == rr[i - 1].y) {
      const int p = z_order ? rr[i - 1].z : std::abs(rr[i - 1].z), q = z_order ? rr[i].z : std::abs(rr[i].z);
      if (q < p) return false;
    }
  }
  size_t next = 0;
  for (const auto& t : tasks) {
    if ((size_t)t[0] != next || t[1] < 1 || t[1] > 32) return false;
    int x1 = rr[t[0]].i1, x2 = rr[t[0]].i2;
    for (int q = t[0]; q < t[0] + t[1]; ++q) {
      if (rr[q].y != rr[t[0]].y) return false;
      x1 = std::min(x1, rr[q].i1);
      x2 = std::max(x2, rr[q].i2);
    }
    if (x1 != t[2] || x2 != t[3]) return false;
    next += t[1];
  }
  return next == rr.size();
}

int main() {
  const int shapes[][3] = {{4, 4, 4},     {5, 7, 6},       {32, 32, 32},   {33, 31, 30},
                           {40, 36, 33},  {64, 64, 64},    {75, 75, 75},   {128, 128, 128},
                           {129, 64, 17}, {200, 192, 188}, {256, 256, 256}};
  const float radii[] = {0.5f, 1.0f, 1.5f, 3.0f, 5.0f, 14.0f, 16.0f, 30.9999f, 31.0f,
                         62.0f, 63.0f, 64.0f, 94.0f, 126.0f, 127.0f, 200.0f, 1000.0f};
  long long cases = 0, bad = 0;
  for (const auto& sh : shapes)
    for (float ri : radii)
      for (int shift = -1; shift <= 1; ++shift) {   // centres off the middle voxel too
        const int nx = sh[0], ny = sh[1], nz = sh[2];
        const int lx = nx / 2 + 1 + shift, ly = ny / 2 + 1, lz = nz / 2 + 1 - shift;
        std::vector<Run> a, b;
        by_voxel(nx, ny, nz, ri, lx, ly, lz, a);
        spi::prepcub_lines(nx, ny, nz, ri, lx, ly, lz, [&](int i1, int i2, int y, int z) { b.push_back(Run{i1, i2, y, z}); });
        ++cases;
        bool same = a.size() == b.size();
        for (size_t i = 0; same && i < a.size(); ++i)
          same = a[i].i1 == b[i].i1 && a[i].i2 == b[i].i2 && a[i].y == b[i].y && a[i].z == b[i].z;
        if (!same) {
          ++bad;
          std::printf("mismatch %dx%dx%d ri=%g shift=%d: %zu vs %zu runs\n", nx, ny, nz, ri, shift, a.size(), b.size());
        }
        for (bool zo : {false, true})
          if (!tasks_ok(b, zo)) {
            ++bad;
            std::printf("bad row tasks %dx%dx%d ri=%g shift=%d z_order=%d\n", nx, ny, nz, ri, shift, (int)zo);
          }
      }
  std::printf("%lld cases, %lld mismatches\n", cases, bad);
  return bad != 0;
}
