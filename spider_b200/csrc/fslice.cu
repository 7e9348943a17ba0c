// FourierSlice: the central-slice operator pair on ONELINE's geometry.
//
// SPIDER's BP 3F inserts each image's spectrum into the 3D Fourier grid as a
// central slice with Kaiser-Bessel weights (ONELINE, oneline.f:38-200) and has
// no extraction with the same kernel.  This file adds the pair a
// differentiable reconstruction needs (no counterpart in the reference):
//
//   E   (forward, extraction):  grid X -> slices T, the exact real-linear
//       adjoint of the insertion below;
//   E^T (adjoint, insertion):   slices T -> grid X, ONELINE's X += BTQ * W
//       with the weight grid dropped;
//   E^T E + lam I (normal):     one fused pass that gathers each pixel's taps
//       and scatters the sum back over the same taps.
//
// Grid: complex float2 [2nx][2nx][nx+1] (i fastest, Fortran X(0:NX,N,N)).
// Slices: float2 [nslice][2nx][nx+1] in the layout and sign of the staged
// spectra the back-projection inserts (cuFFT R2C of the padded, shifted
// image; ONELINE's BI is its conjugate).  Every tap -- voxel, table weight,
// Hermitian flip (x < 0), reflected point (oneline.f:118-150) -- is computed
// exactly as insert_x4_kernel computes it, four lanes per pixel over the
// nonzero window of the table.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/spider_b200.h"
#include "ctx.h"

namespace spi {

struct FsDesc {
  float dm[6];  // DM(1:6) of the slice (CANG, cang.f:44-81)
  int img;      // slice index
  int cols;     // order of the insertion and normal kernels: 0 row by row, 1 by half columns
};
static_assert(sizeof(FsDesc) == 32, "slice descriptor is 32 bytes");

__device__ __forceinline__ int fs_nint_pos(float v) {  // Fortran NINT, v >= 0
  const float f = floorf(v);
  return (int)f + ((__fsub_rn(v, f) >= 0.5f) ? 1 : 0);
}
__device__ __forceinline__ float fs_tap(const float* tab, float v, int k, float fltb) {
  return tab[fs_nint_pos(__fmul_rn(fabsf(__fsub_rn(v, (float)k)), fltb))];
}

// Line r (0 <= r < N) of a slice: row J = r - NX + 1 (pixels consecutive in
// I) or, for a slice marked cols, half of column I = r / 2 (pixels
// consecutive in J; J >= 0 for even r, J < 0 for odd r).  Pixel k of the line
// is (i0 + di k, j0 + dj k), k < cnt: the pixels of the line inside the half
// disc of oneline.f's loops, so every pixel of the slice lies on exactly one
// line in either order.  The host marks slices as the back-projection does
// (bp.cu, insert_line_x4): eight pixels stepping along z scatter into eight
// grid planes 2 MB apart at 256^3.  Only the insertions E^T follow the mark
// (use_cols): at 256^3 with 8,192 slices it took E^T from 158.6 to 111.7 ms,
// while the fused normal operators, which gather before they scatter, were
// 2% slower with it (0.363 against 0.356 s per CG iteration in FP64).
struct FsLine {
  int i0, j0, di, dj, cnt;
};
__device__ __forceinline__ int fs_isqrt_below(int rem) {   // the largest m >= 0 with m * m < rem (rem > 0)
  // approximate square root (no IEEE slow path); the two loops make m exact
  float f;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(f) : "f"((float)(rem - 1)));
  int m = (int)f;
  while (m > 0 && m * m >= rem) --m;
  while ((m + 1) * (m + 1) < rem) ++m;
  return m;
}
__device__ __forceinline__ FsLine fs_line(const FsDesc& sd, int r, int nx, bool use_cols) {
  const int NN4 = nx * nx;
  FsLine l;
  if (!(use_cols && sd.cols)) {
    l.j0 = r - nx + 1; l.i0 = 0; l.di = 1; l.dj = 0;
    l.cnt = (l.j0 * l.j0 < NN4) ? fs_isqrt_below(NN4 - l.j0 * l.j0) + 1 : 0;
  } else {
    l.i0 = r >> 1; l.di = 0;
    const int jm = fs_isqrt_below(NN4 - l.i0 * l.i0);
    if (r & 1) { l.j0 = -1; l.dj = -1; l.cnt = l.i0 == 0 ? 0 : jm; }
    else { l.j0 = 0; l.dj = 1; l.cnt = jm + 1; }
  }
  return l;
}

// The tap window of pixel (I, J) for lane q of its four-lane group (lanes
// gl..gl+3 share the pixel): x tap xs + q, the 4 x 4 (y, z) windows starting
// at ys, zs.  Called by all 32 lanes (the y/z weights are exchanged by
// shuffles).  `ok` is false when the pixel has no taps.
struct FsWin {
  bool ok, flipped;
  int xs, ys, zs;
  float tx;
  float ty[4], tz[4];
};

// LS: lanes per x tap in the pixel's lane group (the y/z weight of window
// position l lives in lane gl + l * LS).
template <int LS = 1>
__device__ __forceinline__ void fs_window(const FsDesc& sd, int I, int J, int nx, const float* tab, float fltb,
                                          int q, int gl, FsWin& w) {
  const int N = 2 * nx, N2 = nx, LN2 = 2, NN4 = N * N / 4;
  const float fN = (float)N;
  bool ok = I <= N2 && (I * I + J * J) < NN4 && !(I == 0 && J < 0);
  const float fI = (float)I, fJ = (float)J;
  float xnew = __fadd_rn(__fmul_rn(fI, sd.dm[0]), __fmul_rn(fJ, sd.dm[3]));
  float ynew = __fadd_rn(__fmul_rn(fI, sd.dm[1]), __fmul_rn(fJ, sd.dm[4]));
  float znew = __fadd_rn(__fmul_rn(fI, sd.dm[2]), __fmul_rn(fJ, sd.dm[5]));
  w.flipped = xnew < 0.0f;
  if (w.flipped) {
    xnew = -xnew; ynew = -ynew; znew = -znew;
  }
  const int ixn = __float2int_rz(__fadd_rn(__fadd_rn(xnew, 0.5f), fN)) - N;
  const int iyn = __float2int_rz(__fadd_rn(__fadd_rn(ynew, 0.5f), fN)) - N;
  const int izn = __float2int_rz(__fadd_rn(__fadd_rn(znew, 0.5f), fN)) - N;
  ok = ok && ixn <= (N2 - LN2 - 1) && iyn >= (-N2 + 2 + LN2) && iyn <= (N2 - LN2 - 1) && izn >= (-N2 + 2 + LN2) &&
       izn <= (N2 - LN2 - 1);
  if (!ok) { xnew = ynew = znew = 0.0f; }   // keeps the lookups below in range; no taps follow
  const int ix0 = ok ? ixn : 0, iy0 = ok ? iyn : 0, iz0 = ok ? izn : 0;
  w.xs = fs_tap(tab, xnew, ix0 - 2, fltb) != 0.0f ? ix0 - 2 : ix0 - 1;
  w.ys = fs_tap(tab, ynew, iy0 - 2, fltb) != 0.0f ? iy0 - 2 : iy0 - 1;
  w.zs = fs_tap(tab, znew, iz0 - 2, fltb) != 0.0f ? iz0 - 2 : iz0 - 1;
  w.tx = fs_tap(tab, xnew, w.xs + q, fltb);
  const float tyq = fs_tap(tab, ynew, w.ys + q, fltb);
  const float tzq = fs_tap(tab, znew, w.zs + q, fltb);
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    w.ty[l] = __shfl_sync(0xffffffffu, tyq, gl + l * LS);
    w.tz[l] = __shfl_sync(0xffffffffu, tzq, gl + l * LS);
  }
  w.ok = ok && w.tx != 0.0f;
}

// Grid index of tap (q, ly, lz) of window w: main tap (ixp, iyp, izp), or
// for ixp < 0 the reflected point (-ixp, -iyp, -izp) (refl = true).
__device__ __forceinline__ size_t fs_voxel(const FsWin& w, int q, int ly, int lz, int nx, bool& refl) {
  const int N = 2 * nx;
  const int ixp = w.xs + q, iyp = w.ys + ly, izp = w.zs + lz;
  const bool r = ixp < 0;
  const int ixa = r ? -ixp : ixp;
  const int iya = r ? ((iyp > 0) ? N - iyp : -iyp) : ((iyp >= 0) ? iyp : N + iyp);
  const int iza = r ? ((izp > 0) ? N - izp : -izp) : ((izp >= 0) ? izp : N + izp);
  refl = r;
  return ((size_t)iza * N + iya) * (size_t)(nx + 1) + ixa;
}

__device__ __forceinline__ float2 fs_cmul(float2 v, float wg, bool conj_) {
  return make_float2(__fmul_rn(v.x, wg), conj_ ? -__fmul_rn(v.y, wg) : __fmul_rn(v.y, wg));
}

// Sum over the lane's 16 taps of wg * X (conj(X) at reflected points)
__device__ __forceinline__ float2 fs_gather(const float2* __restrict__ X, const FsWin& w, int q, int nx) {
  float2 acc = make_float2(0.0f, 0.0f);
  if (!w.ok) return acc;
#pragma unroll
  for (int lz = 0; lz < 4; ++lz) {
    if (w.tz[lz] == 0.0f) continue;
#pragma unroll
    for (int ly = 0; ly < 4; ++ly) {
      const float tyz = __fmul_rn(w.ty[ly], w.tz[lz]);
      if (tyz == 0.0f) continue;
      const float wg = __fmul_rn(w.tx, tyz);
      if (wg == 0.0f) continue;
      bool refl;
      const float2 v = __ldg(X + fs_voxel(w, q, ly, lz, nx, refl));
      const float2 t = fs_cmul(v, wg, refl);
      acc.x = __fadd_rn(acc.x, t.x);
      acc.y = __fadd_rn(acc.y, t.y);
    }
  }
  return acc;
}

// X[v] += wg * b over the lane's taps (conj(b) at reflected points)
__device__ __forceinline__ void fs_scatter(float2* __restrict__ X, const FsWin& w, int q, int nx, float2 b) {
  if (!w.ok) return;
#pragma unroll
  for (int lz = 0; lz < 4; ++lz) {
    if (w.tz[lz] == 0.0f) continue;
#pragma unroll
    for (int ly = 0; ly < 4; ++ly) {
      const float tyz = __fmul_rn(w.ty[ly], w.tz[lz]);
      if (tyz == 0.0f) continue;
      const float wg = __fmul_rn(w.tx, tyz);
      if (wg == 0.0f) continue;
      bool refl;
      const size_t v = fs_voxel(w, q, ly, lz, nx, refl);
      atomicAdd(X + v, fs_cmul(b, wg, refl));
    }
  }
}

__device__ __forceinline__ float2 group_sum4(float2 v) {   // sum over the four lanes of a pixel, in every lane
  v.x = __fadd_rn(v.x, __shfl_xor_sync(0xffffffffu, v.x, 1));
  v.y = __fadd_rn(v.y, __shfl_xor_sync(0xffffffffu, v.y, 1));
  v.x = __fadd_rn(v.x, __shfl_xor_sync(0xffffffffu, v.x, 2));
  v.y = __fadd_rn(v.y, __shfl_xor_sync(0xffffffffu, v.y, 2));
  return v;
}

// MODE 0: extraction E (X -> T), 1: insertion E^T (T -> X), 2: normal E^T E
// (P -> Q, Q pre-set to lam * P).  A warp takes one row J of one slice
// (rows handed out in slice-major order by a grid stride), eight pixels at a
// time.
template <int MODE>
__global__ void __launch_bounds__(256) fs_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                 const FsDesc* __restrict__ slices, int nslices, int nx,
                                                 const float* __restrict__ kbtab, float fltb) {
  extern __shared__ float tab[];
  for (int i = threadIdx.x; i < 5000; i += blockDim.x) tab[i] = kbtab[i];
  __syncthreads();
  const int N = 2 * nx, NN4 = N * N / 4;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3, gl = lane & ~3;
  const long long nitems = (long long)nslices * N;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  const size_t rowlen = (size_t)(nx + 1);
  const size_t plane = (size_t)N * rowlen;
  for (long long item = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < nitems;
       item += warps) {
    const int s = (int)(item / N);
    const FsDesc sd = slices[s];
    if (MODE == 0) {
      // rows only: every pixel of the row is written, zero outside the disc
      const int J = (int)(item % N) - nx + 1;
      const int JP = (J >= 0) ? J : N + J;
      const size_t srow = (size_t)sd.img * plane + (size_t)JP * rowlen;
      int I0 = 0;
      for (; I0 <= nx && I0 * I0 + J * J < NN4; I0 += 8) {   // warp-uniform
        const int I = I0 + g;
        FsWin w;
        fs_window(sd, I, J, nx, tab, fltb, q, gl, w);
        const float2 acc = group_sum4(fs_gather(in, w, q, nx));
        // BI_adj = acc (conj'ed for a flipped pixel); T = conj(BI_adj)
        if (q == 0 && I <= nx) {
          float2 t = make_float2(0.0f, 0.0f);
          if (I * I + J * J < NN4 && !(I == 0 && J < 0)) t = w.flipped ? acc : make_float2(acc.x, -acc.y);
          out[srow + I] = t;
        }
      }
      for (int I = I0 + lane; I <= nx; I += 32) out[srow + I] = make_float2(0.0f, 0.0f);
    } else {
      const FsLine ln = fs_line(sd, (int)(item % N), nx, MODE == 1);
      for (int k0 = 0; k0 < ln.cnt; k0 += 8) {   // warp-uniform
        const int k = k0 + g;
        const int I = ln.i0 + ln.di * k, J = ln.j0 + ln.dj * k;
        FsWin w;
        fs_window(sd, I, J, nx, tab, fltb, q, gl, w);
        if (MODE == 1) {
          // BTQ = BI = conj(T), or conj(BI) = T for a flipped pixel
          float2 b = make_float2(0.0f, 0.0f);
          if (w.ok) {
            const int JP = (J >= 0) ? J : N + J;
            const float2 t = in[(size_t)sd.img * plane + (size_t)JP * rowlen + I];
            b = w.flipped ? t : make_float2(t.x, -t.y);
          }
          fs_scatter(out, w, q, nx, b);
        } else {
          // extraction then insertion of the same pixel: the flips cancel
          const float2 sum = group_sum4(fs_gather(in, w, q, nx));
          fs_scatter(out, w, q, nx, sum);
        }
      }
    }
  }
}

// The normal operator in FP64: the same taps and FP32 table weights, with the
// grids, the pixel sums and the scatter (FP64 atomics) in double precision.
// Late CG iterations apply E^T E to directions whose image is much smaller
// than ||E^T E|| ||p||; FP32 sums would lose that many digits there.
__device__ __forceinline__ double2 fs_gather64(const double2* __restrict__ X, const FsWin& w, int q, int nx) {
  double2 acc = make_double2(0.0, 0.0);
  if (!w.ok) return acc;
#pragma unroll
  for (int lz = 0; lz < 4; ++lz) {
    if (w.tz[lz] == 0.0f) continue;
#pragma unroll
    for (int ly = 0; ly < 4; ++ly) {
      const float tyz = __fmul_rn(w.ty[ly], w.tz[lz]);
      if (tyz == 0.0f) continue;
      const float wg = __fmul_rn(w.tx, tyz);
      if (wg == 0.0f) continue;
      bool refl;
      const double2 v = X[fs_voxel(w, q, ly, lz, nx, refl)];
      const double d = (double)wg;
      acc.x = __dadd_rn(acc.x, __dmul_rn(v.x, d));
      acc.y = refl ? __dsub_rn(acc.y, __dmul_rn(v.y, d)) : __dadd_rn(acc.y, __dmul_rn(v.y, d));
    }
  }
  return acc;
}

__device__ __forceinline__ void fs_scatter64(double2* __restrict__ X, const FsWin& w, int q, int nx, double2 b) {
  if (!w.ok) return;
#pragma unroll
  for (int lz = 0; lz < 4; ++lz) {
    if (w.tz[lz] == 0.0f) continue;
#pragma unroll
    for (int ly = 0; ly < 4; ++ly) {
      const float tyz = __fmul_rn(w.ty[ly], w.tz[lz]);
      if (tyz == 0.0f) continue;
      const float wg = __fmul_rn(w.tx, tyz);
      if (wg == 0.0f) continue;
      bool refl;
      double* v = reinterpret_cast<double*>(X + fs_voxel(w, q, ly, lz, nx, refl));
      const double d = (double)wg;
      atomicAdd(v, __dmul_rn(b.x, d));
      atomicAdd(v + 1, refl ? -__dmul_rn(b.y, d) : __dmul_rn(b.y, d));
    }
  }
}

// NORMAL: E^T E of an FP64 grid; else E^T of FP32 slices (`sl_in`) into an
// FP64 grid.
// In the normal operator the lane's 16 voxel offsets come from four plane and
// four row terms computed once per pixel (32-bit: a grid has < 2^32 voxels up
// to nx = 512) and serve both the gather and the scatter (measured 2-3%
// faster than computing each tap's index twice, 48 instead of 57 registers).
template <bool NORMAL>
__global__ void __launch_bounds__(256) fs_normal64_kernel(const double2* __restrict__ in, const float2* __restrict__ sl_in,
                                                          double2* __restrict__ out,
                                                          const FsDesc* __restrict__ slices, int nslices, int nx,
                                                          const float* __restrict__ kbtab, float fltb) {
  extern __shared__ float tab[];
  for (int i = threadIdx.x; i < 5000; i += blockDim.x) tab[i] = kbtab[i];
  __syncthreads();
  const int N = 2 * nx;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3, gl = lane & ~3;
  const long long nitems = (long long)nslices * N;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long item = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < nitems;
       item += warps) {
    const int s = (int)(item / N);
    const FsDesc sd = slices[s];
    const FsLine ln = fs_line(sd, (int)(item % N), nx, !NORMAL);
    for (int k0 = 0; k0 < ln.cnt; k0 += 8) {   // warp-uniform
      const int k = k0 + g;
      const int I = ln.i0 + ln.di * k, J = ln.j0 + ln.dj * k;
      FsWin w;
      fs_window(sd, I, J, nx, tab, fltb, q, gl, w);
      double2 v;
      if (NORMAL) {
        const int ixp = w.xs + q;
        const bool refl = ixp < 0;
        const unsigned ixa = (unsigned)(refl ? -ixp : ixp);
        unsigned zoff[4], yoff[4];
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const int izp = w.zs + l, iyp = w.ys + l;
          const int iza = refl ? ((izp > 0) ? N - izp : -izp) : ((izp >= 0) ? izp : N + izp);
          const int iya = refl ? ((iyp > 0) ? N - iyp : -iyp) : ((iyp >= 0) ? iyp : N + iyp);
          zoff[l] = (unsigned)iza * (unsigned)N * (unsigned)(nx + 1);
          yoff[l] = (unsigned)iya * (unsigned)(nx + 1) + ixa;
        }
        v = make_double2(0.0, 0.0);
        if (w.ok) {
#pragma unroll
          for (int lz = 0; lz < 4; ++lz) {
            if (w.tz[lz] == 0.0f) continue;
#pragma unroll
            for (int ly = 0; ly < 4; ++ly) {
              const float tyz = __fmul_rn(w.ty[ly], w.tz[lz]);
              if (tyz == 0.0f) continue;
              const float wg = __fmul_rn(w.tx, tyz);
              if (wg == 0.0f) continue;
              const double2 x = in[zoff[lz] + yoff[ly]];
              const double d = (double)wg;
              v.x = __dadd_rn(v.x, __dmul_rn(x.x, d));
              v.y = refl ? __dsub_rn(v.y, __dmul_rn(x.y, d)) : __dadd_rn(v.y, __dmul_rn(x.y, d));
            }
          }
        }
        v.x = __dadd_rn(v.x, __shfl_xor_sync(0xffffffffu, v.x, 1));
        v.y = __dadd_rn(v.y, __shfl_xor_sync(0xffffffffu, v.y, 1));
        v.x = __dadd_rn(v.x, __shfl_xor_sync(0xffffffffu, v.x, 2));
        v.y = __dadd_rn(v.y, __shfl_xor_sync(0xffffffffu, v.y, 2));
        if (!w.ok) continue;
#pragma unroll
        for (int lz = 0; lz < 4; ++lz) {
          if (w.tz[lz] == 0.0f) continue;
#pragma unroll
          for (int ly = 0; ly < 4; ++ly) {
            const float tyz = __fmul_rn(w.ty[ly], w.tz[lz]);
            if (tyz == 0.0f) continue;
            const float wg = __fmul_rn(w.tx, tyz);
            if (wg == 0.0f) continue;
            double* o = reinterpret_cast<double*>(out + (zoff[lz] + yoff[ly]));
            const double d = (double)wg;
            atomicAdd(o, __dmul_rn(v.x, d));
            atomicAdd(o + 1, refl ? -__dmul_rn(v.y, d) : __dmul_rn(v.y, d));
          }
        }
        continue;
      } else {   // BTQ = BI = conj(T), or T for a flipped pixel
        v = make_double2(0.0, 0.0);
        if (w.ok) {
          const int JP = (J >= 0) ? J : N + J;
          const float2 t = sl_in[((size_t)sd.img * N + JP) * (size_t)(nx + 1) + I];
          v = make_double2((double)t.x, w.flipped ? (double)t.y : -(double)t.y);
        }
      }
      fs_scatter64(out, w, q, nx, v);
    }
  }
}

// E^T into an FP64 grid with eight lanes per pixel: lane 8g + 2q + h takes x
// tap q of pixel g and the real (h = 0) or imaginary (h = 1) part.  There is
// no 16-byte FP64 reduction, so in the four-lane form every tap's complex add
// is two 8-byte reductions from one lane, the real parts of a pixel's four
// taps (16 bytes apart) in one instruction and the imaginary parts in
// another; here one instruction adds both parts of four consecutive voxels
// (64 contiguous bytes), half the L2 reduction requests and sectors.
// Measured with 10,000 and 8,192 slices: 71.8 against 84.0 ms at 128^3,
// 239 against 291 ms at 256^3.  The fused normal operator keeps four lanes: its
// gather, with every weight and voxel index computed by two lanes here, made
// it 1.7x slower in this form (0.159 against 0.0945 s per CG iteration), and
// a four-lane gather followed by this scatter in two passes (the windows and
// pixel sums moved across lanes by shuffles) 1.3x slower (0.123 s).
__global__ void __launch_bounds__(256) fs_insert64w_kernel(const float2* __restrict__ sl_in, double* __restrict__ out,
                                                           const FsDesc* __restrict__ slices, int nslices, int nx,
                                                           const float* __restrict__ kbtab, float fltb) {
  extern __shared__ float tab[];
  for (int i = threadIdx.x; i < 5000; i += blockDim.x) tab[i] = kbtab[i];
  __syncthreads();
  const int N = 2 * nx;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 3, q = (lane >> 1) & 3, h = lane & 1, gl = lane & ~7;
  const long long nitems = (long long)nslices * N;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long item = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < nitems;
       item += warps) {
    const int s = (int)(item / N);
    const FsDesc sd = slices[s];
    const FsLine ln = fs_line(sd, (int)(item % N), nx, true);
    for (int k0 = 0; k0 < ln.cnt; k0 += 4) {   // warp-uniform
      const int k = k0 + g;
      const int I = ln.i0 + ln.di * k, J = ln.j0 + ln.dj * k;
      FsWin w;
      fs_window<2>(sd, I, J, nx, tab, fltb, q, gl, w);
      if (!w.ok) continue;
      // BTQ = BI = conj(T), or T for a flipped pixel
      const int JP = (J >= 0) ? J : N + J;
      const float2 t = sl_in[((size_t)sd.img * N + JP) * (size_t)(nx + 1) + I];
      const double v = h ? (w.flipped ? (double)t.y : -(double)t.y) : (double)t.x;
#pragma unroll
      for (int lz = 0; lz < 4; ++lz) {
        if (w.tz[lz] == 0.0f) continue;
#pragma unroll
        for (int ly = 0; ly < 4; ++ly) {
          const float tyz = __fmul_rn(w.ty[ly], w.tz[lz]);
          if (tyz == 0.0f) continue;
          const float wg = __fmul_rn(w.tx, tyz);
          if (wg == 0.0f) continue;
          bool refl;
          const size_t vx = fs_voxel(w, q, ly, lz, nx, refl);
          const double tw = __dmul_rn(v, (double)wg);
          atomicAdd(out + 2 * vx + h, (h && refl) ? -tw : tw);
        }
      }
    }
  }
}

// Extraction E on an FP64 grid into FP64 slices (FP64 sums of the same taps):
// an exact reference of the FP32 extraction for gradient checks.
__global__ void __launch_bounds__(256) fs_extract64_kernel(const double2* __restrict__ in, double2* __restrict__ out,
                                                           const FsDesc* __restrict__ slices, int nslices, int nx,
                                                           const float* __restrict__ kbtab, float fltb) {
  extern __shared__ float tab[];
  for (int i = threadIdx.x; i < 5000; i += blockDim.x) tab[i] = kbtab[i];
  __syncthreads();
  const int N = 2 * nx, NN4 = N * N / 4;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3, gl = lane & ~3;
  const long long nitems = (long long)nslices * N;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long item = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < nitems;
       item += warps) {
    const int s = (int)(item / N);
    const int J = (int)(item % N) - nx + 1;
    const FsDesc sd = slices[s];
    const int JP = (J >= 0) ? J : N + J;
    const size_t srow = ((size_t)sd.img * N + JP) * (size_t)(nx + 1);
    int I0 = 0;
    for (; I0 <= nx && I0 * I0 + J * J < NN4; I0 += 8) {   // warp-uniform
      const int I = I0 + g;
      FsWin w;
      fs_window(sd, I, J, nx, tab, fltb, q, gl, w);
      double2 v = fs_gather64(in, w, q, nx);
      v.x = __dadd_rn(v.x, __shfl_xor_sync(0xffffffffu, v.x, 1));
      v.y = __dadd_rn(v.y, __shfl_xor_sync(0xffffffffu, v.y, 1));
      v.x = __dadd_rn(v.x, __shfl_xor_sync(0xffffffffu, v.x, 2));
      v.y = __dadd_rn(v.y, __shfl_xor_sync(0xffffffffu, v.y, 2));
      if (q == 0 && I <= nx) {
        double2 t = make_double2(0.0, 0.0);
        if (I * I + J * J < NN4 && !(I == 0 && J < 0)) t = w.flipped ? v : make_double2(v.x, -v.y);
        out[srow + I] = t;
      }
    }
    for (int I = I0 + lane; I <= nx; I += 32) out[srow + I] = make_double2(0.0, 0.0);
  }
}

__global__ void fs_scale64_kernel(const double2* __restrict__ p, double lam, double2* __restrict__ q, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = p[i];
    q[i] = make_double2(__dmul_rn(lam, v.x), __dmul_rn(lam, v.y));
  }
}

__global__ void fs_scale_kernel(const float2* __restrict__ p, float lam, float2* __restrict__ q, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float2 v = p[i];
    q[i] = make_float2(__fmul_rn(lam, v.x), __fmul_rn(lam, v.y));
  }
}

// Volume of a grid of spectrum coefficients.  The grid models the volume's
// spectrum as V(k) = sum_v X_v K(k - v) (E samples exactly that), so the
// volume is the inverse transform of X times the transform of the separable
// Kaiser-Bessel kernel, |WKB| of WINDKB2A (bp32f.f:964-1005), where the
// direct gridding of BP 3F divides by it.  Plane i = 0 holds each voxel and
// its Friedel mate; its Hermitian part (X(0,j,k) + conj X(0,-j,-k)) / 2 is
// used.  Then the phase (-1)^(i+j+k), SPIDER's inverse sign (conjugate) and a
// C2R transform; the centred nx^3 is cropped, scaled by 1/n^3 and multiplied
// by |WKB(LR)| inside radius nx/2 and set to zero outside.
__global__ void fs_vol_prep_kernel(const float2* __restrict__ X, float2* __restrict__ out, int nx) {
  const int N = 2 * nx;
  const size_t h = (size_t)(nx + 1);
  const size_t nvox = h * N * N;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nvox; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % h);
    const size_t t = q / h;
    const int j = (int)(t % N), k = (int)(t / N);
    float2 v = X[q];
    if (i == 0) {
      const int jm = (N - j) % N, km = (N - k) % N;
      const float2 m = X[((size_t)km * N + jm) * h];
      v = make_float2(__fmul_rn(0.5f, __fadd_rn(v.x, m.x)), __fmul_rn(0.5f, __fsub_rn(v.y, m.y)));
    }
    const float s = ((i + j + k) & 1) ? -1.0f : 1.0f;
    float2 r = make_float2(s * v.x, -(s * v.y));
    if (q == 0) r.y = 0.0f;
    out[q] = r;
  }
}

__global__ void fs_vol_out_kernel(const float* __restrict__ R, int nx, int ip, float pix, const float* __restrict__ wkb,
                                  float* __restrict__ vol) {
  const int N = 2 * nx, c = nx / 2 + 1;
  const int l2 = (nx / 2) * (nx / 2);
  const size_t total = (size_t)nx * nx * nx;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const size_t t = q / nx;
    const int j = (int)(t % nx), k = (int)(t / nx);
    const int lr = (k + 1 - c) * (k + 1 - c) + (j + 1 - c) * (j + 1 - c) + (i + 1 - c) * (i + 1 - c);
    float o = 0.0f;
    if (lr <= l2) o = __fmul_rn(__fmul_rn(R[((size_t)(ip + k) * N + (ip + j)) * N + (ip + i)], pix), wkb[lr]);
    vol[q] = o;
  }
}

}  // namespace spi

using namespace spi;

struct spi_fslice_plan {
  spi_ctx* ctx = nullptr;
  int device = 0, nx = 0, n = 0, nang = 0, sm_count = 148;
  FsDesc* sl = nullptr;        // [nang]
  float* tab = nullptr;        // KB table, 5000 floats
  float fltb = 0.0f;
  float* wkb = nullptr;        // |WKB(LR)|, LR = 0..(nx/2)^2
  // staging and volume buffers (made on first use; not part of the capturable calls)
  cufftHandle r2c = 0, c2r = 0, r2c_tail = 0;
  int r2c_batch = 0, r2c_tail_batch = 0;
  float* padded = nullptr;     // [r2c_batch][n][n]
  float2* cplx = nullptr;      // [n][n][nx+1]
  float* real3 = nullptr;      // [n][n][n]
};

namespace {

int fs_blocks(const spi_fslice_plan* p) { return p->sm_count * 3; }
// E^T into FP64 with eight lanes per pixel (SPI_FS_LANES=4 selects the four-lane form)
bool fs_w8() {
  const char* e = std::getenv("SPI_FS_LANES");
  return !(e && std::atoi(e) == 4);
}
int fs_grid_blocks(const spi_fslice_plan* p, size_t work) {
  size_t b = (work + 255) / 256, cap = (size_t)p->sm_count * 8;
  return (int)std::max<size_t>(1, std::min(b, cap));
}
size_t fs_grid_elems(const spi_fslice_plan* p) { return (size_t)(p->nx + 1) * p->n * p->n; }
constexpr size_t kFsSmem = 5000 * sizeof(float);

}  // namespace

extern "C" {

int spi_fslice_plan_create(spi_ctx* ctx, int nx, const float* angles, int nang, spi_fslice_plan** out) {
  if (!ctx || !out) return fail(kInvalid, "spi_fslice_plan_create: NULL argument");
  *out = nullptr;
  if (nx < 8 || nx > 512) return fail(kInvalid, "spi_fslice_plan_create: nx = %d must be 8..512", nx);
  if (nang < 1 || !angles) return fail(kInvalid, "spi_fslice_plan_create: %d angles", nang);
  SPI_CUDA(cudaSetDevice(ctx->device));
  KBTab kb;
  fill_kb(2 * nx, kb);
  {
    const int i0 = std::max(0, (int)std::floor(2.0 * kb.fltb) - 1);
    for (int i = i0; i < 5000; ++i)
      if (kb.tab[i] != 0.0f)
        return fail(kInvalid, "spi_fslice_plan_create: the interpolation table of nx = %d has more than four "
                              "nonzero taps per axis", nx);
  }
  std::vector<FsDesc> hs(nang);
  const char* ord = std::getenv("SPI_INSERT_ORDER");
  const int order = !ord ? 1 : std::strcmp(ord, "rows") == 0 ? 0 : std::strcmp(ord, "cols") == 0 ? 2 : 1;
  for (int a = 0; a < nang; ++a) {
    float dm[9];
    cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], dm);   // BUILDM1 (bp3f.f:1287)
    std::memcpy(hs[a].dm, dm, 6 * sizeof(float));
    hs[a].img = a;
    // insertion order (FsLine): the in-plane axis with the smaller z
    // component, for boxes above 192 (as the back-projection chooses)
    hs[a].cols = (order == 2 || (order == 1 && nx > 192 && std::fabs(dm[5]) < std::fabs(dm[2]))) ? 1 : 0;
  }
  std::vector<float> wkb;
  windkb_table(nx, kb, wkb);
  auto* p = new spi_fslice_plan();
  p->ctx = ctx;
  p->device = ctx->device;
  p->sm_count = ctx->sm_count;
  p->nx = nx;
  p->n = 2 * nx;
  p->nang = nang;
  p->fltb = kb.fltb;
  cudaError_t e = cudaMalloc(&p->sl, sizeof(FsDesc) * nang);
  if (e == cudaSuccess) e = cudaMalloc(&p->tab, sizeof(kb.tab));
  if (e == cudaSuccess) e = cudaMalloc(&p->wkb, wkb.size() * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(p->sl, hs.data(), sizeof(FsDesc) * nang, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p->tab, kb.tab, sizeof(kb.tab), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p->wkb, wkb.data(), wkb.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    spi_fslice_plan_destroy(p);
    return fail(kAlloc, "spi_fslice_plan_create: %s", cudaGetErrorString(e));
  }
  *out = p;
  return 0;
}

int spi_fslice_plan_destroy(spi_fslice_plan* p) {
  if (!p) return 0;
  cudaSetDevice(p->device);
  if (p->r2c) cufftDestroy(p->r2c);
  if (p->r2c_tail) cufftDestroy(p->r2c_tail);
  if (p->c2r) cufftDestroy(p->c2r);
  cudaFree(p->sl);
  cudaFree(p->tab);
  cudaFree(p->wkb);
  cudaFree(p->padded);
  cudaFree(p->cplx);
  cudaFree(p->real3);
  delete p;
  return 0;
}

int spi_fslice_stage(spi_fslice_plan* p, const float* imgs, float* slices, void* stream) {
  if (!p || !imgs || !slices) return fail(kInvalid, "spi_fslice_stage: NULL argument");
  SPI_CUDA(cudaSetDevice(p->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nx = p->nx, n = p->n;
  if (!p->r2c) {
    p->r2c_batch = (int)std::max<size_t>(1, std::min<size_t>((size_t)p->nang, (512ull << 20) / ((size_t)n * n * 4)));
    SPI_CUDA(cudaMalloc(&p->padded, (size_t)p->r2c_batch * n * n * sizeof(float)));
    int dims[2] = {n, n};
    SPI_CUFFT(cufftPlanMany(&p->r2c, 2, dims, nullptr, 1, n * n, nullptr, 1, n * (n / 2 + 1), CUFFT_R2C,
                            p->r2c_batch));
  }
  SPI_CUFFT(cufftSetStream(p->r2c, s));
  const size_t plane = (size_t)n * (nx + 1);
  for (int a0 = 0; a0 < p->nang; a0 += p->r2c_batch) {
    const int nb = std::min(p->r2c_batch, p->nang - a0);
    SPI_TRY(stage_images(p->ctx, s, imgs + (size_t)a0 * nx * nx, nx, nb, p->padded));
    cufftHandle plan = p->r2c;
    if (nb < p->r2c_batch) {   // a shorter last batch has a plan of its own
      if (p->r2c_tail_batch != nb) {
        if (p->r2c_tail) cufftDestroy(p->r2c_tail);
        p->r2c_tail = 0;
        p->r2c_tail_batch = 0;
        int dims[2] = {n, n};
        SPI_CUFFT(cufftPlanMany(&p->r2c_tail, 2, dims, nullptr, 1, n * n, nullptr, 1, n * (n / 2 + 1), CUFFT_R2C, nb));
        p->r2c_tail_batch = nb;
      }
      plan = p->r2c_tail;
      SPI_CUFFT(cufftSetStream(plan, s));
    }
    SPI_CUFFT(cufftExecR2C(plan, p->padded, reinterpret_cast<cufftComplex*>(slices) + (size_t)a0 * plane));
  }
  p->ctx->count();
  return 0;
}

int spi_fslice_forward(const spi_fslice_plan* p, const float* grid, float* slices, void* stream) {
  if (!p || !grid || !slices) return fail(kInvalid, "spi_fslice_forward: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  fs_kernel<0><<<fs_blocks(p), 256, kFsSmem, s>>>(reinterpret_cast<const float2*>(grid),
                                                   reinterpret_cast<float2*>(slices), p->sl, p->nang, p->nx, p->tab,
                                                   p->fltb);
  SPI_TRY(check_kernel("fs_kernel<extract>"));
  p->ctx->count();
  return 0;
}

int spi_fslice_adjoint(const spi_fslice_plan* p, const float* slices, float* grid, void* stream) {
  if (!p || !grid || !slices) return fail(kInvalid, "spi_fslice_adjoint: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SPI_CUDA(cudaMemsetAsync(grid, 0, fs_grid_elems(p) * sizeof(float2), s));
  fs_kernel<1><<<fs_blocks(p), 256, kFsSmem, s>>>(reinterpret_cast<const float2*>(slices),
                                                   reinterpret_cast<float2*>(grid), p->sl, p->nang, p->nx, p->tab,
                                                   p->fltb);
  SPI_TRY(check_kernel("fs_kernel<insert>"));
  p->ctx->count();
  return 0;
}

int spi_fslice_normal(const spi_fslice_plan* p, const float* grid_in, float lam, float* grid_out, void* stream) {
  if (!p || !grid_in || !grid_out) return fail(kInvalid, "spi_fslice_normal: NULL argument");
  if (grid_in == grid_out) return fail(kInvalid, "spi_fslice_normal: input and output must differ");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t ne = fs_grid_elems(p);
  fs_scale_kernel<<<fs_grid_blocks(p, ne), 256, 0, s>>>(reinterpret_cast<const float2*>(grid_in), lam,
                                                        reinterpret_cast<float2*>(grid_out), ne);
  SPI_TRY(check_kernel("fs_scale_kernel"));
  fs_kernel<2><<<fs_blocks(p), 256, kFsSmem, s>>>(reinterpret_cast<const float2*>(grid_in),
                                                   reinterpret_cast<float2*>(grid_out), p->sl, p->nang, p->nx, p->tab,
                                                   p->fltb);
  SPI_TRY(check_kernel("fs_kernel<normal>"));
  p->ctx->count(2);
  return 0;
}

int spi_fslice_normal64(const spi_fslice_plan* p, const double* grid_in, double lam, double* grid_out, void* stream) {
  if (!p || !grid_in || !grid_out) return fail(kInvalid, "spi_fslice_normal64: NULL argument");
  if (grid_in == grid_out) return fail(kInvalid, "spi_fslice_normal64: input and output must differ");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t ne = fs_grid_elems(p);
  fs_scale64_kernel<<<fs_grid_blocks(p, ne), 256, 0, s>>>(reinterpret_cast<const double2*>(grid_in), lam,
                                                          reinterpret_cast<double2*>(grid_out), ne);
  SPI_TRY(check_kernel("fs_scale64_kernel"));
  fs_normal64_kernel<true><<<fs_blocks(p), 256, kFsSmem, s>>>(reinterpret_cast<const double2*>(grid_in), nullptr,
                                                              reinterpret_cast<double2*>(grid_out), p->sl, p->nang,
                                                              p->nx, p->tab, p->fltb);
  SPI_TRY(check_kernel("fs_normal64_kernel"));
  p->ctx->count(2);
  return 0;
}

int spi_fslice_forward64(const spi_fslice_plan* p, const double* grid, double* slices, void* stream) {
  if (!p || !grid || !slices) return fail(kInvalid, "spi_fslice_forward64: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  fs_extract64_kernel<<<fs_blocks(p), 256, kFsSmem, s>>>(reinterpret_cast<const double2*>(grid),
                                                         reinterpret_cast<double2*>(slices), p->sl, p->nang, p->nx,
                                                         p->tab, p->fltb);
  SPI_TRY(check_kernel("fs_extract64_kernel"));
  p->ctx->count();
  return 0;
}

int spi_fslice_adjoint64(const spi_fslice_plan* p, const float* slices, double* grid, void* stream) {
  if (!p || !grid || !slices) return fail(kInvalid, "spi_fslice_adjoint64: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SPI_CUDA(cudaMemsetAsync(grid, 0, fs_grid_elems(p) * sizeof(double2), s));
  if (fs_w8())
    fs_insert64w_kernel<<<fs_blocks(p), 256, kFsSmem, s>>>(reinterpret_cast<const float2*>(slices), grid, p->sl,
                                                           p->nang, p->nx, p->tab, p->fltb);
  else
    fs_normal64_kernel<false><<<fs_blocks(p), 256, kFsSmem, s>>>(nullptr, reinterpret_cast<const float2*>(slices),
                                                                 reinterpret_cast<double2*>(grid), p->sl, p->nang,
                                                                 p->nx, p->tab, p->fltb);
  SPI_TRY(check_kernel("fs_normal64_kernel<insert>"));
  p->ctx->count();
  return 0;
}

int spi_fslice_volume(spi_fslice_plan* p, const float* grid, float* vol_out, void* stream) {
  if (!p || !grid || !vol_out) return fail(kInvalid, "spi_fslice_volume: NULL argument");
  SPI_CUDA(cudaSetDevice(p->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nx = p->nx, n = p->n;
  if (!p->c2r) {
    SPI_CUDA(cudaMalloc(&p->cplx, fs_grid_elems(p) * sizeof(float2)));
    SPI_CUDA(cudaMalloc(&p->real3, (size_t)n * n * n * sizeof(float)));
    SPI_CUFFT(cufftPlan3d(&p->c2r, n, n, n, CUFFT_C2R));
  }
  SPI_CUFFT(cufftSetStream(p->c2r, s));
  const size_t ne = fs_grid_elems(p);
  fs_vol_prep_kernel<<<fs_grid_blocks(p, ne), 256, 0, s>>>(reinterpret_cast<const float2*>(grid), p->cplx, nx);
  SPI_TRY(check_kernel("fs_vol_prep_kernel"));
  SPI_CUFFT(cufftExecC2R(p->c2r, reinterpret_cast<cufftComplex*>(p->cplx), p->real3));
  const int ip = (n - nx) / 2 + nx % 2;
  const float pix = 1.0f / (float)((long long)n * n * n);
  fs_vol_out_kernel<<<fs_grid_blocks(p, (size_t)nx * nx * nx), 256, 0, s>>>(p->real3, nx, ip, pix, p->wkb, vol_out);
  SPI_TRY(check_kernel("fs_vol_out_kernel"));
  p->ctx->count(2);
  return 0;
}

}  // extern "C"
