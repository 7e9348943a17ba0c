// Fourier gridding back-projection (SPIDER BP 3F / BP 32F) on sm_100a.
//
// Per chunk of images:   stage (PADD2 + phase as a circular shift, FP64 mean)
//                        -> batched cuFFT R2C
//                        -> insert (ONELINE, one persistent launch per chunk)
// Per volume:            SYMPLANE0 -> NRMW2 (+ADDADA) -> cuFFT C2R -> WINDKB2A
//
// The grid is an array of float4 {Re X, Im X, W, 0} voxels laid out
// [k][j][i], i = 0..nx fastest (Fortran X(0:NX,N,N) with W interleaved), so
// each gridding tap is one 16-byte vector atomic in L2.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <tuple>
#include <mutex>
#include <map>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "../../include/spider_b200.h"
#include "ctx.h"

namespace spi {

struct SliceDesc {
  float dm[6];  // DMS(1:6): first two columns of the (symmetrised) rotation
  int img;      // image index inside the chunk
  short grid;   // target grid (BP 32F half set)
  short cols;   // insertion order of the x4 kernels: 0 row by row, 1 column by column
};
static_assert(sizeof(SliceDesc) == 32, "slice descriptor is 32 bytes");

// ----------------------------------------------------------------------------
// helpers
__device__ __forceinline__ int nint_pos(float v) {  // Fortran NINT, v >= 0
  float f = floorf(v);
  return (int)f + ((__fsub_rn(v, f) >= 0.5f) ? 1 : 0);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// ----------------------------------------------------------------------------
// Stage: PADD2 (bp3f.f:1307-1343) with ASTA_D's FP64 mean outside radius
// nx/2 (asta.f:61-92).  The phase BI*(-1)**(I+J+1) (bp3f.f:453-458) equals a
// circular shift of the padded image by n/2 in both axes, so the padded
// image is written already shifted: pixel i lands at (ip + i - nx) mod n.
// One CTA per image (blockIdx.y splits the padded rows over gridDim.y CTAs,
// each computing the image's border mean itself, when few images fill a
// launch).  Warps take whole rows, lanes consecutive pixels, so no index is
// divided; each value is the same (double)pixel - mean rounded to float.
// Images beyond `nvalid` are written as zeros.
__global__ void __launch_bounds__(256) stage_kernel(const float* __restrict__ imgs, int nx, int n, int ip,
                                                    int nvalid, double klp, float* __restrict__ padded) {
  const int b = blockIdx.x;
  float* out = padded + (size_t)b * n * n;
  __shared__ double red[8];
  __shared__ double qs_sh;
  const bool valid = b < nvalid;
  const float* img = imgs + (size_t)b * nx * nx;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (valid) {
    const float rr = (float)(nx / 2) * (float)(nx / 2);
    const int nc = nx / 2 + 1;
    double s = 0.0;
    for (int j = warp; j < nx; j += nwarps) {
      const float t = (float)(j + 1 - nc);
      const float tt = __fmul_rn(t, t);
      const float* row = img + (size_t)j * nx;
      for (int i = lane; i < nx; i += 32) {
        const float t2 = (float)(i + 1 - nc);
        if (__fadd_rn(tt, __fmul_rn(t2, t2)) > rr) s += (double)__ldg(row + i);
      }
    }
    s = warp_sum(s);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nwarps; ++w) t += red[w];
      qs_sh = t / klp;
    }
    __syncthreads();
  }
  const double qs = valid ? qs_sh : 0.0;
  const int y0 = (int)(((long long)n * blockIdx.y) / gridDim.y);
  const int y1 = (int)(((long long)n * (blockIdx.y + 1)) / gridDim.y);
  for (int y = y0 + warp; y < y1; y += nwarps) {
    int j = y + nx - ip;
    if (j >= n) j -= n;
    float* orow = out + (size_t)y * n;
    if (!valid || j >= nx) {                        // a padding row
      for (int x = lane; x < n; x += 32) orow[x] = 0.0f;
      continue;
    }
    const float* irow = img + (size_t)j * nx;
    int i = lane + nx - ip;                          // source column of x = lane, kept in [0, n)
    if (i >= n) i -= n;
    for (int x = lane; x < n; x += 32) {
      orow[x] = (i < nx) ? __double2float_rn(__dsub_rn((double)__ldg(irow + i), qs)) : 0.0f;
      i += 32;
      if (i >= n) i -= n;
    }
  }
}

// ----------------------------------------------------------------------------
// Staging and the forward 2D transform for power-of-two padded sizes n, in
// two passes (FMRS_2's R2C, fmrs_2.f:54-58, with cuFFT's sign and layout:
// out[y'][k] = sum_y sum_x in[y][x] e^(-2 pi i (k x + y' y) / n), k = 0..n/2).
// Only the nx rows of the padded image that hold image pixels are nonzero,
// so the row pass transforms those rows only and the column pass never
// stores the zero ones.
//
// Pass 1 (stage_rowfft_kernel, one CTA per image as stage_kernel, which it
// replaces): the same staged values (pixel - FP64 border mean, shifted by n/2)
// for each image row j, then a real FFT of length n as a complex FFT of
// length h = n/2 of z[m] = in[2m] + i in[2m+1] (radix-2, in shared memory,
// inputs loaded in bit-reversed order) split into R[k] = E[k] + W^k O[k],
// E = (Z[k] + conj Z[h-k]) / 2, O = (Z[k] - conj Z[h-k]) / 2i, W = e^(-2 pi i/n).
// R (h + 1 values) goes to inter[b][j][.].
// Pass 2 (colfft_kernel): a CTA takes 16 columns k of one image, places row
// j's values at the padded row y = (j + ip - nx) mod n (bit-reversed), zero
// elsewhere, and runs 16 complex FFTs of length n.  Twiddles W^t, t < n/2,
// come from a table computed in FP64 on the host.
constexpr int kRowThreads = 64;   // threads per row FFT in pass 1
constexpr int kColTile = 16;      // columns per CTA in pass 2

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// in-place radix-2 decimation-in-time stages over `len` points (input in
// bit-reversed order) at a[0..len); threads t0..t0+nt-1 of the CTA share the
// work; tw[t] = W_n^t with W_len^u = tw[u * (n / len)]
__device__ __forceinline__ void fft_stages(float2* a, int len, int lg, const float2* tw, int twstep, int t0, int nt,
                                           int tid) {
  for (int st = 1; st <= lg; ++st) {
    const int half = 1 << (st - 1);
    const int tws = (len >> st) * twstep;
    for (int bfly = tid - t0; bfly < (len >> 1); bfly += nt) {
      const int grp = bfly >> (st - 1), k = bfly & (half - 1);
      const int pos = (grp << st) + k;
      const float2 w = tw[k * tws];
      const float2 u = a[pos], v = cmulf(w, a[pos + half]);
      a[pos] = make_float2(__fadd_rn(u.x, v.x), __fadd_rn(u.y, v.y));
      a[pos + half] = make_float2(__fsub_rn(u.x, v.x), __fsub_rn(u.y, v.y));
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int bitrev(int v, int lg) { return (int)(__brev((unsigned)v) >> (32 - lg)); }

__global__ void __launch_bounds__(256) stage_rowfft_kernel(const float* __restrict__ imgs, int nx, int n, int ip,
                                                           int nvalid, double klp, const float2* __restrict__ twg,
                                                           float2* __restrict__ inter, size_t inter_stride) {
  extern __shared__ float2 fsm[];            // tw[n/2], then 4 rows of h complex values
  const int h = n >> 1, lgh = 31 - __clz(h);
  float2* tw = fsm;
  for (int t = threadIdx.x; t < h; t += blockDim.x) tw[t] = twg[t];
  const int b = blockIdx.x;
  if (b >= nvalid) return;                   // uniform per CTA; only valid images are transformed
  __shared__ double red[8];
  __shared__ double qs_sh;
  const float* img = imgs + (size_t)b * nx * nx;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  {
    const float rr = (float)(nx / 2) * (float)(nx / 2);
    const int nc = nx / 2 + 1;
    double s = 0.0;
    for (int j = warp; j < nx; j += nwarps) {
      const float t = (float)(j + 1 - nc);
      const float tt = __fmul_rn(t, t);
      const float* row = img + (size_t)j * nx;
      for (int i = lane; i < nx; i += 32) {
        const float t2 = (float)(i + 1 - nc);
        if (__fadd_rn(tt, __fmul_rn(t2, t2)) > rr) s += (double)__ldg(row + i);
      }
    }
    s = warp_sum(s);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nwarps; ++w) t += red[w];
      qs_sh = t / klp;
    }
    __syncthreads();
  }
  const double qs = qs_sh;
  const int groups = blockDim.x / kRowThreads, grp = threadIdx.x / kRowThreads;
  float2* a = fsm + h + (size_t)grp * h;
  float2* ib = inter + (size_t)b * inter_stride;
  // image rows j0.. of this CTA part (blockIdx.y splits them when few images fill a launch)
  const int j0 = (int)(((long long)nx * blockIdx.y) / gridDim.y), j1 = (int)(((long long)nx * (blockIdx.y + 1)) / gridDim.y);
  const int rounds = (j1 - j0 + groups - 1) / groups;
  for (int rd = 0; rd < rounds; ++rd) {
    const int j = j0 + rd * groups + grp;
    const bool has = j < j1;
    if (has) {
      const float* irow = img + (size_t)j * nx;
      for (int m = threadIdx.x - grp * kRowThreads; m < h; m += kRowThreads) {
        float v2[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int i = 2 * m + e + nx - ip;        // padded column x = 2m + e holds pixel i when i < nx
          if (i >= n) i -= n;
          v2[e] = (i < nx) ? __double2float_rn(__dsub_rn((double)__ldg(irow + i), qs)) : 0.0f;
        }
        a[bitrev(m, lgh)] = make_float2(v2[0], v2[1]);
      }
    }
    __syncthreads();
    fft_stages(a, h, lgh, tw, 2, grp * kRowThreads, kRowThreads, threadIdx.x);
    if (has) {
      float2* orow = ib + (size_t)j * (h + 1);
      for (int k = threadIdx.x - grp * kRowThreads; k <= h; k += kRowThreads) {
        const float2 zk = a[k & (h - 1)], zc = a[(h - k) & (h - 1)];
        // E = (zk + conj zc) / 2, O = (zk - conj zc) / (2i)
        const float2 e = make_float2(__fmul_rn(0.5f, __fadd_rn(zk.x, zc.x)), __fmul_rn(0.5f, __fsub_rn(zk.y, zc.y)));
        const float2 o = make_float2(__fmul_rn(0.5f, __fadd_rn(zk.y, zc.y)), __fmul_rn(-0.5f, __fsub_rn(zk.x, zc.x)));
        const float2 w = (k < h) ? tw[k] : make_float2(-1.0f, 0.0f);
        const float2 wo = cmulf(w, o);
        orow[k] = make_float2(__fadd_rn(e.x, wo.x), __fadd_rn(e.y, wo.y));
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) colfft_kernel(const float2* __restrict__ inter, size_t inter_stride, int nx,
                                                     int n, int ip, int nvalid, const float2* __restrict__ twg,
                                                     float2* __restrict__ out) {
  extern __shared__ float2 fsm[];            // tw[n/2], then kColTile columns of n values, stride n + 1
  const int h = n >> 1, lg = 31 - __clz(n);
  const int cs = n + 1;                      // column stride: the tile's columns start in different banks
  const int tiles = (h + 1 + kColTile - 1) / kColTile;
  const int b = blockIdx.x / tiles, k0 = (blockIdx.x % tiles) * kColTile;
  float2* tw = fsm;
  float2* a = fsm + h;
  for (int t = threadIdx.x; t < h; t += blockDim.x) tw[t] = twg[t];
  if (b >= nvalid) return;
  const int ncol = min(kColTile, h + 1 - k0);
  for (int q = threadIdx.x; q < kColTile * cs; q += blockDim.x) a[q] = make_float2(0.0f, 0.0f);
  __syncthreads();
  const float2* ib = inter + (size_t)b * inter_stride;
  for (int q = threadIdx.x; q < nx * kColTile; q += blockDim.x) {
    const int j = q / kColTile, c = q % kColTile;
    if (c >= ncol) continue;
    int y = j + ip - nx;
    if (y < 0) y += n;
    a[c * cs + bitrev(y, lg)] = ib[(size_t)j * (h + 1) + k0 + c];
  }
  __syncthreads();
  // kColTile transforms of n points; thread t works on column t % kColTile
  const int c = threadIdx.x % kColTile, tpc = blockDim.x / kColTile, sub = threadIdx.x / kColTile;
  float2* col = a + (size_t)c * cs;
  for (int st = 1; st <= lg; ++st) {
    const int half = 1 << (st - 1);
    const int tws = n >> st;
    for (int bfly = sub; bfly < h; bfly += tpc) {
      const int grp = bfly >> (st - 1), k = bfly & (half - 1);
      const int pos = (grp << st) + k;
      const float2 w = tw[k * tws];
      const float2 u = col[pos], v = cmulf(w, col[pos + half]);
      col[pos] = make_float2(__fadd_rn(u.x, v.x), __fadd_rn(u.y, v.y));
      col[pos + half] = make_float2(__fsub_rn(u.x, v.x), __fsub_rn(u.y, v.y));
    }
    __syncthreads();
  }
  float2* ob = out + (size_t)b * n * (h + 1);
  for (int q = threadIdx.x; q < n * kColTile; q += blockDim.x) {
    const int y = q / kColTile, cc = q % kColTile;
    if (cc < ncol) ob[(size_t)y * (h + 1) + k0 + cc] = a[cc * cs + y];
  }
}

// ----------------------------------------------------------------------------
// The same two passes with the transforms in registers (four-step FFT of H =
// 32 P points over one warp: P-point DFTs in each lane's registers, a twiddle
// W_H^(lane k2), then 32-point DFTs across the lanes by shuffles), one warp
// per padded row (pass 1, H = n/2) or per column (pass 2, H = n).  A lane
// starts with x[lane + 32 r], r < P, and ends with X[P brev5(lane) + k2],
// k2 < P.  The radix-2 shared-memory form above is kept for n < 128 and
// n > 512.

// W_n^t for 0 <= t < n from the table of t < n/2 (W_n^(t + n/2) = -W_n^t)
__device__ __forceinline__ float2 tw_full(const float2* tw, int t, int h) {
  return t < h ? tw[t] : make_float2(-tw[t - h].x, -tw[t - h].y);
}

__host__ __device__ constexpr int log2_c(int v) { return v <= 1 ? 0 : 1 + log2_c(v / 2); }
// bit reversal of V over BITS bits as a compile-time constant (register indices
// must fold to constants, or the array goes to local memory)
template <int V, int BITS>
struct BrevT {
  static constexpr int value = ((V & 1) << (BITS - 1)) | BrevT<(V >> 1), BITS - 1>::value;
};
template <int V>
struct BrevT<V, 0> {
  static constexpr int value = 0;
};
template <int K, int P, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (K < P) {
    f(std::integral_constant<int, K>{});
    static_for<K + 1, P>(f);
  }
}

// P-point radix-2 decimation-in-frequency FFT in registers: natural order in,
// a[brev(k)] = X[k] out; W_P^e = tw[e * (n / P)]
template <int P>
__device__ __forceinline__ void reg_fft_dif(float2 (&a)[P], const float2* tw, int n) {
#pragma unroll
  for (int h = P / 2; h >= 1; h >>= 1) {
#pragma unroll
    for (int i = 0; i < P; ++i) {
      if (i & h) continue;
      const float2 u = a[i], v = a[i + h];
      a[i] = make_float2(__fadd_rn(u.x, v.x), __fadd_rn(u.y, v.y));
      const float2 d = make_float2(__fsub_rn(u.x, v.x), __fsub_rn(u.y, v.y));
      const int e = (i & (h - 1)) * (P / (2 * h));
      a[i + h] = e == 0 ? d : cmulf(tw[e * (n / P)], d);
    }
  }
}

// 32-point decimation-in-frequency FFT across the lanes, for each of the P
// values of a lane: lane l ends with the output brev5(l)
template <int P>
__device__ __forceinline__ void warp_fft32_dif(float2 (&a)[P], const float2* tw, int n, int lane) {
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    const bool top = (lane & h) == 0;
    const float2 w = tw[(lane & (h - 1)) * (16 / h) * (n / 32)];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      const float px = __shfl_xor_sync(0xffffffffu, a[k].x, h);
      const float py = __shfl_xor_sync(0xffffffffu, a[k].y, h);
      if (top) a[k] = make_float2(__fadd_rn(a[k].x, px), __fadd_rn(a[k].y, py));
      else a[k] = cmulf(w, make_float2(__fsub_rn(px, a[k].x), __fsub_rn(py, a[k].y)));
    }
  }
}

// H = 32 P point DFT (sign -1) of x[lane + 32 r] = z[r]; z[k2] = X[P brev5(lane) + k2] after
template <int P>
__device__ __forceinline__ void warp_fft(float2 (&z)[P], const float2* tw, int n, int lane) {
  reg_fft_dif<P>(z, tw, n);
  float2 y[P];
  static_for<0, P>([&](auto kc) {
    constexpr int k2 = decltype(kc)::value;
    const float2 v = z[BrevT<k2, log2_c(P)>::value];
    const int t = ((n / (32 * P)) * lane * k2) & (n - 1);   // W_H^(lane k2) = W_n^((n/H) lane k2)
    y[k2] = k2 == 0 ? v : cmulf(tw_full(tw, t, n / 2), v);
  });
  warp_fft32_dif<P>(y, tw, n, lane);
#pragma unroll
  for (int k2 = 0; k2 < P; ++k2) z[k2] = y[k2];
}

__device__ __forceinline__ int brev5(int v) { return (int)(__brev((unsigned)v) >> 27); }

// Pass 1, one warp per image row (P = n / 64): staging as stage_rowfft_kernel,
// the real row as the complex sequence z[m] = in[2m] + i in[2m+1] of h = n/2
// points, R[k] = E[k] + W_n^k O[k] for k <= h into inter[b][j][k].
// the largest d >= 0 with d * d <= rem (rem >= 0)
__device__ __forceinline__ int isqrt_floor(int rem) {
  float f;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(f) : "f"((float)rem));
  int d = (int)f;
  while (d > 0 && d * d > rem) --d;
  while ((d + 1) * (d + 1) <= rem) ++d;
  return d;
}

template <int P>
__global__ void __launch_bounds__(256) stage_rowfft_w_kernel(const float* __restrict__ imgs, int nx, int n, int ip,
                                                             int nvalid, double klp, const float2* __restrict__ twg,
                                                             float2* __restrict__ inter, size_t inter_stride) {
  __shared__ float2 tw[512];
  __shared__ double red[8];
  __shared__ double qs_sh;
  // per warp, a row's outputs R[k] at k + k / P (the lanes' values are P apart;
  // this spreads them over the banks) before the row is written coalesced
  __shared__ float2 rbuf[8][32 * P + 32 + 1];
  const int h = n >> 1;   // = 32 P
  for (int t = threadIdx.x; t < h; t += blockDim.x) tw[t] = twg[t];
  const int b = blockIdx.x;
  if (b >= nvalid) return;   // uniform per CTA
  const float* img = imgs + (size_t)b * nx * nx;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  {
    // ASTA's border mean over the pixels outside the inscribed circle: row j
    // (t = j + 1 - nc) keeps columns with t2 = i + 1 - nc, t^2 + t2^2 > r^2,
    // i.e. all but the run |t2| <= isqrt(r^2 - t^2) (integers, exact)
    const int r2 = (nx / 2) * (nx / 2), nc = nx / 2 + 1;
    double sum = 0.0;
    for (int j = warp; j < nx; j += nwarps) {
      const int t = j + 1 - nc, rem = r2 - t * t;
      const float* row = img + (size_t)j * nx;
      int a0 = nx, b0 = nx;   // border: [0, a0) and [b0, nx)
      if (rem >= 0) {
        const int d = isqrt_floor(rem);
        a0 = max(0, nc - 1 - d);
        b0 = min(nx, nc + d);
      }
      for (int i = lane; i < a0; i += 32) sum += (double)__ldg(row + i);
      for (int i = b0 + lane; i < nx; i += 32) sum += (double)__ldg(row + i);
    }
    sum = warp_sum(sum);
    if (lane == 0) red[warp] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nwarps; ++w) t += red[w];
      qs_sh = t / klp;
    }
    __syncthreads();
  }
  const double qs = qs_sh;
  float2* ib = inter + (size_t)b * inter_stride;
  const int j0 = (int)(((long long)nx * blockIdx.y) / gridDim.y), j1 = (int)(((long long)nx * (blockIdx.y + 1)) / gridDim.y);
  const int k1 = brev5(lane);
  const int lanec0 = brev5((32 - k1) & 31);   // the lane holding Z[h - P k1]
  for (int j = j0 + warp; j < j1; j += nwarps) {   // warp-uniform
    const float* irow = img + (size_t)j * nx;
    float2 z[P];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      // padded columns 2m, 2m + 1 hold pixels i, i + 1 when i < nx (i even:
      // nx - ip = nx / 2 is even for the sizes this kernel takes)
      int i = 2 * (lane + 32 * r) + nx - ip;
      if (i >= n) i -= n;
      z[r] = make_float2(0.0f, 0.0f);
      if (i < nx) {
        const float2 p = __ldg(reinterpret_cast<const float2*>(irow + i));
        z[r] = make_float2(__double2float_rn(__dsub_rn((double)p.x, qs)), __double2float_rn(__dsub_rn((double)p.y, qs)));
      }
    }
    warp_fft<P>(z, tw, n, lane);   // the h-point FFT (tw is the table of W_n)
    float2 zc[P];
    zc[0] = make_float2(__shfl_sync(0xffffffffu, z[0].x, lanec0), __shfl_sync(0xffffffffu, z[0].y, lanec0));
#pragma unroll
    for (int k2 = 1; k2 < P; ++k2)
      zc[k2] = make_float2(__shfl_sync(0xffffffffu, z[P - k2].x, 31 - lane),
                           __shfl_sync(0xffffffffu, z[P - k2].y, 31 - lane));
    float2* rb = rbuf[warp];
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) {
      const int k = P * k1 + k2;
      const float2 zk = z[k2], c = zc[k2];
      const float2 ev = make_float2(__fmul_rn(0.5f, __fadd_rn(zk.x, c.x)), __fmul_rn(0.5f, __fsub_rn(zk.y, c.y)));
      const float2 od = make_float2(__fmul_rn(0.5f, __fadd_rn(zk.y, c.y)), __fmul_rn(-0.5f, __fsub_rn(zk.x, c.x)));
      const float2 wo = cmulf(tw[k], od);
      rb[(P + 1) * k1 + k2] = make_float2(__fadd_rn(ev.x, wo.x), __fadd_rn(ev.y, wo.y));
      if (k == 0) {   // R[h] = E[0] - O[0]
        rb[h + h / P] = make_float2(__fsub_rn(ev.x, od.x), __fsub_rn(ev.y, od.y));
      }
    }
    __syncwarp();
    float2* orow = ib + (size_t)j * (h + 1);
    for (int k = lane; k <= h; k += 32) orow[k] = rb[k + k / P];
    __syncwarp();
  }
}

// Pass 1 at n = 512 (nx = 256): as stage_rowfft_w_kernel, one warp per row,
// but the 256-point transform in three register levels joined by two
// transposes through the warp's shared buffer instead of shuffles: level 1,
// lane t takes x[t + 32 r], an 8-point DFT over r and W_256^(t k2) give
// S[k2][t]; level 2, lane (k2, u) takes S[k2][u + 4 r], an 8-point DFT over r
// and W_32^(u m2) give T[k2][m2][u]; level 3, lane (k2, m2, m2 + 1) takes
// T[k2][m2][u], 4-point DFTs over u give X[64 m1 + 8 m2 + k2] into the buffer,
// from which each lane forms R[k] = E[k] + W_512^k O[k] for k = lane + 32 i
// and writes the row coalesced.  Strides and the swizzle of X (k + k / 4)
// keep every warp access at most 3-way bank-conflicted (checked by
// enumeration).
constexpr int kR512SS = 36, kR512TS = 35, kR512TR = 4, kR512Buf = 320;
__global__ void __launch_bounds__(256) stage_rowfft512_kernel(const float* __restrict__ imgs, int nx, int n, int ip,
                                                              int nvalid, double klp, const float2* __restrict__ twg,
                                                              float2* __restrict__ inter, size_t inter_stride) {
  __shared__ float2 tw[256];
  __shared__ double red[8];
  __shared__ double qs_sh;
  __shared__ float2 wbuf[8][kR512Buf];
  const int h = 256;
  for (int t = threadIdx.x; t < h; t += blockDim.x) tw[t] = twg[t];
  const int b = blockIdx.x;
  if (b >= nvalid) return;   // uniform per CTA
  const float* img = imgs + (size_t)b * nx * nx;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  {
    const int r2 = (nx / 2) * (nx / 2), nc = nx / 2 + 1;
    double sum = 0.0;
    for (int j = warp; j < nx; j += nwarps) {
      const int t = j + 1 - nc, rem = r2 - t * t;
      const float* row = img + (size_t)j * nx;
      int a0 = nx, b0 = nx;
      if (rem >= 0) {
        const int d = isqrt_floor(rem);
        a0 = max(0, nc - 1 - d);
        b0 = min(nx, nc + d);
      }
      for (int i = lane; i < a0; i += 32) sum += (double)__ldg(row + i);
      for (int i = b0 + lane; i < nx; i += 32) sum += (double)__ldg(row + i);
    }
    sum = warp_sum(sum);
    if (lane == 0) red[warp] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nwarps; ++w) t += red[w];
      qs_sh = t / klp;
    }
    __syncthreads();
  }
  const double qs = qs_sh;
  float2* ib = inter + (size_t)b * inter_stride;
  float2* B = wbuf[warp];
  const int k2l = lane >> 2, ul = lane & 3;
  const int j0 = (int)(((long long)nx * blockIdx.y) / gridDim.y), j1 = (int)(((long long)nx * (blockIdx.y + 1)) / gridDim.y);
  // padded columns 2m, 2m + 1 (m = lane + 32 r) hold pixels i, i + 1 when i < nx;
  // a row's pixels are loaded one row ahead of its transform
  auto load_row = [&](int jr, float2 (&pv)[8]) {
    const float* irow = img + (size_t)jr * nx;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      int i = 2 * (lane + 32 * r) + nx - ip;
      if (i >= n) i -= n;
      pv[r] = (i < nx) ? __ldg(reinterpret_cast<const float2*>(irow + i)) : make_float2(0.0f, 0.0f);
    }
  };
  float2 pnext[8];
  if (j0 + warp < j1) load_row(j0 + warp, pnext);
  for (int j = j0 + warp; j < j1; j += nwarps) {   // warp-uniform
    float2 v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      int i = 2 * (lane + 32 * r) + nx - ip;
      if (i >= n) i -= n;
      v[r] = (i < nx) ? make_float2(__double2float_rn(__dsub_rn((double)pnext[r].x, qs)),
                                    __double2float_rn(__dsub_rn((double)pnext[r].y, qs)))
                      : make_float2(0.0f, 0.0f);
    }
    if (j + nwarps < j1) load_row(j + nwarps, pnext);
    // level 1
    reg_fft_dif<8>(v, tw, n);
    static_for<0, 8>([&](auto kc) {
      constexpr int k2 = decltype(kc)::value;
      const float2 val = v[BrevT<k2, 3>::value];
      B[k2 * kR512SS + lane] = k2 == 0 ? val : cmulf(tw_full(tw, 2 * lane * k2, h), val);   // W_256^(t k2)
    });
    __syncwarp();
    // level 2
    float2 w[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) w[r] = B[k2l * kR512SS + ul + 4 * r];
    reg_fft_dif<8>(w, tw, n);
    __syncwarp();
    static_for<0, 8>([&](auto mc) {
      constexpr int m2 = decltype(mc)::value;
      const float2 val = w[BrevT<m2, 3>::value];
      B[k2l * kR512TS + m2 * kR512TR + ul] = m2 == 0 ? val : cmulf(tw_full(tw, 16 * ul * m2, h), val);   // W_32^(u m2)
    });
    __syncwarp();
    // level 3: lane takes (k2, m2) for m2 = 2 (lane & 3) and 2 (lane & 3) + 1
    float2 q0[4], q1[4];
    const int m2a = 2 * ul;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      q0[u] = B[k2l * kR512TS + m2a * kR512TR + u];
      q1[u] = B[k2l * kR512TS + (m2a + 1) * kR512TR + u];
    }
    reg_fft_dif<4>(q0, tw, n);
    reg_fft_dif<4>(q1, tw, n);
    __syncwarp();
    static_for<0, 4>([&](auto mc) {
      constexpr int m1 = decltype(mc)::value;
      const int y0 = 64 * m1 + 8 * m2a + k2l, y1 = y0 + 8;
      B[y0 + (y0 >> 2)] = q0[BrevT<m1, 2>::value];
      B[y1 + (y1 >> 2)] = q1[BrevT<m1, 2>::value];
    });
    __syncwarp();
    float2* orow = ib + (size_t)j * (h + 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = lane + 32 * i, kc = (h - k) & (h - 1);
      const float2 zk = B[k + (k >> 2)], c = B[kc + (kc >> 2)];
      const float2 ev = make_float2(__fmul_rn(0.5f, __fadd_rn(zk.x, c.x)), __fmul_rn(0.5f, __fsub_rn(zk.y, c.y)));
      const float2 od = make_float2(__fmul_rn(0.5f, __fadd_rn(zk.y, c.y)), __fmul_rn(-0.5f, __fsub_rn(zk.x, c.x)));
      const float2 wo = cmulf(tw[k], od);
      orow[k] = make_float2(__fadd_rn(ev.x, wo.x), __fadd_rn(ev.y, wo.y));
      if (k == 0) orow[h] = make_float2(__fsub_rn(ev.x, od.x), __fsub_rn(ev.y, od.y));   // R[h] = E[0] - O[0]
    }
    __syncwarp();
  }
}

// Pass 2 at n = 128 and 256, one warp per column (P = n / 32; the shuffle
// stages made it slower than colfft512_kernel's shared-memory transposes at
// n = 512: 1.48 against 0.97 ms per 1,024 images): a CTA takes kColTileW columns k0..
// of one image; the nx rows of those columns are read row by row (coalesced)
// into shared memory, each warp transforms its columns (padded row y holds
// image row j = (y - ip + nx) mod n when j < nx, else zero) into a second
// tile, and the CTA writes that tile row by row.  256 threads (8 warps, two
// columns each).
constexpr int kColTileW = 16;
template <int P>
__global__ void __launch_bounds__(256) colfft_w_kernel(const float2* __restrict__ inter, size_t inter_stride, int nx,
                                                       int n, int ip, int nvalid, const float2* __restrict__ twg,
                                                       float2* __restrict__ out) {
  extern __shared__ float2 fsm[];   // tw[n/2], inputs [kColTileW][nx + 1], outputs [kColTileW][so]
  const int h = n >> 1;             // n = 32 P
  const int tiles = (h + 1 + kColTileW - 1) / kColTileW;
  const int b = blockIdx.x / tiles, k0 = (blockIdx.x % tiles) * kColTileW;
  // Output y of column c sits at c * so + y + y / P: a warp's 32 lanes store
  // rows P brev5(lane) + k2, P rows apart, which this spreads over the banks
  // (so = n + n / P + 1 = n + 33, 1 mod 16, keeps the row-by-row reads apart
  // too); the input columns have stride nx + 1 for the same reason.
  const int si = nx + 1, so = n + n / P + 1;
  float2* tw = fsm;
  float2* ain = fsm + h;
  float2* aout = ain + (size_t)kColTileW * si;
  for (int t = threadIdx.x; t < h; t += blockDim.x) tw[t] = twg[t];
  if (b >= nvalid) return;          // uniform per CTA
  const int ncol = min(kColTileW, h + 1 - k0);
  const float2* ib = inter + (size_t)b * inter_stride;
  for (int q = threadIdx.x; q < nx * kColTileW; q += blockDim.x) {
    const int j = q / kColTileW, c = q % kColTileW;
    if (c < ncol) ain[c * si + j] = ib[(size_t)j * (h + 1) + k0 + c];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int k1 = brev5(lane);
  for (int c = warp; c < ncol; c += nwarps) {   // warp-uniform
    float2 z[P];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const int y = lane + 32 * r;
      int j = y - ip + nx;
      if (j >= n) j -= n;
      z[r] = (j < nx) ? ain[c * si + j] : make_float2(0.0f, 0.0f);
    }
    warp_fft<P>(z, tw, n, lane);
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) aout[c * so + (P + 1) * k1 + k2] = z[k2];   // y + y / P, y = P k1 + k2
  }
  __syncthreads();
  float2* ob = out + (size_t)b * n * (h + 1);
  for (int q = threadIdx.x; q < n * kColTileW; q += blockDim.x) {
    const int y = q / kColTileW, c = q % kColTileW;
    if (c < ncol) ob[(size_t)y * (h + 1) + k0 + c] = aout[c * so + y + y / P];
  }
}

// Pass 2 at n = 512 (nx = 256), 64 threads per column, three register
// radix-8 levels joined by two shared-memory transposes: level 1, thread t
// takes x[t + 64 r], an 8-point DFT over r and W_512^(t k2) give S[k2][t];
// level 2, thread (k2, u) takes S[k2][u + 8 r], an 8-point DFT over r and
// W_64^(u m2) give T[k2][m2][u]; level 3, thread (k2, m2) takes T[k2][m2][u],
// an 8-point DFT over u gives X[64 m1 + 8 m2 + k2].  A CTA of 256 threads does
// COLS (4 or 8) columns of one image, 4 at a time.  Shared strides are chosen
// so that a warp's accesses hit each bank at most twice (checked by
// enumeration for both column counts).
constexpr int kC512SI = 260, kC512SO = 580, kC512WB = 576;
constexpr size_t colfft512_smem(int cols) { return (size_t)(256 + cols * (kC512SI + kC512SO) + 4 * kC512WB) * 8; }
template <int COLS>
__global__ void __launch_bounds__(256) colfft512_kernel(const float2* __restrict__ inter, size_t inter_stride, int nx,
                                                        int n, int ip, int nvalid, const float2* __restrict__ twg,
                                                        float2* __restrict__ out) {
  constexpr int kC512Cols = COLS;
  extern __shared__ float2 fsm[];   // tw[256], in [8][SI], out [8][SO], work [4][WB]
  const int h = 256;
  const int tiles = (h + 1 + kC512Cols - 1) / kC512Cols;
  const int b = blockIdx.x / tiles, k0 = (blockIdx.x % tiles) * kC512Cols;
  float2* tw = fsm;
  float2* ain = tw + h;
  float2* aout = ain + kC512Cols * kC512SI;
  float2* work = aout + kC512Cols * kC512SO;
  for (int t = threadIdx.x; t < h; t += blockDim.x) tw[t] = twg[t];
  if (b >= nvalid) return;          // uniform per CTA
  const int ncol = min(kC512Cols, h + 1 - k0);
  const float2* ib = inter + (size_t)b * inter_stride;
  {
    // nx * 8 = 2,048 values, 8 per thread: all loads first, then the stores
    constexpr int kPer = 256 * kC512Cols / 256;
    float2 ld[kPer];
#pragma unroll
    for (int e = 0; e < kPer; ++e) {
      const int q = threadIdx.x + 256 * e, j = q / kC512Cols, c = q % kC512Cols;
      ld[e] = (c < ncol) ? __ldg(ib + (size_t)j * (h + 1) + k0 + c) : make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int e = 0; e < kPer; ++e) {
      const int q = threadIdx.x + 256 * e, j = q / kC512Cols, c = q % kC512Cols;
      ain[c * kC512SI + j] = ld[e];
    }
  }
  __syncthreads();
  const int grp = threadIdx.x >> 6, t = threadIdx.x & 63;
  float2* S = work + grp * kC512WB;
  const int g8 = t >> 3, l8 = t & 7;
  for (int c = grp; c < kC512Cols; c += 4) {   // COLS / 4 rounds, the same for every group
    float2 v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      int j = t + 64 * r - ip + nx;
      if (j >= n) j -= n;
      v[r] = (j < nx) ? ain[c * kC512SI + j] : make_float2(0.0f, 0.0f);
    }
    reg_fft_dif<8>(v, tw, n);
    static_for<0, 8>([&](auto kc) {
      constexpr int k2 = decltype(kc)::value;
      const float2 val = v[BrevT<k2, 3>::value];
      S[k2 * 68 + t] = k2 == 0 ? val : cmulf(tw_full(tw, t * k2, h), val);
    });
    __syncthreads();
    float2 w[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) w[r] = S[g8 * 68 + l8 + 8 * r];   // k2 = g8, u = l8
    reg_fft_dif<8>(w, tw, n);
    __syncthreads();                                             // S read; T overwrites it
    static_for<0, 8>([&](auto mc) {
      constexpr int m2 = decltype(mc)::value;
      const float2 val = w[BrevT<m2, 3>::value];
      S[g8 * 72 + 9 * m2 + l8] = m2 == 0 ? val : cmulf(tw_full(tw, 8 * l8 * m2, h), val);
    });
    __syncthreads();
    float2 qv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) qv[u] = S[g8 * 72 + 9 * l8 + u];   // k2 = g8, m2 = l8
    reg_fft_dif<8>(qv, tw, n);
    static_for<0, 8>([&](auto mc) {
      constexpr int m1 = decltype(mc)::value;
      const int y = 64 * m1 + 8 * l8 + g8;
      aout[c * kC512SO + y + (y >> 3)] = qv[BrevT<m1, 3>::value];
    });
    __syncthreads();                                             // before the next round's S
  }
  float2* ob = out + (size_t)b * n * (h + 1);
  for (int q = threadIdx.x; q < n * kC512Cols; q += blockDim.x) {
    const int y = q / kC512Cols, c = q % kC512Cols;
    if (c < ncol) ob[(size_t)y * (h + 1) + k0 + c] = aout[c * kC512SO + y + (y >> 3)];
  }
}

// ----------------------------------------------------------------------------
// RTSQ (rtsq.f:56-140) with QUADRI (quadri.f:83-150): in-plane rotation and
// shift of each image before PADD2, for RB 3F / RB 32F (bp3f.f:406-425).  One
// thread per output pixel; per image the host passes COS and SIN of
// THETA*DGR_TO_RAD (REAL) and the shifts, so every coordinate is the Fortran's.
struct RtsqParm {
  float cod, sid, shx, shy;
};

__device__ __forceinline__ float quadri_dev(float xx, float yy, int nx, int ny, const float* __restrict__ f) {
  float x = xx, y = yy;
  if (x < 1.0f) x = __fadd_rn(x, (float)((1 - __float2int_rz(x) / nx) * nx));
  if (x > __fadd_rn((float)nx, 0.5f)) x = __fadd_rn(fmodf(__fsub_rn(x, 1.0f), (float)nx), 1.0f);
  if (y < 1.0f) y = __fadd_rn(y, (float)((1 - __float2int_rz(y) / ny) * ny));
  if (y > __fadd_rn((float)ny, 0.5f)) y = __fadd_rn(fmodf(__fsub_rn(y, 1.0f), (float)ny), 1.0f);
  const int i = __float2int_rz(x), j = __float2int_rz(y);
  const float dx0 = __fsub_rn(x, (float)i), dy0 = __fsub_rn(y, (float)j);
  int ip1 = i + 1, im1 = i - 1, jp1 = j + 1, jm1 = j - 1;
  if (ip1 > nx) ip1 -= nx;
  if (im1 < 1) im1 += nx;
  if (jp1 > ny) jp1 -= ny;
  if (jm1 < 1) jm1 += ny;
#define QF(a, b) __ldg(f + (size_t)((b) - 1) * nx + ((a) - 1))
  const float f0 = QF(i, j);
  const float c1 = __fsub_rn(QF(ip1, j), f0);
  const float c2 = __fmul_rn(__fadd_rn(__fsub_rn(c1, f0), QF(im1, j)), 0.5f);
  const float c3 = __fsub_rn(QF(i, jp1), f0);
  const float c4 = __fmul_rn(__fadd_rn(__fsub_rn(c3, f0), QF(i, jm1)), 0.5f);
  const float dxb = __fsub_rn(dx0, 1.0f), dyb = __fsub_rn(dy0, 1.0f);
  const float hxc = (float)(int)copysignf(1.0f, dx0);
  const float hyc = (float)(int)copysignf(1.0f, dy0);
  int ic = __float2int_rz(__fadd_rn((float)i, hxc)), jc = __float2int_rz(__fadd_rn((float)j, hyc));
  if (ic > nx) ic -= nx; else if (ic < 1) ic += nx;
  if (jc > ny) jc -= ny; else if (jc < 1) jc += ny;
  float t = __fsub_rn(QF(ic, jc), f0);
  t = __fsub_rn(t, __fmul_rn(hxc, c1));
  t = __fsub_rn(t, __fmul_rn(__fmul_rn(hxc, __fsub_rn(hxc, 1.0f)), c2));
  t = __fsub_rn(t, __fmul_rn(hyc, c3));
  t = __fsub_rn(t, __fmul_rn(__fmul_rn(hyc, __fsub_rn(hyc, 1.0f)), c4));
  const float c5 = __fmul_rn(t, __fmul_rn(hxc, hyc));
#undef QF
  const float a = __fadd_rn(__fadd_rn(c1, __fmul_rn(dxb, c2)), __fmul_rn(dy0, c5));
  const float b = __fadd_rn(c3, __fmul_rn(dyb, c4));
  return __fadd_rn(__fadd_rn(f0, __fmul_rn(dx0, a)), __fmul_rn(dy0, b));
}

__global__ void rtsq_kernel(const float* __restrict__ in, float* __restrict__ out, int nx, int nimg,
                            const RtsqParm* __restrict__ prm) {
  const size_t total = (size_t)nimg * nx * nx;
  const int iycen = nx / 2 + 1, ixcen = nx / 2 + 1;
  const bool even = (nx % 2) == 0;
  const float r1 = (float)(-nx / 2);
  const float r2 = even ? __fsub_rn((float)(nx / 2), 1.0f) : (float)(nx / 2);
  const float re1 = even ? (float)(-nx) : (float)(-nx - 1), re2 = even ? (float)nx : (float)(nx + 1);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(q / ((size_t)nx * nx));
    const int p = (int)(q % ((size_t)nx * nx));
    const int ix = p % nx + 1, iy = p / nx + 1;
    const RtsqParm m = prm[b];
    const float shx = fmodf(m.shx, (float)nx), shy = fmodf(m.shy, (float)nx);
    const float fixcenmshx = __fsub_rn((float)(-ixcen), shx), fiycenmshy = __fsub_rn((float)(-iycen), shy);
    float yi = __fadd_rn((float)iy, fiycenmshy);
    if (yi < r1) yi = fminf(__fadd_rn(yi, re2), r2);
    if (yi > r2) yi = fmaxf(__fadd_rn(yi, re1), r1);
    const float ycod = __fadd_rn(__fmul_rn(yi, m.cod), (float)iycen);
    const float ysid = __fadd_rn(__fmul_rn(-yi, m.sid), (float)ixcen);
    float xi = __fadd_rn((float)ix, fixcenmshx);
    if (xi < r1) xi = fminf(__fadd_rn(xi, re2), r2);
    if (xi > r2) xi = fmaxf(__fadd_rn(xi, re1), r1);
    const float yold = __fadd_rn(__fmul_rn(xi, m.sid), ycod);
    const float xold = __fadd_rn(__fmul_rn(xi, m.cod), ysid);
    out[q] = quadri_dev(xold, yold, nx, nx, in + (size_t)b * nx * nx);
  }
}

// FP32 spectrum -> BF16 spectrum (reduced-precision storage mode)
__global__ void to_bf16_kernel(const float2* __restrict__ in, __nv_bfloat162* __restrict__ out, size_t count) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < count; q += (size_t)gridDim.x * blockDim.x)
    out[q] = __floats2bfloat162_rn(in[q].x, in[q].y);
}

template <bool BF16>
__device__ __forceinline__ float2 load_spec(const void* spec, size_t q) {
  // read-only during the insertion: non-coherent global loads (the
  // multi-class kernel's spectrum pointers come from shared memory)
  if (BF16) {
    __nv_bfloat162 v = __ldg(static_cast<const __nv_bfloat162*>(spec) + q);
    return make_float2(__low2float(v), __high2float(v));
  } else {
    return __ldg(static_cast<const float2*>(spec) + q);
  }
}

// ----------------------------------------------------------------------------
// Insert: ONELINE (oneline.f:38-200) for every row J of every slice.
// One warp per (slice, row); lanes stride over I.  Coordinates, rounding,
// bounds and table lookups follow the Fortran statement by statement with
// explicit round-to-nearest intrinsics (no contraction), so each tap's voxel
// and weight are bit-identical to the CPU restatement; the accumulation is an
// FP32 vector atomic per tap.
template <bool BF16>
__global__ void __launch_bounds__(512) insert_kernel(const void* __restrict__ spec, const SliceDesc* __restrict__ slices,
                                                     int nslices, int nx, const float* __restrict__ kbtab, float fltb,
                                                     float4* __restrict__ g0, float4* __restrict__ g1, int seg_map) {
  extern __shared__ float tab[];
  for (int i = threadIdx.x; i < 5000; i += blockDim.x) tab[i] = kbtab[i];
  __syncthreads();

  const int N = 2 * nx;          // callee N of ONELINE
  const int N2 = nx;             // callee N2 of ONELINE
  const int LN2 = 2;
  const float fN = (float)N;
  const int lane = threadIdx.x & 31;
  const int warps_per_block = blockDim.x >> 5;
  // work item = 32 consecutive pixels (one warp) of one row of one slice,
  // slice-major: the resident warps cover about one slice at a time, so the
  // voxels they update (one thick central plane) stay resident in L2
  const int nseg = seg_map ? (nx + 1 + 31) >> 5 : 1;
  const long long per_slice = (long long)N * nseg;
  const long long nitems = (long long)nslices * per_slice;
  const size_t rowlen = (size_t)(nx + 1);
  const size_t plane = (size_t)N * rowlen;

  for (long long item = (long long)blockIdx.x * warps_per_block + (threadIdx.x >> 5); item < nitems;
       item += (long long)gridDim.x * warps_per_block) {
    const int s = (int)(item / per_slice);
    const int rem = (int)(item % per_slice);
    const int J = rem / nseg - nx + 1;  // J = -NX+1 .. NX
    const int I0 = (rem % nseg) << 5;
    if (I0 * I0 + J * J >= N * N / 4) continue;   // the whole segment lies outside the disk
    const int Iend = seg_map ? min(I0 + 32, N2 + 1) : N2 + 1;
    const SliceDesc sd = slices[s];
    float4* G = sd.grid ? g1 : g0;
    const int JP = (J >= 0) ? J : N + J;
    const size_t specrow = (size_t)sd.img * plane + (size_t)JP * rowlen;
    const float fJ = (float)J;
    const float j3 = __fmul_rn(fJ, sd.dm[3]), j4 = __fmul_rn(fJ, sd.dm[4]), j5 = __fmul_rn(fJ, sd.dm[5]);
    for (int I = I0 + lane; I < Iend; I += 32) {
      if (!((I * I + J * J) < (N * N / 4)) || (I == 0 && J < 0)) continue;
      const float fI = (float)I;
      float xnew = __fadd_rn(__fmul_rn(fI, sd.dm[0]), j3);
      float ynew = __fadd_rn(__fmul_rn(fI, sd.dm[1]), j4);
      float znew = __fadd_rn(__fmul_rn(fI, sd.dm[2]), j5);
      const float2 sp = load_spec<BF16>(spec, specrow + I);
      // SPIDER forward sign = conjugate of the cuFFT R2C output
      float br = sp.x, bi = -sp.y;
      if (xnew < 0.0f) {
        xnew = -xnew; ynew = -ynew; znew = -znew;
        bi = -bi;
      }
      const int ixn = __float2int_rz(__fadd_rn(__fadd_rn(xnew, 0.5f), fN)) - N;
      const int iyn = __float2int_rz(__fadd_rn(__fadd_rn(ynew, 0.5f), fN)) - N;
      const int izn = __float2int_rz(__fadd_rn(__fadd_rn(znew, 0.5f), fN)) - N;
      if (!(ixn <= (N2 - LN2 - 1) && iyn >= (-N2 + 2 + LN2) && iyn <= (N2 - LN2 - 1) &&
            izn >= (-N2 + 2 + LN2) && izn <= (N2 - LN2 - 1)))
        continue;
      float tz[5], ty[5], tx[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        tz[l] = tab[nint_pos(__fmul_rn(fabsf(__fsub_rn(znew, (float)(izn + l - 2))), fltb))];
        ty[l] = tab[nint_pos(__fmul_rn(fabsf(__fsub_rn(ynew, (float)(iyn + l - 2))), fltb))];
        tx[l] = tab[nint_pos(__fmul_rn(fabsf(__fsub_rn(xnew, (float)(ixn + l - 2))), fltb))];
      }
      if (ixn >= 0) {
        const int lb = -min(ixn, LN2);
#pragma unroll
        for (int lz = 0; lz < 5; ++lz) {
          if (tz[lz] == 0.0f) continue;
          const int izp = izn + lz - 2;
          const int iza = (izp >= 0) ? izp : N + izp;
#pragma unroll
          for (int ly = 0; ly < 5; ++ly) {
            const float tyz = __fmul_rn(ty[ly], tz[lz]);
            if (tyz == 0.0f) continue;
            const int iyp = iyn + ly - 2;
            const int iya = (iyp >= 0) ? iyp : N + iyp;
            float4* row = G + ((size_t)iza * N + iya) * rowlen;
#pragma unroll
            for (int lx = 0; lx < 5; ++lx) {
              if (lx - 2 < lb) continue;
              const float wg = __fmul_rn(tx[lx], tyz);
              if (wg != 0.0f)
                atomicAdd(row + (ixn + lx - 2), make_float4(__fmul_rn(br, wg), __fmul_rn(bi, wg), wg, 0.0f));
            }
          }
        }
      }
      if (ixn < LN2) {  // reflected points (oneline.f:118-150)
#pragma unroll
        for (int lz = 0; lz < 5; ++lz) {
          if (tz[lz] == 0.0f) continue;
          const int izp = izn + lz - 2;
          const int izt = (izp > 0) ? N - izp : -izp;
#pragma unroll
          for (int ly = 0; ly < 5; ++ly) {
            const float tyz = __fmul_rn(ty[ly], tz[lz]);
            if (tyz == 0.0f) continue;
            const int iyp = iyn + ly - 2;
            const int iyt = (iyp > 0) ? N - iyp : -iyp;
            float4* row = G + ((size_t)izt * N + iyt) * rowlen;
#pragma unroll
            for (int lx = 0; lx < 2; ++lx) {     // ixp = ixn-2 .. -1
              const int ixp = ixn + lx - 2;
              if (ixp > -1) continue;
              const float wg = __fmul_rn(tx[lx], tyz);
              if (wg != 0.0f)
                atomicAdd(row + (-ixp), make_float4(__fmul_rn(br, wg), __fmul_rn(-bi, wg), wg, 0.0f));
            }
          }
        }
      }
    }
  }
}

// ----------------------------------------------------------------------------
// Insert, lanes over the x taps.  A warp takes one row J of one slice and walks
// it six pixels at a time: lanes 5g..5g+4 share pixel I0+g and lane 5g+LX owns
// the x tap LX, so for each (LY, LZ) pair the five vector atomics of a pixel
// land on 80 contiguous bytes of one grid row (the x axis is the fastest) and
// the L2 receives one or two line requests per pixel instead of five scattered
// ones.  A lane whose tap falls below x = 0 (IXN < LN2) adds the reflected
// point instead (oneline.f:118-150), so every lane issues exactly one atomic
// per (LY, LZ).  Every voxel and weight is computed as in insert_kernel.
//
// Rows are handed out in slice-major order by a work counter (one atomic per
// row and warp) rather than by a fixed grid stride: the warps then stay on
// neighbouring rows of the same few slices for the whole launch, and the
// voxels they update stay resident in L2 (with a fixed stride fast and slow
// warps drift apart and the set of slices in flight grows with the launch).
template <bool BF16>
__global__ void __launch_bounds__(512) insert_xlane_kernel(const void* __restrict__ spec,
                                                           const SliceDesc* __restrict__ slices, int nslices, int nx,
                                                           const float* __restrict__ kbtab, float fltb,
                                                           float4* __restrict__ g0, float4* __restrict__ g1,
                                                           unsigned long long* __restrict__ work) {
  extern __shared__ float tab[];
  for (int i = threadIdx.x; i < 5000; i += blockDim.x) tab[i] = kbtab[i];
  __syncthreads();

  const int N = 2 * nx, N2 = nx, LN2 = 2;
  const int NN4 = N * N / 4;
  const float fN = (float)N;
  const int lane = threadIdx.x & 31;
  const int g = lane / 5;           // pixel of the group of six (g = 6: idle lanes 30, 31)
  const int lx = lane - 5 * g;      // x tap 0..4
  const long long nitems = (long long)nslices * N;
  const size_t rowlen = (size_t)(nx + 1);
  const size_t plane = (size_t)N * rowlen;

  for (;;) {
    unsigned long long it = 0;
    if (lane == 0) it = atomicAdd(work, 1ull);
    const long long item = (long long)__shfl_sync(0xffffffffu, it, 0);
    if (item >= nitems) break;
    const int s = (int)(item / N);
    const int J = (int)(item % N) - nx + 1;  // J = -NX+1 .. NX
    const SliceDesc sd = slices[s];
    float4* G = sd.grid ? g1 : g0;
    const int JP = (J >= 0) ? J : N + J;
    const size_t specrow = (size_t)sd.img * plane + (size_t)JP * rowlen;
    const float fJ = (float)J;
    const float j3 = __fmul_rn(fJ, sd.dm[3]), j4 = __fmul_rn(fJ, sd.dm[4]), j5 = __fmul_rn(fJ, sd.dm[5]);
    for (int I0 = 0; I0 <= N2 && I0 * I0 + J * J < NN4; I0 += 6) {
      const int I = I0 + g;
      if (g == 6 || I > N2 || !((I * I + J * J) < NN4) || (I == 0 && J < 0)) continue;
      const float fI = (float)I;
      float xnew = __fadd_rn(__fmul_rn(fI, sd.dm[0]), j3);
      float ynew = __fadd_rn(__fmul_rn(fI, sd.dm[1]), j4);
      float znew = __fadd_rn(__fmul_rn(fI, sd.dm[2]), j5);
      const float2 sp = load_spec<BF16>(spec, specrow + I);
      float br = sp.x, bi = -sp.y;   // SPIDER forward sign = conjugate of the cuFFT R2C output
      if (xnew < 0.0f) {
        xnew = -xnew; ynew = -ynew; znew = -znew;
        bi = -bi;
      }
      const int ixn = __float2int_rz(__fadd_rn(__fadd_rn(xnew, 0.5f), fN)) - N;
      const int iyn = __float2int_rz(__fadd_rn(__fadd_rn(ynew, 0.5f), fN)) - N;
      const int izn = __float2int_rz(__fadd_rn(__fadd_rn(znew, 0.5f), fN)) - N;
      if (!(ixn <= (N2 - LN2 - 1) && iyn >= (-N2 + 2 + LN2) && iyn <= (N2 - LN2 - 1) &&
            izn >= (-N2 + 2 + LN2) && izn <= (N2 - LN2 - 1)))
        continue;
      float tz[5], ty[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        tz[l] = tab[nint_pos(__fmul_rn(fabsf(__fsub_rn(znew, (float)(izn + l - 2))), fltb))];
        ty[l] = tab[nint_pos(__fmul_rn(fabsf(__fsub_rn(ynew, (float)(iyn + l - 2))), fltb))];
      }
      const int ixp = ixn + lx - 2;
      const float tx = tab[nint_pos(__fmul_rn(fabsf(__fsub_rn(xnew, (float)ixp)), fltb))];
      if (tx == 0.0f) continue;
      // main tap at (ixp, iyp, izp), or for ixp < 0 the reflected point
      // (-ixp, -iyp, -izp) with the conjugate value
      const bool refl = ixp < 0;
      const float bis = refl ? -bi : bi;
      const int ixa = refl ? -ixp : ixp;
#pragma unroll
      for (int lz = 0; lz < 5; ++lz) {
        if (tz[lz] == 0.0f) continue;
        const int izp = izn + lz - 2;
        const int iza = refl ? ((izp > 0) ? N - izp : -izp) : ((izp >= 0) ? izp : N + izp);
#pragma unroll
        for (int ly = 0; ly < 5; ++ly) {
          const float tyz = __fmul_rn(ty[ly], tz[lz]);
          if (tyz == 0.0f) continue;
          const int iyp = iyn + ly - 2;
          const int iya = refl ? ((iyp > 0) ? N - iyp : -iyp) : ((iyp >= 0) ? iyp : N + iyp);
          const float wg = __fmul_rn(tx, tyz);
          if (wg != 0.0f)
            atomicAdd(G + ((size_t)iza * N + iya) * rowlen + ixa,
                      make_float4(__fmul_rn(br, wg), __fmul_rn(bis, wg), wg, 0.0f));
        }
      }
    }
  }
}

// ----------------------------------------------------------------------------
// Insert, four lanes per pixel over the nonzero taps.  The generalised
// Kaiser-Bessel table is zero from distance ~1.8 on (0.9 of the two-voxel
// half width), so along each axis the tap at offset -2 is nonzero only when
// the coordinate lies more than 0.2 below its nearest voxel and the tap at +2
// only when it lies more than 0.2 above: at most four of the five taps are
// nonzero, in the window [-2, 1] or [-1, 2].  A warp takes one row J of one
// slice, eight pixels at a time; lanes 4g..4g+3 share pixel I0+g, lane 4g+q
// owns x tap XS+q of the window, and each lane loops over the 4 x 4 (Y, Z)
// window.  Window starts are read from the same table lookups the taps use
// (offset -2 nonzero => window [-2, 1]); the host verifies that the table is
// zero beyond distance 2, which makes the window exact.  Compared with five
// lanes over all 5 x 5 (Y, Z) taps this issues 2 instead of 4.2 atomic
// instructions per pixel and uses every lane.  Each voxel and weight (and
// the reflected points of oneline.f:118-150) is computed as in insert_kernel;
// taps outside the window have zero weight, which the reference skips too.
__device__ __forceinline__ float kb_tap(const float* tab, float v, int k, float fltb) {
  return tab[nint_pos(__fmul_rn(fabsf(__fsub_rn(v, (float)k)), fltb))];
}
// The same lookup in a table cut after entry `last`, which (like every entry
// after it) is zero: for a table kb_window4_ok accepts, the result is the
// same as kb_tap's.
__device__ __forceinline__ float kb_tap_cut(const float* tab, float v, int k, float fltb, int last) {
  return tab[min(nint_pos(__fmul_rn(fabsf(__fsub_rn(v, (float)k)), fltb)), last)];
}

// G[i] += v as one 16-byte reduction in L2 (red.global.add.v4.f32).  The
// address is converted to the global window explicitly: the multi-class
// kernel takes its grid pointers from shared memory, and on such a generic
// pointer atomicAdd(float4*) was not compiled to the vector reduction
// (measured: 1.9x the instructions and no L2 reduction requests; 205
// against 156 ms for the same 10,000 images at 256^3).
__device__ __forceinline__ void red_add_v4(float4* p, float4 v) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(__cvta_generic_to_global(p)), "f"(v.x),
               "f"(v.y), "f"(v.z), "f"(v.w));
}

// The largest m >= 0 with m * m < rem (rem > 0).
__device__ __forceinline__ int isqrt_below(int rem) {
  // approximate square root (no IEEE slow path); the two loops make m exact
  float f;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(f) : "f"((float)(rem - 1)));
  int m = (int)f;
  while (m > 0 && m * m >= rem) --m;
  while ((m + 1) * (m + 1) < rem) ++m;
  return m;
}

// One line of one slice, eight pixels at a time, as described above: the
// body of insert_x4_kernel and insert_mc_kernel.  Line r (0 <= r < N) is row
// J = r - NX + 1 (pixels consecutive in I), or, for a slice whose
// descriptor says cols, half of column I = r / 2 (pixels consecutive in J:
// J >= 0 for even r, J < 0 for odd r).  The eight pixels of a step then lie
// along the slice's second axis (DMS(4:6)) instead of its first (DMS(1:3)).
// The host picks, per slice, the axis whose z component is smaller: a step
// along z puts the eight pixels' atomics in eight grid planes 2 MB apart
// (measured at 256^3: rows along z 45.5k images/s, along x or y 65k).  Each
// pixel's taps and weights are the same in both orders.
template <bool BF16, int CUT = 0>
__device__ __forceinline__ void insert_line_x4(const void* __restrict__ spec, const SliceDesc& sd,
                                               float4* __restrict__ G, int r, int nx, const float* tab, float fltb,
                                               int g, int q, int gl) {
  // CUT > 0: the table holds entries 0..CUT-1 only (see kb_tap_cut)
  auto tap = [&](float v, int k) { return CUT ? kb_tap_cut(tab, v, k, fltb, CUT - 1) : kb_tap(tab, v, k, fltb); };
  const int N = 2 * nx, N2 = nx, LN2 = 2;
  const int NN4 = N * N / 4;
  const float fN = (float)N;
  const size_t rowlen = (size_t)(nx + 1);
  const size_t plane = (size_t)N * rowlen;
  const size_t spec0 = (size_t)sd.img * plane;
  // pixel k of the line: (I, J) = (i0 + di * k, j0 + dj * k), k < cnt; the
  // pixels inside the half disc of oneline.f's loops (I >= 0, I*I + J*J <
  // NN4, no I = 0 with J < 0)
  int i0, j0, di, dj, cnt;
  if (!sd.cols) {
    j0 = r - nx + 1; i0 = 0; di = 1; dj = 0;                 // J = -NX+1 .. NX
    cnt = (j0 * j0 < NN4) ? isqrt_below(NN4 - j0 * j0) + 1 : 0;
  } else {
    i0 = r >> 1; di = 0;                                      // I = 0 .. NX-1
    const int jm = isqrt_below(NN4 - i0 * i0);
    if (r & 1) { j0 = -1; dj = -1; cnt = i0 == 0 ? 0 : jm; }
    else { j0 = 0; dj = 1; cnt = jm + 1; }
  }
#pragma unroll 1
  for (int k0 = 0; k0 < cnt; k0 += 8) {   // warp-uniform
    const int k = k0 + g;
    const int I = i0 + di * k, J = j0 + dj * k;
    bool ok = k < cnt && !(I == 0 && J < 0);
    const float fI = (float)I, fJ = (float)J;
    float xnew = __fadd_rn(__fmul_rn(fI, sd.dm[0]), __fmul_rn(fJ, sd.dm[3]));
    float ynew = __fadd_rn(__fmul_rn(fI, sd.dm[1]), __fmul_rn(fJ, sd.dm[4]));
    float znew = __fadd_rn(__fmul_rn(fI, sd.dm[2]), __fmul_rn(fJ, sd.dm[5]));
    float br = 0.0f, bi = 0.0f;
    if (ok) {
      const int JP = (J >= 0) ? J : N + J;
      const float2 sp = load_spec<BF16>(spec, spec0 + (size_t)JP * rowlen + I);
      br = sp.x;
      bi = -sp.y;   // SPIDER forward sign = conjugate of the cuFFT R2C output
    }
    if (xnew < 0.0f) {
      xnew = -xnew; ynew = -ynew; znew = -znew;
      bi = -bi;
    }
    const int ixn = __float2int_rz(__fadd_rn(__fadd_rn(xnew, 0.5f), fN)) - N;
    const int iyn = __float2int_rz(__fadd_rn(__fadd_rn(ynew, 0.5f), fN)) - N;
    const int izn = __float2int_rz(__fadd_rn(__fadd_rn(znew, 0.5f), fN)) - N;
    ok = ok && ixn <= (N2 - LN2 - 1) && iyn >= (-N2 + 2 + LN2) && iyn <= (N2 - LN2 - 1) &&
         izn >= (-N2 + 2 + LN2) && izn <= (N2 - LN2 - 1);
    if (!ok) { xnew = ynew = znew = 0.0f; }   // keeps the lookups below in range; no taps follow
    const int ix0 = ok ? ixn : 0, iy0 = ok ? iyn : 0, iz0 = ok ? izn : 0;
    const int xs = tap(xnew, ix0 - 2) != 0.0f ? ix0 - 2 : ix0 - 1;
    const int ys = tap(ynew, iy0 - 2) != 0.0f ? iy0 - 2 : iy0 - 1;
    const int zs = tap(znew, iz0 - 2) != 0.0f ? iz0 - 2 : iz0 - 1;
    const float tx = tap(xnew, xs + q);
    const float tyq = tap(ynew, ys + q);
    const float tzq = tap(znew, zs + q);
    float ty[4], tz[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      ty[l] = __shfl_sync(0xffffffffu, tyq, gl + l);
      tz[l] = __shfl_sync(0xffffffffu, tzq, gl + l);
    }
    if (!ok || tx == 0.0f) continue;
    // main tap at (ixp, iyp, izp), or for ixp < 0 the reflected point
    // (-ixp, -iyp, -izp) with the conjugate value
    const int ixp = xs + q;
    const bool refl = ixp < 0;
    const float bis = refl ? -bi : bi;
    const int ixa = refl ? -ixp : ixp;
#pragma unroll
    for (int lz = 0; lz < 4; ++lz) {
      if (tz[lz] == 0.0f) continue;
      const int izp = zs + lz;
      const int iza = refl ? ((izp > 0) ? N - izp : -izp) : ((izp >= 0) ? izp : N + izp);
#pragma unroll
      for (int ly = 0; ly < 4; ++ly) {
        const float tyz = __fmul_rn(ty[ly], tz[lz]);
        if (tyz == 0.0f) continue;
        const int iyp = ys + ly;
        const int iya = refl ? ((iyp > 0) ? N - iyp : -iyp) : ((iyp >= 0) ? iyp : N + iyp);
        const float wg = __fmul_rn(tx, tyz);
        if (wg != 0.0f)
          red_add_v4(G + ((size_t)iza * N + iya) * rowlen + ixa,
                     make_float4(__fmul_rn(br, wg), __fmul_rn(bis, wg), wg, 0.0f));
      }
    }
  }
}

// 48 registers: 0.6% faster at 256^3 than the compiler's own choice of 64
// (measured), with no spills; launches use at most 512 threads.
template <bool BF16>
__global__ void __maxnreg__(48) insert_x4_kernel(const void* __restrict__ spec, const SliceDesc* __restrict__ slices,
                                                 int nslices, int nx, const float* __restrict__ kbtab, float fltb,
                                                 float4* __restrict__ g0, float4* __restrict__ g1,
                                                 unsigned long long* __restrict__ work) {
  extern __shared__ float tab[];
  for (int i = threadIdx.x; i < 5000; i += blockDim.x) tab[i] = kbtab[i];
  __syncthreads();

  const int N = 2 * nx;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2;          // pixel of the group of eight
  const int q = lane & 3;           // x tap of the window
  const int gl = lane & ~3;         // first lane of the group
  const long long nitems = (long long)nslices * N;

  for (;;) {
    unsigned long long it = 0;
    if (lane == 0) it = atomicAdd(work, 1ull);
    const long long item = (long long)__shfl_sync(0xffffffffu, it, 0);
    if (item >= nitems) break;
    const int s = (int)(item / N);
    const SliceDesc sd = slices[s];
    insert_line_x4<BF16>(spec, sd, sd.grid ? g1 : g0, (int)(item % N), nx, tab, fltb, g, q, gl);
  }
}

// ----------------------------------------------------------------------------
// Insert for several classes of different box sizes in one launch (BP 32F of
// each class, the image loop bp32f.f:802-913 run for all classes together).
// The work items are the rows of every class's slices, class after class;
// a row finds its class by its item index and takes that class's box size,
// table (one shared-memory copy per distinct box size), spectra and grids.
// Each row is inserted exactly as insert_x4_kernel inserts it.
struct McClass {
  const void* spec;            // spectra of the class's images in this launch
  const SliceDesc* slices;     // the class's slice descriptors
  float4* g0;                  // grids the taps go to (half-set 1 and 2)
  float4* g1;
  long long item0;             // first work item (row) of the class
  int nx, nslices, tab, pad;   // box size, slices, table index
};
static_assert(sizeof(McClass) == 56, "class descriptor is 56 bytes");
constexpr int kMcMaxClass = 16, kMcMaxTab = 8;
// Entries of a table the multi-class kernel keeps: a table kb_window4_ok
// accepts is zero from floor(2 * FLTB) - 1 = 3331 on (FLTB = 4999/3), so
// 3,332 entries (13 KB) hold every nonzero value and a zero to clamp to;
// eight tables then fit two CTAs per SM.
constexpr int kMcTab = 3332;

template <bool BF16>
__global__ void __launch_bounds__(512) insert_mc_kernel(const McClass* __restrict__ cls, int ncls, long long nitems,
                                                        const float* __restrict__ tabs, const float* __restrict__ fltbs,
                                                        int ntab, unsigned long long* __restrict__ work) {
  extern __shared__ float tab[];   // [ntab][kMcTab]
  __shared__ McClass sc[kMcMaxClass];
  __shared__ float sfl[kMcMaxTab];
  for (int i = threadIdx.x; i < kMcTab * ntab; i += blockDim.x) tab[i] = tabs[(i / kMcTab) * 5000 + i % kMcTab];
  if (threadIdx.x < ncls) sc[threadIdx.x] = cls[threadIdx.x];
  if (threadIdx.x < ntab) sfl[threadIdx.x] = fltbs[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3, gl = lane & ~3;
  for (;;) {
    unsigned long long it = 0;
    if (lane == 0) it = atomicAdd(work, 1ull);
    const long long item = (long long)__shfl_sync(0xffffffffu, it, 0);
    if (item >= nitems) break;
    int c = 0;
    while (c + 1 < ncls && sc[c + 1].item0 <= item) ++c;
    const McClass& C = sc[c];
    const int N = 2 * C.nx;
    const long long local = item - C.item0;
    const SliceDesc sd = C.slices[local / N];
    insert_line_x4<BF16, kMcTab>(C.spec, sd, sd.grid ? C.g1 : C.g0, (int)(local % N), C.nx, tab + kMcTab * C.tab,
                                 sfl[C.tab], g, q, gl);
  }
}

// True when the table is zero for every distance >= 2 (index nint(2*fltb)
// and above, less one for rounding), the condition under which at most four
// consecutive taps of the five are nonzero (insert_x4_kernel).
static bool kb_window4_ok(const KBTab& kb) {
  const int i0 = std::max(0, (int)std::floor(2.0 * kb.fltb) - 1);
  for (int i = i0; i < 5000; ++i)
    if (kb.tab[i] != 0.0f) return false;
  return true;
}

// ----------------------------------------------------------------------------
// Insert, tile-privatised form.  A CTA takes a 16 (I) x 8 (J) tile of pixels
// of one slice; 256 threads = 2 per pixel, splitting the z taps (LZ = -2..0
// and 1..2).  The tile's taps land in a thin slab whose bounding box (at most
// 7182 voxels over all orientations for this tile shape) is accumulated in
// shared memory with FP32 shared atomics and flushed with one global vector
// atomic per touched voxel, instead of one per tap (each voxel receives ~13
// taps per image).  Tiles whose pixels straddle the x = 0 flip (two separate
// clusters) or whose box would not fit use direct global atomics; reflected
// taps (IXN < LN2, oneline.f:118-150) always do.  Every tap's voxel and weight
// are computed exactly as in insert_kernel.  With FX the box holds int32
// fixed point (scaled per tile by the largest spectrum value) and the
// shared adds are native integer atomics instead of float ones.
constexpr int kTileI = 16, kTileJ = 8, kTileCap = 7296;

// shared-memory reduction without a returned value (no scoreboard wait)
__device__ __forceinline__ void red_shared_add(float* p, float v) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}

template <bool BF16, bool FX>
__global__ void __launch_bounds__(256, 2) insert_tile_kernel(const void* __restrict__ spec, const SliceDesc* __restrict__ slices,
                                                             int nslices, int nx, const float* __restrict__ tab, float fltb,
                                                             float4* __restrict__ g0, float4* __restrict__ g1) {
  extern __shared__ float sm[];
  float* s_re = sm;
  float* s_im = sm + kTileCap;
  float* s_w = sm + 2 * kTileCap;
  int* f_re = reinterpret_cast<int*>(s_re);   // FX: the same words as int32 fixed point
  int* f_im = reinterpret_cast<int*>(s_im);
  int* f_w = reinterpret_cast<int*>(s_w);
  __shared__ int s_box[8];   // xmin,ymin,zmin,-xmax,-ymax,-zmax, flipped-any, unflipped-any
  __shared__ unsigned s_vmax; // FX: max |Re|, |Im| of the tile's spectrum values (float bits)

  const int N = 2 * nx, N2 = nx, LN2 = 2;
  const float fN = (float)N;
  const size_t rowlen = (size_t)(nx + 1);
  const size_t plane = (size_t)N * rowlen;
  const int tiles_i = (nx + 1 + kTileI - 1) / kTileI;
  const int tiles_j = (N + kTileJ - 1) / kTileJ;
  const int tiles_per_slice = tiles_i * tiles_j;
  const long long nitems = (long long)nslices * tiles_per_slice;
  const int t = threadIdx.x;
  const int p = t & 127, half = t >> 7;
  const int lz0 = half ? 3 : 0, lz1 = half ? 5 : 3;

  for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int s = (int)(item / tiles_per_slice);
    const int tl = (int)(item % tiles_per_slice);
    const int I0 = (tl % tiles_i) * kTileI;
    const int J0 = (tl / tiles_i) * kTileJ - nx + 1;
    // skip tiles entirely outside the disk I^2 + J^2 < NX^2
    {
      const int ci = I0, cj = (J0 > 0) ? J0 : ((J0 + kTileJ - 1 < 0) ? J0 + kTileJ - 1 : 0);
      if (ci * ci + cj * cj >= N * N / 4) continue;   // uniform across the CTA
    }
    const SliceDesc sd = slices[s];
    float4* G = sd.grid ? g1 : g0;
    const int I = I0 + (p & (kTileI - 1));
    const int J = J0 + (p >> 4);
    bool ok = (I <= N2) && (J <= nx) && ((I * I + J * J) < (N * N / 4)) && !(I == 0 && J < 0);
    float xnew = 0.f, ynew = 0.f, znew = 0.f, br = 0.f, bi = 0.f;
    int ixn = 0, iyn = 0, izn = 0;
    bool flipped = false;
    if (ok) {
      const float fI = (float)I, fJ = (float)J;
      xnew = __fadd_rn(__fmul_rn(fI, sd.dm[0]), __fmul_rn(fJ, sd.dm[3]));
      ynew = __fadd_rn(__fmul_rn(fI, sd.dm[1]), __fmul_rn(fJ, sd.dm[4]));
      znew = __fadd_rn(__fmul_rn(fI, sd.dm[2]), __fmul_rn(fJ, sd.dm[5]));
      const int JP = (J >= 0) ? J : N + J;
      const float2 sp = load_spec<BF16>(spec, (size_t)sd.img * plane + (size_t)JP * rowlen + I);
      br = sp.x;
      bi = -sp.y;
      if (xnew < 0.0f) {
        xnew = -xnew; ynew = -ynew; znew = -znew;
        bi = -bi;
        flipped = true;
      }
      ixn = __float2int_rz(__fadd_rn(__fadd_rn(xnew, 0.5f), fN)) - N;
      iyn = __float2int_rz(__fadd_rn(__fadd_rn(ynew, 0.5f), fN)) - N;
      izn = __float2int_rz(__fadd_rn(__fadd_rn(znew, 0.5f), fN)) - N;
      ok = (ixn <= (N2 - LN2 - 1) && iyn >= (-N2 + 2 + LN2) && iyn <= (N2 - LN2 - 1) &&
            izn >= (-N2 + 2 + LN2) && izn <= (N2 - LN2 - 1));
    }
    // tile bounding box of the main taps
    if (t < 8) s_box[t] = (t < 6) ? 0x7fffffff : 0;
    if (FX && t == 0) s_vmax = 0u;
    __syncthreads();
    if (FX && ok) atomicMax(&s_vmax, __float_as_uint(fmaxf(fabsf(br), fabsf(bi))));
    if (ok && half == 0) {
      atomicMin(&s_box[0], ixn);
      atomicMin(&s_box[1], iyn);
      atomicMin(&s_box[2], izn);
      atomicMin(&s_box[3], -ixn);
      atomicMin(&s_box[4], -iyn);
      atomicMin(&s_box[5], -izn);
      if (flipped) s_box[6] = 1; else s_box[7] = 1;
    }
    __syncthreads();
    const int bx0 = max(s_box[0] - 2, 0), by0 = s_box[1] - 2, bz0 = s_box[2] - 2;
    const int bx = -s_box[3] + 2 - bx0 + 1, by = -s_box[4] + 2 - by0 + 1, bz = -s_box[5] + 2 - bz0 + 1;
    const bool any = s_box[0] != 0x7fffffff;
    const bool mixed = s_box[6] && s_box[7];
    const bool priv = any && !mixed && (long long)bx * by * bz <= kTileCap;
    __syncthreads();      // every thread has read the box before it is reused
    if (!any) continue;   // uniform: no valid pixel in this tile
    const int bsize = priv ? bx * by * bz : 0;
    // FX scales: a voxel receives from at most 64 pixels of one tile (the
    // table is zero beyond 1.8 voxels, so a voxel's support in the slice
    // plane is at most the largest cross-section of a 3.6-voxel cube, ~22
    // pixels), each adding a weight <= 1 times a value <= vmax
    const float vmax = FX ? __uint_as_float(s_vmax) : 0.0f;
    const float sc_v = (FX && vmax > 0.0f) ? 0.95f * 2147483648.0f / (64.0f * vmax) : 0.0f;
    const float sc_w = 0.95f * 2147483648.0f / 64.0f;
    if (priv) {
      for (int q = t; q < bsize; q += blockDim.x) {
        if (FX) { f_re[q] = 0; f_im[q] = 0; f_w[q] = 0; }
        else { s_re[q] = 0.f; s_im[q] = 0.f; s_w[q] = 0.f; }
      }
      __syncthreads();
    }
    if (ok) {
      float tz[5], ty[5], tx[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        tz[l] = __ldg(tab + nint_pos(__fmul_rn(fabsf(__fsub_rn(znew, (float)(izn + l - 2))), fltb)));
        ty[l] = __ldg(tab + nint_pos(__fmul_rn(fabsf(__fsub_rn(ynew, (float)(iyn + l - 2))), fltb)));
        tx[l] = __ldg(tab + nint_pos(__fmul_rn(fabsf(__fsub_rn(xnew, (float)(ixn + l - 2))), fltb)));
      }
      const int lb = -min(ixn, LN2);
#pragma unroll
      for (int lz = 0; lz < 5; ++lz) {
        if (lz < lz0 || lz >= lz1 || tz[lz] == 0.0f) continue;
        const int izp = izn + lz - 2;
#pragma unroll
        for (int ly = 0; ly < 5; ++ly) {
          const float tyz = __fmul_rn(ty[ly], tz[lz]);
          if (tyz == 0.0f) continue;
          const int iyp = iyn + ly - 2;
          if (priv) {
            const int rowq = ((izp - bz0) * by + (iyp - by0)) * bx - bx0;
#pragma unroll
            for (int lx = 0; lx < 5; ++lx) {
              if (lx - 2 < lb) continue;
              const float wg = __fmul_rn(tx[lx], tyz);
              if (wg != 0.0f) {
                const int q = rowq + ixn + lx - 2;
                if (FX) {
                  atomicAdd(f_re + q, __float2int_rn(__fmul_rn(br, wg) * sc_v));
                  atomicAdd(f_im + q, __float2int_rn(__fmul_rn(bi, wg) * sc_v));
                  atomicAdd(f_w + q, __float2int_rn(wg * sc_w));
                } else {
                  red_shared_add(s_re + q, __fmul_rn(br, wg));
                  red_shared_add(s_im + q, __fmul_rn(bi, wg));
                  red_shared_add(s_w + q, wg);
                }
              }
            }
          } else {
            const int iza = (izp >= 0) ? izp : N + izp;
            const int iya = (iyp >= 0) ? iyp : N + iyp;
            float4* row = G + ((size_t)iza * N + iya) * rowlen;
#pragma unroll
            for (int lx = 0; lx < 5; ++lx) {
              if (lx - 2 < lb) continue;
              const float wg = __fmul_rn(tx[lx], tyz);
              if (wg != 0.0f)
                atomicAdd(row + (ixn + lx - 2), make_float4(__fmul_rn(br, wg), __fmul_rn(bi, wg), wg, 0.0f));
            }
          }
        }
      }
      if (ixn < LN2) {  // reflected points (oneline.f:118-150), direct
#pragma unroll
        for (int lz = 0; lz < 5; ++lz) {
          if (lz < lz0 || lz >= lz1 || tz[lz] == 0.0f) continue;
          const int izp = izn + lz - 2;
          const int izt = (izp > 0) ? N - izp : -izp;
#pragma unroll
          for (int ly = 0; ly < 5; ++ly) {
            const float tyz = __fmul_rn(ty[ly], tz[lz]);
            if (tyz == 0.0f) continue;
            const int iyp = iyn + ly - 2;
            const int iyt = (iyp > 0) ? N - iyp : -iyp;
            float4* row = G + ((size_t)izt * N + iyt) * rowlen;
#pragma unroll
            for (int lx = 0; lx < 2; ++lx) {
              const int ixp = ixn + lx - 2;
              if (ixp > -1) continue;
              const float wg = __fmul_rn(tx[lx], tyz);
              if (wg != 0.0f)
                atomicAdd(row + (-ixp), make_float4(__fmul_rn(br, wg), __fmul_rn(-bi, wg), wg, 0.0f));
            }
          }
        }
      }
    }
    if (priv) {
      __syncthreads();
      const float inv_v = sc_v > 0.0f ? 1.0f / sc_v : 0.0f, inv_w = 1.0f / sc_w;
      for (int q = t; q < bsize; q += blockDim.x) {
        float4 v;
        bool any;
        if (FX) {
          const int qr = f_re[q], qi = f_im[q], qw = f_w[q];
          any = (qr | qi | qw) != 0;
          v = make_float4((float)qr * inv_v, (float)qi * inv_v, (float)qw * inv_w, 0.0f);
        } else {
          v = make_float4(s_re[q], s_im[q], s_w[q], 0.0f);
          any = v.z != 0.0f;
        }
        if (any) {
          const int ix = q % bx;
          const int r = q / bx;
          const int iyp = by0 + r % by, izp = bz0 + r / by;
          const int iza = (izp >= 0) ? izp : N + izp;
          const int iya = (iyp >= 0) ? iyp : N + iyp;
          atomicAdd(G + ((size_t)iza * N + iya) * rowlen + (bx0 + ix), v);
        }
      }
    }
    __syncthreads();   // shared box and accumulators are reused by the next tile
  }
}

// ----------------------------------------------------------------------------
// SYMPLANE0 (bp32f.f:1051-1088) on plane I = 0.  The updated positions of
// different (IYA, IZA) are disjoint, so every pair runs in its own thread.
__device__ __forceinline__ float4 conj4(float4 v) { return make_float4(v.x, -v.y, v.z, v.w); }
__device__ __forceinline__ float4 addconj4(float4 a, float4 b) {  // a + conj(b), W added
  return make_float4(__fadd_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fadd_rn(a.z, b.z), 0.0f);
}

__global__ void symplane0_kernel(float4* __restrict__ G, int nx) {
  const int N = 2 * nx, m = nx - 1;
  const size_t rowlen = (size_t)(nx + 1);
  auto at = [&](int a, int b) -> float4& { return G[((size_t)(b - 1) * N + (a - 1)) * rowlen]; };
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < m * m) {
    int a = 2 + t % m, b = 2 + t / m;
    int ar = N - a + 2, br = N - b + 2;
    float4 v1 = addconj4(at(a, b), at(ar, br));
    at(a, b) = v1;
    at(ar, br) = conj4(v1);
    float4 v3 = addconj4(at(ar, b), at(a, br));
    at(ar, b) = v3;
    at(a, br) = conj4(v3);
  } else if (t < m * m + m) {
    int a = 2 + (t - m * m);
    float4 v = addconj4(at(a, 1), at(N - a + 2, 1));
    at(a, 1) = v;
    at(N - a + 2, 1) = conj4(v);
  } else if (t < m * m + 2 * m) {
    int b = 2 + (t - m * m - m);
    float4 v = addconj4(at(1, b), at(1, N - b + 2));
    at(1, b) = v;
    at(1, N - b + 2) = conj4(v);
  }
}

// ----------------------------------------------------------------------------
// NRMW2 (bp3f.f:1347-1371): X*(-1)**(I+J+K)/W where W > 0.1, else 0, with
// the division in FP64; optional ADDADA of a second grid first
// (bp32f.f:345-346); output conjugated for SPIDER's inverse sign
// (fftw3.f:426-437).  The DC imaginary part, which a real inverse transform
// ignores, is written as zero so the C2R input is exactly Hermitian.
__global__ void nrmw2_kernel(const float4* __restrict__ g0, const float4* __restrict__ g1, float2* __restrict__ out,
                             int nx) {
  const int N = 2 * nx;
  const size_t h = (size_t)(nx + 1);
  const size_t nvox = h * N * N;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nvox; q += (size_t)gridDim.x * blockDim.x) {
    float4 g = g0[q];
    if (g1) {
      float4 o = g1[q];
      g.x = __fadd_rn(g.x, o.x);
      g.y = __fadd_rn(g.y, o.y);
      g.z = __fadd_rn(g.z, o.z);
    }
    float2 r = make_float2(0.0f, 0.0f);
    if (g.z > 0.1f) {
      int i = (int)(q % h);
      size_t t = q / h;
      int j = (int)(t % N), k = (int)(t / N);
      double s = ((i + j + k) & 1) ? -1.0 : 1.0;
      double w = (double)g.z;
      r.x = __double2float_rn(__ddiv_rn(s * (double)g.x, w));
      r.y = -__double2float_rn(__ddiv_rn(s * (double)g.y, w));
    }
    if (q == 0) r.y = 0.0f;
    out[q] = r;
  }
}

// ----------------------------------------------------------------------------
// WINDKB2A (bp32f.f:945-1045).  The padded inverse transform R[n][n][n] is
// cropped at offset ip, scaled by 1/n^3 (FFTW3_USEPLAN's SPIDER scale,
// fftw3.f:443-449), divided by |WKB(LR)|; the mean TNR of the shell
// (nx/2-1)^2 <= LR <= (nx/2)^2 is subtracted inside the sphere, and the
// outside is zeroed.  Pass 1 sums the shell in FP64 into acc[0].
__global__ void windkb_shell_kernel(const float* __restrict__ R, int nx, int ip, float pix,
                                    const float* __restrict__ wkb, double* __restrict__ acc) {
  const int N = 2 * nx, c = nx / 2 + 1;
  const int l2 = (nx / 2) * (nx / 2), l2p = (nx / 2 - 1) * (nx / 2 - 1);
  const size_t total = (size_t)nx * nx * nx;
  double s = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(q % nx);
    size_t t = q / nx;
    int j = (int)(t % nx), k = (int)(t / nx);
    int lr = (k + 1 - c) * (k + 1 - c) + (j + 1 - c) * (j + 1 - c) + (i + 1 - c) * (i + 1 - c);
    if (lr >= l2p && lr <= l2) {
      float v = __fmul_rn(R[((size_t)(ip + k) * N + (ip + j)) * N + (ip + i)], pix);
      v = __fdiv_rn(v, wkb[lr]);
      s += (double)v;
    }
  }
  __shared__ double red[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) atomicAdd(acc, v);
  }
}

__global__ void windkb_out_kernel(const float* __restrict__ R, int nx, int ip, float pix,
                                  const float* __restrict__ wkb, const double* __restrict__ acc, double m,
                                  float* __restrict__ vol) {
  const int N = 2 * nx, c = nx / 2 + 1;
  const int l2 = (nx / 2) * (nx / 2);
  const size_t total = (size_t)nx * nx * nx;
  const float tnr = __double2float_rn(acc[0] / m);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(q % nx);
    size_t t = q / nx;
    int j = (int)(t % nx), k = (int)(t / nx);
    int lr = (k + 1 - c) * (k + 1 - c) + (j + 1 - c) * (j + 1 - c) + (i + 1 - c) * (i + 1 - c);
    float o = 0.0f;
    if (lr <= l2) {
      float v = __fmul_rn(R[((size_t)(ip + k) * N + (ip + j)) * N + (ip + i)], pix);
      v = __fdiv_rn(v, wkb[lr]);
      o = __fsub_rn(v, tnr);
    }
    vol[q] = o;
  }
}

// ----------------------------------------------------------------------------
// SYMVOL (symvol.f:39-180, SP_MP branch) with TRIQDF/TRIQUAD (symvol.f:230-252,
// triquad.f): q2 = sum over symmetries, in order, of q1 sampled at RM^T x with
// triquadratic interpolation inside radius sqrt(IRADI) and q1 itself outside.
// Same DOUBLE/REAL mix and operation order as the Fortran.
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }

__device__ float triquad_dev(double r, double s, double t, const float* f) {
  const float c2 = 0.5f, c4 = 0.25f, c8 = 0.125f;
  const float rs = __double2float_rn(__dmul_rn(r, s)), st = __double2float_rn(__dmul_rn(s, t));
  const float rt = __double2float_rn(__dmul_rn(r, t));
  const float rst = __double2float_rn(__dmul_rn(r, (double)st));
  const float rsq = __double2float_rn(__dsub_rn(1.0, __dmul_rn(r, r)));
  const float ssq = __double2float_rn(__dsub_rn(1.0, __dmul_rn(s, s)));
  const float tsq = __double2float_rn(__dsub_rn(1.0, __dmul_rn(t, t)));
  const float rm1 = __double2float_rn(__dsub_rn(1.0, r)), sm1 = __double2float_rn(__dsub_rn(1.0, s));
  const float tm1 = __double2float_rn(__dsub_rn(1.0, t));
  const float rp1 = __double2float_rn(__dadd_rn(1.0, r)), sp1 = __double2float_rn(__dadd_rn(1.0, s));
  const float tp1 = __double2float_rn(__dadd_rn(1.0, t));
  const float R = __double2float_rn(r), S = __double2float_rn(s), T = __double2float_rn(t);
  float v = fm(fm(fm(fm(fm(-c8, rst), rm1), sm1), tm1), f[0]);
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c4, st), rsq), sm1), tm1), f[1]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c8, rst), rp1), sm1), tm1), f[2]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c4, rt), rm1), ssq), tm1), f[3]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c2, T), rsq), ssq), tm1), f[4]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c4, rt), rp1), ssq), tm1), f[5]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c8, rst), rm1), sp1), tm1), f[6]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c4, st), rsq), sp1), tm1), f[7]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c8, rst), rp1), sp1), tm1), f[8]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c4, rs), rm1), sm1), tsq), f[9]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c2, S), rsq), sm1), tsq), f[10]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c4, rs), rp1), sm1), tsq), f[11]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c2, R), rm1), ssq), tsq), f[12]));
  v = __fadd_rn(v, fm(fm(fm(rsq, ssq), tsq), f[13]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c2, R), rp1), ssq), tsq), f[14]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c4, rs), rm1), sp1), tsq), f[15]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c2, S), rsq), sp1), tsq), f[16]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c4, rs), rp1), sp1), tsq), f[17]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c8, rst), rm1), sm1), tp1), f[18]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c4, st), rsq), sm1), tp1), f[19]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c8, rst), rp1), sm1), tp1), f[20]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c4, rt), rm1), ssq), tp1), f[21]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c2, T), rsq), ssq), tp1), f[22]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c4, rt), rp1), ssq), tp1), f[23]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(-c8, rst), rm1), sp1), tp1), f[24]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c4, st), rsq), sp1), tp1), f[25]));
  v = __fadd_rn(v, fm(fm(fm(fm(fm(c8, rst), rp1), sp1), tp1), f[26]));
  return v;
}

__global__ void symvol_kernel(const float* __restrict__ q1, float* __restrict__ q2, int nx,
                              const float* __restrict__ rm, int nsym) {
  const int klx = -nx / 2, knx = (nx % 2 == 0) ? nx / 2 - 1 : nx / 2;
  const int mn = min(abs(klx), abs(knx));
  const int iradi = (mn - 1) * (mn - 1);
  const size_t nv = (size_t)nx * nx * nx;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nv; q += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(q % nx) + klx;
    const size_t t = q / nx;
    const int iy = (int)(t % nx) + klx, iz = (int)(t / nx) + klx;
    float o = 0.0f;
    for (int is = 0; is < nsym; ++is) {
      const float* R = rm + 9 * is;
      if (R[0] == 1.0f && R[4] == 1.0f && R[8] == 1.0f) {
        o = __fadd_rn(o, q1[q]);
        continue;
      }
      const int icrd = ix * ix + iy * iy + iz * iz;
      if (icrd <= iradi) {
        const float fy = (float)iy, fz = (float)iz, fx = (float)ix;
        const double qr0 = __dadd_rn((double)__fadd_rn(fm(R[1], fy), fm(R[2], fz)), (double)fm(R[0], fx));
        const double qr1 = __dadd_rn((double)__fadd_rn(fm(R[4], fy), fm(R[5], fz)), (double)fm(R[3], fx));
        const double qr2 = __dadd_rn((double)__fadd_rn(fm(R[7], fy), fm(R[8], fz)), (double)fm(R[6], fx));
        const int iox = (int)floor(qr0), ioy = (int)floor(qr1), ioz = (int)floor(qr2);
        const double dx = __dsub_rn(qr0, (double)iox), dy = __dsub_rn(qr1, (double)ioy), dz = __dsub_rn(qr2, (double)ioz);
        float f[27];
#pragma unroll
        for (int l = 0; l < 27; ++l) {
          const int X = l % 3 - 1, Y = (l / 3) % 3 - 1, Z = l / 9 - 1;
          f[l] = __ldg(q1 + ((size_t)(ioz + Z - klx) * nx + (ioy + Y - klx)) * nx + (iox + X - klx));
        }
        o = __fadd_rn(o, triquad_dev(dx, dy, dz, f));
      } else {
        o = __fadd_rn(o, q1[q]);
      }
    }
    q2[q] = o;
  }
}

// ----------------------------------------------------------------------------
// BP 3F P / M helpers: float4 grid <-> (X interleaved complex, W)
__global__ void grid_split_kernel(const float4* __restrict__ G, float2* __restrict__ X, float* __restrict__ W, size_t nvox) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nvox; q += (size_t)gridDim.x * blockDim.x) {
    float4 g = G[q];
    X[q] = make_float2(g.x, g.y);
    W[q] = g.z;
  }
}
__global__ void grid_add_kernel(float4* __restrict__ G, const float2* __restrict__ X, const float* __restrict__ W, size_t nvox) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nvox; q += (size_t)gridDim.x * blockDim.x) {
    float4 g = G[q];
    float2 x = X[q];
    g.x = __fadd_rn(g.x, x.x);
    g.y = __fadd_rn(g.y, x.y);
    g.z = __fadd_rn(g.z, W[q]);
    G[q] = g;
  }
}

// ----------------------------------------------------------------------------
// Compensated accumulation.  The insertion adds the taps of a run of images
// into a partial grid P (plain FP32 vector atomics); every `fold_every`
// images P is folded into the running grid H with an error-free two-sum
// (Knuth: s = h + p, e = (h - (s - b)) + (p - b) with b = s - h), whose
// rounding errors e accumulate in a compensation grid C, and P is cleared.
// H + C then carries the sum to about twice single precision, so the error
// of the total grows with the images per fold instead of with all images.
// COLLAPSE (before SYMPLANE0 / NRMW2 or a partial read-out) ends the
// accumulation: H = fl(H + C), one rounding, and C is cleared.
__device__ __forceinline__ void two_sum(float& h, float p, float& c) {
  const float s = __fadd_rn(h, p);
  const float b = __fsub_rn(s, h);
  const float e = __fadd_rn(__fsub_rn(h, __fsub_rn(s, b)), __fsub_rn(p, b));
  h = s;
  c = __fadd_rn(c, e);
}

template <bool COLLAPSE>
__global__ void fold_kernel(float4* __restrict__ P, float4* __restrict__ H, float4* __restrict__ C, size_t nvox) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nvox; q += (size_t)gridDim.x * blockDim.x) {
    const float4 d = P[q];
    const bool any = d.x != 0.0f || d.y != 0.0f || d.z != 0.0f;
    if (!COLLAPSE && !any) continue;
    float4 c = C[q];
    const bool has_c = c.x != 0.0f || c.y != 0.0f || c.z != 0.0f;
    if (!any && !has_c) continue;
    float4 h = H[q];
    if (any) {
      two_sum(h.x, d.x, c.x);
      two_sum(h.y, d.y, c.y);
      two_sum(h.z, d.z, c.z);
      P[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (COLLAPSE) {
      h.x = __fadd_rn(h.x, c.x);
      h.y = __fadd_rn(h.y, c.y);
      h.z = __fadd_rn(h.z, c.z);
      c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    H[q] = h;
    C[q] = c;
  }
}

// ============================================================================
// host side

int check_kernel(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(kCuda, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return 0;
}

int DevBuf::ensure(size_t want) {
  if (want <= bytes && p) return 0;
  release();
  if (want == 0) return 0;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    return fail(kAlloc, "cudaMalloc(%zu bytes) failed: %s", want, cudaGetErrorString(e));
  }
  bytes = want;
  return 0;
}
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}
int HostBuf::ensure(size_t want) {
  if (want <= bytes && p) return 0;
  release();
  if (want == 0) return 0;
  cudaError_t e = cudaMallocHost(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    return fail(kAlloc, "cudaMallocHost(%zu bytes) failed: %s", want, cudaGetErrorString(e));
  }
  bytes = want;
  return 0;
}
void HostBuf::release() {
  if (p) cudaFreeHost(p);
  p = nullptr;
  bytes = 0;
}

void bp_release(spi_ctx* c) {
  for (auto& g : c->grid) g.release();
  for (auto& g : c->part) g.release();
  for (auto& g : c->comp) g.release();
  c->unfolded = 0;
  c->comp_dirty = false;
  c->gptr[0] = c->gptr[1] = nullptr;
  c->wkb_nx = 0;
  c->imgs.release();
  c->imgs2.release();
  c->rtsq_prm.release();
  rtsf_release(c);
  c->padded.release();
  c->fft_tw.release();
  c->spectra.release();
  c->spec_tmp.release();
  c->slices.release();
  c->workctr.release();
  c->mc_params.release();
  c->mc_host.release();
  c->cplx.release();
  c->real3.release();
  c->wkb.release();
  c->volbuf.release();
  c->symtmp.release();
  c->hslices.release();
  if (c->plan2d) cufftDestroy(c->plan2d);
  if (c->plan3d) cufftDestroy(c->plan3d);
  c->plan2d = 0;
  c->plan3d = 0;
  c->plan2d_n = c->plan2d_batch = c->plan3d_n = 0;
  c->nx = c->n = c->ngrids = 0;
  c->pending_sym0[0] = c->pending_sym0[1] = false;
  c->merged = false;
}

static int grid_blocks(const spi_ctx* c, size_t work, int threads) {
  size_t b = (work + threads - 1) / threads;
  size_t cap = (size_t)c->sm_count * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

static size_t grid_voxels(const spi_ctx* c) { return (size_t)(c->nx + 1) * c->n * c->n; }

// The grid the insertion adds into: the partial grid with compensated
// accumulation, else the grid itself.
static float4* insert_target(spi_ctx* c, int g) { return c->accum ? c->part[g].as<float4>() : c->gptr[g]; }

// Fold the partial grids into the grids (two-sum, compensation kept), or with
// `collapse` also add the compensation into the grids and clear it; a no-op
// without compensated accumulation or pending sums.
static int fold_grids(spi_ctx* c, bool collapse) {
  if (!c->accum || c->ngrids == 0) return 0;
  if (c->unfolded == 0 && !(collapse && c->comp_dirty)) return 0;
  const size_t nvox = grid_voxels(c);
  int ev = c->phase_begin(8);
  for (int g = 0; g < c->ngrids; ++g) {
    float4 *P = c->part[g].as<float4>(), *H = c->gptr[g], *C = c->comp[g].as<float4>();
    if (collapse)
      fold_kernel<true><<<grid_blocks(c, nvox, 256), 256, 0, c->stream>>>(P, H, C, nvox);
    else
      fold_kernel<false><<<grid_blocks(c, nvox, 256), 256, 0, c->stream>>>(P, H, C, nvox);
    SPI_TRY(check_kernel("fold_kernel"));
    c->count();
  }
  c->phase_end(ev);
  c->unfolded = 0;
  c->comp_dirty = !collapse;
  return 0;
}

static int env_int(const char* name, int dflt) {
  const char* s = getenv(name);
  if (!s || !*s) return dflt;
  return atoi(s);
}

// PADD2 + ASTA_D + phase shift (stage_kernel) of nimg device images of box
// nx into padded[b][2nx][2nx] on stream s: the input of the batched R2C.
int stage_images(const spi_ctx* c, cudaStream_t s, const float* imgs, int nx, int nimg, float* padded) {
  if (nimg <= 0) return 0;
  const int n = 2 * nx;
  int klp_count = 0;
  const float rr = (float)(nx / 2) * (float)(nx / 2);
  const int nc = nx / 2 + 1;
  for (int j = 1; j <= nx; ++j)
    for (int i = 1; i <= nx; ++i) {
      const float t = (float)(j - nc), t2 = (float)(i - nc);
      if (t * t + t2 * t2 > rr) ++klp_count;
    }
  const int ip = (n - nx) / 2 + nx % 2;
  const int parts = std::max(1, std::min(8, (4 * c->sm_count + nimg - 1) / nimg));
  stage_kernel<<<dim3(nimg, parts), 256, 0, s>>>(imgs, nx, n, ip, nimg, (double)(float)klp_count, padded);
  return check_kernel("stage_kernel");
}

}  // namespace spi

using namespace spi;

int spi_ctx::phase_begin(int phase, cudaStream_t s) {
  if (!timing) return -1;
  if (!s) s = stream;
  cudaEvent_t a, b;
  if (ev_pool.size() >= 2) {
    a = ev_pool.back(); ev_pool.pop_back();
    b = ev_pool.back(); ev_pool.pop_back();
  } else {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  cudaEventRecord(a, s);
  ev_pending.push_back(PhaseEv{a, b, phase, s});
  return (int)ev_pending.size() - 1;
}

void spi_ctx::phase_end(int slot) {
  if (slot < 0) return;
  cudaEventRecord(ev_pending[slot].b, ev_pending[slot].s);
}

void spi_ctx::phase_collect() {
  for (auto& e : ev_pending) {
    float ms = 0.0f;
    cudaEventSynchronize(e.b);
    if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
      phase_ms[e.phase] += ms;
      phase_n[e.phase] += 1;
    }
    ev_pool.push_back(e.a);
    ev_pool.push_back(e.b);
  }
  ev_pending.clear();
}

long long spi_ctx::device_bytes() const {
  long long t = 0;
  const DevBuf* bufs[] = {&grid[0], &grid[1], &part[0], &part[1], &comp[0], &comp[1], &kbtab, &imgs, &padded, &spectra, &spec_tmp, &slices, &cplx, &real3,
                          &workctr,
                          &wkb, &acc, &volbuf, &pj_vol, &pj_out, &pj_runs, &pj_dm, &pj_rows, &pj_v4, &pj_fbs};
  for (auto b : bufs) t += (long long)b->bytes;
  for (auto& b : cg_buf) t += (long long)b.bytes;
  return t;
}

extern "C" {

int spi_version(void) { return 100; }

int spi_kb_table(int n2, float* tab, float* fltb) {
  if (!tab || n2 < 16) return fail(kInvalid, "spi_kb_table: n2 = %d", n2);
  KBTab t;
  fill_kb(n2, t);
  memcpy(tab, t.tab, sizeof(t.tab));
  if (fltb) *fltb = t.fltb;
  return 0;
}

const char* spi_last_error(void) { return last_error_cstr(); }

int spi_ctx_create(int device, spi_ctx** out) {
  if (!out) return fail(kInvalid, "spi_ctx_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  SPI_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(kInvalid, "spi_ctx_create: device %d of %d", device, ndev);
  SPI_CUDA(cudaSetDevice(device));
  spi_ctx* c = new spi_ctx();
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->sm_count = prop.multiProcessorCount;
  if (prop.major < 10) {
    delete c;
    return fail(kDevice, "spi_ctx_create: device %d is sm_%d%d; this library is built for sm_100a", device,
                prop.major, prop.minor);
  }
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(kCuda, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  e = cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return fail(kCuda, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  int st = c->acc.ensure(64);
  if (st) {
    cudaStreamDestroy(c->stream2);
    cudaStreamDestroy(c->stream);
    delete c;
    return st;
  }
  c->pipeline = env_int("SPI_PIPELINE", 1) ? 1 : 0;
  c->first_piece = env_int("SPI_FIRST_PIECE", 1) ? 1 : 0;
  c->accum = env_int("SPI_BP_ACCUM", 1) ? 1 : 0;
  *out = c;
  return 0;
}

int spi_ctx_destroy(spi_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  bp_release(c);
  pj_release(c);
  cg_release(c);
  c->kbtab.release();
  c->acc.release();
  c->hbuf.release();
  c->phase_collect();
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  for (auto e : c->ev_ready) cudaEventDestroy(e);
  for (auto e : c->ev_done) cudaEventDestroy(e);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  cudaStreamSynchronize(c->stream2);
  cudaStreamDestroy(c->stream2);
  cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

long long spi_ctx_launch_count(const spi_ctx* c) { return c ? c->launches : 0; }

void* spi_ctx_stream(const spi_ctx* c) { return c ? (void*)c->stream : nullptr; }

int spi_ctx_set_timing(spi_ctx* c, int on) {
  if (!c) return fail(kInvalid, "NULL context");
  c->phase_collect();
  c->timing = on != 0;
  return 0;
}

int spi_ctx_timing(spi_ctx* c, double* ms_out, long long* count_out) {
  if (!c) return fail(kInvalid, "NULL context");
  SPI_CUDA(cudaSetDevice(c->device));
  c->phase_collect();
  for (int i = 0; i < SPI_NPHASE; ++i) {
    if (ms_out) ms_out[i] = c->phase_ms[i];
    if (count_out) count_out[i] = c->phase_n[i];
    c->phase_ms[i] = 0.0;
    c->phase_n[i] = 0;
  }
  return 0;
}
long long spi_ctx_device_bytes(const spi_ctx* c) { return c ? c->device_bytes() : 0; }

int spi_bp_open(spi_ctx* c, int nx, int ngrids, const float* sym_angles, int nsym) {
  if (!c) return fail(kInvalid, "spi_bp_open: NULL context");
  if (nx < 8 || nx > 512) return fail(kInvalid, "spi_bp_open: nx = %d must be 8..512", nx);
  if (ngrids != 1 && ngrids != 2) return fail(kInvalid, "spi_bp_open: ngrids = %d must be 1 or 2", ngrids);
  if (nsym > 1 && !sym_angles) return fail(kInvalid, "spi_bp_open: nsym = %d but no symmetry angles", nsym);
  SPI_CUDA(cudaSetDevice(c->device));
  if (c->nx != nx) {
    SPI_CUDA(cudaStreamSynchronize(c->stream));   // insertions may still be running
    bp_release(c);   // buffers are sized by nx; same-size reopens keep them
  } else {
    c->pending_sym0[0] = c->pending_sym0[1] = false;
    c->merged = false;
  }
  c->nx = nx;
  c->n = 2 * nx;
  c->ngrids = ngrids;
  c->inserted = false;
  c->nsym = nsym > 1 ? nsym : 1;
  c->sym_dm.assign((size_t)9 * c->nsym, 0.0f);
  if (nsym > 1)
    for (int s = 0; s < nsym; ++s)  // BUILDS: CANG(phi, theta, psi) per symmetry (builds.f:52)
      cang(sym_angles[3 * s + 2], sym_angles[3 * s + 1], sym_angles[3 * s + 0], &c->sym_dm[9 * s]);
  fill_kb(c->n, c->kb);
  SPI_TRY(c->kbtab.ensure(sizeof(c->kb.tab)));
  SPI_CUDA(cudaMemcpyAsync(c->kbtab.p, c->kb.tab, sizeof(c->kb.tab), cudaMemcpyHostToDevice, c->stream));
  const size_t gbytes = grid_voxels(c) * sizeof(float4);
  for (int g = 0; g < ngrids; ++g) {
    if (c->ext_grid[g]) {
      c->gptr[g] = c->ext_grid[g];
    } else {
      SPI_TRY(c->grid[g].ensure(gbytes));
      c->gptr[g] = c->grid[g].as<float4>();
    }
    SPI_CUDA(cudaMemsetAsync(c->gptr[g], 0, gbytes, c->stream));
    if (c->accum) {
      SPI_TRY(c->part[g].ensure(gbytes));
      SPI_TRY(c->comp[g].ensure(gbytes));
      SPI_CUDA(cudaMemsetAsync(c->part[g].p, 0, gbytes, c->stream));
      SPI_CUDA(cudaMemsetAsync(c->comp[g].p, 0, gbytes, c->stream));
    }
  }
  c->unfolded = 0;
  c->comp_dirty = false;
  if (c->fold_every <= 0) c->fold_every = env_int("SPI_BP_FOLD", 4096);
  // chunk sizes: spectra of one chunk <= ~4.3 GB FP32
  const size_t spec_per_img = (size_t)c->n * (nx + 1) * sizeof(float2);
  int chunk = (int)std::min<size_t>(8192, std::max<size_t>(64, (size_t)4400000000ull / spec_per_img));
  chunk = env_int("SPI_BP_CHUNK", chunk);
  {
    const char* m = getenv("SPI_INSERT");
    const int def_mode = kb_window4_ok(c->kb) ? 3 : 2;
    c->insert_mode = !m ? def_mode : strcmp(m, "tile") == 0 ? 0 : strcmp(m, "direct") == 0 ? 1
                   : strcmp(m, "xlane") == 0 ? 2 : strcmp(m, "tilefx") == 0 ? 4 : def_mode;
    const char* o = getenv("SPI_SLICE_ORDER");
    c->slice_order = (o && strcmp(o, "input") == 0) ? 0 : 1;
    const char* lo = getenv("SPI_INSERT_ORDER");
    c->line_order = !lo ? 1 : strcmp(lo, "rows") == 0 ? 0 : strcmp(lo, "cols") == 0 ? 2 : 1;
    const char* mp = getenv("SPI_INSERT_MAP");
    c->insert_seg_map = (mp && strcmp(mp, "seg") == 0) ? 1 : 0;
    // The insertion is limited by L2 atomics, not by occupancy.  Measured on
    // 4,096 images: the x-lane kernel is best at 24 warps/SM for 128^3 and 16
    // for 64^3 and 256^3; the direct kernel at 24 warps/SM for 64^3, 8 for
    // 128^3-192^3 and 4 for 256^3.
    int def_threads = 256, def_bps = (nx > 96 && nx <= 160) ? 3 : 2;
    if (c->insert_mode == 1) {
      def_threads = nx <= 96 ? 256 : 128;
      def_bps = nx <= 96 ? 3 : nx <= 224 ? 2 : 1;
    }
    c->insert_threads = env_int("SPI_INSERT_THREADS", def_threads);
    if (c->insert_threads != 64 && c->insert_threads != 128 && c->insert_threads != 256 && c->insert_threads != 512)
      c->insert_threads = def_threads;
    c->insert_blocks_per_sm = env_int("SPI_INSERT_BLOCKS_PER_SM", def_bps);
  }
  // FFT sub-batch (and insert launch): padded images <= 1 GB.  Larger batches
  // transform faster and, with the dynamic row counter, launch size no longer
  // costs insertion speed (measured at 256^3: 1,024 and 4,096 alike).
  int sub = (int)std::min<size_t>((size_t)chunk, std::max<size_t>(8, (size_t)1073741824ull / ((size_t)c->n * c->n * 4)));
  sub = std::max(1, std::min(chunk, env_int("SPI_BP_SUB", sub)));
  c->sub = sub;
  c->sort_group = std::max(1, std::min(sub, env_int("SPI_SORT_GROUP", sub)));
  c->upload_images = std::max(0, env_int("SPI_UPLOAD_IMAGES", 0));   // 0: pieces of ~64 MB
  // n = 512 column pass: 4 columns per CTA (47 KB of shared memory, 4 CTAs
  // per SM) measured 69.64-69.69 ms per 4,096-image step against
  // 69.96-70.32 ms with 8 (74 KB, 3 CTAs per SM), two alternations at 256^3
  c->col512 = env_int("SPI_COLFFT_COLS", 4) == 8 ? 8 : 4;
  {
    // The own two-pass R2C is the default at n = 512 (nx = 256), where its
    // register passes (stage_rowfft512_kernel + colfft512_kernel) measured
    // 1.22 ms per 1,024 images against 1.36 ms for PADD2 + cuFFT; elsewhere
    // PADD2 + cuFFT.  SPI_FFT=cufft / own / own2 choose explicitly (own: the
    // register passes at n = 128-512, radix-2 elsewhere; own2: radix-2).
    const char* f = getenv("SPI_FFT");
    const bool pow2 = (c->n & (c->n - 1)) == 0 && c->n >= 16 && c->n <= 1024;
    if (f && strcmp(f, "own") == 0) c->fft_own = pow2 ? 1 : 0;
    else if (f && strcmp(f, "own2") == 0) c->fft_own = pow2 ? 2 : 0;
    else if (f && strcmp(f, "cufft") == 0) c->fft_own = 0;
    else c->fft_own = c->n == 512 ? 1 : 0;
  }
  c->chunk = ((chunk + sub - 1) / sub) * sub;
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int spi_bp_attach_grids(spi_ctx* c, void* g0, void* g1) {
  if (!c) return fail(kInvalid, "NULL context");
  if (c->ngrids) return fail(kInvalid, "spi_bp_attach_grids: call before spi_bp_open");
  c->ext_grid[0] = static_cast<float4*>(g0);
  c->ext_grid[1] = static_cast<float4*>(g1);
  return 0;
}

int spi_bp_grid_bytes(int nx, long long* bytes) {
  if (!bytes || nx < 8 || nx > 512) return fail(kInvalid, "spi_bp_grid_bytes: nx = %d", nx);
  *bytes = (long long)(nx + 1) * (2LL * nx) * (2LL * nx) * 16;
  return 0;
}

int spi_bp_set_spectrum_precision(spi_ctx* c, int bf16) {
  if (!c) return fail(kInvalid, "NULL context");
  c->bf16 = bf16 ? 1 : 0;
  return 0;
}

int spi_bp_set_accumulation(spi_ctx* c, int compensated, int fold_every) {
  if (!c) return fail(kInvalid, "NULL context");
  if (c->ngrids) return fail(kInvalid, "spi_bp_set_accumulation: call before spi_bp_open");
  if (fold_every < 0) return fail(kInvalid, "spi_bp_set_accumulation: fold_every = %d", fold_every);
  c->accum = compensated ? 1 : 0;
  c->fold_every = fold_every;
  return 0;
}

int spi_bp_flush(spi_ctx* c) {
  if (!c || c->ngrids == 0) return fail(kInvalid, "spi_bp_flush: no open reconstruction");
  SPI_CUDA(cudaSetDevice(c->device));
  SPI_TRY(fold_grids(c, true));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// Twiddles of the own R2C: W_n^t = e^(-2 pi i t / n), t < n/2, computed in FP64.
// The register-FFT passes exist for n = 128, 256 and 512 (SPI_FFT=own; at n =
// 512 the column pass is colfft512_kernel); the shared-memory radix-2 passes
// take the other sizes (and SPI_FFT=own2).
static bool fft_warp_form(const spi_ctx* c) { return c->fft_own == 1 && (c->n == 128 || c->n == 256 || c->n == 512); }

static int launch_rowfft(spi_ctx* c, cudaStream_t st, const float* src, int np, int parts, double klp, float2* inter) {
  const int nx = c->nx, n = c->n, ip = (n - nx) / 2 + nx % 2;
  const float2* tw = c->fft_tw.as<float2>();
  const size_t istride = (size_t)n * n / 2;
  if (fft_warp_form(c)) {
    const dim3 g(np, parts);
    if (n == 128) stage_rowfft_w_kernel<2><<<g, 256, 0, st>>>(src, nx, n, ip, np, klp, tw, inter, istride);
    else if (n == 256) stage_rowfft_w_kernel<4><<<g, 256, 0, st>>>(src, nx, n, ip, np, klp, tw, inter, istride);
    else stage_rowfft512_kernel<<<g, 256, 0, st>>>(src, nx, n, ip, np, klp, tw, inter, istride);
    return check_kernel("stage_rowfft_w_kernel");
  }
  const size_t smem = (size_t)(n / 2) * 5 * sizeof(float2);
  stage_rowfft_kernel<<<dim3(np, parts), 256, smem, st>>>(src, nx, n, ip, np, klp, tw, inter, istride);
  return check_kernel("stage_rowfft_kernel");
}

static int launch_colfft(spi_ctx* c, cudaStream_t st, const float2* inter, int nvalid, float2* out) {
  const int nx = c->nx, n = c->n, ip = (n - nx) / 2 + nx % 2;
  const float2* tw = c->fft_tw.as<float2>();
  const size_t istride = (size_t)n * n / 2;
  if (fft_warp_form(c)) {
    const int tiles = (n / 2 + 1 + kColTileW - 1) / kColTileW;
    const size_t smem = ((size_t)(n / 2) + (size_t)kColTileW * ((nx + 1) + (n + 33))) * sizeof(float2);
    if (n == 128) {
      colfft_w_kernel<4><<<nvalid * tiles, 256, smem, st>>>(inter, istride, nx, n, ip, nvalid, tw, out);
    } else if (n == 256) {
      colfft_w_kernel<8><<<nvalid * tiles, 256, smem, st>>>(inter, istride, nx, n, ip, nvalid, tw, out);
    } else {
      const int cols = c->col512;
      const int t512 = (n / 2 + 1 + cols - 1) / cols;
      if (cols == 4)
        colfft512_kernel<4><<<nvalid * t512, 256, colfft512_smem(4), st>>>(inter, istride, nx, n, ip, nvalid, tw, out);
      else
        colfft512_kernel<8><<<nvalid * t512, 256, colfft512_smem(8), st>>>(inter, istride, nx, n, ip, nvalid, tw, out);
    }
    return check_kernel("colfft_w_kernel");
  }
  const int tiles = (n / 2 + 1 + kColTile - 1) / kColTile;
  const size_t smem = ((size_t)(n / 2) + (size_t)kColTile * (n + 1)) * sizeof(float2);
  colfft_kernel<<<nvalid * tiles, 256, smem, st>>>(inter, istride, nx, n, ip, nvalid, tw, out);
  return check_kernel("colfft_kernel");
}

static int ensure_fft_twiddles(spi_ctx* c) {
  const int n = c->n, h = n / 2;
  if (c->fft_tw.p && c->fft_tw.bytes >= (size_t)h * sizeof(float2)) return 0;
  std::vector<float2> tw(h);
  for (int t = 0; t < h; ++t) {
    const double a = -2.0 * M_PI * (double)t / (double)n;
    tw[t] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  SPI_TRY(c->fft_tw.ensure((size_t)h * sizeof(float2)));
  SPI_CUDA(cudaMemcpy(c->fft_tw.p, tw.data(), (size_t)h * sizeof(float2), cudaMemcpyHostToDevice));
  static std::mutex mu;
  static unsigned long long done = 0;
  std::lock_guard<std::mutex> lk(mu);
  const unsigned long long bit = 1ull << (c->device & 63);
  if (!(done & bit)) {   // the column pass holds 16 columns of up to 1,024 points
    SPI_CUDA(cudaFuncSetAttribute(colfft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)((512 + kColTile * 1025) * sizeof(float2))));
    const int wsm = (int)((128 + kColTileW * (129 + 256 + 33)) * sizeof(float2));   // n = 256
    SPI_CUDA(cudaFuncSetAttribute(colfft_w_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, wsm));
    SPI_CUDA(cudaFuncSetAttribute(colfft_w_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, wsm));
    SPI_CUDA(cudaFuncSetAttribute(colfft512_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)colfft512_smem(4)));
    SPI_CUDA(cudaFuncSetAttribute(colfft512_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)colfft512_smem(8)));
    done |= bit;
  }
  return 0;
}

static int ensure_chunk_buffers(spi_ctx* c) {
  const int nx = c->nx, n = c->n;
  if (c->fft_own) SPI_TRY(ensure_fft_twiddles(c));
  SPI_TRY(c->imgs.ensure((size_t)c->chunk * nx * nx * sizeof(float)));
  SPI_TRY(c->padded.ensure((size_t)c->sub * n * n * sizeof(float)));
  const size_t plane = (size_t)n * (nx + 1);
  if (c->bf16) {
    SPI_TRY(c->spectra.ensure((size_t)c->chunk * plane * sizeof(__nv_bfloat162)));
    SPI_TRY(c->spec_tmp.ensure((size_t)c->sub * plane * sizeof(float2)));
  } else {
    SPI_TRY(c->spectra.ensure((size_t)c->chunk * plane * sizeof(float2)));
  }
  SPI_TRY(c->slices.ensure((size_t)c->chunk * c->nsym * sizeof(SliceDesc)));
  if (c->plan2d == 0 || c->plan2d_n != n || c->plan2d_batch != c->sub) {
    if (c->plan2d) cufftDestroy(c->plan2d);
    c->plan2d = 0;
    int dims[2] = {n, n};
    SPI_CUFFT(cufftPlanMany(&c->plan2d, 2, dims, nullptr, 1, n * n, nullptr, 1, n * (n / 2 + 1), CUFFT_R2C, c->sub));
    SPI_CUFFT(cufftSetStream(c->plan2d, c->stream));
    c->plan2d_n = n;
    c->plan2d_batch = c->sub;
  }
  return 0;
}

static int bp_insert_impl(spi_ctx* c, const float* imgs, int nimg, const float* angles, const float* inplane,
                          const uint8_t* half, int imgs_on_device);

int spi_bp_insert(spi_ctx* c, const float* imgs, int nimg, const float* angles, const uint8_t* half,
                  int imgs_on_device) {
  return bp_insert_impl(c, imgs, nimg, angles, nullptr, half, imgs_on_device);
}

int spi_bp_insert_rb(spi_ctx* c, const float* imgs, int nimg, const float* angles, const float* inplane,
                     const uint8_t* half, int imgs_on_device) {
  if (nimg > 0 && !inplane) return fail(kInvalid, "spi_bp_insert_rb: in-plane parameters are required");
  return bp_insert_impl(c, imgs, nimg, angles, inplane, half, imgs_on_device);
}

}  // extern "C"

// Launch the configured insertion kernel over `nslices` slice descriptors
// (on the library stream), persistent: sm_count x blocks-per-SM CTAs.
template <typename K>
static int insert_blocks(spi_ctx* c, K kernel, int threads, size_t smem, int cap) {
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (cap > 0) per_sm = std::min(per_sm, cap);
  return c->sm_count * std::max(per_sm, 1);
}

static int launch_insert(spi_ctx* c, const SliceDesc* sl, int nslices, float4* g1) {
  const void* spec = c->spectra.p;
  const int nx = c->nx;
  const float* tab = c->kbtab.as<float>();
  const float fltb = c->kb.fltb;
  float4* g0 = insert_target(c, 0);
  int ev_ins = c->phase_begin(2);
  if (c->insert_mode >= 1 && c->insert_mode <= 3) {
    const size_t smem = 5000 * sizeof(float);
    const int threads = c->insert_threads;
    if (c->insert_mode == 1) {
      if (c->bf16)
        insert_kernel<true><<<insert_blocks(c, insert_kernel<true>, threads, smem, c->insert_blocks_per_sm), threads,
                              smem, c->stream>>>(spec, sl, nslices, nx, tab, fltb, g0, g1, c->insert_seg_map);
      else
        insert_kernel<false><<<insert_blocks(c, insert_kernel<false>, threads, smem, c->insert_blocks_per_sm),
                               threads, smem, c->stream>>>(spec, sl, nslices, nx, tab, fltb, g0, g1,
                                                           c->insert_seg_map);
    } else if (c->insert_mode == 3) {
      SPI_TRY(c->workctr.ensure(sizeof(unsigned long long)));
      auto* work = c->workctr.as<unsigned long long>();
      SPI_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned long long), c->stream));
      if (c->bf16)
        insert_x4_kernel<true><<<insert_blocks(c, insert_x4_kernel<true>, threads, smem, c->insert_blocks_per_sm),
                                 threads, smem, c->stream>>>(spec, sl, nslices, nx, tab, fltb, g0, g1, work);
      else
        insert_x4_kernel<false><<<insert_blocks(c, insert_x4_kernel<false>, threads, smem, c->insert_blocks_per_sm),
                                  threads, smem, c->stream>>>(spec, sl, nslices, nx, tab, fltb, g0, g1, work);
    } else {
      // row counter of this launch (launches on the library stream are serialised)
      SPI_TRY(c->workctr.ensure(sizeof(unsigned long long)));
      auto* work = c->workctr.as<unsigned long long>();
      SPI_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned long long), c->stream));
      if (c->bf16)
        insert_xlane_kernel<true><<<insert_blocks(c, insert_xlane_kernel<true>, threads, smem,
                                                  c->insert_blocks_per_sm),
                                    threads, smem, c->stream>>>(spec, sl, nslices, nx, tab, fltb, g0, g1, work);
      else
        insert_xlane_kernel<false><<<insert_blocks(c, insert_xlane_kernel<false>, threads, smem,
                                                   c->insert_blocks_per_sm),
                                     threads, smem, c->stream>>>(spec, sl, nslices, nx, tab, fltb, g0, g1, work);
    }
  } else {
    const size_t smem = 3 * kTileCap * sizeof(float);
    const bool fx = c->insert_mode == 4;
    // the attribute is per device; set once per device (several threads may race here harmlessly)
    static std::atomic<unsigned long long> attr_done{0};
    const unsigned long long bit = 1ull << (c->device & 63);
    if (!(attr_done.load() & bit)) {
      cudaFuncSetAttribute(insert_tile_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(insert_tile_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(insert_tile_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(insert_tile_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      attr_done.fetch_or(bit);
    }
#define SPI_TILE(B, F)                                                                                    \
  insert_tile_kernel<B, F><<<insert_blocks(c, insert_tile_kernel<B, F>, 256, smem, 0), 256, smem, c->stream>>>( \
      spec, sl, nslices, nx, tab, fltb, g0, g1)
    if (c->bf16) {
      if (fx) SPI_TILE(true, true); else SPI_TILE(true, false);
    } else {
      if (fx) SPI_TILE(false, true); else SPI_TILE(false, false);
    }
#undef SPI_TILE
  }
  SPI_TRY(check_kernel("insert_kernel"));
  c->phase_end(ev_ins);
  c->count();
  return 0;
}

// Events of the staging/insertion pipeline, one pair per FFT sub-batch slot.
static int ensure_pipeline_events(spi_ctx* c, int nsubs) {
  if (!c->ev_fork) {
    SPI_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    SPI_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  }
  while ((int)c->ev_ready.size() < nsubs) {
    cudaEvent_t r, d;
    SPI_CUDA(cudaEventCreateWithFlags(&r, cudaEventDisableTiming));
    if (cudaEventCreateWithFlags(&d, cudaEventDisableTiming) != cudaSuccess) {
      cudaEventDestroy(r);
      return fail(kCuda, "cudaEventCreate failed");
    }
    c->ev_ready.push_back(r);
    c->ev_done.push_back(d);
  }
  return 0;
}

// Insertion order of a slice for the x4 kernels (SliceDesc::cols): along the
// in-plane axis, DMS(1:3) (rows) or DMS(4:6) (columns), whose z component is
// smaller, unless the context fixes one order.  Boxes up to 192 keep rows:
// there a grid plane is at most 1.2 MB and the choice measured neutral
// (192^3: 113.8k against 114.1k images/s of random orientations) or slower
// (128^3: 260.1k against 262.4k), while at 256^3 it gains 5%.
static short line_cols(const spi_ctx* c, const float* dms) {
  if (c->line_order != 1) return c->line_order == 2 ? 1 : 0;
  if (c->nx <= 192) return 0;
  return std::fabs(dms[5]) < std::fabs(dms[2]) ? 1 : 0;
}

// Slice descriptors of nimg images: CANG of each angle triple (BUILDM1,
// bp3f.f:1287), its products with the symmetry matrices (bp3f.f:460-466) and
// the grid its half-set mask routes it to; image index a % chunk.  With slice
// ordering on, the slices of each group of `group` images are ordered by the
// normal of their central plane (boustrophedon over rings of the polar
// angle), so the slices in flight together touch overlapping voxels and
// their atomics hit in L2; the order only changes the FP32 summation order.
// Groups lie inside the FFT sub-batches of a chunk (its first `first`
// images, then `sub` at a time), so an insertion launch, which takes one
// sub-batch, only meets slices of images it has staged.
static void build_slices(const spi_ctx* c, const float* angles, const uint8_t* half, int nimg, int chunk, int first,
                         int sub, int group, SliceDesc* hs) {
  const int nsym = c->nsym;
  for (int a = 0; a < nimg; ++a) {
    float dm[9];
    cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], dm);  // BUILDM1 (bp3f.f:1287)
    int g = (c->ngrids == 2 && half) ? (half[a] ? 0 : 1) : 0;
    for (int s = 0; s < nsym; ++s) {
      float dms[9];
      if (nsym > 1) matmul33(&c->sym_dm[9 * s], dm, dms);
      else memcpy(dms, dm, sizeof(dms));
      SliceDesc& d = hs[(size_t)a * nsym + s];
      memcpy(d.dm, dms, 6 * sizeof(float));
      d.img = a % chunk;
      d.grid = (short)g;
      d.cols = line_cols(c, dms);
    }
  }
  if (!c->slice_order) return;
  for (int a0 = 0; a0 < nimg; a0 += chunk) {
    const int a1 = std::min(nimg, a0 + chunk);
    for (int s0 = a0, bi = 0; s0 < a1; s0 += (bi == 0 ? first : sub), ++bi) {
      const int s1 = std::min(a1, s0 + (bi == 0 ? first : sub));
      for (int b0 = s0; b0 < s1; b0 += group) {
        const int nb = std::min(group, s1 - b0);
        SliceDesc* base = hs + (size_t)b0 * nsym;
        const int m = nb * nsym;
        const int rings = std::max(1, (int)std::sqrt((double)m / 2.0));
        std::vector<std::pair<double, int>> key(m);
        for (int q = 0; q < m; ++q) {
          const float* d = base[q].dm;
          double cx = (double)d[1] * d[5] - (double)d[2] * d[4];
          double cy = (double)d[2] * d[3] - (double)d[0] * d[5];
          double cz = (double)d[0] * d[4] - (double)d[1] * d[3];
          if (cz < 0 || (cz == 0 && (cy < 0 || (cy == 0 && cx < 0)))) { cx = -cx; cy = -cy; cz = -cz; }
          const double th = std::acos(std::min(1.0, std::max(-1.0, cz)));      // 0..pi/2
          const double ph = std::atan2(cy, cx);                                 // -pi..pi
          int ring = std::min(rings - 1, (int)(th / (M_PI / 2) * rings));
          double u = (ph + M_PI) / (2 * M_PI);
          if (ring & 1) u = 1.0 - u;
          key[q] = {ring + u, q};
        }
        std::sort(key.begin(), key.end());
        std::vector<SliceDesc> tmp(base, base + m);
        for (int q = 0; q < m; ++q) base[q] = tmp[key[q].second];
      }
    }
  }
}

static int bp_insert_impl(spi_ctx* c, const float* imgs, int nimg, const float* angles, const float* inplane,
                          const uint8_t* half, int imgs_on_device) {
  if (!c || c->ngrids == 0) return fail(kInvalid, "spi_bp_insert: no open reconstruction (spi_bp_open)");
  if (nimg < 0 || (nimg > 0 && (!imgs || !angles))) return fail(kInvalid, "spi_bp_insert: bad image arguments");
  if (c->merged) return fail(kInvalid, "spi_bp_insert: images cannot follow spi_bp_partial_add");
  if (nimg == 0) return 0;
  SPI_CUDA(cudaSetDevice(c->device));
  SPI_TRY(ensure_chunk_buffers(c));
  c->inserted = true;
  const int nx = c->nx, n = c->n, nsym = c->nsym;
  // slice descriptors for the whole call (host, pinned)
  const size_t nsl = (size_t)nimg * nsym;
  SPI_TRY(c->hslices.ensure(nsl * sizeof(SliceDesc)));
  SliceDesc* hs = c->hslices.as<SliceDesc>();
  const bool copy_pipe = !imgs_on_device && c->pipeline;
  // images per upload piece: at most ~64 MB unless the context sets a count
  const int piece = c->upload_images > 0 ? c->upload_images
                                         : (int)((64ull << 20) / ((size_t)nx * nx * sizeof(float)));
  const int up = imgs_on_device ? c->sub : std::max(1, std::min(c->sub, piece));
  // With host images in a call of one chunk, the first FFT sub-batch is one
  // upload piece, so the first insertion starts once that piece has arrived
  // rather than a whole sub-batch (at 256^3: 256 images, 1.2 ms of upload at
  // 55 GB/s, instead of 1,024 images, 4.8 ms); the later sub-batches' uploads
  // still run ahead under the compute.  Only where a sub-batch writes the
  // spectra of its own images alone (the own R2C, or BF16 spectra through
  // the FFT scratch): cuFFT's FP32 path transforms a full batch of c->sub
  // images into the chunk's spectra, which a shifted last sub-batch would
  // overrun.
  const int first_sub =
      (copy_pipe && c->first_piece && nimg <= c->chunk && (c->fft_own || c->bf16)) ? up : c->sub;
  build_slices(c, angles, half, nimg, c->chunk, first_sub, c->sub, c->sort_group, hs);
  int klp_count = 0;
  {
    float rr = (float)(nx / 2) * (float)(nx / 2);
    int nc = nx / 2 + 1;
    for (int j = 1; j <= nx; ++j)
      for (int i = 1; i <= nx; ++i) {
        float t = (float)(j - nc), t2 = (float)(i - nc);
        if (t * t + t2 * t2 > rr) ++klp_count;
      }
  }
  const double klp = (double)(float)klp_count;
  const int ip = (n - nx) / 2 + nx % 2;
  const size_t spec_plane = (size_t)n * (nx + 1);
  std::vector<RtsqParm> rprm;
  const bool rtsf = inplane && c->rb_fbs;
  if (inplane) {
    // COS/SIN(THETA*DGR_TO_RAD) in REAL, as RTSQ computes them (rtsq.f:111-112)
    const float dgr = 3.14159265358979323846f / 180.0f;
    rprm.resize(nimg);
    for (int a = 0; a < nimg; ++a) {
      const float th = inplane[3 * a];
      rprm[a] = RtsqParm{std::cos(th * dgr), std::sin(th * dgr), inplane[3 * a + 1], inplane[3 * a + 2]};
      if (rtsf) {
        // RTSF: THETA = THETAT * PI / 180, COS/SIN in REAL; SHX, SHY = MODULO(SH, NX)
        // (rtsf.f:158-168), Fortran MODULO as fmod with the sign of NX
        const float theta = th * 3.14159265358979323846f / 180.0f;
        auto modulo = [&](float v) {
          float r = std::fmod(v, (float)nx);
          if (r != 0.0f && r < 0.0f) r += (float)nx;
          return r;
        };
        rprm[a] = RtsqParm{std::cos(theta), std::sin(theta), modulo(inplane[3 * a + 1]), modulo(inplane[3 * a + 2])};
      }
    }
    SPI_TRY(c->imgs2.ensure((size_t)c->chunk * nx * nx * sizeof(float)));
    SPI_TRY(c->rtsq_prm.ensure((size_t)c->chunk * sizeof(RtsqParm)));
  }
  // Copy pipeline.  With host images, the copy stream uploads the chunk in
  // pieces of `up` images (<= ~64 MB) and records ev_ready per piece; the
  // library stream waits for each piece, rotates (RTSQ) and pads it, then
  // transforms and inserts the FFT sub-batch and records ev_done for it once
  // its images have been padded; the upload into the same sub-batch slot in
  // the next chunk waits for that.  Uploads thus run under the transforms and
  // the insertion, and only the first piece of a call is exposed.  (Staging
  // and transforming FFT sub-batches on a third stream beside the insertion
  // was measured slower: each insertion launch took 21.1-21.3 instead of
  // 15.7-15.8 ms of 1,024 images at 256^3 while a transform ran beside it,
  // 46.2-46.6k instead of 57.5-58.3k images/s device-resident.)
  const int nsubs = (c->chunk + c->sub - 1) / c->sub + (first_sub < c->sub ? 1 : 0);
  auto sub_len = [&](int bi) { return bi == 0 ? first_sub : c->sub; };   // images of sub-batch bi
  const int ppsub = (c->sub + up - 1) / up;
  SPI_TRY(ensure_pipeline_events(c, nsubs * ppsub));
  cudaStream_t cs = copy_pipe ? c->stream2 : c->stream;
  if (copy_pipe) {
    SPI_CUDA(cudaEventRecord(c->ev_fork, c->stream));
    SPI_CUDA(cudaStreamWaitEvent(cs, c->ev_fork, 0));
  }
  SPI_CUFFT(cufftSetStream(c->plan2d, c->stream));
  std::vector<char> done_valid(nsubs, 0);
  float4* g1 = insert_target(c, c->ngrids == 2 ? 1 : 0);
  for (int a0 = 0; a0 < nimg; a0 += c->chunk) {
    const int nb = std::min(c->chunk, nimg - a0);
    if (inplane)
      SPI_CUDA(cudaMemcpyAsync(c->rtsq_prm.p, rprm.data() + a0, (size_t)nb * sizeof(RtsqParm), cudaMemcpyHostToDevice,
                               c->stream));
    SPI_CUDA(cudaMemcpyAsync(c->slices.p, hs + (size_t)a0 * nsym, (size_t)nb * nsym * sizeof(SliceDesc),
                             cudaMemcpyHostToDevice, c->stream));
    if (!imgs_on_device) {   // uploads of the whole chunk, ahead of the compute
      for (int b0 = 0, bi = 0; b0 < nb; b0 += sub_len(bi), ++bi) {
        const int nvalid = std::min(sub_len(bi), nb - b0);
        if (done_valid[bi]) SPI_CUDA(cudaStreamWaitEvent(cs, c->ev_done[bi], 0));
        for (int p0 = b0, pi = 0; p0 < b0 + nvalid; p0 += up, ++pi) {
          const int np = std::min(up, b0 + nvalid - p0);
          // (no timing events on the copy stream: recording them there was
          // measured to serialise the uploads with the compute)
          int ev = copy_pipe ? -1 : c->phase_begin(7, cs);
          SPI_CUDA(cudaMemcpyAsync(c->imgs.as<float>() + (size_t)p0 * nx * nx, imgs + ((size_t)a0 + p0) * nx * nx,
                                   (size_t)np * nx * nx * sizeof(float), cudaMemcpyHostToDevice, cs));
          c->phase_end(ev);
          SPI_CUDA(cudaEventRecord(c->ev_ready[(size_t)bi * ppsub + pi], cs));
        }
      }
    }
    for (int b0 = 0, bi = 0; b0 < nb; b0 += sub_len(bi), ++bi) {
      const int nvalid = std::min(sub_len(bi), nb - b0);
      for (int p0 = b0, pi = 0; p0 < b0 + nvalid; p0 += up, ++pi) {
        const int np = std::min(up, b0 + nvalid - p0);
        const bool last = p0 + up >= b0 + nvalid;
        const float* src;
        if (!imgs_on_device) {
          if (copy_pipe) SPI_CUDA(cudaStreamWaitEvent(c->stream, c->ev_ready[(size_t)bi * ppsub + pi], 0));
          src = c->imgs.as<float>() + (size_t)p0 * nx * nx;
        } else {
          src = imgs + ((size_t)a0 + p0) * nx * nx;
        }
        if (inplane) {
          int ev = c->phase_begin(0);
          float* dst = c->imgs2.as<float>() + (size_t)p0 * nx * nx;
          if (rtsf) {
            static_assert(sizeof(RtsqParm) == sizeof(float4), "RTSF reads the parameters as float4");
            SPI_TRY(rtsf_images(c, src, dst, nx, np, reinterpret_cast<const float4*>(c->rtsq_prm.as<RtsqParm>() + p0)));
          } else {
            rtsq_kernel<<<grid_blocks(c, (size_t)np * nx * nx, 256), 256, 0, c->stream>>>(
                src, dst, nx, np, c->rtsq_prm.as<RtsqParm>() + p0);
            SPI_TRY(check_kernel("rtsq_kernel"));
            c->count();
          }
          c->phase_end(ev);
          src = dst;
        }
        int ev = c->phase_begin(0);
        if (c->fft_own) {
          // pass 1 of the own R2C: staged rows transformed into padded, used as
          // the row-spectrum buffer (n*n/2 complex slots per image)
          const int parts = std::max(1, std::min(8, (4 * c->sm_count + np - 1) / std::max(np, 1)));
          SPI_TRY(launch_rowfft(c, c->stream, src, np, parts, klp,
                                c->padded.as<float2>() + (size_t)(p0 - b0) * n * n / 2));
        } else {
          // the last piece also zero-pads the unused tail of the FFT batch
          const int blocks = last ? c->sub - (p0 - b0) : np;
          const int parts = std::max(1, std::min(8, (4 * c->sm_count + blocks - 1) / std::max(blocks, 1)));
          stage_kernel<<<dim3(blocks, parts), 256, 0, c->stream>>>(src, nx, n, ip, np, klp,
                                                                   c->padded.as<float>() + (size_t)(p0 - b0) * n * n);
          SPI_TRY(check_kernel("stage_kernel"));
        }
        c->phase_end(ev);
        c->count();
      }
      SPI_CUDA(cudaEventRecord(c->ev_done[bi], c->stream));   // the uploaded images are consumed
      done_valid[bi] = 1;
      float2* fout = c->bf16 ? c->spec_tmp.as<float2>() : c->spectra.as<float2>() + (size_t)b0 * spec_plane;
      int ev = c->phase_begin(1);
      if (c->fft_own) {   // pass 2: the columns of the valid images
        SPI_TRY(launch_colfft(c, c->stream, c->padded.as<float2>(), nvalid, fout));
        c->count();
      } else {
        SPI_CUFFT(cufftExecR2C(c->plan2d, c->padded.as<cufftReal>(), reinterpret_cast<cufftComplex*>(fout)));
      }
      c->phase_end(ev);
      if (c->bf16) {
        const size_t cnt = (size_t)nvalid * spec_plane;
        to_bf16_kernel<<<grid_blocks(c, cnt, 256), 256, 0, c->stream>>>(
            fout, reinterpret_cast<__nv_bfloat162*>(c->spectra.p) + (size_t)b0 * spec_plane, cnt);
        SPI_TRY(check_kernel("to_bf16_kernel"));
        c->count();
      }
      SPI_TRY(launch_insert(c, c->slices.as<SliceDesc>() + (size_t)b0 * nsym, nvalid * nsym, g1));
      c->unfolded += nvalid;
      if (c->unfolded >= c->fold_every) SPI_TRY(fold_grids(c, false));
    }
  }
  if (copy_pipe) {   // join
    SPI_CUDA(cudaEventRecord(c->ev_join, cs));
    SPI_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
  }
  c->pending_sym0[0] = true;
  if (c->ngrids == 2) c->pending_sym0[1] = true;
  // The call returns when its work is done.  Returning as soon as the inputs
  // were consumed (the last staging kernel) was measured 1% faster with
  // device images but 12% slower end to end with host images: the next
  // chunk's uploads then run under this chunk's last insertion.
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// ----------------------------------------------------------------------------
// Multi-class insertion: the images of several open reconstructions (one
// context per class, each opened with its own box size) in one call whose
// insertion is one launch per round over the slices of every class.  All work
// runs on the first context's stream: while the call runs, the other
// classes' contexts use that stream (their own are idle and restored after).
namespace {
struct StreamSwap {
  std::vector<spi_ctx*> ctxs;
  std::vector<cudaStream_t> saved;
  ~StreamSwap() {
    for (size_t i = 0; i < ctxs.size(); ++i) ctxs[i]->stream = saved[i];
  }
};
}  // namespace

static int bp_insert_multi_impl(spi_ctx* const* ctxs, int ncls, const float* const* imgs, const int* nimg,
                                const float* const* angles, const uint8_t* const* half, int imgs_on_device) {
  if (!ctxs || ncls < 1 || ncls > kMcMaxClass || !imgs || !nimg || !angles)
    return fail(kInvalid, "spi_bp_insert_multi: %d classes (1..%d) or NULL arrays", ncls, kMcMaxClass);
  spi_ctx* lead = ctxs[0];
  for (int k = 0; k < ncls; ++k) {
    spi_ctx* c = ctxs[k];
    if (!c || c->ngrids == 0) return fail(kInvalid, "spi_bp_insert_multi: class %d has no open reconstruction", k);
    if (c->merged) return fail(kInvalid, "spi_bp_insert_multi: class %d follows spi_bp_partial_add", k);
    if (c->device != lead->device || c->bf16 != lead->bf16)
      return fail(kInvalid, "spi_bp_insert_multi: class %d is on another device or spectrum precision", k);
    if (nimg[k] < 0 || (nimg[k] > 0 && (!imgs[k] || !angles[k])))
      return fail(kInvalid, "spi_bp_insert_multi: bad images of class %d", k);
    for (int j = 0; j < k; ++j)
      if (ctxs[j] == c) return fail(kInvalid, "spi_bp_insert_multi: class %d repeats a context", k);
  }
  // one table per distinct box size
  std::vector<int> tab_nx, cls_tab(ncls);
  for (int k = 0; k < ncls; ++k) {
    auto it = std::find(tab_nx.begin(), tab_nx.end(), ctxs[k]->nx);
    if (it == tab_nx.end()) {
      if ((int)tab_nx.size() == kMcMaxTab)
        return fail(kInvalid, "spi_bp_insert_multi: more than %d distinct box sizes", kMcMaxTab);
      cls_tab[k] = (int)tab_nx.size();
      tab_nx.push_back(ctxs[k]->nx);
    } else {
      cls_tab[k] = (int)(it - tab_nx.begin());
    }
    if (!kb_window4_ok(ctxs[k]->kb))
      return fail(kInvalid, "spi_bp_insert_multi: the table of nx = %d is not a four-tap window", ctxs[k]->nx);
  }
  const int ntab = (int)tab_nx.size();
  SPI_CUDA(cudaSetDevice(lead->device));
  StreamSwap swap;
  for (int k = 0; k < ncls; ++k) {
    SPI_CUDA(cudaStreamSynchronize(ctxs[k]->stream));
    swap.ctxs.push_back(ctxs[k]);
    swap.saved.push_back(ctxs[k]->stream);
  }
  cudaStream_t st = lead->stream;
  for (int k = 1; k < ncls; ++k) ctxs[k]->stream = st;
  // rounds and slice counts (the FFT sub-batch of each class was set by spi_bp_open)
  int rounds = 0;
  std::vector<size_t> sl_off(ncls + 1, 0);
  for (int k = 0; k < ncls; ++k) {
    rounds = std::max(rounds, (nimg[k] + ctxs[k]->sub - 1) / ctxs[k]->sub);
    sl_off[k + 1] = sl_off[k] + (size_t)nimg[k] * ctxs[k]->nsym;
  }
  // Everything the host copies during the call sits in one pinned buffer
  // (copies from pageable memory would synchronise the stream every round):
  // the slice descriptors of every class, one class table per round, the
  // tables and their FLTB.
  const size_t cls_bytes = sizeof(McClass) * kMcMaxClass;
  const size_t h_sl = 0, h_cls = h_sl + sl_off[ncls] * sizeof(SliceDesc);
  const size_t h_tab = h_cls + (size_t)std::max(rounds, 1) * cls_bytes;
  SPI_TRY(lead->mc_host.ensure(h_tab + sizeof(float) * (5000 + 1) * kMcMaxTab));
  SliceDesc* hs_all = reinterpret_cast<SliceDesc*>(lead->mc_host.as<char>() + h_sl);
  McClass* hc_all = reinterpret_cast<McClass*>(lead->mc_host.as<char>() + h_cls);
  float* ht = reinterpret_cast<float*>(lead->mc_host.as<char>() + h_tab);
  float* hf = ht + 5000 * kMcMaxTab;
  // launch parameters on the device: class table, then the tables and their FLTB
  SPI_TRY(lead->mc_params.ensure(cls_bytes + sizeof(float) * (5000 + 1) * kMcMaxTab + sizeof(unsigned long long)));
  auto* d_cls = lead->mc_params.as<McClass>();
  float* d_tabs = reinterpret_cast<float*>(lead->mc_params.as<char>() + cls_bytes);
  float* d_fl = d_tabs + 5000 * kMcMaxTab;
  auto* d_work = reinterpret_cast<unsigned long long*>(d_fl + kMcMaxTab);
  for (int t = 0; t < ntab; ++t)
    for (int k = 0; k < ncls; ++k)
      if (cls_tab[k] == t) {
        memcpy(ht + (size_t)5000 * t, ctxs[k]->kb.tab, 5000 * sizeof(float));
        hf[t] = ctxs[k]->kb.fltb;
        break;
      }
  SPI_CUDA(cudaMemcpyAsync(d_tabs, ht, (size_t)5000 * ntab * sizeof(float), cudaMemcpyHostToDevice, st));
  SPI_CUDA(cudaMemcpyAsync(d_fl, hf, ntab * sizeof(float), cudaMemcpyHostToDevice, st));
  const size_t smem = (size_t)kMcTab * ntab * sizeof(float);
  // every table must be zero from entry kMcTab - 1 on (checked above by kb_window4_ok: zero from 3331)
  static_assert(kMcTab >= 3332, "the cut table must keep entries 0..3331");
  {
    static std::mutex mu;
    static unsigned long long done = 0;
    std::lock_guard<std::mutex> lk(mu);
    const unsigned long long bit = 1ull << (lead->device & 63);
    if (!(done & bit)) {
      SPI_CUDA(cudaFuncSetAttribute(insert_mc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kMcTab * kMcMaxTab * sizeof(float))));
      SPI_CUDA(cudaFuncSetAttribute(insert_mc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kMcTab * kMcMaxTab * sizeof(float))));
      done |= bit;
    }
  }
  // per class: buffers (room for two FFT sub-batches: round r stages into
  // half r % 2 while round r - 1's insertion reads the other), slice
  // descriptors of all its images, staging constants
  std::vector<double> klp(ncls);
  for (int k = 0; k < ncls; ++k) {
    spi_ctx* c = ctxs[k];
    SPI_TRY(ensure_chunk_buffers(c));
    const size_t two = (size_t)std::max(c->chunk, 2 * c->sub);
    const size_t plane = (size_t)c->n * (c->nx + 1);
    SPI_TRY(c->spectra.ensure(two * plane * (c->bf16 ? sizeof(__nv_bfloat162) : sizeof(float2))));
    SPI_TRY(c->slices.ensure(two * c->nsym * sizeof(SliceDesc)));
    if (!imgs_on_device) SPI_TRY(c->imgs.ensure(two * c->nx * c->nx * sizeof(float)));
    if (nimg[k] > 0)
      build_slices(c, angles[k], half ? half[k] : nullptr, nimg[k], c->sub, c->sub, c->sub, c->sub, hs_all + sl_off[k]);
    const int nx = c->nx;
    int cnt = 0;
    const float rr = (float)(nx / 2) * (float)(nx / 2);
    const int nc = nx / 2 + 1;
    for (int j = 1; j <= nx; ++j)
      for (int i = 1; i <= nx; ++i) {
        const float t = (float)(j - nc), t2 = (float)(i - nc);
        if (t * t + t2 * t2 > rr) ++cnt;
      }
    klp[k] = (double)(float)cnt;
    if (nimg[k] > 0) c->inserted = true;
  }
  // rounds: every class stages its next FFT sub-batch on the staging stream,
  // then one launch on the compute stream inserts them all
  cudaStream_t s2 = lead->stream2;
  SPI_TRY(ensure_pipeline_events(lead, 2));   // ev_ready[h]: half h staged; ev_done[h]: half h inserted
  SPI_CUDA(cudaEventRecord(lead->ev_fork, st));
  SPI_CUDA(cudaStreamWaitEvent(s2, lead->ev_fork, 0));
  for (int k = 0; k < ncls; ++k) SPI_CUFFT(cufftSetStream(ctxs[k]->plan2d, s2));
  for (int r = 0; r < rounds; ++r) {
    const int h = r & 1;
    McClass* hc = hc_all + (size_t)r * kMcMaxClass;
    int nc = 0;
    long long items = 0;
    if (r >= 2) SPI_CUDA(cudaStreamWaitEvent(s2, lead->ev_done[h], 0));   // round r - 2 read this half
    for (int k = 0; k < ncls; ++k) {
      spi_ctx* c = ctxs[k];
      const int nx = c->nx, n = c->n;
      const int a0 = r * c->sub, nb = std::min(c->sub, nimg[k] - a0);
      if (nb <= 0) continue;
      const size_t plane = (size_t)n * (nx + 1);
      const size_t hoff = (size_t)h * c->sub;   // first image of this half
      const float* src = imgs[k] + (size_t)a0 * nx * nx;
      if (!imgs_on_device) {
        float* dst = c->imgs.as<float>() + hoff * nx * nx;
        SPI_CUDA(cudaMemcpyAsync(dst, src, (size_t)nb * nx * nx * sizeof(float), cudaMemcpyHostToDevice, s2));
        src = dst;
      }
      const int ip = (n - nx) / 2 + nx % 2;
      const int parts = std::max(1, std::min(8, (4 * c->sm_count + c->sub - 1) / c->sub));
      float2* fout = c->bf16 ? c->spec_tmp.as<float2>() : c->spectra.as<float2>() + hoff * plane;
      if (c->fft_own) {   // the own R2C (the class's box takes the same default as spi_bp_insert)
        const int rparts = std::max(1, std::min(8, (4 * c->sm_count + nb - 1) / std::max(nb, 1)));
        SPI_TRY(launch_rowfft(c, s2, src, nb, rparts, klp[k], c->padded.as<float2>()));
        SPI_TRY(launch_colfft(c, s2, c->padded.as<float2>(), nb, fout));
        c->count(2);
      } else {
        stage_kernel<<<dim3(c->sub, parts), 256, 0, s2>>>(src, nx, n, ip, nb, klp[k], c->padded.as<float>());
        SPI_TRY(check_kernel("stage_kernel"));
        c->count();
        SPI_CUFFT(cufftExecR2C(c->plan2d, c->padded.as<cufftReal>(), reinterpret_cast<cufftComplex*>(fout)));
      }
      if (c->bf16) {
        const size_t cntv = (size_t)nb * plane;
        to_bf16_kernel<<<grid_blocks(c, cntv, 256), 256, 0, s2>>>(
            fout, reinterpret_cast<__nv_bfloat162*>(c->spectra.p) + hoff * plane, cntv);
        SPI_TRY(check_kernel("to_bf16_kernel"));
        c->count();
      }
      const size_t nsl = (size_t)nb * c->nsym;
      SliceDesc* dsl = c->slices.as<SliceDesc>() + hoff * c->nsym;
      SPI_CUDA(cudaMemcpyAsync(dsl, hs_all + sl_off[k] + (size_t)a0 * c->nsym, nsl * sizeof(SliceDesc),
                               cudaMemcpyHostToDevice, s2));
      McClass m{};
      m.spec = c->bf16 ? (const void*)(reinterpret_cast<__nv_bfloat162*>(c->spectra.p) + hoff * plane)
                       : (const void*)(c->spectra.as<float2>() + hoff * plane);
      m.slices = dsl;
      m.g0 = insert_target(c, 0);
      m.g1 = insert_target(c, c->ngrids == 2 ? 1 : 0);
      m.item0 = items;
      m.nx = nx;
      m.nslices = (int)nsl;
      m.tab = cls_tab[k];
      hc[nc++] = m;
      items += (long long)nsl * n;
    }
    SPI_CUDA(cudaEventRecord(lead->ev_ready[h], s2));
    if (nc == 0) continue;
    SPI_CUDA(cudaStreamWaitEvent(st, lead->ev_ready[h], 0));
    SPI_CUDA(cudaMemcpyAsync(d_cls, hc, nc * sizeof(McClass), cudaMemcpyHostToDevice, st));
    SPI_CUDA(cudaMemsetAsync(d_work, 0, sizeof(unsigned long long), st));
    int per_sm = 1;
    if (lead->bf16)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, insert_mc_kernel<true>, 512, smem);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, insert_mc_kernel<false>, 512, smem);
    const int blocks = lead->sm_count * std::max(1, std::min(per_sm, env_int("SPI_MC_BLOCKS_PER_SM", 2)));
    int ev = lead->phase_begin(2, st);
    if (lead->bf16)
      insert_mc_kernel<true><<<blocks, 512, smem, st>>>(d_cls, nc, items, d_tabs, d_fl, ntab, d_work);
    else
      insert_mc_kernel<false><<<blocks, 512, smem, st>>>(d_cls, nc, items, d_tabs, d_fl, ntab, d_work);
    SPI_TRY(check_kernel("insert_mc_kernel"));
    lead->phase_end(ev);
    lead->count();
    SPI_CUDA(cudaEventRecord(lead->ev_done[h], st));
    for (int k = 0; k < ncls; ++k) {
      spi_ctx* c = ctxs[k];
      const int nb = std::min(c->sub, nimg[k] - r * c->sub);
      if (nb <= 0) continue;
      c->unfolded += nb;
      if (c->unfolded >= c->fold_every) SPI_TRY(fold_grids(c, false));
    }
    // the staging buffers and descriptors of every class are reused next round
  }
  for (int k = 0; k < ncls; ++k) {
    if (nimg[k] <= 0) continue;
    ctxs[k]->pending_sym0[0] = true;
    if (ctxs[k]->ngrids == 2) ctxs[k]->pending_sym0[1] = true;
  }
  SPI_CUDA(cudaStreamSynchronize(s2));
  SPI_CUDA(cudaStreamSynchronize(st));
  return 0;
}

extern "C" int spi_bp_insert_multi(spi_ctx* const* ctxs, int nclass, const float* const* imgs, const int* nimg,
                                   const float* const* angles, const uint8_t* const* half, int imgs_on_device) {
  return bp_insert_multi_impl(ctxs, nclass, imgs, nimg, angles, half, imgs_on_device);
}

// ----------------------------------------------------------------------------
// Autotuner of the insertion launch.  For the open reconstruction it times
// each candidate (kernel variant x threads per CTA x CTAs per SM) on one
// sub-batch of synthetic slices (orientations on a spiral over the sphere,
// zero spectra: the cost of a launch does not depend on the values), keeps
// the fastest, and zeroes the grids again.  Results are cached per (device,
// nx, grids, spectrum precision, symmetry count) for the process.
struct TuneVal {
  int mode, threads, bps;
  float ms;
};
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int, int>, TuneVal> g_tune;

static int bp_autotune_impl(spi_ctx* c, int force) {
  if (!c || c->ngrids == 0) return fail(kInvalid, "spi_bp_autotune: no open reconstruction (spi_bp_open)");
  if (c->inserted || c->merged)
    return fail(kInvalid, "spi_bp_autotune: call it right after spi_bp_open, before any image is inserted");
  SPI_CUDA(cudaSetDevice(c->device));
  const auto key = std::make_tuple(c->device, c->nx, c->ngrids, c->bf16, c->nsym);
  if (!force) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      c->insert_mode = it->second.mode;
      c->insert_threads = it->second.threads;
      c->insert_blocks_per_sm = it->second.bps;
      c->tuned_ms = it->second.ms;
      return 0;
    }
  }
  SPI_TRY(ensure_chunk_buffers(c));
  const int nx = c->nx, nsym = c->nsym;
  const int sample = std::min(c->sub, 512);
  const size_t nsl = (size_t)sample * nsym;
  SPI_TRY(c->hslices.ensure(nsl * sizeof(SliceDesc)));
  SliceDesc* hs = c->hslices.as<SliceDesc>();
  for (int a = 0; a < sample; ++a) {
    const double th = std::acos(1.0 - 2.0 * (a + 0.5) / sample) * 180.0 / M_PI;
    const float phi = (float)std::fmod(a * 137.50776405, 360.0), psi = (float)std::fmod(a * 222.4922359, 360.0);
    float dm[9];
    cang(phi, (float)th, psi, dm);
    for (int sy = 0; sy < nsym; ++sy) {
      float dms[9];
      if (nsym > 1) matmul33(&c->sym_dm[9 * sy], dm, dms);
      else memcpy(dms, dm, sizeof(dms));
      SliceDesc& d = hs[(size_t)a * nsym + sy];
      memcpy(d.dm, dms, 6 * sizeof(float));
      d.img = a;
      d.grid = (c->ngrids == 2) ? (short)(a & 1) : 0;
      d.cols = line_cols(c, dms);
    }
  }
  SPI_CUDA(cudaMemcpyAsync(c->slices.p, hs, nsl * sizeof(SliceDesc), cudaMemcpyHostToDevice, c->stream));
  const size_t plane = (size_t)c->n * (nx + 1);
  SPI_CUDA(cudaMemsetAsync(c->spectra.p, 0, (size_t)sample * plane * (c->bf16 ? 4 : 8), c->stream));
  float4* g1 = insert_target(c, c->ngrids == 2 ? 1 : 0);
  const int modes[2] = {kb_window4_ok(c->kb) ? 3 : 2, 2};
  const int shapes[5][2] = {{256, 2}, {256, 3}, {512, 2}, {128, 4}, {512, 1}};
  cudaEvent_t e0, e1;
  SPI_CUDA(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(kCuda, "cudaEventCreate failed");
  }
  const bool timing = c->timing;
  c->timing = false;
  TuneVal best{c->insert_mode, c->insert_threads, c->insert_blocks_per_sm, 1e30f};
  int st = 0;
  // two passes over the candidates, each shape's best pass counts (shapes
  // within ~1% of one another at 256^3 were otherwise picked by noise)
  float tmin[2][5];
  for (auto& row : tmin)
    for (float& v : row) v = 1e30f;
  for (int pass = 0; pass < 2 && !st; ++pass)
    for (int mi = 0; mi < 2 && !st; ++mi) {
      if (mi == 1 && modes[0] == modes[1]) break;
      for (int si = 0; si < 5; ++si) {
        c->insert_mode = modes[mi];
        c->insert_threads = shapes[si][0];
        c->insert_blocks_per_sm = shapes[si][1];
        if ((st = launch_insert(c, c->slices.as<SliceDesc>(), (int)nsl, g1))) break;   // warm-up
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 2 && !st; ++r) st = launch_insert(c, c->slices.as<SliceDesc>(), (int)nsl, g1);
        cudaEventRecord(e1, c->stream);
        if (st || (st = (cudaEventSynchronize(e1) == cudaSuccess) ? 0 : kCuda)) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        tmin[mi][si] = std::min(tmin[mi][si], 0.5f * ms);
      }
    }
  for (int mi = 0; mi < 2; ++mi)
    for (int si = 0; si < 5; ++si)
      if (tmin[mi][si] < best.ms) best = TuneVal{modes[mi], shapes[si][0], shapes[si][1], tmin[mi][si]};
  c->timing = timing;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->insert_mode = best.mode;
  c->insert_threads = best.threads;
  c->insert_blocks_per_sm = best.bps;
  c->tuned_ms = best.ms;
  if (st) return st;
  const size_t gbytes = grid_voxels(c) * sizeof(float4);
  for (int g = 0; g < c->ngrids; ++g) {
    SPI_CUDA(cudaMemsetAsync(c->gptr[g], 0, gbytes, c->stream));
    if (c->accum) SPI_CUDA(cudaMemsetAsync(c->part[g].p, 0, gbytes, c->stream));
  }
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  return 0;
}

extern "C" {

int spi_bp_autotune(spi_ctx* c, int force) { return bp_autotune_impl(c, force); }

int spi_bp_get_launch(const spi_ctx* c, int* kernel, int* threads, int* blocks_per_sm, float* tuned_ms) {
  if (!c) return fail(kInvalid, "NULL context");
  if (kernel) *kernel = c->insert_mode;
  if (threads) *threads = c->insert_threads;
  if (blocks_per_sm) *blocks_per_sm = c->insert_blocks_per_sm;
  if (tuned_ms) *tuned_ms = c->tuned_ms;
  return 0;
}

static int apply_sym0(spi_ctx* c, int g) {
  SPI_TRY(fold_grids(c, true));   // the grids hold the complete sums from here on
  if (!c->pending_sym0[g]) return 0;
  const int m = c->nx - 1;
  const int work = m * m + 2 * m;
  int ev = c->phase_begin(3);
  symplane0_kernel<<<(work + 255) / 256, 256, 0, c->stream>>>(c->gptr[g], c->nx);
  SPI_TRY(check_kernel("symplane0_kernel"));
  c->phase_end(ev);
  c->count();
  c->pending_sym0[g] = false;
  return 0;
}

// NRMW2 + inverse FFT + WINDKB2A of (grid ga [+ grid gb]) into vol (device)
static int finish_one(spi_ctx* c, int ga, int gb, float* dvol) {
  const int nx = c->nx, n = c->n;
  const size_t nvox = grid_voxels(c);
  SPI_TRY(c->cplx.ensure(nvox * sizeof(float2)));
  SPI_TRY(c->real3.ensure((size_t)n * n * n * sizeof(float)));
  if (c->plan3d == 0 || c->plan3d_n != n) {
    if (c->plan3d) cufftDestroy(c->plan3d);
    c->plan3d = 0;
    SPI_CUFFT(cufftPlan3d(&c->plan3d, n, n, n, CUFFT_C2R));
    SPI_CUFFT(cufftSetStream(c->plan3d, c->stream));
    c->plan3d_n = n;
  }
  int ev = c->phase_begin(4);
  nrmw2_kernel<<<grid_blocks(c, nvox, 256), 256, 0, c->stream>>>(
      c->gptr[ga], gb >= 0 ? c->gptr[gb] : nullptr, c->cplx.as<float2>(), nx);
  SPI_TRY(check_kernel("nrmw2_kernel"));
  c->phase_end(ev);
  c->count();
  ev = c->phase_begin(5);
  SPI_CUFFT(cufftExecC2R(c->plan3d, reinterpret_cast<cufftComplex*>(c->cplx.p), c->real3.as<cufftReal>()));
  c->phase_end(ev);
  // WINDKB2A: |WKB| table and shell voxel count depend on nx only
  if (c->wkb_nx != nx) {
    std::vector<float> wkb;
    windkb_table(nx, c->kb, wkb);
    SPI_TRY(c->wkb.ensure(wkb.size() * sizeof(float)));
    SPI_CUDA(cudaMemcpyAsync(c->wkb.p, wkb.data(), wkb.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    const int l2 = (nx / 2) * (nx / 2), l2p = (nx / 2 - 1) * (nx / 2 - 1), cc = nx / 2 + 1;
    long m = 0;
    for (int k = 1; k <= nx; ++k)
      for (int j = 1; j <= nx; ++j) {
        const int base = (k - cc) * (k - cc) + (j - cc) * (j - cc);
        if (base > l2) continue;
        for (int i = 1; i <= nx; ++i) {
          int lr = base + (i - cc) * (i - cc);
          if (lr >= l2p && lr <= l2) ++m;
        }
      }
    c->wkb_m = m;
    c->wkb_nx = nx;
  }
  const long m = c->wkb_m;
  const int ip = (n - nx) / 2 + nx % 2;
  const float pix = 1.0f / (float)((long long)n * n * n);
  const size_t total = (size_t)nx * nx * nx;
  ev = c->phase_begin(6);
  SPI_CUDA(cudaMemsetAsync(c->acc.p, 0, sizeof(double), c->stream));
  windkb_shell_kernel<<<grid_blocks(c, total, 256), 256, 0, c->stream>>>(c->real3.as<float>(), nx, ip, pix,
                                                                         c->wkb.as<float>(), c->acc.as<double>());
  SPI_TRY(check_kernel("windkb_shell_kernel"));
  windkb_out_kernel<<<grid_blocks(c, total, 256), 256, 0, c->stream>>>(c->real3.as<float>(), nx, ip, pix,
                                                                       c->wkb.as<float>(), c->acc.as<double>(),
                                                                       (double)(float)m, dvol);
  SPI_TRY(check_kernel("windkb_out_kernel"));
  c->phase_end(ev);
  c->count(2);
  if (c->nsym > 1) {
    // real-space symmetrisation (bp3f.f:252-279): SYMVOL(TEMP = volume) -> volume
    const size_t vbytes = total * sizeof(float);
    SPI_TRY(c->symtmp.ensure(vbytes + 9 * sizeof(float) * (size_t)c->nsym));
    float* q1 = c->symtmp.as<float>();
    float* rm = q1 + total;
    SPI_CUDA(cudaMemcpyAsync(q1, dvol, vbytes, cudaMemcpyDeviceToDevice, c->stream));
    SPI_CUDA(cudaMemcpyAsync(rm, c->sym_dm.data(), 9 * sizeof(float) * (size_t)c->nsym, cudaMemcpyHostToDevice,
                             c->stream));
    symvol_kernel<<<grid_blocks(c, total, 256), 256, 0, c->stream>>>(q1, dvol, nx, rm, c->nsym);
    SPI_TRY(check_kernel("symvol_kernel"));
    c->count();
  }
  return 0;
}

int spi_bp_finish(spi_ctx* c, float* vol_all, float* vol_1, float* vol_2, int out_on_device) {
  if (!c || c->ngrids == 0) return fail(kInvalid, "spi_bp_finish: no open reconstruction");
  SPI_CUDA(cudaSetDevice(c->device));
  for (int g = 0; g < c->ngrids; ++g) SPI_TRY(apply_sym0(c, g));
  const size_t vbytes = (size_t)c->nx * c->nx * c->nx * sizeof(float);
  struct Job { float* out; int ga, gb; } jobs[3];
  int nj = 0;
  if (c->ngrids == 1) {
    if (vol_all) jobs[nj++] = {vol_all, 0, -1};
  } else {
    if (vol_1) jobs[nj++] = {vol_1, 0, -1};
    if (vol_all) jobs[nj++] = {vol_all, 0, 1};
    if (vol_2) jobs[nj++] = {vol_2, 1, -1};
  }
  // Host outputs: each volume gets its own staging buffer, and its copy to
  // the host runs on the second stream while the next volume is computed.
  if (!out_on_device) {
    SPI_TRY(c->volbuf.ensure((size_t)std::max(nj, 1) * vbytes));
    SPI_TRY(ensure_pipeline_events(c, 3));
  }
  for (int t = 0; t < nj; ++t) {
    float* dst = out_on_device ? jobs[t].out : c->volbuf.as<float>() + (size_t)t * (vbytes / sizeof(float));
    SPI_TRY(finish_one(c, jobs[t].ga, jobs[t].gb, dst));
    if (!out_on_device) {
      SPI_CUDA(cudaEventRecord(c->ev_ready[t], c->stream));
      SPI_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_ready[t], 0));
      SPI_CUDA(cudaMemcpyAsync(jobs[t].out, dst, vbytes, cudaMemcpyDeviceToHost, c->stream2));
    }
  }
  if (!out_on_device) SPI_CUDA(cudaStreamSynchronize(c->stream2));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int spi_bp_partial_out(spi_ctx* c, int g, float* x_out, float* w_out) {
  if (!c || c->ngrids == 0 || g < 0 || g >= c->ngrids) return fail(kInvalid, "spi_bp_partial_out: bad grid");
  SPI_CUDA(cudaSetDevice(c->device));
  SPI_TRY(apply_sym0(c, g));
  const size_t nvox = grid_voxels(c);
  SPI_TRY(c->cplx.ensure(nvox * sizeof(float2)));
  SPI_TRY(c->real3.ensure(std::max(nvox * sizeof(float), (size_t)c->n * c->n * c->n * sizeof(float))));
  grid_split_kernel<<<grid_blocks(c, nvox, 256), 256, 0, c->stream>>>(c->gptr[g], c->cplx.as<float2>(),
                                                                      c->real3.as<float>(), nvox);
  SPI_TRY(check_kernel("grid_split_kernel"));
  c->count();
  if (x_out) SPI_CUDA(cudaMemcpyAsync(x_out, c->cplx.p, nvox * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
  if (w_out) SPI_CUDA(cudaMemcpyAsync(w_out, c->real3.p, nvox * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int spi_bp_partial_add(spi_ctx* c, int g, const float* x_in, const float* w_in) {
  if (!c || c->ngrids == 0 || g < 0 || g >= c->ngrids) return fail(kInvalid, "spi_bp_partial_add: bad grid");
  if (!x_in || !w_in) return fail(kInvalid, "spi_bp_partial_add: NULL partial");
  SPI_CUDA(cudaSetDevice(c->device));
  SPI_TRY(apply_sym0(c, g));  // inserted images are symmetrised before the merge
  const size_t nvox = grid_voxels(c);
  SPI_TRY(c->cplx.ensure(nvox * sizeof(float2)));
  SPI_TRY(c->real3.ensure(std::max(nvox * sizeof(float), (size_t)c->n * c->n * c->n * sizeof(float))));
  SPI_CUDA(cudaMemcpyAsync(c->cplx.p, x_in, nvox * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
  SPI_CUDA(cudaMemcpyAsync(c->real3.p, w_in, nvox * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  grid_add_kernel<<<grid_blocks(c, nvox, 256), 256, 0, c->stream>>>(c->gptr[g], c->cplx.as<float2>(),
                                                                    c->real3.as<float>(), nvox);
  SPI_TRY(check_kernel("grid_add_kernel"));
  c->count();
  c->merged = true;
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int spi_bp_close(spi_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  bp_release(c);
  return 0;
}

int spi_bp3f(spi_ctx* c, const float* imgs, int nx, int nang, const float* angles, const float* sym_angles,
             int nsym, float* vol_out) {
  SPI_TRY(spi_bp_open(c, nx, 1, sym_angles, nsym));
  SPI_TRY(spi_bp_insert(c, imgs, nang, angles, nullptr, 0));
  SPI_TRY(spi_bp_finish(c, vol_out, nullptr, nullptr, 0));
  return spi_bp_close(c);
}

int spi_bp32f(spi_ctx* c, const float* imgs, int nx, int nang, const float* angles, const float* sym_angles,
              int nsym, const uint8_t* half, float* vol_all, float* vol_1, float* vol_2) {
  if (!half) return fail(kInvalid, "spi_bp32f: half-set mask is required");
  SPI_TRY(spi_bp_open(c, nx, 2, sym_angles, nsym));
  SPI_TRY(spi_bp_insert(c, imgs, nang, angles, half, 0));
  SPI_TRY(spi_bp_finish(c, vol_all, vol_1, vol_2, 0));
  return spi_bp_close(c);
}

}  // extern "C"
