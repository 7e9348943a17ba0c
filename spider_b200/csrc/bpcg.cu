// BP CG, linear interpolation (BPCG bpcg.f:70 -> BPCG_2 bpcg.f:425-814 ->
// HIANG hiang.f:40-112 -> BPCG_3_LIN bpcg.f:818-1238) on sm_100a.
//
// Operators (voxel runs from PREPCUB_S, prepcub_s.f:54-111):
//   A   = PRJCQ_N (prjcq.f:48-82): every sphere voxel splats bilinearly into
//         the projection.  One CTA per projection keeps the image in shared
//         memory (n <= 224) and walks whole runs with the reference's
//         sequential XB = XB + DM(1) accumulation, so sample positions are
//         bit-identical; shared-memory atomics accumulate.
//   A^T = BCKPJ_LIN (bckpj.f:59-94, SP_MP branch): every sphere voxel
//         gathers from each projection through the PROJT difference table
//         (bpcg.f:732-742), computed on the fly from four pixels with the
//         same float operations.  One thread per voxel sums the projections
//         in image order, the order of the reference's image loop, so the
//         back-projection is bit-identical to the CPU form.
// CG scalars (DELSQ, AKDEN, P, Q) are FP64 device scalars; the vectors and
// projections are FP64 by default and FP32 (the reference's REAL) on request.
// One CG iteration is a fixed kernel sequence captured once as a CUDA graph.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "../../include/spider_b200.h"
#include "ctx.h"

namespace spi {

struct CgRun {
  int l1, l2;   // first/last 1-based linear index of the run
  int x, y, z;  // 1-based coordinates of the first voxel
};

struct CgDM {
  float d[6];
};

static void prepcub_s(int n, float ri, int ldp, std::vector<CgRun>& runs) {
  const float r = ri * ri;
  int nmat = 0;
  runs.clear();
  for (int i1 = 1; i1 <= n; ++i1) {
    float t = (float)(i1 - ldp);
    float xx = t * t;
    for (int i2 = 1; i2 <= n; ++i2) {
      float t2 = (float)(i2 - ldp);
      float yy = t2 * t2 + xx;
      bool first = true;
      for (int i3 = 1; i3 <= n; ++i3) {
        ++nmat;
        float t3 = (float)(i3 - ldp);
        float rc = t3 * t3 + yy;
        if (first) {
          if (rc > r) continue;
          first = false;
          runs.push_back(CgRun{nmat, nmat, i3, i2, i1});
        } else if (rc <= r) {
          runs.back().l2 = nmat;
        }
      }
    }
  }
}

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void block_add_d(double v, double* dst) {
  __shared__ double red[32];
  v = warp_sum_d(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    w = warp_sum_d(w);
    if (threadIdx.x == 0) atomicAdd(dst, w);
  }
  __syncthreads();
}

// run of a voxel: index of the run containing linear voxel q (0-based), via
// the per-line run table line_run[(z-1)*n + (y-1)] (-1 when the line is empty)

// round-to-nearest arithmetic without contraction, for FP32 and FP64
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }

#include "bpcg_fbs.cuh"

// ---------------------------------------------------------------------------
// ASTASQ (bpcg.f:1244-1274): FP64 sums per image; counts are host constants.
__global__ void astasq_kernel(const float* __restrict__ projs, int n, float r2, double* __restrict__ acc) {
  const float* x = projs + (size_t)blockIdx.x * n * n;
  const int nc = n / 2 + 1;
  double aba = 0.0, ssq = 0.0, sus = 0.0;
  for (int p = threadIdx.x; p < n * n; p += blockDim.x) {
    int i = p % n + 1, j = p / n + 1;
    float t = (float)(j - nc), t2 = (float)(i - nc);
    float rr = __fadd_rn(__fmul_rn(t, t), __fmul_rn(t2, t2));
    float v = x[p];
    if (rr > r2) aba += (double)v;
    else { ssq += (double)v * (double)v; sus += (double)v; }
  }
  block_add_d(aba, acc + 0);
  block_add_d(ssq, acc + 1);
  block_add_d(sus, acc + 2);
}

// ---------------------------------------------------------------------------
// A^T: BCKPJ_LIN gather.  Threads own voxels of the run list (flattened
// through run_of[]); each adds projections [k0, k1) in order.
template <class T>
__global__ void __launch_bounds__(256) bckpj_kernel(T* __restrict__ cube, const CgRun* __restrict__ runs,
                                                    const int* __restrict__ vox_run, const int* __restrict__ vox_off,
                                                    long long nvox, const T* __restrict__ projs,
                                                    const CgDM* __restrict__ dms, const int* __restrict__ lb,
                                                    int k0, int k1, int n, int ldp) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const CgRun r = runs[vox_run[v]];
    const int jt = vox_off[v];
    const size_t lin = (size_t)r.l1 - 1 + jt;
    T c = cube[lin];
    const float fx = (float)(r.x - ldp), fy = (float)(r.y - ldp), fz = (float)(r.z - ldp), fj = (float)jt;
    for (int k = k0; k < k1; ++k) {
      const CgDM dm = dms[k];
      // XB = ((X-LDP)*DM1 + (Y-LDP)*DM2 + (Z-LDP)*DM3) + LDPNM ; XBB = XB + JT*DM1
      const float xb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[0]), __fmul_rn(fy, dm.d[1])), __fmul_rn(fz, dm.d[2])), (float)ldp);
      const float yb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[3]), __fmul_rn(fy, dm.d[4])), __fmul_rn(fz, dm.d[5])), (float)ldp);
      const float xbb = __fadd_rn(xb, __fmul_rn(fj, dm.d[0]));
      const float ybb = __fadd_rn(yb, __fmul_rn(fj, dm.d[3]));
      const int iqx = __float2int_rz(xbb), iqy = __float2int_rz(ybb);
      const T* P = projs + (size_t)k * n * n;
      const int I = (iqy - 1) * n + iqx;  // PROJT column, 1-based
      T b1 = 0, b2 = 0, b3 = 0, b4 = 0;
      if (I >= 1 && I <= n * n - n - 1) {
        T p00 = P[I - 1], p01 = P[I + n - 1], p10 = P[I], p11 = P[I + n];
        if (lb) {
          const int w = lb[k];
          if (w > 1) {
            const T fw = (T)w;
            p00 = rmul(p00, fw); p01 = rmul(p01, fw); p10 = rmul(p10, fw); p11 = rmul(p11, fw);
          }
        }
        b1 = p00;
        b2 = rsub(p01, p00);
        b3 = rsub(p10, p00);
        b4 = rsub(rsub(p11, p10), b2);
      }
      const T dy = (T)__fsub_rn(ybb, (float)iqy), dx = (T)__fsub_rn(xbb, (float)iqx);
      c = radd(radd(radd(c, b1), rmul(dy, b2)), rmul(dx, radd(b3, rmul(dy, b4))));
    }
    cube[lin] = c;
  }
}

// ---------------------------------------------------------------------------
// PRJCQ_N splat of one voxel run into an image in shared memory.  Positions
// follow the reference's sequential walk XB = XB + DM(1), YB = YB + DM(4)
// (prjcq.f:64-80), so every sample lands where the reference puts it.  Along
// a run the 2 x 2 target cell moves by at most one pixel per voxel (|DM(1)|,
// |DM(4)| <= 1), so the four pixel sums of the current cell are kept in
// registers; pixels the next cell shares move with it and only the others
// are added to shared memory.  Every weight goes to the same pixel as in the
// reference; only the grouping of the sums differs.
template <class T, class A>
__device__ __forceinline__ void splat_run(A* img, const T* __restrict__ cube, const CgRun& r, const CgDM& dm, int n,
                                          int ldp) {
  const float fx = (float)(r.x - ldp), fy = (float)(r.y - ldp), fz = (float)(r.z - ldp);
  float xb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[0]), __fmul_rn(fy, dm.d[1])), __fmul_rn(fz, dm.d[2])), (float)ldp);
  float yb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[3]), __fmul_rn(fy, dm.d[4])), __fmul_rn(fz, dm.d[5])), (float)ldp);
  int cx = -4, cy = -4;                 // cached cell (none)
  A a00 = 0, a10 = 0, a01 = 0, a11 = 0; // sums at (cx,cy), (cx+1,cy), (cx,cy+1), (cx+1,cy+1)
  auto flush_to = [&](int qx, int qy) {
    A n00 = 0, n10 = 0, n01 = 0, n11 = 0;
    auto move = [&](A v, int ox, int oy) {
      const int ex = ox - qx, ey = oy - qy;
      if (ex == 0 && ey == 0) n00 += v;
      else if (ex == 1 && ey == 0) n10 += v;
      else if (ex == 0 && ey == 1) n01 += v;
      else if (ex == 1 && ey == 1) n11 += v;
      else if (v != (A)0) atomicAdd(img + (oy - 1) * n + (ox - 1), v);
    };
    move(a00, cx, cy);
    move(a10, cx + 1, cy);
    move(a01, cx, cy + 1);
    move(a11, cx + 1, cy + 1);
    a00 = n00; a10 = n10; a01 = n01; a11 = n11;
    cx = qx; cy = qy;
  };
  for (int j = r.l1; j <= r.l2; ++j) {
    const int iqx = __float2int_rz(xb), iqy = __float2int_rz(yb);
    if (iqx >= 1 && iqx < n && iqy >= 1 && iqy < n) {
      const T cv = cube[(size_t)j - 1];
      const T dx = (T)__fsub_rn(xb, (float)iqx);
      const T dy = rmul((T)__fsub_rn(yb, (float)iqy), cv);
      const T dx1m = rsub((T)1, dx);
      const T dy1m = rsub(cv, dy);
      if (iqx != cx || iqy != cy) flush_to(iqx, iqy);
      a00 += (A)rmul(dx1m, dy1m);
      a10 += (A)rmul(dx, dy1m);
      a01 += (A)rmul(dx1m, dy);
      a11 += (A)rmul(dx, dy);
    }
    xb = __fadd_rn(xb, dm.d[0]);
    yb = __fadd_rn(yb, dm.d[3]);
  }
  flush_to(-4, -4);
}

// ---------------------------------------------------------------------------
// A: PRJCQ_N splat, one CTA per projection, image privatised in shared memory.
// T is the type of the volume and projections, A that of the shared-memory
// accumulator (A = float with T = double: FP32 native shared atomics, a third
// of the shared memory, FP64 everywhere else).
template <class T, class A>
__global__ void __launch_bounds__(512) prjcq_smem_kernel(const T* __restrict__ cube, const CgRun* __restrict__ runs,
                                                         int nruns, const CgDM* __restrict__ dms, int n, int ldp,
                                                         T* __restrict__ projs) {
  extern __shared__ __align__(16) unsigned char smraw[];
  A* img = reinterpret_cast<A*>(smraw);
  const int k = blockIdx.x;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) img[i] = (A)0;
  __syncthreads();
  const CgDM dm = dms[k];
  for (int ri = threadIdx.x; ri < nruns; ri += blockDim.x) splat_run<T, A>(img, cube, runs[ri], dm, n, ldp);
  __syncthreads();
  T* out = projs + (size_t)k * n * n;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) out[i] = (T)img[i];
}

// ---------------------------------------------------------------------------
// Mixed-precision operators (precision modes 2 and 3).  Projections live only
// as the reference's PROJT four-term table (bpcg.f:732-742), one entry
// {B1, B2, B3, B4} per pixel column I: B1 = P(I), B2 = P(I+N) - P(I),
// B3 = P(I+1) - P(I), B4 = P(I+N+1) - P(I+1) - B2 (1-based, with the HIANG
// weight LB applied to the four pixels first), so A^T reads one vector per
// (voxel, image) instead of four scattered values.  The terms are formed in
// FP64 and stored in FP64 (mode 4) or rounded once to FP32 (modes 2, 3).
// Tables are made per chunk of images and consumed right away.
template <bool WIDE> struct ProjtEntry;
template <> struct ProjtEntry<false> { float4 v; };
template <> struct ProjtEntry<true> { double2 a, b; };

template <bool WIDE>
__device__ __forceinline__ void projt_store(ProjtEntry<WIDE>* out, double b1, double b2, double b3, double b4);
template <>
__device__ __forceinline__ void projt_store<false>(ProjtEntry<false>* out, double b1, double b2, double b3, double b4) {
  out->v = make_float4((float)b1, (float)b2, (float)b3, (float)b4);
}
template <>
__device__ __forceinline__ void projt_store<true>(ProjtEntry<true>* out, double b1, double b2, double b3, double b4) {
  out->a = make_double2(b1, b2);
  out->b = make_double2(b3, b4);
}
__device__ __forceinline__ void projt_load(const ProjtEntry<false>* p, double& b1, double& b2, double& b3, double& b4) {
  const float4 v = __ldg(&p->v);
  b1 = v.x; b2 = v.y; b3 = v.z; b4 = v.w;
}
__device__ __forceinline__ void projt_load(const ProjtEntry<true>* p, double& b1, double& b2, double& b3, double& b4) {
  const double2 a = __ldg(&p->a), b = __ldg(&p->b);
  b1 = a.x; b2 = a.y; b3 = b.x; b4 = b.y;
}

// the four terms at column I from pixel values val(i) (0-based) and weight w
template <bool WIDE, class V>
__device__ __forceinline__ void projt_make(ProjtEntry<WIDE>* out, V val, int I, int n, double w) {
  if (I < 1 || I > n * n - n - 1) {
    projt_store<WIDE>(out, 0.0, 0.0, 0.0, 0.0);
    return;
  }
  double p00 = val(I - 1), p01 = val(I + n - 1), p10 = val(I), p11 = val(I + n);
  if (w > 1.0) { p00 *= w; p01 *= w; p10 *= w; p11 *= w; }
  const double b2 = p01 - p00;
  projt_store<WIDE>(out, p00, b2, p10 - p00, (p11 - p10) - b2);
}

// PROJT of input images [nimg][n*n] (weight 1)
template <bool WIDE>
__global__ void projt_images_kernel(const float* __restrict__ imgs, int n, int nimg, ProjtEntry<WIDE>* __restrict__ projt) {
  const long long total = (long long)nimg * n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t / ((long long)n * n));
    const int I = (int)(t % ((long long)n * n)) + 1;
    const float* P = imgs + (size_t)k * n * n;
    projt_make<WIDE>(projt + t, [P](int i) { return (double)P[i]; }, I, n, 1.0);
  }
}

// max |x| over the sphere voxels, as the bit pattern of a non-negative
// double (which orders like the unsigned integer), for the fixed-point scale
template <class T>
__global__ void absmax_kernel(const T* __restrict__ x, const CgRun* __restrict__ runs, const int* __restrict__ vr,
                              const int* __restrict__ vo, long long nvox, unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs((double)x[(size_t)runs[vr[v]].l1 - 1 + vo[v]]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// PRJCQ_N of projections kbase .. kbase+gridDim.x-1, accumulated in fixed
// point in shared memory with native 32-bit integer atomics (exact and order
// independent), written out as PROJT with the HIANG weights lb[k].
//
// Scale: every voxel whose projection can reach a pixel lies in a 2 x 2 x
// (2 RI) prism, whose lattice points number at most the volume of the prism
// grown by the half-diagonal of a unit cube, pi (sqrt 2 + sqrt 3 / 2)^2
// (2 RI + sqrt 3) = `mcap`; each adds at most max|x| (bilinear weights
// <= 1).  Mode 3 rounds each contribution to q = w * 0.95 * 2^31 / (mcap *
// max|x|) in one int32 word per pixel (a step of ~1e-6 max|x|).  Modes 2
// and 4 (WIDE) round to a 2^16 finer grid, q = w * 0.95 * 2^47 / (mcap * max|x|)
// in 64 bits, and adds q >> 16 and q & 0xffff into two int32 words per
// pixel: the high sum stays within 0.95 * 2^31 + mcap, the low one within
// mcap * 65535, and the pixel is hi * 65536 + lo exactly (a step of ~1e-11
// max|x|).
template <class T, bool WIDE, bool WT>
__global__ void __launch_bounds__(512) prjcq_projt_kernel(const T* __restrict__ cube, const CgRun* __restrict__ runs,
                                                          int nruns, const CgDM* __restrict__ dms,
                                                          const int* __restrict__ lb, int kbase, int n, int ldp,
                                                          const unsigned long long* __restrict__ maxabs_bits,
                                                          float mcap, ProjtEntry<WT>* __restrict__ projt) {
  extern __shared__ __align__(16) unsigned char smraw[];
  int* hi = reinterpret_cast<int*>(smraw);
  int* lo = hi + n * n;   // WIDE only
  const int k = kbase + blockIdx.x;
  for (int i = threadIdx.x; i < n * n * (WIDE ? 2 : 1); i += blockDim.x) hi[i] = 0;
  const double maxabs = __longlong_as_double((long long)*maxabs_bits);
  const double full = WIDE ? 0.95 * 140737488355328.0 : 0.95 * 2147483648.0;   // 2^47 or 2^31
  const double scale = maxabs > 0.0 ? full / ((double)mcap * maxabs) : 0.0;
  __syncthreads();
  const CgDM dm = dms[k];
  auto add = [&](int* p, double w) {
    if (WIDE) {
      const long long q = __double2ll_rn(w * scale);
      atomicAdd(p, (int)(q >> 16));
      atomicAdd(p + n * n, (int)(q & 0xffff));
    } else {
      atomicAdd(p, __double2int_rn(w * scale));
    }
  };
  for (int ri = threadIdx.x; ri < nruns; ri += blockDim.x) {
    const CgRun r = runs[ri];
    const float fx = (float)(r.x - ldp), fy = (float)(r.y - ldp), fz = (float)(r.z - ldp);
    float xb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[0]), __fmul_rn(fy, dm.d[1])), __fmul_rn(fz, dm.d[2])), (float)ldp);
    float yb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[3]), __fmul_rn(fy, dm.d[4])), __fmul_rn(fz, dm.d[5])), (float)ldp);
    T cnext = cube[(size_t)r.l1 - 1];   // the next voxel's value, loaded one step ahead
    for (int j = r.l1; j <= r.l2; ++j) {
      const T cv = cnext;
      if (j < r.l2) cnext = cube[(size_t)j];
      const int iqx = __float2int_rz(xb), iqy = __float2int_rz(yb);
      if (iqx >= 1 && iqx < n && iqy >= 1 && iqy < n) {
        const T dx = (T)__fsub_rn(xb, (float)iqx);
        const T dy = rmul((T)__fsub_rn(yb, (float)iqy), cv);
        const T dx1m = rsub((T)1, dx);
        const T dy1m = rsub(cv, dy);
        int* p = hi + (iqy - 1) * n + (iqx - 1);
        add(p, (double)rmul(dx1m, dy1m));
        add(p + 1, (double)rmul(dx, dy1m));
        add(p + n, (double)rmul(dx1m, dy));
        add(p + n + 1, (double)rmul(dx, dy));
      }
      xb = __fadd_rn(xb, dm.d[0]);
      yb = __fadd_rn(yb, dm.d[3]);
    }
  }
  __syncthreads();
  const double inv = scale > 0.0 ? 1.0 / scale : 0.0;
  const double w = lb ? (double)lb[k] : 1.0;
  ProjtEntry<WT>* out = projt + (size_t)blockIdx.x * n * n;
  auto val = [&](int i) {
    return WIDE ? ((double)hi[i] * 65536.0 + (double)lo[i]) * inv : (double)hi[i] * inv;
  };
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) projt_make<WT>(out + i, val, i + 1, n, w);
}

// The same projector for images too large for one CTA's shared memory: C
// CTAs per projection, CTA b owning the pixel rows [b R, b R + R) (R =
// ceil(n / C)) and accumulating rows [b R, b R + R + 2) of the fixed-point
// image, the two extra rows being what its PROJT entries read beyond the
// band (I + N, and I + 1 wrapping to the next row at the last column).  Every
// CTA walks all runs with the reference's sequential XB/YB steps and splats
// only into its rows, so all atomics stay in its own shared memory; the
// voxels of other bands cost four instructions each.  Integer sums make the
// tables identical to those of the one-CTA kernel.  (A 2-4 CTA cluster
// adding into one another's bands through distributed shared memory was
// measured 3-8x slower at n = 256.)
template <class T, bool WIDE, bool WT>
__global__ void __launch_bounds__(512) prjcq_projt_band_kernel(
    const T* __restrict__ cube, const CgRun* __restrict__ runs, int nruns, const CgDM* __restrict__ dms,
    const int* __restrict__ lb, int kbase, int n, int ldp, int C, const unsigned long long* __restrict__ maxabs_bits,
    float mcap, ProjtEntry<WT>* __restrict__ projt) {
  const int R = (n + C - 1) / C;
  const int proj = blockIdx.x / C, b = blockIdx.x % C;
  const int r0 = b * R;
  const int r1 = min(n, r0 + R);             // owned rows [r0, r1)
  const int h1 = min(n, r0 + R + 2);         // accumulated rows [r0, h1)
  const int words = (R + 2) * n;             // per array
  extern __shared__ __align__(16) unsigned char smraw[];
  int* hi = reinterpret_cast<int*>(smraw);   // lo = hi + words (WIDE)
  const int k = kbase + proj;
  for (int i = threadIdx.x; i < words * (WIDE ? 2 : 1); i += blockDim.x) hi[i] = 0;
  const double maxabs = __longlong_as_double((long long)*maxabs_bits);
  const double full = WIDE ? 0.95 * 140737488355328.0 : 0.95 * 2147483648.0;   // 2^47 or 2^31
  const double scale = maxabs > 0.0 ? full / ((double)mcap * maxabs) : 0.0;
  __syncthreads();
  auto add = [&](int local, double w) {
    if (WIDE) {
      const long long q = __double2ll_rn(w * scale);
      atomicAdd(hi + local, (int)(q >> 16));
      atomicAdd(hi + words + local, (int)(q & 0xffff));
    } else {
      atomicAdd(hi + local, __double2int_rn(w * scale));
    }
  };
  const CgDM dm = dms[k];
  const float ystep = dm.d[3];
  for (int ri = threadIdx.x; ri < nruns; ri += blockDim.x) {
    const CgRun r = runs[ri];
    const float fx = (float)(r.x - ldp), fy = (float)(r.y - ldp), fz = (float)(r.z - ldp);
    float xb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[0]), __fmul_rn(fy, dm.d[1])), __fmul_rn(fz, dm.d[2])), (float)ldp);
    float yb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[3]), __fmul_rn(fy, dm.d[4])), __fmul_rn(fz, dm.d[5])), (float)ldp);
    // A run whose rows all miss the band is skipped: its YB is linear in the
    // step up to the walk's rounding (well under the 2-row margin).
    const float ye = yb + (float)(r.l2 - r.l1) * ystep;
    if (fmaxf(yb, ye) + 2.0f < (float)r0 || fminf(yb, ye) - 2.0f > (float)(h1 + 1)) continue;
    for (int j = r.l1; j <= r.l2; ++j) {
      const int iqy = __float2int_rz(yb);
      // rows iqy-1 and iqy (0-based) of the splat; skip unless one is accumulated here
      if (iqy >= r0 && iqy - 1 < h1) {
        const int iqx = __float2int_rz(xb);
        if (iqx >= 1 && iqx < n && iqy >= 1 && iqy < n) {
          const T cv = cube[(size_t)j - 1];
          const T dx = (T)__fsub_rn(xb, (float)iqx);
          const T dy = rmul((T)__fsub_rn(yb, (float)iqy), cv);
          const T dx1m = rsub((T)1, dx);
          const T dy1m = rsub(cv, dy);
          const int ya = iqy - 1, yb1 = iqy;   // pixel rows, 0-based
          if (ya >= r0 && ya < h1) {
            const int l = (ya - r0) * n + (iqx - 1);
            add(l, (double)rmul(dx1m, dy1m));
            add(l + 1, (double)rmul(dx, dy1m));
          }
          if (yb1 >= r0 && yb1 < h1) {
            const int l = (yb1 - r0) * n + (iqx - 1);
            add(l, (double)rmul(dx1m, dy));
            add(l + 1, (double)rmul(dx, dy));
          }
        }
      } else if ((ystep > 0.0f && iqy > h1) || (ystep < 0.0f && iqy < r0)) {
        // past the band: adding DM(4) of one sign moves YB (and its
        // truncation) one way only, so no later voxel of the run reaches it
        break;
      }
      xb = __fadd_rn(xb, dm.d[0]);
      yb = __fadd_rn(yb, dm.d[3]);
    }
  }
  __syncthreads();
  const double inv = scale > 0.0 ? 1.0 / scale : 0.0;
  const double w = lb ? (double)lb[k] : 1.0;
  ProjtEntry<WT>* out = projt + (size_t)proj * n * n;
  auto val = [&](int pix) {
    const int l = pix - r0 * n;
    return WIDE ? ((double)hi[l] * 65536.0 + (double)hi[words + l]) * inv : (double)hi[l] * inv;
  };
  for (int i = r0 * n + threadIdx.x; i < r1 * n; i += blockDim.x) projt_make<WT>(out + i, val, i + 1, n, w);
}

// BCKPJ_LIN from PROJT tables of images [k0, k1) (table of image k at
// projt + (k - kbase) * n * n), accumulating in T.
template <class T, bool WIDE>
__global__ void __launch_bounds__(256) bckpj_projt_kernel(T* __restrict__ cube, const CgRun* __restrict__ runs,
                                                          const int* __restrict__ vox_run, const int* __restrict__ vox_off,
                                                          long long nvox, const ProjtEntry<WIDE>* __restrict__ projt,
                                                          const CgDM* __restrict__ dms, int kbase, int k0, int k1, int n,
                                                          int ldp) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const CgRun r = runs[vox_run[v]];
    const int jt = vox_off[v];
    const size_t lin = (size_t)r.l1 - 1 + jt;
    T c = cube[lin];
    const float fx = (float)(r.x - ldp), fy = (float)(r.y - ldp), fz = (float)(r.z - ldp), fj = (float)jt;
    for (int k = k0; k < k1; ++k) {
      const CgDM dm = dms[k];
      const float xb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[0]), __fmul_rn(fy, dm.d[1])), __fmul_rn(fz, dm.d[2])), (float)ldp);
      const float yb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[3]), __fmul_rn(fy, dm.d[4])), __fmul_rn(fz, dm.d[5])), (float)ldp);
      const float xbb = __fadd_rn(xb, __fmul_rn(fj, dm.d[0]));
      const float ybb = __fadd_rn(yb, __fmul_rn(fj, dm.d[3]));
      const int iqx = __float2int_rz(xbb), iqy = __float2int_rz(ybb);
      const int I = (iqy - 1) * n + iqx;  // PROJT column, 1-based
      double b1 = 0.0, b2 = 0.0, b3 = 0.0, b4 = 0.0;
      if (I >= 1 && I <= n * n - n - 1) projt_load(projt + (size_t)(k - kbase) * n * n + (I - 1), b1, b2, b3, b4);
      const T dy = (T)__fsub_rn(ybb, (float)iqy), dx = (T)__fsub_rn(xbb, (float)iqx);
      c = radd(radd(radd(c, (T)b1), rmul(dy, (T)b2)), rmul(dx, radd((T)b3, rmul(dy, (T)b4))));
    }
    cube[lin] = c;
  }
}

// Same splat with global atomics, for images that exceed shared memory.
template <class T>
__global__ void __launch_bounds__(256) prjcq_global_kernel(const T* __restrict__ cube, const CgRun* __restrict__ runs,
                                                           int nruns, const CgDM* __restrict__ dms, int nang, int n,
                                                           int ldp, T* __restrict__ projs) {
  const long long total = (long long)nruns * nang;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t / nruns);
    const CgRun r = runs[t % nruns];
    const CgDM dm = dms[k];
    T* img = projs + (size_t)k * n * n;
    const float fx = (float)(r.x - ldp), fy = (float)(r.y - ldp), fz = (float)(r.z - ldp);
    float xb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[0]), __fmul_rn(fy, dm.d[1])), __fmul_rn(fz, dm.d[2])), (float)ldp);
    float yb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[3]), __fmul_rn(fy, dm.d[4])), __fmul_rn(fz, dm.d[5])), (float)ldp);
    for (int j = r.l1; j <= r.l2; ++j) {
      const int iqx = __float2int_rz(xb), iqy = __float2int_rz(yb);
      const T cv = cube[(size_t)j - 1];
      const T dx = (T)__fsub_rn(xb, (float)iqx);
      const T dy = rmul((T)__fsub_rn(yb, (float)iqy), cv);
      const T dx1m = rsub((T)1, dx);
      const T dy1m = rsub(cv, dy);
      if (iqx >= 1 && iqx < n && iqy >= 1 && iqy < n) {
        T* p = img + (iqy - 1) * n + (iqx - 1);
        atomicAdd(p, rmul(dx1m, dy1m));
        atomicAdd(p + 1, rmul(dx, dy1m));
        atomicAdd(p + n, rmul(dx1m, dy));
        atomicAdd(p + n + 1, rmul(dx, dy));
      }
      xb = __fadd_rn(xb, dm.d[0]);
      yb = __fadd_rn(yb, dm.d[3]);
    }
  }
}

// ---------------------------------------------------------------------------
// vector kernels over the sphere voxels (flattened run list)
__device__ __forceinline__ size_t vox_lin(const CgRun* runs, const int* vr, const int* vo, long long v) {
  return (size_t)runs[vr[v]].l1 - 1 + vo[v];
}

// CB -= QT inside the sphere (bpcg.f:780-790); acc[0] += CB^2 (BNORM)
template <class T>
__global__ void cb_background_kernel(T* __restrict__ cb, const CgRun* __restrict__ runs, const int* __restrict__ vr,
                                     const int* __restrict__ vo, long long nvox, T qt, double* __restrict__ acc) {
  double s = 0.0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const size_t q = vox_lin(runs, vr, vo, v);
    const T c = rsub(cb[q], qt);
    cb[q] = c;
    s += (double)c * (double)c;
  }
  block_add_d(s, acc);
}

// acc[0] += sum a*b over the sphere (FP64)
template <class T>
__global__ void dot_kernel(const T* __restrict__ a, const T* __restrict__ b, const CgRun* __restrict__ runs,
                           const int* __restrict__ vr, const int* __restrict__ vo, long long nvox,
                           double* __restrict__ acc) {
  double s = 0.0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const size_t q = vox_lin(runs, vr, vo, v);
    s += (double)a[q] * (double)b[q];
  }
  block_add_d(s, acc);
}

// CG scalar state, all FP64, on the device
struct CgScal {
  double delsq, akden, q, p, err, chi2, bnorm, pad;
};

// Q = Q*DELSQ (bpcg.f:1160), then BCKP = CB - Q*BCKP inside the sphere
template <class T>
__global__ void dir_update_kernel(T* __restrict__ p, const T* __restrict__ cb, const CgRun* __restrict__ runs,
                                  const int* __restrict__ vr, const int* __restrict__ vo, long long nvox,
                                  const CgScal* __restrict__ sc) {
  const double qd = sc->q * sc->delsq;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const size_t i = vox_lin(runs, vr, vo, v);
    p[i] = (T)((double)cb[i] - qd * (double)p[i]);
  }
}

// after the direction update: Q = -1/DELSQ (bpcg.f:1168)
__global__ void scal_after_dir_kernel(CgScal* sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sc->q = -1.0 / sc->delsq;
}

// P = DELSQ/AKDEN; ERR = DELSQ/BNORM; CHI2 = CHI2 - P*DELSQ (bpcg.f:1197-1212)
__global__ void scal_step_kernel(CgScal* sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    sc->p = sc->delsq / sc->akden;
    sc->err = sc->delsq / sc->bnorm;
    sc->chi2 = sc->chi2 - sc->p * sc->delsq;
  }
}

// BCKN += P*BCKP ; CB -= P*BCKE inside the sphere
template <class T>
__global__ void step_kernel(T* __restrict__ x, T* __restrict__ cb, const T* __restrict__ p, const T* __restrict__ e,
                            const CgRun* __restrict__ runs, const int* __restrict__ vr, const int* __restrict__ vo,
                            long long nvox, const CgScal* __restrict__ sc) {
  const double s = sc->p;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const size_t i = vox_lin(runs, vr, vo, v);
    x[i] = (T)((double)x[i] + s * (double)p[i]);
    cb[i] = (T)((double)cb[i] - s * (double)e[i]);
  }
}

// FIXEDGE (bpcg.f:1278-1517), part 1: zero outside the sphere runs
template <class T>
__global__ void zero_outside_kernel(T* __restrict__ p, int n, int ldp, float r2) {
  const size_t nnn = (size_t)n * n * n;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nnn; q += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % n) + 1;
    const size_t t = q / n;
    const int y = (int)(t % n) + 1, z = (int)(t / n) + 1;
    const float tz = (float)(z - ldp), ty = (float)(y - ldp), tx = (float)(x - ldp);
    const float rc = __fadd_rn(__fmul_rn(tx, tx), __fadd_rn(__fmul_rn(ty, ty), __fmul_rn(tz, tz)));
    if (rc > r2) p[q] = (T)0;
  }
}

// FIXEDGE part 2: extend the first/last nonzero of every line along `axis`
// by 1, 2 or 3 voxels (mode 1/2/3); one thread per line, the reference scans.
template <class T>
__global__ void fixedge_axis_kernel(T* __restrict__ p, int n, int axis, int mode) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= n * n) return;
  const int a = line / n, b = line % n;  // a, b: the other two coordinates (0-based)
  size_t base, stride;
  if (axis == 0) { base = ((size_t)a * n + b) * n; stride = 1; }                       // K=a, J=b
  else if (axis == 1) { base = (size_t)a * n * n + b; stride = (size_t)n; }             // K=a, I=b
  else { base = (size_t)a * n + b; stride = (size_t)n * n; }                            // J=a, I=b
  auto L = [&](int t) -> T& { return p[base + (size_t)(t - 1) * stride]; };
  const T z = (T)0;
  if (mode == 1) {
    for (int t = 1; t <= n - 1; ++t) if (L(t + 1) != z) { L(t) = L(t + 1); break; }
    for (int t = n; t >= 2; --t) if (L(t - 1) != z) { L(t) = L(t - 1); break; }
  } else if (mode == 2) {
    for (int t = 2; t <= n - 1; ++t) if (L(t + 1) != z) { T v = L(t + 1); L(t) = v; L(t - 1) = v; break; }
    for (int t = n - 1; t >= 2; --t) if (L(t - 1) != z) { T v = L(t - 1); L(t) = v; L(t + 1) = v; break; }
  } else {
    for (int t = 3; t <= n - 1; ++t) if (L(t + 1) != z) { T v = L(t + 1); L(t) = v; L(t - 1) = v; L(t - 2) = v; break; }
    for (int t = n - 2; t >= 2; --t) if (L(t - 1) != z) { T v = L(t - 1); L(t) = v; L(t + 1) = v; L(t + 2) = v; break; }
  }
}

// BFIRSTS / BSECOND / BTHIRD (bpcg.f:1521-1588): BCKE += lambda * D^k BCKP
template <class T>
__global__ void regularize_kernel(T* __restrict__ e, const T* __restrict__ p, const CgRun* __restrict__ runs,
                                  const int* __restrict__ vr, const int* __restrict__ vo, long long nvox, int n,
                                  T lam, int mode) {
  const long sx = 1, sy = n, sz = (long)n * n;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const long q = (long)vox_lin(runs, vr, vo, v);
    T t;
    if (mode == 1) {
      T s = radd(radd(radd(radd(radd(p[q + sx], p[q + sy]), p[q + sz]), p[q - sx]), p[q - sy]), p[q - sz]);
      t = rsub(rmul((T)6, p[q]), s);
    } else if (mode == 2) {
      t = rmul((T)18, p[q]);
      const long st[3] = {sx, sy, sz};
      for (int d = 0; d < 3; ++d) {
        t = radd(rsub(t, rmul((T)4, p[q + st[d]])), p[q + 2 * st[d]]);
        t = radd(rsub(t, rmul((T)4, p[q - st[d]])), p[q - 2 * st[d]]);
      }
    } else {
      t = rmul((T)60, p[q]);
      const long st[3] = {sx, sy, sz};
      for (int d = 0; d < 3; ++d) {
        t = rsub(radd(rsub(t, rmul((T)15, p[q + st[d]])), rmul((T)6, p[q + 2 * st[d]])), p[q + 3 * st[d]]);
        t = rsub(radd(rsub(t, rmul((T)15, p[q - st[d]])), rmul((T)6, p[q - 2 * st[d]])), p[q - 3 * st[d]]);
      }
    }
    e[q] = radd(e[q], rmul(lam, t));
  }
}

// float -> T widening copy
template <class T>
__global__ void widen_kernel(const float* __restrict__ in, T* __restrict__ out, size_t count) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < count; q += (size_t)gridDim.x * blockDim.x)
    out[q] = (T)in[q];
}

void cg_release(spi_ctx* c) {
  for (auto& b : c->cg_buf) b.release();
  for (auto& b : c->cg_fbs) b.release();
}

// Device-side problem description shared by the entry points
struct CgProblem {
  int n, ldp;
  float ri;
  std::vector<CgRun> runs;
  long long nvox = 0;
};

static int cg_setup(spi_ctx* c, int n, float ri, CgProblem& pb) {
  pb.n = n;
  pb.ldp = n / 2 + 1;
  pb.ri = ri;
  prepcub_s(n, ri, pb.ldp, pb.runs);
  std::vector<int> vr, vo;
  for (size_t r = 0; r < pb.runs.size(); ++r)
    for (int j = pb.runs[r].l1; j <= pb.runs[r].l2; ++j) {
      vr.push_back((int)r);
      vo.push_back(j - pb.runs[r].l1);
    }
  pb.nvox = (long long)vr.size();
  // cg_buf[0] runs, [1] vox_run, [2] vox_off
  SPI_TRY(c->cg_buf[0].ensure(std::max<size_t>(1, pb.runs.size()) * sizeof(CgRun)));
  SPI_TRY(c->cg_buf[1].ensure(std::max<size_t>(1, vr.size()) * sizeof(int)));
  SPI_TRY(c->cg_buf[2].ensure(std::max<size_t>(1, vo.size()) * sizeof(int)));
  if (!pb.runs.empty()) {
    SPI_CUDA(cudaMemcpyAsync(c->cg_buf[0].p, pb.runs.data(), pb.runs.size() * sizeof(CgRun), cudaMemcpyHostToDevice, c->stream));
    SPI_CUDA(cudaMemcpyAsync(c->cg_buf[1].p, vr.data(), vr.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    SPI_CUDA(cudaMemcpyAsync(c->cg_buf[2].p, vo.data(), vo.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  }
  return 0;
}

static int blocks_for(const spi_ctx* c, long long work, int threads) {
  long long b = (work + threads - 1) / threads;
  long long cap = (long long)c->sm_count * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

// A: projections of `cube` for dms[0..nang) into projs
template <class T>
static int launch_project(spi_ctx* c, const CgProblem& pb, const T* cube, const CgDM* dms, int nang, T* projs) {
  const int n = pb.n;
  // FP32 shared-memory accumulation of FP64 projections in the mixed mode
  const bool acc32 = sizeof(T) == 8 && c->cg_fp64 == 2;
  const size_t smem = (size_t)n * n * (acc32 ? sizeof(float) : sizeof(T));
  if (nang <= 0) return 0;
  const size_t smem_cap = 200 * 1024;
  if (smem <= smem_cap) {
    // the attribute is per device; set once per device (several threads may race here harmlessly)
    static std::atomic<unsigned long long> attr_set{0};
    const unsigned long long bit = 1ull << (c->device & 63);
    if (!(attr_set.load() & bit)) {
      cudaFuncSetAttribute(prjcq_smem_kernel<T, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap);
      cudaFuncSetAttribute(prjcq_smem_kernel<T, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap);
      attr_set.fetch_or(bit);
    }
    if (acc32)
      prjcq_smem_kernel<T, float><<<nang, 512, smem, c->stream>>>(cube, c->cg_buf[0].as<CgRun>(),
                                                                  (int)pb.runs.size(), dms, n, pb.ldp, projs);
    else
      prjcq_smem_kernel<T, T><<<nang, 512, smem, c->stream>>>(cube, c->cg_buf[0].as<CgRun>(), (int)pb.runs.size(),
                                                              dms, n, pb.ldp, projs);
    SPI_TRY(check_kernel("prjcq_smem_kernel"));
  } else {
    SPI_CUDA(cudaMemsetAsync(projs, 0, (size_t)nang * n * n * sizeof(T), c->stream));
    long long work = (long long)pb.runs.size() * nang;
    prjcq_global_kernel<T><<<blocks_for(c, work, 256), 256, 0, c->stream>>>(cube, c->cg_buf[0].as<CgRun>(),
                                                                           (int)pb.runs.size(), dms, nang, n,
                                                                           pb.ldp, projs);
    SPI_TRY(check_kernel("prjcq_global_kernel"));
  }
  c->count();
  return 0;
}

// A^T: cube += back-projection of projs (image order, chunks of 64 images)
template <class T>
static int launch_backproject(spi_ctx* c, const CgProblem& pb, T* cube, const T* projs, const CgDM* dms,
                              const int* lb, int nang) {
  const int kchunk = 64;
  for (int k0 = 0; k0 < nang; k0 += kchunk) {
    int k1 = std::min(nang, k0 + kchunk);
    bckpj_kernel<T><<<blocks_for(c, pb.nvox, 256), 256, 0, c->stream>>>(
        cube, c->cg_buf[0].as<CgRun>(), c->cg_buf[1].as<int>(), c->cg_buf[2].as<int>(), pb.nvox, projs, dms, lb, k0,
        k1, pb.n, pb.ldp);
    SPI_TRY(check_kernel("bckpj_kernel"));
    c->count();
  }
  return 0;
}


// images per PROJT chunk of the mixed modes: tables of <= ~1 GB
static int projt_chunk(int n, int nang, size_t entry) {
  const long long per = (long long)n * n * (long long)entry;
  return (int)std::max<long long>(64, std::min<long long>(nang, (1ll << 30) / per));
}

// The mixed modes keep the fixed-point projection in shared memory, split
// into C row bands (1, 2, 4 or 8 CTAs per projection) when one CTA's 200 KB
// do not hold it; 0 when no split does.  A split image takes twice the
// fewest bands that fit: smaller bands put 3 CTAs on an SM instead of 1,
// which outweighs walking every run once more per band (256^3, 2,000
// images: mode 3 0.230 s per iteration with 4 bands against 0.254 s with 2
// and 0.313 s with 8; mode 2 0.365 s with 8 against 0.411 s with 4).
// SPI_CG_BANDS forces a C at least the fewest that fit.
static size_t band_bytes(int n, int C, bool wide) {
  if (C == 1) return (size_t)n * n * (wide ? 8 : 4);
  return (size_t)((n + C - 1) / C + 2) * n * (wide ? 8 : 4);
}
static int mixed_bands(int n, bool wide) {
  const size_t cap = 200 * 1024;
  int cmin = 1;
  while (cmin <= 8 && band_bytes(n, cmin, wide) > cap) cmin *= 2;
  if (cmin > 8) return 0;
  int C = cmin > 1 ? std::min(8, 2 * cmin) : 1;
  if (const char* e = getenv("SPI_CG_BANDS")) {
    const int f = atoi(e);
    if ((f == 1 || f == 2 || f == 4 || f == 8) && f >= cmin && f <= n / 2) C = f;
  }
  return C;
}
static bool mixed_fits(int n, bool wide) { return mixed_bands(n, wide) > 0; }

// A^T from PROJT tables of images [k0, k1), 64 images per launch
template <class T, bool WIDE>
static int launch_backproject_projt(spi_ctx* c, const CgProblem& pb, T* cube, const ProjtEntry<WIDE>* projt,
                                    const CgDM* dms, int kbase, int k0, int k1) {
  for (int a = k0; a < k1; a += 64) {
    const int b = std::min(k1, a + 64);
    bckpj_projt_kernel<T, WIDE><<<blocks_for(c, pb.nvox, 256), 256, 0, c->stream>>>(
        cube, c->cg_buf[0].as<CgRun>(), c->cg_buf[1].as<int>(), c->cg_buf[2].as<int>(), pb.nvox, projt, dms, kbase, a,
        b, pb.n, pb.ldp);
    SPI_TRY(check_kernel("bckpj_projt_kernel"));
    c->count();
  }
  return 0;
}

// A then A^T (BCKE += A^T A BCKP) chunk by chunk through PROJT tables
template <class T, bool WIDE, bool WT>
static int launch_normal_projt(spi_ctx* c, const CgProblem& pb, const T* x, T* out, const CgDM* dms, const int* lb,
                               int nang, ProjtEntry<WT>* projt, unsigned long long* maxabs) {
  const int n = pb.n;
  const int K = projt_chunk(n, nang, sizeof(ProjtEntry<WT>));
  const size_t smem = (size_t)n * n * (WIDE ? 8 : 4);
  // fixed-point scale of the projector: max |x| over the sphere
  SPI_CUDA(cudaMemsetAsync(maxabs, 0, sizeof(unsigned long long), c->stream));
  absmax_kernel<T><<<blocks_for(c, pb.nvox, 256), 256, 0, c->stream>>>(x, c->cg_buf[0].as<CgRun>(), c->cg_buf[1].as<int>(),
                                                                      c->cg_buf[2].as<int>(), pb.nvox, maxabs);
  SPI_TRY(check_kernel("absmax_kernel"));
  c->count();
  const float mcap = (float)(M_PI * std::pow(std::sqrt(2.0) + std::sqrt(3.0) / 2.0, 2.0) *
                             (2.0 * pb.ri + std::sqrt(3.0)));
  static std::atomic<unsigned long long> attr_set{0};
  const unsigned long long bit = 1ull << (c->device & 63);
  if (!(attr_set.load() & bit)) {
    cudaFuncSetAttribute(prjcq_projt_kernel<T, WIDE, WT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(prjcq_projt_band_kernel<T, WIDE, WT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set.fetch_or(bit);
  }
  const int C = mixed_bands(n, WIDE);
  if (C < 1) return fail(kInvalid, "BP CG: n = %d too large for the mixed precision modes", n);
  for (int k0 = 0; k0 < nang; k0 += K) {
    const int kc = std::min(K, nang - k0);
    if (C == 1)
      prjcq_projt_kernel<T, WIDE, WT><<<kc, 512, smem, c->stream>>>(x, c->cg_buf[0].as<CgRun>(), (int)pb.runs.size(), dms,
                                                                 lb, k0, n, pb.ldp, maxabs, mcap, projt);
    else
      prjcq_projt_band_kernel<T, WIDE, WT><<<kc * C, 512, band_bytes(n, C, WIDE), c->stream>>>(
          x, c->cg_buf[0].as<CgRun>(), (int)pb.runs.size(), dms, lb, k0, n, pb.ldp, C, maxabs, mcap, projt);
    SPI_TRY(check_kernel("prjcq_projt_kernel"));
    c->count();
    SPI_TRY((launch_backproject_projt<T, WT>(c, pb, out, projt, dms, k0, k0, k0 + kc)));
  }
  return 0;
}

// setup A^T of the input images through PROJT tables
template <class T, bool WIDE>
static int backproject_images_projt(spi_ctx* c, const CgProblem& pb, T* cb, const float* imgs, const CgDM* dms,
                                    int nang, ProjtEntry<WIDE>* projt) {
  const int n = pb.n;
  const int K = projt_chunk(n, nang, sizeof(ProjtEntry<WIDE>));
  for (int k0 = 0; k0 < nang; k0 += K) {
    const int kc = std::min(K, nang - k0);
    projt_images_kernel<WIDE><<<blocks_for(c, (long long)kc * n * n, 256), 256, 0, c->stream>>>(
        imgs + (size_t)k0 * n * n, n, kc, projt);
    SPI_TRY(check_kernel("projt_images_kernel"));
    c->count();
    SPI_TRY((launch_backproject_projt<T, WIDE>(c, pb, cb, projt, dms, k0, k0, k0 + kc)));
  }
  return 0;
}

static void dms_from_angles(const float* angles, int nang, std::vector<CgDM>& out) {
  out.resize((size_t)std::max(nang, 1));
  for (int k = 0; k < nang; ++k) {
    float dm[9];
    cang(angles[3 * k + 2], angles[3 * k + 1], angles[3 * k + 0], dm);  // CANG(phi, theta, psi)
    memcpy(out[k].d, dm, 6 * sizeof(float));
  }
}

// HIANG (hiang.f:40-112).  ang[3*i] = phi, [3*i+1] = theta, [3*i+2] = psi.
// Duplicates (after the fold and the 0.01 degree truncation of phi) merge into
// their first occurrence, exactly as the reference's pairwise scan does.
// dm9 (FBS only) receives all nine DM entries per merged angle.
static int hiang(std::vector<float>& ang, int nang, std::vector<CgDM>& dms, std::vector<int>& lb,
                 std::vector<float>* dm9 = nullptr) {
  for (int i = 0; i < nang; ++i) {
    if (ang[3 * i + 1] >= 90.0f) {
      ang[3 * i + 1] = 180.0f - ang[3 * i + 1];
      ang[3 * i] = ang[3 * i] + 180.0f;
      if (ang[3 * i] >= 360.0f) ang[3 * i] = ang[3 * i] - 360.0f;
    }
  }
  for (int i = 0; i < nang; ++i) {
    int jjj = (int)(100.0f * ang[3 * i]);
    ang[3 * i] = (float)jjj / 100.0f;
  }
  std::unordered_map<uint64_t, int> first;
  std::vector<int> order;
  lb.clear();
  for (int i = 0; i < nang; ++i) {
    uint32_t a, b;
    float fa = ang[3 * i], fb = ang[3 * i + 1];
    if (fa == 0.0f) fa = 0.0f;  // +0 and -0 compare equal in the reference
    if (fb == 0.0f) fb = 0.0f;
    memcpy(&a, &fa, 4);
    memcpy(&b, &fb, 4);
    uint64_t key = ((uint64_t)a << 32) | b;
    auto it = first.find(key);
    if (it == first.end()) {
      first.emplace(key, (int)order.size());
      order.push_back(i);
      lb.push_back(1);
    } else {
      lb[it->second] += 1;
    }
  }
  const int lo = (int)order.size();
  const double quadpi = (double)3.14159265358979323846f;
  const double d2r = quadpi / 180.0;
  dms.resize((size_t)std::max(lo, 1));
  for (int o = 0; o < lo; ++o) {
    const int i = order[o];
    double cphi = std::cos((double)ang[3 * i] * d2r), sphi = std::sin((double)ang[3 * i] * d2r);
    double cthe = std::cos((double)ang[3 * i + 1] * d2r), sthe = std::sin((double)ang[3 * i + 1] * d2r);
    double cpsi = 1.0, spsi = 0.0;
    float* d = dms[o].d;
    d[0] = (float)(cphi * cthe * cpsi - sphi * spsi);
    d[1] = (float)(sphi * cthe * cpsi + cphi * spsi);
    d[2] = (float)(-sthe * cpsi);
    d[3] = (float)(-cphi * cthe * spsi - sphi * cpsi);
    d[4] = (float)(-sphi * cthe * spsi + cphi * cpsi);
    d[5] = (float)(sthe * spsi);
    if (dm9) {
      if (o == 0) dm9->assign((size_t)9 * lo, 0.0f);
      float* e = dm9->data() + (size_t)9 * o;
      memcpy(e, d, 6 * sizeof(float));
      e[6] = (float)(sthe * cphi);
      e[7] = (float)(sthe * sphi);
      e[8] = (float)(cthe);
    }
  }
  return lo;
}

// ---------------------------------------------------------------------------
// FBS2_PREP for batches of K images: cuFFT plans and FP64 scratch.
struct Fbs2Work {
  int n = 0, K = 0;
  float a4 = 0.0f;          // A4 = PI2 / N in REAL
  cufftHandle fwd = 0, inv = 0;
  double* dbl = nullptr;    // [K][n][n] FFT input
  double2* F = nullptr;     // [K][n][h]
  double2* W = nullptr;     // [3][K][n][h]
  double* D = nullptr;      // [3][K][n][n]
  void destroy() {
    if (fwd) cufftDestroy(fwd);
    if (inv) cufftDestroy(inv);
    fwd = inv = 0;
  }
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// bytes of the scratch of K images (the four arrays, each 256-byte aligned)
static size_t fbs2_work_bytes(int n, size_t K) {
  const size_t nn = (size_t)n * n, s2 = (size_t)n * (n / 2 + 1);
  return align256(K * nn * 8) + align256(K * s2 * 16) + align256(3 * K * s2 * 16) + align256(3 * K * nn * 8);
}

// carve the scratch from p and (with `plans`) create the plans on stream s
static int fbs2_work_init(Fbs2Work& w, int n, int K, char* p, cudaStream_t s, bool plans = true) {
  const size_t nn = (size_t)n * n, s2 = (size_t)n * (n / 2 + 1);
  w.n = n;
  w.K = K;
  w.a4 = 6.28318530717958647692f / (float)n;
  w.dbl = reinterpret_cast<double*>(p); p += align256((size_t)K * nn * 8);
  w.F = reinterpret_cast<double2*>(p); p += align256((size_t)K * s2 * 16);
  w.W = reinterpret_cast<double2*>(p); p += align256(3 * (size_t)K * s2 * 16);
  w.D = reinterpret_cast<double*>(p);
  if (!plans) return 0;
  int d2[2] = {n, n};
  SPI_CUFFT(cufftPlanMany(&w.fwd, 2, d2, nullptr, 1, (int)nn, nullptr, 1, (int)s2, CUFFT_D2Z, K));
  SPI_CUFFT(cufftPlanMany(&w.inv, 2, d2, nullptr, 1, (int)s2, nullptr, 1, (int)nn, CUFFT_Z2D, 3 * K));
  SPI_CUFFT(cufftSetStream(w.fwd, s));
  SPI_CUFFT(cufftSetStream(w.inv, s));
  return 0;
}

// FBS2_PREP of kc <= K images src[kc][n][n] (S = float images or the
// vector type's projections) into the interleaved tables P2[kc][n*n][4] of
// type TT
template <class S, class TT>
static int fbs2_prepare(spi_ctx* c, const Fbs2Work& w, const S* src, int kc, TT* P2) {
  const int n = w.n;
  const size_t nn = (size_t)n * n, count = (size_t)kc * nn, padded = (size_t)w.K * nn;
  fbs_to_double_kernel<S, S><<<blocks_for(c, (long long)padded, 256), 256, 0, c->stream>>>(src, w.dbl, count, padded);
  SPI_TRY(check_kernel("fbs_to_double_kernel"));
  SPI_CUFFT(cufftExecD2Z(w.fwd, w.dbl, reinterpret_cast<cufftDoubleComplex*>(w.F)));
  const size_t spec = (size_t)w.K * n * (n / 2 + 1);
  fbs2_spec_kernel<<<blocks_for(c, (long long)spec, 256), 256, 0, c->stream>>>(w.F, w.W, n, w.K, w.a4,
                                                                              1.0 / ((double)n * n));
  SPI_TRY(check_kernel("fbs2_spec_kernel"));
  SPI_CUFFT(cufftExecZ2D(w.inv, reinterpret_cast<cufftDoubleComplex*>(w.W), w.D));
  fbs2_pack_kernel<S, TT><<<blocks_for(c, (long long)count, 256), 256, 0, c->stream>>>(src, w.D, P2, count, padded);
  SPI_TRY(check_kernel("fbs2_pack_kernel"));
  c->count(3);
  return 0;
}

// ---------------------------------------------------------------------------
// RTSF of nimg device images src -> dst (RB 3F / RB 32F in FBS mode).  The
// plans and scratch (batches of up to K images, about 256 MB) stay with the
// context for the next call of the same size.
void rtsf_release(spi_ctx* c) {
  if (c->rtsf_plan[0]) cufftDestroy(c->rtsf_plan[0]);
  if (c->rtsf_plan[1]) cufftDestroy(c->rtsf_plan[1]);
  c->rtsf_plan[0] = c->rtsf_plan[1] = 0;
  c->rtsf_n = c->rtsf_k = 0;
  c->rtsf_buf.release();
}

int rtsf_images(spi_ctx* c, const float* src, float* dst, int nx, int nimg, const float4* prm) {
  if (nimg <= 0) return 0;
  const size_t nn = (size_t)nx * nx;
  const size_t per = fbs2_work_bytes(nx, 1) + nn * 4 * sizeof(float);
  const int K = (int)std::max<size_t>(1, std::min<size_t>(1024, (size_t(256) << 20) / per));
  Fbs2Work w;
  if (c->rtsf_n != nx || c->rtsf_k != K) {
    rtsf_release(c);
    SPI_TRY(c->rtsf_buf.ensure(fbs2_work_bytes(nx, K) + align256((size_t)K * nn * 4 * sizeof(float))));
    const int st = fbs2_work_init(w, nx, K, c->rtsf_buf.as<char>(), c->stream);
    if (st != 0) {
      w.destroy();
      return st;
    }
    c->rtsf_plan[0] = w.fwd;
    c->rtsf_plan[1] = w.inv;
    c->rtsf_n = nx;
    c->rtsf_k = K;
  } else {
    SPI_TRY(fbs2_work_init(w, nx, K, c->rtsf_buf.as<char>(), c->stream, false));
    w.fwd = c->rtsf_plan[0];
    w.inv = c->rtsf_plan[1];
    SPI_CUFFT(cufftSetStream(w.fwd, c->stream));
    SPI_CUFFT(cufftSetStream(w.inv, c->stream));
  }
  float* P2 = reinterpret_cast<float*>(c->rtsf_buf.as<char>() + fbs2_work_bytes(nx, K));
  for (int b0 = 0; b0 < nimg; b0 += K) {
    const int kb = std::min(K, nimg - b0);
    SPI_TRY((fbs2_prepare<float, float>(c, w, src + (size_t)b0 * nn, kb, P2)));
    rtsf_kernel<<<blocks_for(c, (long long)kb * nn, 256), 256, 0, c->stream>>>(P2, dst + (size_t)b0 * nn, nx, kb,
                                                                             prm + b0);
    SPI_TRY(check_kernel("rtsf_kernel"));
    c->count();
  }
  return 0;
}

// ---------------------------------------------------------------------------
// FBS3_PREP of one n^3 volume: cuFFT plans and FP64 scratch.
struct Fbs3Work {
  int n = 0;
  float a4 = 0.0f;          // A4 = PI2 / N in REAL
  cufftHandle fwd = 0, inv = 0;
  double* dbl = nullptr;    // [n^3] FFT input
  double2* F = nullptr;     // [n][n][h] forward spectrum
  double2* W = nullptr;     // [7][n][n][h] derivative spectra
  double* D = nullptr;      // [7][n^3] derivatives
  void destroy() {
    if (fwd) cufftDestroy(fwd);
    if (inv) cufftDestroy(inv);
    fwd = inv = 0;
  }
};

static size_t fbs3_work_bytes(int n) {
  const size_t nnn = (size_t)n * n * n, s3 = (size_t)n * n * (n / 2 + 1);
  return align256(nnn * 8) + align256(s3 * 16) + align256(7 * s3 * 16) + align256(7 * nnn * 8);
}

static int fbs3_work_init(Fbs3Work& w, int n, char* p, cudaStream_t s, bool plans = true) {
  const size_t nnn = (size_t)n * n * n, s3 = (size_t)n * n * (n / 2 + 1);
  w.n = n;
  w.a4 = 6.28318530717958647692f / (float)n;
  w.dbl = reinterpret_cast<double*>(p); p += align256(nnn * 8);
  w.F = reinterpret_cast<double2*>(p); p += align256(s3 * 16);
  w.W = reinterpret_cast<double2*>(p); p += align256(7 * s3 * 16);
  w.D = reinterpret_cast<double*>(p);
  if (!plans) return 0;
  int d3[3] = {n, n, n};
  SPI_CUFFT(cufftPlan3d(&w.fwd, n, n, n, CUFFT_D2Z));
  SPI_CUFFT(cufftPlanMany(&w.inv, 3, d3, nullptr, 1, (int)s3, nullptr, 1, (int)nnn, CUFFT_Z2D, 7));
  SPI_CUFFT(cufftSetStream(w.fwd, s));
  SPI_CUFFT(cufftSetStream(w.inv, s));
  return 0;
}

// FBS3_PREP of the cube into the interleaved table V[n^3][8] of type TT
template <class T, class TT>
static int fbs3_prepare(spi_ctx* c, const Fbs3Work& w, const T* cube, TT* V) {
  const int n = w.n;
  const size_t nnn = (size_t)n * n * n;
  fbs_to_double_kernel<T, T><<<blocks_for(c, (long long)nnn, 256), 256, 0, c->stream>>>(cube, w.dbl, nnn, nnn);
  SPI_TRY(check_kernel("fbs_to_double_kernel"));
  SPI_CUFFT(cufftExecD2Z(w.fwd, w.dbl, reinterpret_cast<cufftDoubleComplex*>(w.F)));
  const size_t spec = (size_t)n * n * (n / 2 + 1);
  fbs3_spec_kernel<<<blocks_for(c, (long long)spec, 256), 256, 0, c->stream>>>(w.F, w.W, n, w.a4,
                                                                              1.0 / ((double)n * n * n));
  SPI_TRY(check_kernel("fbs3_spec_kernel"));
  SPI_CUFFT(cufftExecZ2D(w.inv, reinterpret_cast<cufftDoubleComplex*>(w.W), w.D));
  fbs3_pack_kernel<T, TT><<<blocks_for(c, (long long)nnn, 256), 256, 0, c->stream>>>(cube, w.D, V, nnn);
  SPI_TRY(check_kernel("fbs3_pack_kernel"));
  c->count(3);
  return 0;
}

// ---------------------------------------------------------------------------
// FBS operators: cuFFT plans and scratch for one BP CG solve.  Projections are
// processed in chunks of K (the 2D plans' batch).
struct FbsState {
  int n = 0, K = 0;
  Fbs2Work w2;              // FBS2_PREP of K images
  Fbs3Work w3;              // FBS3_PREP of the direction
  void* V = nullptr;        // TT [n^3][8] interleaved FBS3 table
  void* P2 = nullptr;       // T [K][n*n][4] interleaved FBS2 tables
  void* pt = nullptr;       // T [K][n][n] projections of the iteration
  int2* segs = nullptr;     // {run, first offset} per BCKPJ_FBS segment
  long long nseg = 0;
  int seg = kFbsSeg;        // voxels per BCKPJ_FBS segment
  float* dm9 = nullptr;     // 9 floats per merged angle
  size_t tsz = 8;           // bytes per table value (FP32 tables in precision modes 2 and 3)
  FbsState() = default;
  FbsState(const FbsState&) = delete;
  FbsState& operator=(const FbsState&) = delete;
  ~FbsState() {
    w2.destroy();
    w3.destroy();
  }
};

template <class T>
static int fbs_setup(spi_ctx* c, const CgProblem& pb, int nang, FbsState& fs, size_t tsz) {
  const int n = pb.n;
  const size_t nn = (size_t)n * n, nnn = nn * n;
  fs.n = n;
  fs.tsz = tsz;
  // chunk: about 1 GiB of 2D scratch, at most 16384 projections
  const size_t per_img = fbs2_work_bytes(n, 1) + nn * 4 * tsz + nn * sizeof(T);
  fs.K = (int)std::max<size_t>(1, std::min<size_t>({(size_t)nang, (size_t)16384, (size_t(1) << 30) / per_img}));
  if (const char* e = getenv("SPI_FBS_CHUNK")) {   // smaller chunks (tests of the chunk loop)
    const int k = atoi(e);
    if (k > 0 && k < fs.K) fs.K = k;
  }
  const size_t K = (size_t)fs.K;
  if (const char* e = getenv("SPI_FBS_SEG")) {   // 2, 4 or 8 voxels per back-projector thread
    const int v = atoi(e);
    if (v == 2 || v == 4 || v == 8) fs.seg = v;
  }
  std::vector<int2> segs;
  for (size_t r = 0; r < pb.runs.size(); ++r) {
    const int len = pb.runs[r].l2 - pb.runs[r].l1 + 1;
    for (int o = 0; o < len; o += fs.seg) segs.push_back(make_int2((int)r, o));
  }
  fs.nseg = (long long)segs.size();
  const size_t b3[2] = {fbs3_work_bytes(n), align256(nnn * 8 * tsz)};
  const size_t w2b = fbs2_work_bytes(n, K);
  const size_t b2[3] = {w2b, align256(K * nn * 4 * tsz), align256(K * nn * sizeof(T))};
  size_t t3 = 0, t2 = 0;
  for (size_t b : b3) t3 += b;
  for (size_t b : b2) t2 += b;
  SPI_TRY(c->cg_fbs[0].ensure(t3));
  SPI_TRY(c->cg_fbs[1].ensure(t2));
  SPI_TRY(c->cg_fbs[2].ensure(std::max<size_t>(1, segs.size()) * sizeof(int2)));
  SPI_TRY(c->cg_fbs[3].ensure((size_t)9 * std::max(nang, 1) * sizeof(float)));
  char* p = c->cg_fbs[0].as<char>();
  SPI_TRY(fbs3_work_init(fs.w3, n, p, c->stream));
  fs.V = p + b3[0];
  p = c->cg_fbs[1].as<char>();
  SPI_TRY(fbs2_work_init(fs.w2, n, fs.K, p, c->stream));
  p += b2[0];
  fs.P2 = p; p += b2[1];
  fs.pt = p;
  fs.segs = c->cg_fbs[2].as<int2>();
  fs.dm9 = c->cg_fbs[3].as<float>();
  if (!segs.empty())
    SPI_CUDA(cudaMemcpyAsync(fs.segs, segs.data(), segs.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  return 0;
}

// PRJCQ_FBS3 of fs.V for merged angles [k0, k0 + kc) into fs.pt, scaled by LB
template <class T, class TT>
static int fbs_project(spi_ctx* c, FbsState& fs, const int* dlb, int k0, int kc) {
  const int n = fs.n;
  const int threads = (n + 31) / 32 * 32;
  const size_t smem = (size_t)threads * (kFbsIC + 1) * sizeof(T);
  auto launch = [&](auto kern) -> int {
    if (smem > 48 * 1024)
      SPI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<dim3(n, kc), threads, smem, c->stream>>>(static_cast<const TT*>(fs.V), fs.dm9, dlb, k0, n,
                                                    static_cast<T*>(fs.pt));
    return 0;
  };
  // a 256-thread bound lets the FP64 form keep its registers (n <= 256)
  if (threads <= 256) SPI_TRY(launch(prjcq_fbs3_kernel<T, TT, 256>));
  else SPI_TRY(launch(prjcq_fbs3_kernel<T, TT, 512>));
  SPI_TRY(check_kernel("prjcq_fbs3_kernel"));
  c->count();
  return 0;
}

// BCKPJ_FBS of kc prepared tables P2 (angles dms[0..kc)) summed into cube
template <class T, class TT>
static int fbs_backproject(spi_ctx* c, const CgProblem& pb, FbsState& fs, T* cube, const TT* P2, const CgDM* dms,
                           int kc) {
  if (fs.nseg == 0 || kc <= 0) return 0;
  auto launch = [&](auto kern) {
    kern<<<blocks_for(c, fs.nseg, 256), 256, 0, c->stream>>>(cube, c->cg_buf[0].as<CgRun>(), fs.segs, fs.nseg, P2,
                                                             dms, kc, pb.n, pb.ldp);
  };
  if (fs.seg == 2) launch(bckpj_fbs_kernel<T, TT, 2>);
  else if (fs.seg == 8) launch(bckpj_fbs_kernel<T, TT, 8>);
  else launch(bckpj_fbs_kernel<T, TT, 4>);
  SPI_TRY(check_kernel("bckpj_fbs_kernel"));
  c->count();
  return 0;
}

// CB = A^T b with FBS (bpcg.f:713-731): FBS2_PREP and BCKPJ_FBS of every
// image, in order, chunk by chunk
template <class T, class TT>
static int fbs_backproject_images(spi_ctx* c, const CgProblem& pb, FbsState& fs, T* cb, const float* imgs, int nang,
                                  const CgDM* dms) {
  const size_t nn = (size_t)pb.n * pb.n;
  for (int k0 = 0; k0 < nang; k0 += fs.K) {
    const int kc = std::min(fs.K, nang - k0);
    SPI_TRY((fbs2_prepare<float, TT>(c, fs.w2, imgs + (size_t)k0 * nn, kc, static_cast<TT*>(fs.P2))));
    SPI_TRY((fbs_backproject<T, TT>(c, pb, fs, cb, static_cast<const TT*>(fs.P2), dms + k0, kc)));
  }
  return 0;
}

// BCKE += A^T A BCKP with FBS (BPCG_3_FBS, bpcg.f:1760-1822): FBS3_PREP of
// the direction, then per chunk of merged angles PRJCQ_FBS3 (scaled by LB),
// FBS2_PREP of the projections and BCKPJ_FBS
template <class T, class TT>
static int fbs_normal(spi_ctx* c, const CgProblem& pb, FbsState& fs, const T* bckp, T* bcke, const int* dlb, int kb,
                      int ke, const CgDM* dms) {
  SPI_TRY((fbs3_prepare<T, TT>(c, fs.w3, bckp, static_cast<TT*>(fs.V))));
  for (int k0 = kb; k0 < ke; k0 += fs.K) {
    const int kc = std::min(fs.K, ke - k0);
    SPI_TRY((fbs_project<T, TT>(c, fs, dlb, k0, kc)));
    SPI_TRY((fbs2_prepare<T, TT>(c, fs.w2, static_cast<const T*>(fs.pt), kc, static_cast<TT*>(fs.P2))));
    SPI_TRY((fbs_backproject<T, TT>(c, pb, fs, bcke, static_cast<const TT*>(fs.P2), dms + k0, kc)));
  }
  return 0;
}

// One rank's share of a BP CG solve over several processes (the reference's
// MPI form, bpcg.f:522-672, 855-1080): its images are [first, first+count) of
// the angle list, its merged angles the SETPART block of HIANG's list, and
// `reduce` sums a device array over the ranks in place (ALLREDUCE_MPI).
struct CgShard {
  int first = 0, count = 0;
  int rank = 0, world = 1;
  spi_allreduce_fn reduce = nullptr;
  void* user = nullptr;
  int sum(spi_ctx* c, void* data, long long n, bool fp64) const {
    if (!reduce) return 0;
    const int st = reduce(data, n, fp64 ? 1 : 0, c->stream, user);
    if (st != 0) return fail(kInvalid, "BP CG: the all-reduce callback returned %d", st);
    return 0;
  }
};

// BPCG_2 + HIANG + BPCG_3_LIN with vectors and projections stored as T;
// nang angles in all, this rank's images `projs` = sh.count of them.
template <class T>
static int bpcg_run(spi_ctx* c, const float* projs, int n, int nang, const float* angles, float ri, float errm,
                    float chim, int maxit, int mode, float lambda, float* vol_out, float* log_out, int* niter_out,
                    const CgShard& sh) {
  CgProblem pb;
  SPI_TRY(cg_setup(c, n, ri, pb));
  const size_t nnn = (size_t)n * n * n;
  const size_t vb = nnn * sizeof(T);
  const int nimg = sh.count;
  const size_t pcount = (size_t)nimg * n * n;
  // mixed mode (FP64 vectors, FP32 PROJT tables made per chunk of images)
  // modes 2 and 4: 47-bit fixed-point projections; mode 4 also keeps FP64
  // PROJT tables (mode 2 FP32 tables, mode 3 31-bit and FP32 tables)
  // FBS interpolation keeps T for the vectors and projections (FP64 in modes 1-4)
  const bool fbs = c->cg_interp == 1;
  if (fbs && n > 512) return fail(kInvalid, "BP CG FBS: n = %d above 512", n);
  const bool wide = c->cg_fp64 == 2 || c->cg_fp64 == 4;
  const bool mixed = !fbs && sizeof(T) == 8 && c->cg_fp64 >= 2 && mixed_fits(n, wide);
  const bool wtab = c->cg_fp64 == 4;
  const size_t pentry = wtab ? sizeof(ProjtEntry<true>) : sizeof(ProjtEntry<false>);
  // ---- HIANG (hiang.f:40-112) over all the angles, and this rank's block of
  // the merged list.  ang[3*i] = phi, [3*i+1] = theta, [3*i+2] = psi.
  std::vector<float> ang((size_t)3 * nang);
  for (int k = 0; k < nang; ++k) {
    ang[3 * k] = angles[3 * k + 2];
    ang[3 * k + 1] = angles[3 * k + 1];
    ang[3 * k + 2] = angles[3 * k];
  }
  std::vector<CgDM> mdms;
  std::vector<int> lb;
  std::vector<float> dm9;
  const int lo = hiang(ang, nang, mdms, lb, fbs ? &dm9 : nullptr);
  // SETPART (setpart.f:4-29): blocks of lo / world, the first lo % world ranks one more
  const int kq = lo / sh.world, kr = lo % sh.world;
  const int kb = sh.rank * kq + std::min(sh.rank, kr);
  const int kc_all = kq + (sh.rank < kr ? 1 : 0);
  const int ke = kb + kc_all;
  const int K = projt_chunk(n, std::max(nimg, kc_all), pentry);
  const int pj_rows = std::max(nimg, kc_all);   // projections of the images, then of the merged block
  // buffers: [3] dms, [4] CB, [5] projections (T) + float staging (mixed: float images + PROJT chunk),
  // [6] BCKN|BCKP|BCKE, [7] scalars + lb
  std::vector<CgDM> dms;
  dms_from_angles(angles + 3 * (size_t)sh.first, nimg, dms);
  SPI_TRY(c->cg_buf[3].ensure(std::max(dms.size(), mdms.size()) * sizeof(CgDM)));
  SPI_TRY(c->cg_buf[4].ensure(vb));
  if (fbs)
    SPI_TRY(c->cg_buf[5].ensure(std::max<size_t>(pcount, 1) * sizeof(float)));
  else if (mixed)
    SPI_TRY(c->cg_buf[5].ensure(pcount * sizeof(float) + (size_t)K * n * n * pentry + 32));
  else
    SPI_TRY(c->cg_buf[5].ensure((size_t)pj_rows * n * n * sizeof(T) +
                                (sizeof(T) != sizeof(float) ? pcount * sizeof(float) : 0) + 4));
  SPI_TRY(c->cg_buf[6].ensure(3 * vb));
  SPI_TRY(c->cg_buf[7].ensure(sizeof(CgScal) + 64 + (size_t)nang * sizeof(int)));
  T* cb = c->cg_buf[4].as<T>();
  T* pj = c->cg_buf[5].as<T>();
  float* pj32 = (mixed || fbs) ? c->cg_buf[5].as<float>()
                      : (sizeof(T) != sizeof(float)) ? reinterpret_cast<float*>(pj + (size_t)pj_rows * n * n)
                                                     : reinterpret_cast<float*>(pj);
  void* projt = mixed ? (void*)(c->cg_buf[5].as<char>() + ((pcount * sizeof(float) + 31) & ~size_t(31))) : nullptr;
  T* bckn = c->cg_buf[6].as<T>();
  T* bckp = bckn + nnn;
  T* bcke = bckp + nnn;
  CgScal* sc = c->cg_buf[7].as<CgScal>();
  double* acc = reinterpret_cast<double*>(reinterpret_cast<char*>(c->cg_buf[7].p) + sizeof(CgScal));
  int* dlb = reinterpret_cast<int*>(reinterpret_cast<char*>(c->cg_buf[7].p) + sizeof(CgScal) + 64);
  SPI_CUDA(cudaMemcpyAsync(c->cg_buf[3].p, dms.data(), dms.size() * sizeof(CgDM), cudaMemcpyHostToDevice, c->stream));
  if (pcount) SPI_CUDA(cudaMemcpyAsync(pj32, projs, pcount * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  // ---- BPCG_2: statistics, CB = A^T b, background correction
  SPI_CUDA(cudaMemsetAsync(acc, 0, 64, c->stream));
  if (nimg > 0) {
    astasq_kernel<<<nimg, 256, 0, c->stream>>>(pj32, n, ri * ri, acc);
    SPI_TRY(check_kernel("astasq_kernel"));
    c->count();
  }
  SPI_CUDA(cudaMemsetAsync(cb, 0, vb, c->stream));
  FbsState fs;
  // FBS interpolation tables: FP32 in precision modes 2 and 3 (FP64 vectors
  // and arithmetic), the vector type otherwise
  const bool fbs32 = fbs && sizeof(T) == 8 && (c->cg_fp64 == 2 || c->cg_fp64 == 3);
  if (fbs) {
    SPI_TRY(fbs_setup<T>(c, pb, std::max(std::max(nimg, lo), 1), fs, fbs32 ? sizeof(float) : sizeof(T)));
    if (fbs32)
      SPI_TRY((fbs_backproject_images<T, float>(c, pb, fs, cb, pj32, nimg, c->cg_buf[3].as<CgDM>())));
    else
      SPI_TRY((fbs_backproject_images<T, T>(c, pb, fs, cb, pj32, nimg, c->cg_buf[3].as<CgDM>())));
  } else if (mixed) {
    if (wtab)
      SPI_TRY((backproject_images_projt<T, true>(c, pb, cb, pj32, c->cg_buf[3].as<CgDM>(), nimg,
                                                static_cast<ProjtEntry<true>*>(projt))));
    else
      SPI_TRY((backproject_images_projt<T, false>(c, pb, cb, pj32, c->cg_buf[3].as<CgDM>(), nimg,
                                                 static_cast<ProjtEntry<false>*>(projt))));
  } else {
    if (sizeof(T) != sizeof(float) && pcount) {
      widen_kernel<T><<<blocks_for(c, (long long)pcount, 256), 256, 0, c->stream>>>(pj32, pj, pcount);
      SPI_TRY(check_kernel("widen_kernel"));
      c->count();
    }
    SPI_TRY(launch_backproject<T>(c, pb, cb, pj, c->cg_buf[3].as<CgDM>(), nullptr, nimg));
  }
  // the ranks' CB and ASTASQ sums (bpcg.f:653-663)
  SPI_TRY(sh.sum(c, cb, (long long)nnn, sizeof(T) == 8));
  SPI_TRY(sh.sum(c, acc, 3, true));
  double hacc[3];
  SPI_CUDA(cudaMemcpyAsync(hacc, acc, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  // pixel counts outside / inside the circle (ASTASQ's D_KLP, D_KLS)
  double klp = 0, kls = 0;
  {
    const float r2 = ri * ri;
    const int nc = n / 2 + 1;
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i) {
        float t = (float)(j - nc), t2 = (float)(i - nc);
        if (t * t + t2 * t2 > r2) klp += 1; else kls += 1;
      }
    klp *= nang;
    kls *= nang;
  }
  const double d_aba = hacc[0] / klp;
  const double d_ssq = hacc[1], d_sus = hacc[2];
  const T qt = (sizeof(T) == sizeof(float)) ? (T)(float)(d_aba * nang) : (T)(d_aba * nang);
  SPI_CUDA(cudaMemsetAsync(acc, 0, 64, c->stream));
  cb_background_kernel<T><<<blocks_for(c, pb.nvox, 256), 256, 0, c->stream>>>(
      cb, c->cg_buf[0].as<CgRun>(), c->cg_buf[1].as<int>(), c->cg_buf[2].as<int>(), pb.nvox, qt, acc);
  SPI_TRY(check_kernel("cb_background_kernel"));
  c->count();
  double bnorm = 0;
  SPI_CUDA(cudaMemcpyAsync(&bnorm, acc, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  const double chi2 = d_ssq - d_aba * (2 * d_sus - d_aba * kls);
  const float di = (float)(n / 2);
  // bpcg.f:269-290: FBS needs RI + MODE <= N/2, linear RI + MODE + 1 <= N/2
  const float extra = fbs ? 0.0f : 1.0f;
  if ((mode == 1 && (ri + 1.0f + extra) > di) || (mode == 2 && (ri + 2.0f + extra) > di) ||
      (mode == 3 && (ri + 3.0f + extra) > di))
    return fail(kMissing, "RADIUS TOO LARGE (%d)", (int)ri);
  if (fbs)
    SPI_CUDA(cudaMemcpyAsync(fs.dm9, dm9.data(), dm9.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  SPI_CUDA(cudaMemcpyAsync(c->cg_buf[3].p, mdms.data(), (size_t)lo * sizeof(CgDM), cudaMemcpyHostToDevice, c->stream));
  SPI_CUDA(cudaMemcpyAsync(dlb, lb.data(), (size_t)lo * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  // ---- BPCG_3_LIN
  SPI_CUDA(cudaMemsetAsync(bckn, 0, 2 * vb, c->stream));  // BCKN, BCKP
  CgScal hs{};
  hs.q = 0.0;
  hs.chi2 = chi2;
  hs.bnorm = bnorm;
  SPI_CUDA(cudaMemcpyAsync(sc, &hs, sizeof(CgScal), cudaMemcpyHostToDevice, c->stream));
  const CgRun* runs = c->cg_buf[0].as<CgRun>();
  const int* vr = c->cg_buf[1].as<int>();
  const int* vo = c->cg_buf[2].as<int>();
  const int nb = blocks_for(c, pb.nvox, 256);
  const float r2 = ri * ri;
  const int nnn_b = blocks_for(c, (long long)nnn, 256);
  const T lam = (T)lambda;
  auto iteration = [&]() -> int {
    // DELSQ = sum CB^2
    SPI_CUDA(cudaMemsetAsync(&sc->delsq, 0, sizeof(double), c->stream));
    dot_kernel<T><<<nb, 256, 0, c->stream>>>(cb, cb, runs, vr, vo, pb.nvox, &sc->delsq);
    dir_update_kernel<T><<<nb, 256, 0, c->stream>>>(bckp, cb, runs, vr, vo, pb.nvox, sc);
    scal_after_dir_kernel<<<1, 32, 0, c->stream>>>(sc);
    SPI_CUDA(cudaMemsetAsync(bcke, 0, vb, c->stream));
    c->count(3);
    // this rank's merged angles [kb, ke) (all of them on one rank)
    const CgDM* mdm = c->cg_buf[3].as<CgDM>() + kb;
    const int* mlb = dlb + kb;
    const int mc = ke - kb;
    if (fbs32) {
      SPI_TRY((fbs_normal<T, float>(c, pb, fs, bckp, bcke, dlb, kb, ke, c->cg_buf[3].as<CgDM>())));
    } else if (fbs) {
      SPI_TRY((fbs_normal<T, T>(c, pb, fs, bckp, bcke, dlb, kb, ke, c->cg_buf[3].as<CgDM>())));
    } else if (mixed) {
      auto* mx = reinterpret_cast<unsigned long long*>(acc + 7);
      if (wide && wtab)
        SPI_TRY((launch_normal_projt<T, true, true>(c, pb, bckp, bcke, mdm, mlb, mc,
                                                    static_cast<ProjtEntry<true>*>(projt), mx)));
      else if (wide)
        SPI_TRY((launch_normal_projt<T, true, false>(c, pb, bckp, bcke, mdm, mlb, mc,
                                                     static_cast<ProjtEntry<false>*>(projt), mx)));
      else
        SPI_TRY((launch_normal_projt<T, false, false>(c, pb, bckp, bcke, mdm, mlb, mc,
                                                      static_cast<ProjtEntry<false>*>(projt), mx)));
    } else {
      SPI_TRY(launch_project<T>(c, pb, bckp, mdm, mc, pj));
      SPI_TRY(launch_backproject<T>(c, pb, bcke, pj, mdm, mlb, mc));
    }
    // the ranks' BCKE (bpcg.f:1031-1032)
    SPI_TRY(sh.sum(c, bcke, (long long)nnn, sizeof(T) == 8));
    zero_outside_kernel<T><<<nnn_b, 256, 0, c->stream>>>(bckp, n, pb.ldp, r2);
    for (int axis = 0; axis < 3; ++axis)
      fixedge_axis_kernel<T><<<(n * n + 127) / 128, 128, 0, c->stream>>>(bckp, n, axis, mode);
    regularize_kernel<T><<<nb, 256, 0, c->stream>>>(bcke, bckp, runs, vr, vo, pb.nvox, n, lam, mode);
    SPI_CUDA(cudaMemsetAsync(&sc->akden, 0, sizeof(double), c->stream));
    dot_kernel<T><<<nb, 256, 0, c->stream>>>(bckp, bcke, runs, vr, vo, pb.nvox, &sc->akden);
    scal_step_kernel<<<1, 32, 0, c->stream>>>(sc);
    step_kernel<T><<<nb, 256, 0, c->stream>>>(bckn, cb, bckp, bcke, runs, vr, vo, pb.nvox, sc);
    SPI_TRY(check_kernel("cg iteration"));
    c->count(9);
    return 0;
  };
  // capture one iteration as a CUDA graph, then replay it
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // the FBS iteration runs cuFFT plans and is launched directly
  bool use_graph = !fbs && !sh.reduce && getenv("SPI_CG_NOGRAPH") == nullptr;
  if (use_graph && cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    use_graph = false;
    cudaGetLastError();
  }
  long long per_iter_launches = 0;
  if (use_graph) {
    const long long before = c->launches;
    const int st = iteration();
    per_iter_launches = c->launches - before;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (st != 0) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      graph = nullptr;
      use_graph = false;
      cudaGetLastError();
    }
    c->launches = before;  // counted per replay below
  }
  int done = 0;
  for (int iter = 1; iter <= maxit; ++iter) {
    if (use_graph) {
      SPI_CUDA(cudaGraphLaunch(exec, c->stream));
      c->launches += per_iter_launches;
    } else {
      SPI_TRY(iteration());
    }
    CgScal s;
    SPI_CUDA(cudaMemcpyAsync(&s, sc, sizeof(CgScal), cudaMemcpyDeviceToHost, c->stream));
    SPI_CUDA(cudaStreamSynchronize(c->stream));
    if (log_out) {
      log_out[3 * (iter - 1)] = (float)iter;
      log_out[3 * (iter - 1) + 1] = (float)s.err;
      log_out[3 * (iter - 1) + 2] = (float)s.chi2;
    }
    done = iter;
    if (std::fabs(s.err) <= errm || std::fabs(s.chi2) <= chim) break;
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (niter_out) *niter_out = done;
  // BCKN -> float volume (staged in the float projection buffer)
  if (sizeof(T) == sizeof(float)) {
    SPI_CUDA(cudaMemcpyAsync(vol_out, bckn, nnn * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  } else {
    std::vector<T> tmp(nnn);
    SPI_CUDA(cudaMemcpyAsync(tmp.data(), bckn, vb, cudaMemcpyDeviceToHost, c->stream));
    SPI_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < nnn; ++i) vol_out[i] = (float)tmp[i];
  }
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

}  // namespace spi

using namespace spi;

extern "C" {

int spi_pj3f(spi_ctx* c, const float* vol, int nx, int ny, int nz, float ri, const float* angles, int nang,
             float* proj_out, int on_device) {
  if (!c) return fail(kInvalid, "NULL context");
  if (nx != ny || nx != nz) return fail(kInvalid, "PJ 3F: cubic volumes only (%dx%dx%d)", nx, ny, nz);
  if (nx > 1024) return fail(kInvalid, "PJ 3F: n = %d above 1024", nx);
  int nruns = 0, ntasks = 0;
  SPI_TRY(pj_common(c, nx, ny, nz, ri, angles, nang, &nruns, &ntasks));
  if (!vol || !proj_out) return fail(kInvalid, "PJ 3F: NULL buffer");
  const int n = nx;
  const size_t nnn = (size_t)n * n * n, vbytes = nnn * sizeof(float);
  const size_t pbytes = (size_t)nang * n * n * sizeof(float);
  const float* dvol = vol;
  float* dout = proj_out;
  if (!on_device) {
    SPI_TRY(c->pj_vol.ensure(vbytes));
    SPI_TRY(c->pj_out.ensure(std::max<size_t>(pbytes, 4)));
    SPI_CUDA(cudaMemcpyAsync(c->pj_vol.p, vol, vbytes, cudaMemcpyHostToDevice, c->stream));
    dvol = c->pj_vol.as<float>();
    dout = c->pj_out.as<float>();
  }
  if (nang == 0) return 0;
  // FBS3_PREP of the volume (writpro_n.f:154-185), REAL tables
  const size_t wb = fbs3_work_bytes(n);
  SPI_TRY(c->pj_fbs.ensure(wb + align256(nnn * 8 * sizeof(float))));
  // the FBS3_PREP plans stay with the context for the next call of this n
  Fbs3Work w;
  int st = 0;
  if (c->pjf_n != n) {
    if (c->pjf_plan[0]) cufftDestroy(c->pjf_plan[0]);
    if (c->pjf_plan[1]) cufftDestroy(c->pjf_plan[1]);
    c->pjf_plan[0] = c->pjf_plan[1] = 0;
    c->pjf_n = 0;
    st = fbs3_work_init(w, n, c->pj_fbs.as<char>(), c->stream);
    if (st != 0) {
      w.destroy();
      return st;
    }
    c->pjf_plan[0] = w.fwd;
    c->pjf_plan[1] = w.inv;
    c->pjf_n = n;
  } else {
    SPI_TRY(fbs3_work_init(w, n, c->pj_fbs.as<char>(), c->stream, false));
    w.fwd = c->pjf_plan[0];
    w.inv = c->pjf_plan[1];
    SPI_CUFFT(cufftSetStream(w.fwd, c->stream));
    SPI_CUFFT(cufftSetStream(w.inv, c->stream));
  }
  float* V = reinterpret_cast<float*>(c->pj_fbs.as<char>() + wb);
  if (st == 0) st = fbs3_prepare<float, float>(c, w, dvol, V);
  if (st == 0) {
    const cudaError_t e = cudaMemsetAsync(dout, 0, pbytes, c->stream);
    if (e != cudaSuccess) st = fail(kCuda, "PJ 3F: %s", cudaGetErrorString(e));
  }
  if (st == 0) {
    const int nocheck = (2.0f * (ri + 1.0f) + 1.0f) <= (float)n;
    if (ntasks > 0) {
      const size_t toff = pj_tasks_offset(nruns);
      const long long warps = (long long)ntasks * nang;
      const int blocks = (int)std::min<long long>((warps + 3) / 4, (long long)c->sm_count * 16);
      wpro_fbs_warp_kernel<float, float><<<blocks, 128, 0, c->stream>>>(
          V, n, c->pj_rows.as<PjRun>(), reinterpret_cast<const int4*>(c->pj_rows.as<char>() + toff), ntasks,
          c->pj_dm.as<PjDM>(), nang, n / 2 + 1, nocheck, dout);
      st = check_kernel("wpro_fbs_warp_kernel");
      c->count();
    }
  }
  if (st == 0 && !on_device) {
    const cudaError_t e = cudaMemcpyAsync(proj_out, dout, pbytes, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) st = fail(kCuda, "PJ 3F: %s", cudaGetErrorString(e));
  }
  const cudaError_t e = cudaStreamSynchronize(c->stream);
  if (st == 0 && e != cudaSuccess) st = fail(kCuda, "PJ 3F: %s", cudaGetErrorString(e));
  return st;
}

int spi_ctx_set_rb_interpolation(spi_ctx* c, int fbs) {
  if (!c) return fail(kInvalid, "NULL context");
  if (fbs != 0 && fbs != 1) return fail(kInvalid, "spi_ctx_set_rb_interpolation: %d must be 0 (RTSQ) or 1 (RTSF)", fbs);
  c->rb_fbs = fbs;
  return 0;
}

int spi_ctx_set_cg_interpolation(spi_ctx* c, int fbs) {
  if (!c) return fail(kInvalid, "NULL context");
  if (fbs != 0 && fbs != 1) return fail(kInvalid, "spi_ctx_set_cg_interpolation: %d must be 0 (linear) or 1 (FBS)", fbs);
  c->cg_interp = fbs;
  return 0;
}

int spi_ctx_set_cg_precision(spi_ctx* c, int mode) {
  if (!c) return fail(kInvalid, "NULL context");
  if (mode < 0 || mode > 4) return fail(kInvalid, "spi_ctx_set_cg_precision: mode %d must be 0 .. 4", mode);
  c->cg_fp64 = mode;
  return 0;
}

int spi_cg_project(spi_ctx* c, const float* vol, int n, float ri, const float* angles, int nang, float* projs,
                   int on_device) {
  if (!c || !vol || !projs || (nang > 0 && !angles)) return fail(kInvalid, "spi_cg_project: bad arguments");
  if (n < 8) return fail(kInvalid, "spi_cg_project: n = %d too small", n);
  SPI_CUDA(cudaSetDevice(c->device));
  CgProblem pb;
  SPI_TRY(cg_setup(c, n, ri, pb));
  std::vector<CgDM> dms;
  dms_from_angles(angles, nang, dms);
  const size_t vb = (size_t)n * n * n * sizeof(float), pbytes = (size_t)nang * n * n * sizeof(float);
  SPI_TRY(c->cg_buf[3].ensure(dms.size() * sizeof(CgDM)));
  SPI_CUDA(cudaMemcpyAsync(c->cg_buf[3].p, dms.data(), dms.size() * sizeof(CgDM), cudaMemcpyHostToDevice, c->stream));
  const float* dv = vol;
  float* dp = projs;
  if (!on_device) {
    SPI_TRY(c->cg_buf[4].ensure(vb));
    SPI_TRY(c->cg_buf[5].ensure(std::max<size_t>(pbytes, 4)));
    SPI_CUDA(cudaMemcpyAsync(c->cg_buf[4].p, vol, vb, cudaMemcpyHostToDevice, c->stream));
    dv = c->cg_buf[4].as<float>();
    dp = c->cg_buf[5].as<float>();
  }
  SPI_TRY(launch_project<float>(c, pb, dv, c->cg_buf[3].as<CgDM>(), nang, dp));
  if (!on_device && pbytes) SPI_CUDA(cudaMemcpyAsync(projs, dp, pbytes, cudaMemcpyDeviceToHost, c->stream));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int spi_cg_backproject(spi_ctx* c, const float* projs, int n, float ri, const float* angles, int nang, float* vol,
                       int on_device) {
  if (!c || !vol || !projs || (nang > 0 && !angles)) return fail(kInvalid, "spi_cg_backproject: bad arguments");
  if (n < 8) return fail(kInvalid, "spi_cg_backproject: n = %d too small", n);
  SPI_CUDA(cudaSetDevice(c->device));
  CgProblem pb;
  SPI_TRY(cg_setup(c, n, ri, pb));
  std::vector<CgDM> dms;
  dms_from_angles(angles, nang, dms);
  const size_t vb = (size_t)n * n * n * sizeof(float), pbytes = (size_t)nang * n * n * sizeof(float);
  SPI_TRY(c->cg_buf[3].ensure(dms.size() * sizeof(CgDM)));
  SPI_CUDA(cudaMemcpyAsync(c->cg_buf[3].p, dms.data(), dms.size() * sizeof(CgDM), cudaMemcpyHostToDevice, c->stream));
  const float* dp = projs;
  float* dv = vol;
  if (!on_device) {
    SPI_TRY(c->cg_buf[4].ensure(vb));
    SPI_TRY(c->cg_buf[5].ensure(std::max<size_t>(pbytes, 4)));
    if (pbytes) SPI_CUDA(cudaMemcpyAsync(c->cg_buf[5].p, projs, pbytes, cudaMemcpyHostToDevice, c->stream));
    dv = c->cg_buf[4].as<float>();
    dp = c->cg_buf[5].as<float>();
  }
  SPI_CUDA(cudaMemsetAsync(dv, 0, vb, c->stream));
  SPI_TRY(launch_backproject<float>(c, pb, dv, dp, c->cg_buf[3].as<CgDM>(), nullptr, nang));
  if (!on_device) SPI_CUDA(cudaMemcpyAsync(vol, dv, vb, cudaMemcpyDeviceToHost, c->stream));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int spi_bpcg(spi_ctx* c, const float* projs, int n, int nang, const float* angles, float ri, float errm, float chim,
             int maxit, int mode, float lambda, float* vol_out, float* log_out, int* niter_out) {
  if (!c || !projs || !angles || !vol_out) return fail(kInvalid, "spi_bpcg: NULL argument");
  if (n < 8 || nang <= 0) return fail(kInvalid, "spi_bpcg: n = %d, nang = %d", n, nang);
  if (mode < 1 || mode > 3) return fail(kInvalid, "spi_bpcg: mode %d must be 1, 2 or 3", mode);
  SPI_CUDA(cudaSetDevice(c->device));
  if (niter_out) *niter_out = 0;
  CgShard sh;   // one process: every image and merged angle, nothing to sum
  sh.count = nang;
  if (c->cg_fp64)
    return bpcg_run<double>(c, projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol_out, log_out,
                            niter_out, sh);
  return bpcg_run<float>(c, projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol_out, log_out, niter_out,
                         sh);
}

int spi_bpcg_shard(spi_ctx* c, const float* projs, int first, int count, int n, int nang, const float* angles,
                   float ri, float errm, float chim, int maxit, int mode, float lambda, int rank, int world,
                   spi_allreduce_fn allreduce, void* user, float* vol_out, float* log_out, int* niter_out) {
  if (!c || !angles || !vol_out || (count > 0 && !projs)) return fail(kInvalid, "spi_bpcg_shard: NULL argument");
  if (n < 8 || nang <= 0) return fail(kInvalid, "spi_bpcg_shard: n = %d, nang = %d", n, nang);
  if (first < 0 || count < 0 || first + count > nang)
    return fail(kInvalid, "spi_bpcg_shard: images [%d, %d) outside the %d angles", first, first + count, nang);
  if (world < 1 || rank < 0 || rank >= world) return fail(kInvalid, "spi_bpcg_shard: rank %d of %d", rank, world);
  if (world > 1 && !allreduce) return fail(kInvalid, "spi_bpcg_shard: %d ranks need an all-reduce callback", world);
  if (mode < 1 || mode > 3) return fail(kInvalid, "spi_bpcg_shard: mode %d must be 1, 2 or 3", mode);
  SPI_CUDA(cudaSetDevice(c->device));
  if (niter_out) *niter_out = 0;
  CgShard sh;
  sh.first = first;
  sh.count = count;
  sh.rank = rank;
  sh.world = world;
  sh.reduce = allreduce;
  sh.user = user;
  if (c->cg_fp64)
    return bpcg_run<double>(c, projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol_out, log_out,
                            niter_out, sh);
  return bpcg_run<float>(c, projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol_out, log_out, niter_out,
                         sh);
}

}  // extern "C"
