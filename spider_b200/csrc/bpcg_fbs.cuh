// BP CG with FBS interpolation (the 'F' answer of BP CG): BPCG_3_FBS
// (bpcg.f:1760-1822) with FBS2_PREP (fbs2.f:182-247), FBS3_PREP
// (fbs3.f:294-407), FBS2 / FBS3 (fbs2.f:94-180, fbs3.f:60-290), PRJCQ_FBS3
// (prjcq.f:97-167) and BCKPJ_FBS (bckpj.f:123-164).  Included by bpcg.cu
// inside namespace spi, after CgRun, CgDM and the round-to-nearest helpers.
//
// Derivatives.  The reference multiplies the SPIDER-sign spectrum (the
// conjugate of the usual forward transform, no scale) by -i*w along each
// axis and transforms back with SPIDER's inverse (conjugate, c2r, 1/N).  Its
// c2r takes only the real part of the x = 0 and x = n/2 bins after the
// complex passes along y (and z).  The derivative spectra are not Hermitian
// in those planes, so here each such plane (column, in 2D) is replaced by its
// Hermitian part (G(k) + conj G(-k)) / 2 before cuFFT's Z2D: the inverse of
// that part is exactly the real part the reference keeps.  The transforms
// run in FP64 for both vector precisions, as the CPU restatement does.
//
// Layout.  The interpolation tables are interleaved: 8 values per voxel
// {F, X1, Y1, XY2, Z1, XZ2, YZ2, XYZ} and 4 per pixel {P, X1, Y1, XY2}, so a
// cubic's two x-neighbours are one contiguous span (128 bytes in FP64).
//
// Sample positions follow the reference's sequential walks (XB = XB + DM(1)
// along an I line of PRJCQ_FBS3, along a voxel run of BCKPJ_FBS), and every
// cubic is evaluated with the reference's operation order in
// round-to-nearest arithmetic without contraction.
#pragma once

// I samples per line between two row reductions (PRJCQ_FBS3): the shared
// tile takes L1 from the gathers, and 16 measured as fast as 8 and faster than 32
constexpr int kFbsIC = 16;
// run voxels per BCKPJ_FBS thread: 4 measured fastest over 128^3 and 256^3
// (2 is 4% faster at 128^3 and 8% slower at 256^3; 8 and 16 are slower)
constexpr int kFbsSeg = 4;

template <class T> struct FbsQuad { T a, b, c, d; };

__device__ __forceinline__ FbsQuad<float> fbs_ldq(const float* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return {v.x, v.y, v.z, v.w};
}
// one 256-bit read-only load (sm_100); every FP64 quad starts on a 32-byte
// boundary (tables are 256-byte aligned, quads 32 bytes apart)
__device__ __forceinline__ FbsQuad<double> fbs_ldq(const double* p) {
  FbsQuad<double> q;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(q.a), "=d"(q.b), "=d"(q.c), "=d"(q.d) : "l"(p));
  return q;
}

// one voxel of an FBS3 table: its value quad {F, X1, Y1, XY2} and its
// z-derivative quad {Z1, XZ2, YZ2, XYZ}.  An FP32 voxel is one 32-byte
// sector, read by one 256-bit load; an FP64 voxel by two.
template <class T>
__device__ __forceinline__ void fbs_ldvox(const float* p, FbsQuad<T>& val, FbsQuad<T>& der) {
  float a[8];
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]), "=f"(a[7])
      : "l"(p));
  val = {(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
  der = {(T)a[4], (T)a[5], (T)a[6], (T)a[7]};
}
template <class T>
__device__ __forceinline__ void fbs_ldvox(const double* p, FbsQuad<T>& val, FbsQuad<T>& der) {
  const FbsQuad<double> u = fbs_ldq(p), w = fbs_ldq(p + 4);
  val = {(T)u.a, (T)u.b, (T)u.c, (T)u.d};
  der = {(T)w.a, (T)w.b, (T)w.c, (T)w.d};
}

// a table quad (type TT) widened to the arithmetic type T
template <class T, class TT>
__device__ __forceinline__ FbsQuad<T> fbs_ld(const TT* p) {
  const FbsQuad<TT> q = fbs_ldq(p);
  return {(T)q.a, (T)q.b, (T)q.c, (T)q.d};
}

// One cubic from values and derivatives at 0 and 1 (fbs2.f:150-170):
// A2 = 3(F1-F0) - 2D0 - D1, A3 = 2(-F1+F0) + D0 + D1, F0 + D0 DX + A2 DX^2 + A3 DX^3.
template <class T>
__device__ __forceinline__ T fbs_cub(T f0, T d0, T f1, T d1, T dx, T dx2, T dx3) {
  const T a2 = rsub(rsub(rmul((T)3, rsub(f1, f0)), rmul((T)2, d0)), d1);
  const T a3 = radd(radd(rmul((T)2, radd(-f1, f0)), d0), d1);
  return radd(radd(radd(f0, rmul(d0, dx)), rmul(a2, dx2)), rmul(a3, dx3));
}

// Bicubic from the quads {F, FX, FY, FXY} at (i2,j2), (i3,j2), (i2,j3), (i3,j3).
template <class T>
__device__ __forceinline__ T fbs_bicubic(const FbsQuad<T>& q00, const FbsQuad<T>& q10, const FbsQuad<T>& q01,
                                         const FbsQuad<T>& q11, T dx, T dx2, T dx3, T dy, T dy2, T dy3) {
  const T adx = fbs_cub(q00.a, q00.b, q10.a, q10.b, dx, dx2, dx3);
  const T bdx = fbs_cub(q01.a, q01.b, q11.a, q11.b, dx, dx2, dx3);
  const T dadx = fbs_cub(q00.c, q00.d, q10.c, q10.d, dx, dx2, dx3);
  const T dbdx = fbs_cub(q01.c, q01.d, q11.c, q11.d, dx, dx2, dx3);
  return fbs_cub(adx, dadx, bdx, dbdx, dy, dy2, dy3);
}

__device__ __forceinline__ int fbs_mod(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}

// FBS2 with CHKBOUND (indices wrapped): P = [n*n][4] {P, X1, Y1, XY2} of
// type TT, arithmetic in T.  Every index is reduced modulo n, so any
// position reads inside the table.
template <class T, class TT>
__device__ __forceinline__ T fbs2_eval(float x, float y, int n, const TT* __restrict__ P) {
  const int i = __float2int_rd(x), j = __float2int_rd(y);
  const T dx = (T)__fsub_rn(x, (float)i), dy = (T)__fsub_rn(y, (float)j);
  const T dx2 = rmul(dx, dx), dx3 = rmul(dx2, dx), dy2 = rmul(dy, dy), dy3 = rmul(dy2, dy);
  const int i2 = fbs_mod(i - 1, n), j2 = fbs_mod(j - 1, n), i3 = fbs_mod(i, n), j3 = fbs_mod(j, n);
  const FbsQuad<T> q00 = fbs_ld<T>(P + ((size_t)j2 * n + i2) * 4);
  const FbsQuad<T> q10 = fbs_ld<T>(P + ((size_t)j2 * n + i3) * 4);
  const FbsQuad<T> q01 = fbs_ld<T>(P + ((size_t)j3 * n + i2) * 4);
  const FbsQuad<T> q11 = fbs_ld<T>(P + ((size_t)j3 * n + i3) * 4);
  return fbs_bicubic(q00, q10, q01, q11, dx, dx2, dx3, dy, dy2, dy3);
}

// FBS3 at (x, y, z) with i = IFIX(x), j = IFIX(y), l = IFIX(z) all in
// [1, n-1] (the PRJCQ_FBS3 bounds check): the corners are (i-1, i) etc.,
// 0-based, with no wrap.  V = [n^3][8] {F, X1, Y1, XY2, Z1, XZ2, YZ2, XYZ}
// of type TT, arithmetic in T.
template <class T, class TT>
__device__ __forceinline__ T fbs3_eval(float x, float y, float z, int i, int j, int l, int n,
                                       const TT* __restrict__ V) {
  const T dx = (T)__fsub_rn(x, (float)i), dy = (T)__fsub_rn(y, (float)j), dz = (T)__fsub_rn(z, (float)l);
  const T dx2 = rmul(dx, dx), dx3 = rmul(dx2, dx), dy2 = rmul(dy, dy), dy3 = rmul(dy2, dy);
  const T dz2 = rmul(dz, dz), dz3 = rmul(dz2, dz);
  const size_t v0 = (((size_t)(l - 1) * n + (j - 1)) * n + (i - 1)) * 8;
  const size_t sy = (size_t)n * 8, sz = (size_t)n * n * 8;
  T c[2], dc[2];
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const TT* b = V + v0 + p * sz;
    // value plane: F, X1, Y1, XY2; z-derivative plane: Z1, XZ2, YZ2, XYZ
    FbsQuad<T> v00, v10, v01, v11, d00, d10, d01, d11;
    fbs_ldvox<T>(b, v00, d00);
    fbs_ldvox<T>(b + 8, v10, d10);
    fbs_ldvox<T>(b + sy, v01, d01);
    fbs_ldvox<T>(b + sy + 8, v11, d11);
    c[p] = fbs_bicubic(v00, v10, v01, v11, dx, dx2, dx3, dy, dy2, dy3);
    dc[p] = fbs_bicubic(d00, d10, d01, d11, dx, dx2, dx3, dy, dy2, dy3);
  }
  return fbs_cub(c[0], dc[0], c[1], dc[1], dz, dz2, dz3);
}

// FBS3 at any position with wrapped indices (FBS3 as WPRO_FBS calls it,
// fbs3.f:60-290): i = FLOOR(x), corners MODULO(i-1, n) and the next one
// modulo n, and likewise for y and z.
template <class T, class TT>
__device__ __forceinline__ T fbs3_eval_wrap(float x, float y, float z, int n, const TT* __restrict__ V) {
  const int i = __float2int_rd(x), j = __float2int_rd(y), l = __float2int_rd(z);
  const int i2 = fbs_mod(i - 1, n), j2 = fbs_mod(j - 1, n), l2 = fbs_mod(l - 1, n);
  const int i3 = (i2 + 1) % n, j3 = (j2 + 1) % n, l3 = (l2 + 1) % n;
  const T dx = (T)__fsub_rn(x, (float)i), dy = (T)__fsub_rn(y, (float)j), dz = (T)__fsub_rn(z, (float)l);
  const T dx2 = rmul(dx, dx), dx3 = rmul(dx2, dx), dy2 = rmul(dy, dy), dy3 = rmul(dy2, dy);
  const T dz2 = rmul(dz, dz), dz3 = rmul(dz2, dz);
  auto at = [&](int ii, int jj, int ll) { return V + (((size_t)ll * n + jj) * n + ii) * 8; };
  T c[2], dc[2];
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const int ll = p ? l3 : l2;
    FbsQuad<T> v00, v10, v01, v11, d00, d10, d01, d11;
    fbs_ldvox<T>(at(i2, j2, ll), v00, d00);
    fbs_ldvox<T>(at(i3, j2, ll), v10, d10);
    fbs_ldvox<T>(at(i2, j3, ll), v01, d01);
    fbs_ldvox<T>(at(i3, j3, ll), v11, d11);
    c[p] = fbs_bicubic(v00, v10, v01, v11, dx, dx2, dx3, dy, dy2, dy3);
    dc[p] = fbs_bicubic(d00, d10, d01, d11, dx, dx2, dx3, dy, dy2, dy3);
  }
  return fbs_cub(c[0], dc[0], c[1], dc[1], dz, dz2, dz3);
}

// ---------------------------------------------------------------------------
// WPRO_FBS (wpro_fbs.f:1-150), PJ 3F, by row tasks as PJ 3Q's
// wpro_warp_kernel: a warp walks up to 32 runs of one output row K = Y + LDP
// (tasks int4 {first run, runs, x1, x2} over the runs in (y, |z|) order) in
// step over x, each lane its run as WPRO_N does (XB = XB + DM(1), ...), every
// sample FBS3 with wrapped indices, and one lane adds the warp's sum of the
// pixel's samples (1.06x the speed of one thread per run with an atomic per
// sample at 128^3, 1.56x at 256^3).  nocheck: the sphere fits
// (2(RI+1)+1 <= N); otherwise samples whose IFIX lies outside 1..N are
// skipped (wpro_fbs.f:138-144).
template <class T, class TT>
__global__ void __launch_bounds__(128) wpro_fbs_warp_kernel(const TT* __restrict__ V, int n,
                                                            const PjRun* __restrict__ runs,
                                                            const int4* __restrict__ tasks, int ntasks,
                                                            const PjDM* __restrict__ dms, int nang, int ldp,
                                                            int nocheck, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long long nwork = (long long)ntasks * nang;
  const long long stride = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long wk = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; wk < nwork; wk += stride) {
    const int a = (int)(wk / ntasks);
    const int4 tk = tasks[wk % ntasks];
    const bool live = lane < tk.y;
    const PjRun r = runs[tk.x + (live ? lane : 0)];
    const int i1 = live ? r.i1 : 1, i2 = live ? r.i2 : 0;
    const PjDM dm = dms[a];
    float* row = out + (size_t)a * n * n + (size_t)(r.y + ldp - 1) * n;
    auto start = [&](float da, float db, float dc) {
      return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn((float)r.x, da), __fmul_rn((float)r.y, db)),
                                 __fmul_rn((float)r.z, dc)),
                       (float)ldp);
    };
    float xb = start(dm.d[0], dm.d[3], dm.d[6]);
    float yb = start(dm.d[1], dm.d[4], dm.d[7]);
    float zb = start(dm.d[2], dm.d[5], dm.d[8]);
    for (int j = tk.z; j <= tk.w; ++j) {
      float v = 0.0f;
      if (j >= i1 && j <= i2) {
        const int iox = __float2int_rz(xb), ioy = __float2int_rz(yb), ioz = __float2int_rz(zb);
        if (nocheck || (iox > 0 && iox <= n && ioy > 0 && ioy <= n && ioz > 0 && ioz <= n))
          v = (float)fbs3_eval_wrap<T, TT>(xb, yb, zb, n, V);
        xb = __fadd_rn(xb, dm.d[0]);
        yb = __fadd_rn(yb, dm.d[1]);
        zb = __fadd_rn(zb, dm.d[2]);
      }
#pragma unroll
      for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
      if (lane == 0 && v != 0.0f) atomicAdd(row + (j - 1), v);
    }
  }
}

// ---------------------------------------------------------------------------
// PRJCQ_FBS3: CTA (row J, projection k); thread t walks line K = t+1 of the
// cube along I.  The samples of IC consecutive I go to shared memory and
// the pixel (I, J) sums them over K in order, as the reference's loop nest
// does; then the HIANG multiplicity LB scales the pixel (bpcg.f:1790-1796).
template <class T, class TT, int MAXT>
__global__ void __launch_bounds__(MAXT) prjcq_fbs3_kernel(const TT* __restrict__ V, const float* __restrict__ dm9,
                                                         const int* __restrict__ lb, int k0, int n,
                                                         T* __restrict__ projs) {
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int IC = kFbsIC;
  T* tile = reinterpret_cast<T*>(smraw);   // [blockDim.x][IC + 1]
  const int k = blockIdx.y;
  const int j = blockIdx.x + 1;
  const int kk = threadIdx.x + 1;
  const bool live = kk <= n;
  const float* dm = dm9 + (size_t)9 * (k0 + k);
  const int h = n / 2;
  const float fh = (float)h, fj = (float)(j - h - 1), fk = (float)(kk - h - 1);
  // -N/2*DM(a) + (J-N/2-1)*DM(b) + (K-N/2-1)*DM(c) + N/2 + 1, left to right
  auto start = [&](float a, float b, float c) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(-__fmul_rn(fh, a), __fmul_rn(fj, b)), __fmul_rn(fk, c)), fh), 1.0f);
  };
  float xb = start(dm[0], dm[3], dm[6]);
  float yb = start(dm[1], dm[4], dm[7]);
  float zb = start(dm[2], dm[5], dm[8]);
  const float d0 = dm[0], d1 = dm[1], d2 = dm[2];
  const int w = lb ? lb[k0 + k] : 1;
  T* out = projs + (size_t)k * n * n + (size_t)(j - 1) * n;
  for (int i0 = 1; i0 <= n; i0 += IC) {
    const int m = min(IC, n - i0 + 1);
    if (live) {
      for (int ii = 0; ii < m; ++ii) {
        T s = (T)0;
        const int iox = __float2int_rz(xb), ioy = __float2int_rz(yb), ioz = __float2int_rz(zb);
        if (iox >= 1 && iox < n && ioy >= 1 && ioy < n && ioz >= 1 && ioz < n)
          s = fbs3_eval<T, TT>(xb, yb, zb, iox, ioy, ioz, n, V);
        tile[threadIdx.x * (IC + 1) + ii] = s;
        xb = __fadd_rn(xb, d0);
        yb = __fadd_rn(yb, d1);
        zb = __fadd_rn(zb, d2);
      }
    }
    __syncthreads();
    if ((int)threadIdx.x < m) {
      T acc = (T)0;
      for (int t = 0; t < n; ++t) acc = radd(acc, tile[t * (IC + 1) + threadIdx.x]);
      if (w > 1) acc = rmul(acc, (T)w);
      out[i0 - 1 + threadIdx.x] = acc;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// BCKPJ_FBS: thread per segment of up to SEG voxels of a run.  For each
// projection, in order, the thread repeats the run's sequential walk up to
// its segment, then adds FBS2 at each of its voxels.  segs[s] = {run, first
// offset within the run}.
template <class T, class TT, int SEG>
__global__ void __launch_bounds__(256) bckpj_fbs_kernel(T* __restrict__ cube, const CgRun* __restrict__ runs,
                                                        const int2* __restrict__ segs, long long nseg,
                                                        const TT* __restrict__ P2, const CgDM* __restrict__ dms,
                                                        int kc, int n, int ldp) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nseg; s += (long long)gridDim.x * blockDim.x) {
    const int2 sg = segs[s];
    const CgRun r = runs[sg.x];
    const int o0 = sg.y;
    const int len = min(SEG, r.l2 - r.l1 + 1 - o0);
    const size_t lin = (size_t)r.l1 - 1 + o0;
    T c[SEG];
#pragma unroll
    for (int t = 0; t < SEG; ++t) c[t] = t < len ? cube[lin + t] : (T)0;
    const float fx = (float)(r.x - ldp), fy = (float)(r.y - ldp), fz = (float)(r.z - ldp);
    for (int k = 0; k < kc; ++k) {
      const CgDM dm = dms[k];
      float xb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[0]), __fmul_rn(fy, dm.d[1])), __fmul_rn(fz, dm.d[2])), (float)ldp);
      float yb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, dm.d[3]), __fmul_rn(fy, dm.d[4])), __fmul_rn(fz, dm.d[5])), (float)ldp);
      for (int t = 0; t < o0; ++t) {
        xb = __fadd_rn(xb, dm.d[0]);
        yb = __fadd_rn(yb, dm.d[3]);
      }
      const TT* P = P2 + (size_t)k * n * n * 4;
#pragma unroll
      for (int t = 0; t < SEG; ++t) {
        if (t < len) c[t] = radd(c[t], fbs2_eval<T, TT>(xb, yb, n, P));
        xb = __fadd_rn(xb, dm.d[0]);
        yb = __fadd_rn(yb, dm.d[3]);
      }
    }
#pragma unroll
    for (int t = 0; t < SEG; ++t)
      if (t < len) cube[lin + t] = c[t];
  }
}

// ---------------------------------------------------------------------------
// Derivative preparation

// dst[q] = (double)(T)src[q] for q < count, zero up to padded
template <class S, class T>
__global__ void fbs_to_double_kernel(const S* __restrict__ src, double* __restrict__ dst, size_t count, size_t padded) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < padded; q += (size_t)gridDim.x * blockDim.x)
    dst[q] = q < count ? (double)(T)src[q] : 0.0;
}

// -i*w*v in the interleaved form of FBS2_PREP / FBS3_PREP: (re, im) -> (im w, -re w)
__device__ __forceinline__ double2 fbs_mul_mi(double2 v, double w) {
  return make_double2(__dmul_rn(v.y, w), -__dmul_rn(v.x, w));
}

// A4 * k with A4 = 2 pi / n in REAL, k the signed frequency of index kk
__device__ __forceinline__ double fbs_w(int kk, int n, float a4) {
  return (double)__fmul_rn((float)(kk <= n / 2 ? kk : kk - n), a4);
}

// FBS2_PREP spectra.  F = [B][n][h] forward spectra (cuFFT sign); W = [3][B][n][h]
// = {X1, Y1, XY2} ready for the inverse: conjugated (SPIDER's inverse sign),
// scaled by 1/n^2, Hermitian part in the x = 0 and x = n/2 columns.
// WY(n/2) keeps its value (FBS2_PREP does not zero its Nyquist frequency).
__global__ void fbs2_spec_kernel(const double2* __restrict__ F, double2* __restrict__ W, int n, int B, float a4,
                                 double scale) {
  const int h = n / 2 + 1;
  const size_t per = (size_t)n * h, total = per * B;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % h);
    const int j = (int)((q / h) % n);
    const size_t b = q / per;
    const double wx = (double)__fmul_rn((float)i, a4);
    auto der = [&](int jj, double2* d) {
      const double2 f = F[b * per + (size_t)jj * h + i];
      const double2 fs = make_double2(f.x, -f.y);   // SPIDER sign
      const double wy = fbs_w(jj, n, a4);
      d[0] = fbs_mul_mi(fs, wx);
      d[1] = fbs_mul_mi(fs, wy);
      d[2] = fbs_mul_mi(d[0], wy);
    };
    double2 d[3];
    der(j, d);
    if (i == 0 || 2 * i == n) {
      double2 e[3];
      der((n - j) % n, e);
#pragma unroll
      for (int m = 0; m < 3; ++m) d[m] = make_double2((d[m].x + e[m].x) * 0.5, (d[m].y - e[m].y) * 0.5);
    }
#pragma unroll
    for (int m = 0; m < 3; ++m)
      W[((size_t)m * B + b) * per + (size_t)j * h + i] = make_double2(d[m].x * scale, -d[m].y * scale);
  }
}

// FBS3_PREP spectra.  F = [n][n][h]; W = [7][n][n][h] = {X1, Y1, Z1, XY2, XZ2,
// YZ2, XYZ}, prepared for the inverse as in fbs2_spec_kernel.  WY and WZ are
// zero at the Nyquist index (fbs3.f:330-345); XZ2 takes X1's real part for
// both components (fbs3.f:379-380), as the reference has it.
__global__ void fbs3_spec_kernel(const double2* __restrict__ F, double2* __restrict__ W, int n, float a4,
                                 double scale) {
  const int h = n / 2 + 1;
  const size_t per = (size_t)n * n * h;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < per; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % h);
    const int j = (int)((q / h) % n);
    const int l = (int)(q / ((size_t)n * h));
    const double wx = (double)__fmul_rn((float)i, a4);
    auto wsig = [&](int kk) -> double { return (n % 2 == 0 && 2 * kk == n) ? 0.0 : fbs_w(kk, n, a4); };
    auto der = [&](int jj, int ll, double2* d) {
      const double2 f = F[((size_t)ll * n + jj) * h + i];
      const double2 fs = make_double2(f.x, -f.y);
      const double wy = wsig(jj), wz = wsig(ll);
      const double2 x1 = fbs_mul_mi(fs, wx), y1 = fbs_mul_mi(fs, wy), xy2 = fbs_mul_mi(x1, wy);
      d[0] = x1;
      d[1] = y1;
      d[2] = fbs_mul_mi(fs, wz);
      d[3] = xy2;
      d[4] = make_double2(__dmul_rn(x1.x, wz), -__dmul_rn(x1.x, wz));
      d[5] = fbs_mul_mi(y1, wz);
      d[6] = fbs_mul_mi(xy2, wz);
    };
    double2 d[7];
    der(j, l, d);
    if (i == 0 || 2 * i == n) {
      double2 e[7];
      der((n - j) % n, (n - l) % n, e);
#pragma unroll
      for (int m = 0; m < 7; ++m) d[m] = make_double2((d[m].x + e[m].x) * 0.5, (d[m].y - e[m].y) * 0.5);
    }
#pragma unroll
    for (int m = 0; m < 7; ++m) W[(size_t)m * per + q] = make_double2(d[m].x * scale, -d[m].y * scale);
  }
}

// P[q] = {(T)src[q], (T)D[q], (T)D[ds+q], (T)D[2 ds+q]} (value, X1, Y1, XY2)
template <class S, class T>
__global__ void fbs2_pack_kernel(const S* __restrict__ src, const double* __restrict__ D, T* __restrict__ P,
                                 size_t count, size_t dstride) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < count; q += (size_t)gridDim.x * blockDim.x) {
    T* o = P + q * 4;
    o[0] = (T)src[q];
    o[1] = (T)D[q];
    o[2] = (T)D[dstride + q];
    o[3] = (T)D[2 * dstride + q];
  }
}

// V[v] = {F, X1, Y1, XY2, Z1, XZ2, YZ2, XYZ} of type TT; D = [7][n^3] in the
// order X1, Y1, Z1, XY2, XZ2, YZ2, XYZ
template <class T, class TT>
__global__ void fbs3_pack_kernel(const T* __restrict__ cube, const double* __restrict__ D, TT* __restrict__ V,
                                 size_t nnn) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nnn; q += (size_t)gridDim.x * blockDim.x) {
    TT* o = V + q * 8;
    o[0] = (TT)cube[q];
    o[1] = (TT)D[q];
    o[2] = (TT)D[nnn + q];
    o[3] = (TT)D[3 * nnn + q];
    o[4] = (TT)D[2 * nnn + q];
    o[5] = (TT)D[4 * nnn + q];
    o[6] = (TT)D[5 * nnn + q];
    o[7] = (TT)D[6 * nnn + q];
  }
}

// ---------------------------------------------------------------------------
// RTSF (rtsf.f:109-205), the SCLI = 1 branch that RB 3F / RB 32F take with
// SPIDER's FBS mode on (bp3f.f:412-417): output pixel (IX, IY) is FBS2 (with
// wrapped indices) of the image at its rotated and shifted source position.
// prm[b] = {COS(THETA), SIN(THETA), MODULO(SHX, NX), MODULO(SHY, NX)} in REAL,
// computed by the host; P2 = [nimg][nx*nx][4] FBS2 tables of the images.
__global__ void rtsf_kernel(const float* __restrict__ P2, float* __restrict__ out, int nx, int nimg,
                            const float4* __restrict__ prm) {
  const size_t nn = (size_t)nx * nx, total = (size_t)nimg * nn;
  const float fn = (float)nx, fc = (float)(nx / 2 + 1);   // CX = CY = NX/2 + 1
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(q / nn);
    const int p = (int)(q % nn);
    const int ix = p % nx + 1, iy = p / nx + 1;
    const float4 m = prm[b];
    // FY = IY + FY0, replaced by IY + FY1 / IY + FY2 across the shifted edge
    float fy = __fadd_rn((float)iy, __fsub_rn(-m.w, fc));
    if ((float)(iy - 1) < m.w) fy = __fadd_rn((float)iy, __fsub_rn(__fadd_rn(-m.w, fn), fc));
    if ((float)(iy - 1) >= __fadd_rn(m.w, fn)) fy = __fadd_rn((float)iy, __fsub_rn(__fsub_rn(-m.w, fn), fc));
    float fx = __fadd_rn((float)ix, __fsub_rn(-m.z, fc));
    if ((float)(ix - 1) < m.z) fx = __fadd_rn((float)ix, __fsub_rn(__fadd_rn(-m.z, fn), fc));
    if ((float)(ix - 1) >= __fadd_rn(m.z, fn)) fx = __fadd_rn((float)ix, __fsub_rn(__fsub_rn(-m.z, fn), fc));
    const float ycod = __fadd_rn(__fmul_rn(m.x, fy), fc);
    const float ysid = __fadd_rn(__fmul_rn(-m.y, fy), fc);
    const float xold = __fadd_rn(__fmul_rn(m.x, fx), ysid);
    const float yold = __fadd_rn(__fmul_rn(m.y, fx), ycod);
    out[q] = fbs2_eval<float, float>(xold, yold, nx, P2 + (size_t)b * nn * 4);
  }
}
