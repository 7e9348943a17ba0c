// PJ 3Q: real-space trilinear projection (WPRO_N, wpro_n.f:44-150) and its
// exact adjoint (trilinear insertion), on sm_100a.
//
// PREPCUB (prepcub.f:54-109) turns the sphere of radius RI into runs of
// voxels along x.  WPRO_N walks each run accumulating the sample position
// with XB = XB + DM(1) (sequential float additions), so one GPU thread owns
// one (projection, run) pair and walks it in the same order: every sample
// position and every trilinear weight is bit-identical to the CPU form.  The
// forward projection gives a warp up to 32 runs of one output row and sums
// their samples at each x before one atomic add (wpro_warp_kernel); the
// adjoint walks the runs in PREPCUB's (z, y) order, one per thread.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "../../include/spider_b200.h"
#include "ctx.h"
#include "pj_runs.h"

namespace spi {

// PREPCUB's runs, in its (z, y) order
static void prepcub(int nsam, int nrow, int nslice, float ri, int ldpx, int ldpy, int ldpz, std::vector<PjRun>& runs) {
  runs.clear();
  prepcub_lines(nsam, nrow, nslice, ri, ldpx, ldpy, ldpz, [&](int a, int b, int y, int z) {
    runs.push_back(PjRun{a, b, a - ldpx, y - ldpy, z - ldpz});
  });
}

// Start position of a run: IPCUBE(3)*DM(1) + IPCUBE(4)*DM(4) + IPCUBE(5)*DM(7) + LDPX
__device__ __forceinline__ float run_start(const PjRun& r, float a, float b, float c, int ldp) {
  return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn((float)r.x, a), __fmul_rn((float)r.y, b)), __fmul_rn((float)r.z, c)),
                   (float)ldp);
}

// a[o] for a run-time corner index o, by selects (no local memory)
__device__ __forceinline__ float sel8(const float (&a)[8], int o) {
  float v = a[0];
#pragma unroll
  for (int i = 1; i < 8; ++i) v = (o == i) ? a[i] : v;
  return v;
}

// One WPRO_N sample at (xb, yb, zb): the trilinear value when IFIX of every
// coordinate lies in 1..n-1 (wpro_n.f:93-98), else 0 (the reference adds
// nothing).  FORM (PjForm) selects the plain volume (eight floats), quads
// (two 16-byte loads) or cells (one 32-byte load); all give the same bits.
template <int FORM>
__device__ __forceinline__ float wpro_sample(const float* __restrict__ cube, const float4* __restrict__ v4, int nsam,
                                             int nrow, int nslice, float xb, float yb, float zb) {
  const int iox = __float2int_rz(xb), ioy = __float2int_rz(yb), ioz = __float2int_rz(zb);
  if (!(iox >= 1 && iox < nsam && ioy >= 1 && ioy < nrow && ioz >= 1 && ioz < nslice)) return 0.0f;
  const size_t sy = (size_t)nsam, sz = (size_t)nsam * nrow;
  const size_t o = (size_t)(ioz - 1) * sz + (size_t)(ioy - 1) * sy + (iox - 1);
  const float dx = __fsub_rn(xb, (float)iox), dy = __fsub_rn(yb, (float)ioy), dz = __fsub_rn(zb, (float)ioz);
  float c000, c100, c010, c110, c001, c101, c011, c111;
  if (FORM == 2) {
    float a[8];
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]), "=f"(a[7])
        : "l"(v4 + 2 * o));
    c000 = a[0]; c100 = a[1]; c010 = a[2]; c110 = a[3];
    c001 = a[4]; c101 = a[5]; c011 = a[6]; c111 = a[7];
  } else if (FORM == 1) {
    const float4 q0 = __ldg(v4 + o), q1 = __ldg(v4 + o + sz);
    c000 = q0.x; c100 = q0.y; c010 = q0.z; c110 = q0.w;
    c001 = q1.x; c101 = q1.y; c011 = q1.z; c111 = q1.w;
  } else {
    const float* c0 = cube + o;
    c000 = __ldg(c0); c100 = __ldg(c0 + 1); c010 = __ldg(c0 + sy); c110 = __ldg(c0 + sy + 1);
    c001 = __ldg(c0 + sz); c101 = __ldg(c0 + sz + 1); c011 = __ldg(c0 + sz + sy); c111 = __ldg(c0 + sz + sy + 1);
  }
  // A1..A8 exactly as wpro_n.f:103-114
  const float a1 = c000;
  const float a2 = __fsub_rn(c100, a1);
  const float a3 = __fsub_rn(c010, a1);
  const float a4 = __fsub_rn(c001, a1);
  const float a5 = __fadd_rn(__fsub_rn(-a2, c010), c110);
  const float a61 = __fadd_rn(-c001, c101);
  const float a6 = __fadd_rn(-a2, a61);
  const float a7 = __fadd_rn(__fsub_rn(-a3, c001), c011);
  const float a8 = __fadd_rn(__fsub_rn(__fsub_rn(-a5, a61), c011), c111);
  // A1 + DZ*(A4 + A6*DX + (A7 + A8*DX)*DY) + A3*DY + DX*(A2 + A5*DY)
  const float inner = __fadd_rn(__fadd_rn(a4, __fmul_rn(a6, dx)), __fmul_rn(__fadd_rn(a7, __fmul_rn(a8, dx)), dy));
  float v = __fadd_rn(a1, __fmul_rn(dz, inner));
  v = __fadd_rn(v, __fmul_rn(a3, dy));
  return __fadd_rn(v, __fmul_rn(dx, __fadd_rn(a2, __fmul_rn(a5, dy))));
}

// Forward projection by row tasks: a warp takes up to 32 runs of one output
// row K = y + LDPY (tasks = int4 {first run, runs, x1, x2}, runs in order of
// |z| so their x ranges nest) and walks them in step over x = x1..x2, every
// lane its own run with the reference's sequential XB = XB + DM(1) while x
// lies in its range.  The lanes' samples at one x all belong to pixel (x, K),
// so the warp sums them with shuffles and one lane adds the sum: one L2
// atomic per 32 samples instead of one per sample (at 128^3 the L2
// reductions fall from 64M to 2.4M per 64 projections).  Reads the packed
// volume (FORM: quads or cells); sample values are the bits of wpro_kernel's,
// only the order of the sum over z differs.  SLAB: only samples whose IOZ
// lies in zlo <= IOZ < zhi are taken, so a packed volume larger than L2 is
// read slab by slab (the row tasks then hold consecutive z); a run whose ZB
// misses the slab sits out, a lane stops at the slab's far side (ZB moves one
// way along a run), and the warp leaves the task once all lanes have.
template <int FORM, bool SLAB>
__global__ void __launch_bounds__(128) wpro_warp_kernel(const float4* __restrict__ v4, int nsam, int nrow, int nslice,
                                                        const PjRun* __restrict__ runs,
                                                        const int4* __restrict__ tasks, int ntasks,
                                                        const PjDM* __restrict__ dms, int nang, int ldpx, int ldpy,
                                                        int ldpz, int zlo, int zhi, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long long nwork = (long long)ntasks * nang;
  const long long stride = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; w < nwork; w += stride) {
    const int a = (int)(w / ntasks);
    const int4 tk = tasks[w % ntasks];
    const bool live = lane < tk.y;
    const PjRun r = runs[tk.x + (live ? lane : 0)];
    int i1 = live ? r.i1 : 1, i2 = live ? r.i2 : 0;
    const PjDM dm = dms[a];
    float* row = out + (size_t)a * nsam * nrow + (size_t)(r.y + ldpy - 1) * nsam;
    float xb = run_start(r, dm.d[0], dm.d[3], dm.d[6], ldpx);
    float yb = run_start(r, dm.d[1], dm.d[4], dm.d[7], ldpy);
    float zb = run_start(r, dm.d[2], dm.d[5], dm.d[8], ldpz);
    if (SLAB) {
      // a run whose ZB (linear along it; 2-voxel margin for the walk's
      // rounding) misses the slab takes no part in this pass
      const float ze = zb + (float)(i2 - i1) * dm.d[2];
      if (fmaxf(zb, ze) + 2.0f < (float)zlo || fminf(zb, ze) - 2.0f > (float)zhi) i2 = i1 - 1;
      if (!__any_sync(0xffffffffu, i2 >= i1)) continue;
    }
    if constexpr (!SLAB && FORM == 2) {
      // one pass on cells: each lane stores its sample in the warp's 32 x 33
      // tile (row = lane's run, column = step); every 32 steps lane l adds
      // up column l, one pixel, and the warp's atomics cover 32 consecutive
      // pixels.  Padded rows keep stores and column reads conflict-free.
      // Plans of 2,000 projections at 128^3: 231k projections/s against
      // 189k with the shuffle sums; on quads (192^3, 1,000 projections) the
      // tile was slower, 35.6k against 42.4k, so quads keep the shuffles.
      __shared__ float wtile[4][32][33];   // one tile per warp of the 128-thread CTA
      float(*tile)[33] = wtile[threadIdx.x >> 5];
      int j0 = tk.z;
      for (int j = tk.z; j <= tk.w; ++j) {
        float v = 0.0f;
        if (j >= i1 && j <= i2) {
          v = wpro_sample<FORM>(nullptr, v4, nsam, nrow, nslice, xb, yb, zb);
          xb = __fadd_rn(xb, dm.d[0]);
          yb = __fadd_rn(yb, dm.d[1]);
          zb = __fadd_rn(zb, dm.d[2]);
        }
        tile[lane][j - j0] = v;
        if (j - j0 == 31 || j == tk.w) {
          __syncwarp();
          if (lane <= j - j0) {
            float acc = 0.0f;
#pragma unroll 8
            for (int q = 0; q < 32; ++q) acc += tile[q][lane];
            if (acc != 0.0f) atomicAdd(row + (j0 + lane - 1), acc);
          }
          __syncwarp();
          j0 = j + 1;
        }
      }
    } else {
    for (int j = tk.z; j <= tk.w; ++j) {
      float v = 0.0f;
      if (j >= i1 && j <= i2) {
        if (SLAB) {
          const int ioz = __float2int_rz(zb);
          if ((dm.d[2] > 0.0f && ioz >= zhi) || (dm.d[2] < 0.0f && ioz < zlo)) {
            i2 = j - 1;   // past the slab: ZB moves one way along the run
          } else if (ioz >= zlo && ioz < zhi) {
            v = wpro_sample<FORM>(nullptr, v4, nsam, nrow, nslice, xb, yb, zb);
          }
        } else {
          v = wpro_sample<FORM>(nullptr, v4, nsam, nrow, nslice, xb, yb, zb);
        }
        xb = __fadd_rn(xb, dm.d[0]);
        yb = __fadd_rn(yb, dm.d[1]);
        zb = __fadd_rn(zb, dm.d[2]);
      }
      // SLAB: every lane has finished its run or passed the slab after this step
      const bool finished = SLAB && __all_sync(0xffffffffu, j >= i2);
      if (!SLAB || __any_sync(0xffffffffu, v != 0.0f)) {
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
        if (lane == 0 && v != 0.0f) atomicAdd(row + (j - 1), v);
      }
      if (finished) break;
    }
    }
  }
}

__global__ void __launch_bounds__(128) wpro_kernel(const float* __restrict__ cube, int nsam, int nrow, int nslice,
                                                   const PjRun* __restrict__ runs, int nruns,
                                                   const PjDM* __restrict__ dms, int nang, int ldpx, int ldpy,
                                                   int ldpz, float* __restrict__ out) {
  const long long total = (long long)nruns * nang;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t / nruns);
    const PjRun r = runs[t % nruns];
    const PjDM dm = dms[a];
    float* b = out + (size_t)a * nsam * nrow + (size_t)(r.y + ldpy - 1) * nsam;
    float xb = run_start(r, dm.d[0], dm.d[3], dm.d[6], ldpx);
    float yb = run_start(r, dm.d[1], dm.d[4], dm.d[7], ldpy);
    float zb = run_start(r, dm.d[2], dm.d[5], dm.d[8], ldpz);
    for (int j = r.i1; j <= r.i2; ++j) {
      const float v = wpro_sample<0>(cube, nullptr, nsam, nrow, nslice, xb, yb, zb);
      if (v != 0.0f) atomicAdd(b + (j - 1), v);
      xb = __fadd_rn(xb, dm.d[0]);
      yb = __fadd_rn(yb, dm.d[1]);
      zb = __fadd_rn(zb, dm.d[2]);
    }
  }
}

// Packed volumes for the forward projection.  Quads {f(x,y,z), f(x+1,y,z),
// f(x,y+1,z), f(x+1,y+1,z)} (16 bytes per voxel, 0 past the last x or y):
// a trilinear sample reads two quads (planes z and z+1) instead of eight
// scattered floats.  Cells (32 bytes per voxel: the quads of planes z and
// z+1 side by side, 0 past the last z): one 256-bit load per sample.
// Measured with plans of 2,000 (128^3) and 500 (256^3) projections, against
// one thread per run on the plain volume (97k and 8.7k projections/s):
// wpro_warp_kernel on cells 189k at 128^3 (67 MB, inside L2) but 11.0k at
// 256^3 (537 MB); on quads 153k and 13.1k.  So cells while they take at most
// kCellMaxBytes, quads up to quad_fwd_max(), then the plain volume.  The
// adjoint accumulates into quads under the same cap, in z slabs of at most
// kSlabBytes so that each slab's quads stay in L2.
constexpr size_t kCellMaxBytes = size_t(96) << 20;
constexpr size_t kSlabBytes = size_t(64) << 20;
// 8 GB of packed volume or quad accumulator (quads of volumes up to about
// 800^3); SPI_PJ_QUADMAX (MiB) overrides, 0 keeps the forward projection on
// the plain volume and the adjoint on scalar atomics.
static size_t quad_fwd_max() {
  const char* e = getenv("SPI_PJ_QUADMAX");
  return e ? (size_t)std::max(0LL, atoll(e)) << 20 : size_t(8) << 30;
}
// z slabs of the forward projection for a packed volume of `bytes`: one pass
// up to twice kCellMaxBytes, above that slabs of at most kCellMaxBytes whose
// quads stay in L2 (wpro_warp_kernel<FORM, true>).  Plans at 256^3 (268 MB
// of quads, 3 slabs), 500 projections: 15.0k against 13.4k projections/s in
// one pass (64 MB slabs 14.4k, 32 MB 11.0k; cells in 96 MB slabs 12.5k); at
// 192^3 (113 MB of quads) two slabs were 9% slower than one pass.
static int fwd_slabs(size_t bytes) {
  if (bytes <= 2 * kCellMaxBytes) return 1;
  return (int)((bytes + kCellMaxBytes - 1) / kCellMaxBytes);
}
enum PjForm { kPjPlain = 0, kPjQuads = 1, kPjCells = 2 };
static int pj_fwd_form(size_t nvox) {
  const size_t cap = quad_fwd_max();
  if (nvox * 32 <= std::min(cap, kCellMaxBytes)) return kPjCells;
  return nvox * 16 <= cap ? kPjQuads : kPjPlain;
}
static size_t pj_packed_bytes(int form, size_t nvox) { return form == kPjCells ? nvox * 32 : form == kPjQuads ? nvox * 16 : 0; }

__global__ void pj_pack4_kernel(const float* __restrict__ cube, int nsam, int nrow, int nslice,
                                float4* __restrict__ v4) {
  const size_t total = (size_t)nsam * nrow * nslice;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % nsam);
    const int y = (int)((q / nsam) % nrow);
    const bool bx = x + 1 < nsam, by = y + 1 < nrow;
    v4[q] = make_float4(__ldg(cube + q), bx ? __ldg(cube + q + 1) : 0.0f, by ? __ldg(cube + q + nsam) : 0.0f,
                        (bx && by) ? __ldg(cube + q + nsam + 1) : 0.0f);
  }
}

// cell of voxel q: v8[2q] = quad of plane z, v8[2q + 1] = quad of plane z + 1
__global__ void pj_pack_cells_kernel(const float* __restrict__ cube, int nsam, int nrow, int nslice,
                                     float4* __restrict__ v8) {
  const size_t total = (size_t)nsam * nrow * nslice, sz = (size_t)nsam * nrow;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % nsam);
    const int y = (int)((q / nsam) % nrow);
    const int z = (int)(q / sz);
    const bool bx = x + 1 < nsam, by = y + 1 < nrow;
    float4 lo = make_float4(__ldg(cube + q), bx ? __ldg(cube + q + 1) : 0.0f, by ? __ldg(cube + q + nsam) : 0.0f,
                            (bx && by) ? __ldg(cube + q + nsam + 1) : 0.0f);
    float4 hi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (z + 1 < nslice) {
      const float* c1 = cube + q + sz;
      hi = make_float4(__ldg(c1), bx ? __ldg(c1 + 1) : 0.0f, by ? __ldg(c1 + nsam) : 0.0f,
                       (bx && by) ? __ldg(c1 + nsam + 1) : 0.0f);
    }
    v8[2 * q] = lo;
    v8[2 * q + 1] = hi;
  }
}

// Transpose of wpro_kernel: every sample spreads its projection value into
// the 8 neighbouring voxels with the trilinear weights of the same position.
// Along a run the 2 x 2 x 2 cell moves by at most one voxel per axis and
// step (each row of the rotation has unit length), so the eight sums of the
// current cell are kept in registers; when the cell moves, the corners the
// next cell shares move with it and only the others go to memory as atomic
// adds (about half the atomics; each weight still goes to the same voxel).
__global__ void __launch_bounds__(128) wpro_adjoint_kernel(const float* __restrict__ proj, int nsam, int nrow, int nslice,
                                                           const PjRun* __restrict__ runs, int nruns,
                                                           const PjDM* __restrict__ dms, int nang, int ldpx, int ldpy,
                                                           int ldpz, float* __restrict__ cube) {
  const long long total = (long long)nruns * nang;
  const size_t sy = (size_t)nsam, sz = (size_t)nsam * nrow;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t / nruns);
    const PjRun r = runs[t % nruns];
    const PjDM dm = dms[a];
    const float* b = proj + (size_t)a * nsam * nrow;
    const int k = r.y + ldpy;
    float xb = run_start(r, dm.d[0], dm.d[3], dm.d[6], ldpx);
    float yb = run_start(r, dm.d[1], dm.d[4], dm.d[7], ldpy);
    float zb = run_start(r, dm.d[2], dm.d[5], dm.d[8], ldpz);
    int cx = -8, cy = -8, cz = -8;   // cached cell (none); corner o = i + 2 j + 4 l at (cx+i, cy+j, cz+l)
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    auto move_to = [&](int qx, int qy, int qz) {
      const int dx = qx - cx, dy = qy - cy, dz = qz - cz;
      float nw[8];
#pragma unroll
      for (int o = 0; o < 8; ++o) {   // old corner o lands in new corner (i-dx, j-dy, l-dz) or is flushed
        const int i = o & 1, j = (o >> 1) & 1, l = o >> 2;
        const int ni = i - dx, nj = j - dy, nl = l - dz;
        const bool keep = (unsigned)ni < 2u && (unsigned)nj < 2u && (unsigned)nl < 2u;
        if (!keep && acc[o] != 0.0f)
          atomicAdd(cube + (size_t)(cz + l - 1) * sz + (size_t)(cy + j - 1) * sy + (cx + i - 1), acc[o]);
      }
#pragma unroll
      for (int o = 0; o < 8; ++o) {   // new corner o takes old corner (i+dx, j+dy, l+dz) when it exists
        const int oi = (o & 1) + dx, oj = ((o >> 1) & 1) + dy, ol = (o >> 2) + dz;
        const bool has = (unsigned)oi < 2u && (unsigned)oj < 2u && (unsigned)ol < 2u;
        nw[o] = has ? sel8(acc, oi + 2 * oj + 4 * ol) : 0.0f;
      }
#pragma unroll
      for (int o = 0; o < 8; ++o) acc[o] = nw[o];
      cx = qx; cy = qy; cz = qz;
    };
    for (int j = r.i1; j <= r.i2; ++j) {
      const int iox = __float2int_rz(xb), ioy = __float2int_rz(yb), ioz = __float2int_rz(zb);
      if (iox >= 1 && iox < nsam && ioy >= 1 && ioy < nrow && ioz >= 1 && ioz < nslice) {
        const float p = __ldg(b + (size_t)(k - 1) * nsam + (j - 1));
        if (p != 0.0f) {
          const float dx = __fsub_rn(xb, (float)iox), dy = __fsub_rn(yb, (float)ioy), dz = __fsub_rn(zb, (float)ioz);
          const float ex = 1.0f - dx, ey = 1.0f - dy, ez = 1.0f - dz;
          if (iox != cx || ioy != cy || ioz != cz) move_to(iox, ioy, ioz);
          acc[0] += p * ex * ey * ez;
          acc[1] += p * dx * ey * ez;
          acc[2] += p * ex * dy * ez;
          acc[3] += p * dx * dy * ez;
          acc[4] += p * ex * ey * dz;
          acc[5] += p * dx * ey * dz;
          acc[6] += p * ex * dy * dz;
          acc[7] += p * dx * dy * dz;
        }
      }
      xb = __fadd_rn(xb, dm.d[0]);
      yb = __fadd_rn(yb, dm.d[1]);
      zb = __fadd_rn(zb, dm.d[2]);
    }
    move_to(-8, -8, -8);   // flush
  }
}

// The adjoint into x/y-neighbour quads: a sample's eight trilinear weights
// are two float4 adds (planes z and z+1) to the quad of its cell, whose
// origin is the cell's lowest corner; the two quads of the current cell stay
// in registers while the walk stays in it.  Every weight is the one
// wpro_adjoint_kernel adds to the same voxel; pj_unfold4_kernel then sums
// the four quads that hold a voxel.  Two 16-byte vector atomics per cell
// instead of about 3.6 scalar L2 requests per sample (measured at 128^3,
// where the adjoint is bound by L2 throughput).
//
// Only cells whose lowest corner lies in planes zlo <= IOZ < zhi are added
// (the whole volume: 1, nslice), so an accumulator larger than L2 is done in
// slabs that each stay in L2.  Runs whose ZB (linear along the run, with a
// 2-voxel margin for the walk's rounding) misses the slab are skipped, and a
// walk stops once ZB has passed it: adding DM(3) of one sign moves ZB, and
// its truncation, one way only.
__global__ void __launch_bounds__(128) wpro_adjoint4_kernel(const float* __restrict__ proj, int nsam, int nrow,
                                                            int nslice, const PjRun* __restrict__ runs, int nruns,
                                                            const PjDM* __restrict__ dms, int nang, int ldpx,
                                                            int ldpy, int ldpz, int zlo, int zhi, int order,
                                                            float4* __restrict__ q4) {
  const long long total = (long long)nruns * nang;
  const size_t sy = (size_t)nsam, sz = (size_t)nsam * nrow;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t / nruns);
    const PjDM dm = dms[a];
    // neighbouring threads take neighbouring runs: in (z, y) order their
    // walks lie DM(4:6) apart in the volume, in (y, z) order DM(7:9) apart
    bool yz = order == 3;
    if (order == 1) yz = fabsf(dm.d[6]) > fabsf(dm.d[3]);        // the larger x component
    else if (order == 2) yz = fabsf(dm.d[8]) < fabsf(dm.d[5]);   // the smaller z component
    const PjRun r = runs[(yz ? nruns : 0) + t % nruns];
    const float* b = proj + (size_t)a * nsam * nrow;
    const int k = r.y + ldpy;
    float xb = run_start(r, dm.d[0], dm.d[3], dm.d[6], ldpx);
    float yb = run_start(r, dm.d[1], dm.d[4], dm.d[7], ldpy);
    float zb = run_start(r, dm.d[2], dm.d[5], dm.d[8], ldpz);
    const float ze = zb + (float)(r.i2 - r.i1) * dm.d[2];
    if (fmaxf(zb, ze) + 2.0f < (float)zlo || fminf(zb, ze) - 2.0f > (float)zhi) continue;
    int cx = 0, cy = 0, cz = 0;   // cached cell (1-based lowest corner; 0 = none)
    float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
    auto flush = [&]() {
      if (cx > 0) {
        float4* p0 = q4 + (size_t)(cz - 1) * sz + (size_t)(cy - 1) * sy + (cx - 1);
        atomicAdd(p0, a0);
        atomicAdd(p0 + sz, a1);
      }
    };
    for (int j = r.i1; j <= r.i2; ++j) {
      const int iox = __float2int_rz(xb), ioy = __float2int_rz(yb), ioz = __float2int_rz(zb);
      if ((dm.d[2] > 0.0f && ioz >= zhi) || (dm.d[2] < 0.0f && ioz < zlo)) break;
      if (iox >= 1 && iox < nsam && ioy >= 1 && ioy < nrow && ioz >= zlo && ioz < zhi) {
        const float p = __ldg(b + (size_t)(k - 1) * nsam + (j - 1));
        if (p != 0.0f) {
          const float dx = __fsub_rn(xb, (float)iox), dy = __fsub_rn(yb, (float)ioy), dz = __fsub_rn(zb, (float)ioz);
          const float ex = 1.0f - dx, ey = 1.0f - dy, ez = 1.0f - dz;
          if (iox != cx || ioy != cy || ioz != cz) {
            flush();
            cx = iox; cy = ioy; cz = ioz;
            a0 = make_float4(0.f, 0.f, 0.f, 0.f);
            a1 = a0;
          }
          a0.x += p * ex * ey * ez;
          a0.y += p * dx * ey * ez;
          a0.z += p * ex * dy * ez;
          a0.w += p * dx * dy * ez;
          a1.x += p * ex * ey * dz;
          a1.y += p * dx * ey * dz;
          a1.z += p * ex * dy * dz;
          a1.w += p * dx * dy * dz;
        }
      }
      xb = __fadd_rn(xb, dm.d[0]);
      yb = __fadd_rn(yb, dm.d[1]);
      zb = __fadd_rn(zb, dm.d[2]);
    }
    flush();
  }
}

// voxel (x, y, z) = its share of the quads with origins (x, y), (x-1, y),
// (x, y-1) and (x-1, y-1) in plane z
__global__ void pj_unfold4_kernel(const float4* __restrict__ q4, int nsam, int nrow, int nslice,
                                  float* __restrict__ cube) {
  const size_t total = (size_t)nsam * nrow * nslice;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % nsam);
    const int y = (int)((q / nsam) % nrow);
    float v = q4[q].x;
    if (x > 0) v += q4[q - 1].y;
    if (y > 0) v += q4[q - nsam].z;
    if (x > 0 && y > 0) v += q4[q - nsam - 1].w;
    cube[q] = v;
  }
}

void pj_release(spi_ctx* c) {
  c->pj_vol.release();
  c->pj_out.release();
  c->pj_runs.release();
  c->pj_dm.release();
  c->pj_fbs.release();
  c->pj_v4.release();
  c->pj_rows.release();
  if (c->pjf_plan[0]) cufftDestroy(c->pjf_plan[0]);
  if (c->pjf_plan[1]) cufftDestroy(c->pjf_plan[1]);
  c->pjf_plan[0] = c->pjf_plan[1] = 0;
  c->pjf_n = 0;
}


int pj_common(spi_ctx* c, int nx, int ny, int nz, float ri, const float* angles, int nang, int* nruns_out,
              int* ntasks_out, bool z_order) {
  if (!c) return fail(kInvalid, "NULL context");
  if (nx < 4 || ny < 4 || nz < 4) return fail(kInvalid, "PJ 3Q: volume %dx%dx%d too small", nx, ny, nz);
  if (nang < 0 || (nang > 0 && !angles)) return fail(kInvalid, "PJ 3Q: bad angle list");
  if (!(ri > 0.0f)) return fail(kInvalid, "PJ 3Q: radius %g must be positive", (double)ri);
  SPI_CUDA(cudaSetDevice(c->device));
  const int ldpx = nx / 2 + 1, ldpy = ny / 2 + 1, ldpz = nz / 2 + 1;
  std::vector<PjRun> runs;
  prepcub(nx, ny, nz, ri, ldpx, ldpy, ldpz, runs);
  std::vector<PjDM> dms((size_t)std::max(nang, 1));
  for (int a = 0; a < nang; ++a)  // WPRO_N(PHI=reg3, THETA=reg2, PSI=reg1), writpro_n.f:214-216
    cang_pj(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], dms[a].d);
  // the runs twice: PREPCUB's (z, y) order, then (y, z) order (adjoint lanes, see pj_adjoint)
  std::vector<PjRun> both(runs);
  both.insert(both.end(), runs.begin(), runs.end());
  std::stable_sort(both.begin() + runs.size(), both.end(),
                   [](const PjRun& u, const PjRun& v) { return u.y != v.y ? u.y < v.y : u.z < v.z; });
  SPI_TRY(c->pj_runs.ensure(std::max<size_t>(1, both.size()) * sizeof(PjRun)));
  SPI_TRY(c->pj_dm.ensure(dms.size() * sizeof(PjDM)));
  if (!both.empty())
    SPI_CUDA(cudaMemcpyAsync(c->pj_runs.p, both.data(), both.size() * sizeof(PjRun), cudaMemcpyHostToDevice, c->stream));
  SPI_CUDA(cudaMemcpyAsync(c->pj_dm.p, dms.data(), dms.size() * sizeof(PjDM), cudaMemcpyHostToDevice, c->stream));
  std::vector<PjRun> rowruns;
  std::vector<std::array<int, 4>> tasks;
  row_tasks(runs, z_order, rowruns, tasks);
  static_assert(sizeof(std::array<int, 4>) == sizeof(int4), "row tasks are uploaded as int4");
  const size_t rbytes = rowruns.size() * sizeof(PjRun), toff = pj_tasks_offset((int)rowruns.size());
  SPI_TRY(c->pj_rows.ensure(toff + std::max<size_t>(1, tasks.size()) * sizeof(int4)));
  if (!rowruns.empty()) {
    SPI_CUDA(cudaMemcpyAsync(c->pj_rows.p, rowruns.data(), rbytes, cudaMemcpyHostToDevice, c->stream));
    SPI_CUDA(cudaMemcpyAsync(static_cast<char*>(c->pj_rows.p) + toff, tasks.data(), tasks.size() * sizeof(int4),
                             cudaMemcpyHostToDevice, c->stream));
  }
  *nruns_out = (int)runs.size();
  if (ntasks_out) *ntasks_out = (int)tasks.size();
  return 0;
}

// row-task view of pj_rows
static const int4* pj_tasks_of(const void* rows, int nruns) {
  return reinterpret_cast<const int4*>(static_cast<const char*>(rows) + pj_tasks_offset(nruns));
}

// Forward projection of vol (device, nx*ny*nz) into the zeroed out, in the
// given PjForm: packs the volume into packed (quads or cells), then the warp
// row-task kernel; the plain form runs one thread per run on vol.
static int pj_forward(spi_ctx* c, cudaStream_t st, const float* vol, int form, float4* packed, int nx, int ny, int nz,
                      const PjRun* runs, int nruns, const void* rows, int ntasks, const PjDM* dms, int nang,
                      float* out) {
  if (nruns == 0 || nang == 0) return 0;
  const size_t nvox = (size_t)nx * ny * nz;
  const int ldpx = nx / 2 + 1, ldpy = ny / 2 + 1, ldpz = nz / 2 + 1;
  if (form == kPjPlain) {
    const long long total = (long long)nruns * nang;
    const int blocks = (int)std::min<long long>((total + 127) / 128, (long long)c->sm_count * 16);
    wpro_kernel<<<blocks, 128, 0, st>>>(vol, nx, ny, nz, runs, nruns, dms, nang, ldpx, ldpy, ldpz, out);
    SPI_TRY(check_kernel("wpro_kernel"));
    c->count();
    return 0;
  }
  const int pblocks = (int)std::min<size_t>((nvox + 255) / 256, (size_t)c->sm_count * 16);
  if (form == kPjCells)
    pj_pack_cells_kernel<<<pblocks, 256, 0, st>>>(vol, nx, ny, nz, packed);
  else
    pj_pack4_kernel<<<pblocks, 256, 0, st>>>(vol, nx, ny, nz, packed);
  SPI_TRY(check_kernel("pj_pack_kernel"));
  const long long warps = (long long)ntasks * nang;
  const int blocks = (int)std::min<long long>((warps + 3) / 4, (long long)c->sm_count * 16);
  const PjRun* rr = static_cast<const PjRun*>(rows);
  const int4* tk = pj_tasks_of(rows, nruns);
  const int S = fwd_slabs(pj_packed_bytes(form, nvox));
  if (S == 1) {
    if (form == kPjCells)
      wpro_warp_kernel<kPjCells, false><<<blocks, 128, 0, st>>>(packed, nx, ny, nz, rr, tk, ntasks, dms, nang, ldpx,
                                                                ldpy, ldpz, 1, nz, out);
    else
      wpro_warp_kernel<kPjQuads, false><<<blocks, 128, 0, st>>>(packed, nx, ny, nz, rr, tk, ntasks, dms, nang, ldpx,
                                                                ldpy, ldpz, 1, nz, out);
    SPI_TRY(check_kernel("wpro_warp_kernel"));
    c->count(2);
    return 0;
  }
  // cells have IOZ = 1 .. nz-1; S slabs of T planes each
  const int T = (nz - 1 + S - 1) / S;
  for (int zlo = 1; zlo < nz; zlo += T) {
    const int zhi = std::min(nz, zlo + T);
    if (form == kPjCells)
      wpro_warp_kernel<kPjCells, true><<<blocks, 128, 0, st>>>(packed, nx, ny, nz, rr, tk, ntasks, dms, nang, ldpx,
                                                               ldpy, ldpz, zlo, zhi, out);
    else
      wpro_warp_kernel<kPjQuads, true><<<blocks, 128, 0, st>>>(packed, nx, ny, nz, rr, tk, ntasks, dms, nang, ldpx,
                                                               ldpy, ldpz, zlo, zhi, out);
    SPI_TRY(check_kernel("wpro_warp_kernel"));
    c->count();
  }
  c->count();
  return 0;
}

// Adjoint of projs (device, nang*nx*ny) into vol (device): with q4 (a quad
// accumulator of nx*ny*nz float4), wpro_adjoint4_kernel in z slabs of at most
// kSlabBytes of quads and the unfold; without, one thread per run with
// scalar atomics into vol.  Plans of 1,000 (192^3) and 500 (256^3)
// projections: 30.6k and 12.7k projections/s in slabs (2 and 5), against
// 13.1k and 5.6k with scalar atomics; at 128^3 one slab, 112k against 43k.
// Order of the runs among the adjoint's threads (SPI_PJ_ADJ_ORDER): 0 (z, y),
// 3 (y, z), 1 per projection the one whose neighbouring walks differ more
// in x, 2 per projection the one whose neighbouring walks differ less in z.
static int env_order() {
  const char* e = std::getenv("SPI_PJ_ADJ_ORDER");
  return e ? std::atoi(e) : 1;
}

static int pj_adjoint(spi_ctx* c, cudaStream_t st, const float* projs, float4* q4, int nx, int ny, int nz,
                      const PjRun* runs, int nruns, const PjDM* dms, int nang, float* vol) {
  const size_t nvox = (size_t)nx * ny * nz;
  const long long total = (long long)nruns * nang;
  const int blocks = (int)std::min<long long>((total + 127) / 128, (long long)c->sm_count * 16);
  const int ldpx = nx / 2 + 1, ldpy = ny / 2 + 1, ldpz = nz / 2 + 1;
  if (blocks == 0) {
    SPI_CUDA(cudaMemsetAsync(vol, 0, nvox * sizeof(float), st));
    return 0;
  }
  if (!q4) {
    SPI_CUDA(cudaMemsetAsync(vol, 0, nvox * sizeof(float), st));
    wpro_adjoint_kernel<<<blocks, 128, 0, st>>>(projs, nx, ny, nz, runs, nruns, dms, nang, ldpx, ldpy, ldpz, vol);
    SPI_TRY(check_kernel("wpro_adjoint_kernel"));
    c->count();
    return 0;
  }
  SPI_CUDA(cudaMemsetAsync(q4, 0, nvox * sizeof(float4), st));
  const int adj_order = env_order();
  // cells have IOZ = 1 .. nz-1; S slabs of T planes each
  const int S = (int)std::max<size_t>(1, (nvox * sizeof(float4) + kSlabBytes - 1) / kSlabBytes);
  const int T = (nz - 1 + S - 1) / S;
  for (int zlo = 1; zlo < nz; zlo += T) {
    wpro_adjoint4_kernel<<<blocks, 128, 0, st>>>(projs, nx, ny, nz, runs, nruns, dms, nang, ldpx, ldpy, ldpz, zlo,
                                                 std::min(nz, zlo + T), adj_order, q4);
    SPI_TRY(check_kernel("wpro_adjoint4_kernel"));
    c->count();
  }
  pj_unfold4_kernel<<<(int)std::min<size_t>((nvox + 255) / 256, (size_t)c->sm_count * 16), 256, 0, st>>>(q4, nx, ny,
                                                                                                       nz, vol);
  SPI_TRY(check_kernel("pj_unfold4_kernel"));
  c->count();
  return 0;
}

}  // namespace spi

using namespace spi;

extern "C" {

int spi_pj3q(spi_ctx* c, const float* vol, int nx, int ny, int nz, float ri, const float* angles, int nang,
             float* proj_out, int on_device) {
  int nruns = 0, ntasks = 0;
  const int form = pj_fwd_form((size_t)nx * ny * nz);
  const bool slabbed = form != kPjPlain && fwd_slabs(pj_packed_bytes(form, (size_t)nx * ny * nz)) > 1;
  SPI_TRY(pj_common(c, nx, ny, nz, ri, angles, nang, &nruns, &ntasks, slabbed));
  if (!vol || !proj_out) return fail(kInvalid, "PJ 3Q: NULL buffer");
  const size_t vbytes = (size_t)nx * ny * nz * sizeof(float);
  const size_t pbytes = (size_t)nang * nx * ny * sizeof(float);
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
  SPI_CUDA(cudaMemsetAsync(dout, 0, pbytes, c->stream));
  const size_t nvox = (size_t)nx * ny * nz;
  float4* packed = nullptr;
  if (nruns > 0 && form != kPjPlain) {
    SPI_TRY(c->pj_v4.ensure(pj_packed_bytes(form, nvox)));
    packed = c->pj_v4.as<float4>();
  }
  SPI_TRY(pj_forward(c, c->stream, dvol, form, packed, nx, ny, nz, c->pj_runs.as<PjRun>(), nruns, c->pj_rows.p, ntasks,
                     c->pj_dm.as<PjDM>(), nang, dout));
  if (!on_device) SPI_CUDA(cudaMemcpyAsync(proj_out, dout, pbytes, cudaMemcpyDeviceToHost, c->stream));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int spi_pj3q_adjoint(spi_ctx* c, const float* projs, int nx, int ny, int nz, float ri, const float* angles,
                     int nang, float* vol_out, int on_device) {
  int nruns = 0;
  SPI_TRY(pj_common(c, nx, ny, nz, ri, angles, nang, &nruns));
  if (!projs || !vol_out) return fail(kInvalid, "PJ 3Q adjoint: NULL buffer");
  const size_t vbytes = (size_t)nx * ny * nz * sizeof(float);
  const size_t pbytes = (size_t)nang * nx * ny * sizeof(float);
  const float* dp = projs;
  float* dvol = vol_out;
  if (!on_device) {
    SPI_TRY(c->pj_vol.ensure(vbytes));
    SPI_TRY(c->pj_out.ensure(std::max<size_t>(pbytes, 4)));
    if (pbytes) SPI_CUDA(cudaMemcpyAsync(c->pj_out.p, projs, pbytes, cudaMemcpyHostToDevice, c->stream));
    dp = c->pj_out.as<float>();
    dvol = c->pj_vol.as<float>();
  }
  const size_t nvox = (size_t)nx * ny * nz;
  float4* q4 = nullptr;
  if (nruns > 0 && nvox * sizeof(float4) <= quad_fwd_max()) {
    SPI_TRY(c->pj_v4.ensure(nvox * sizeof(float4)));
    q4 = c->pj_v4.as<float4>();
  }
  SPI_TRY(pj_adjoint(c, c->stream, dp, q4, nx, ny, nz, c->pj_runs.as<PjRun>(), nruns, c->pj_dm.as<PjDM>(), nang,
                     dvol));
  if (!on_device) SPI_CUDA(cudaMemcpyAsync(vol_out, dvol, vbytes, cudaMemcpyDeviceToHost, c->stream));
  SPI_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// ---------------------------------------------------------------------------
// PJ 3Q plans: the voxel runs (PREPCUB) and rotation matrices of one volume
// shape, radius and angle list, uploaded once; forward and adjoint are then
// pure launches on a caller stream (no allocation, no host synchronisation),
// so an iterative solver can capture them in a CUDA graph.
}  // extern "C"

struct spi_pj3q_plan {
  spi_ctx* ctx = nullptr;
  int device = 0, nx = 0, ny = 0, nz = 0, nang = 0, nruns = 0, ntasks = 0, form = 0;
  float ri = 0.0f;
  PjRun* runs = nullptr;  // 2 x nruns: (z, y) order, then (y, z) order
  void* rows = nullptr;   // runs in (y, |z|) order, then the row tasks (forward)
  PjDM* dms = nullptr;
  float4* v4 = nullptr;   // packed volume of the forward projection (quads or cells, by form)
  float4* q4 = nullptr;   // quad accumulator of the adjoint
};

extern "C" {

int spi_pj3q_plan_create(spi_ctx* c, int nx, int ny, int nz, float ri, const float* angles, int nang,
                         spi_pj3q_plan** out) {
  if (!out) return fail(kInvalid, "spi_pj3q_plan_create: out is NULL");
  *out = nullptr;
  if (nang <= 0) return fail(kInvalid, "spi_pj3q_plan_create: nang = %d", nang);
  int nruns = 0, ntasks = 0;
  const size_t nvox = (size_t)nx * ny * nz;
  const int form = pj_fwd_form(nvox);
  const bool slabbed = form != kPjPlain && fwd_slabs(pj_packed_bytes(form, nvox)) > 1;
  // runs, row tasks and matrices into the context's buffers
  SPI_TRY(pj_common(c, nx, ny, nz, ri, angles, nang, &nruns, &ntasks, slabbed));
  auto* p = new spi_pj3q_plan();
  p->ctx = c;
  p->device = c->device;
  p->nx = nx; p->ny = ny; p->nz = nz; p->nang = nang; p->nruns = nruns; p->ntasks = ntasks; p->ri = ri;
  const size_t rows_bytes = pj_tasks_offset(nruns) + std::max(1, ntasks) * sizeof(int4);
  cudaError_t e = cudaMalloc(&p->runs, std::max<size_t>(1, 2 * (size_t)nruns) * sizeof(PjRun));
  if (e == cudaSuccess) e = cudaMalloc(&p->dms, (size_t)nang * sizeof(PjDM));
  if (e == cudaSuccess) e = cudaMalloc(&p->rows, rows_bytes);
  p->form = nruns ? form : kPjPlain;
  if (e == cudaSuccess && p->form != kPjPlain) e = cudaMalloc(&p->v4, pj_packed_bytes(p->form, nvox));
  if (e == cudaSuccess && nruns && nvox * sizeof(float4) <= quad_fwd_max()) e = cudaMalloc(&p->q4, nvox * sizeof(float4));
  if (e == cudaSuccess && nruns)
    e = cudaMemcpyAsync(p->runs, c->pj_runs.p, 2 * (size_t)nruns * sizeof(PjRun), cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(p->dms, c->pj_dm.p, (size_t)nang * sizeof(PjDM), cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess && nruns)
    e = cudaMemcpyAsync(p->rows, c->pj_rows.p, rows_bytes, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    cudaFree(p->runs);
    cudaFree(p->rows);
    cudaFree(p->dms);
    cudaFree(p->v4);
    cudaFree(p->q4);
    delete p;
    return fail(kCuda, "spi_pj3q_plan_create: %s", cudaGetErrorString(e));
  }
  *out = p;
  return 0;
}

int spi_pj3q_plan_forward(const spi_pj3q_plan* p, const float* vol, float* proj_out, void* stream) {
  if (!p || !vol || !proj_out) return fail(kInvalid, "spi_pj3q_plan_forward: NULL argument");
  auto st = static_cast<cudaStream_t>(stream);
  SPI_CUDA(cudaMemsetAsync(proj_out, 0, (size_t)p->nang * p->nx * p->ny * sizeof(float), st));
  return pj_forward(p->ctx, st, vol, p->form, p->v4, p->nx, p->ny, p->nz, p->runs, p->nruns, p->rows, p->ntasks, p->dms,
                    p->nang, proj_out);
}

int spi_pj3q_plan_adjoint(const spi_pj3q_plan* p, const float* projs, float* vol_out, void* stream) {
  if (!p || !projs || !vol_out) return fail(kInvalid, "spi_pj3q_plan_adjoint: NULL argument");
  return pj_adjoint(p->ctx, static_cast<cudaStream_t>(stream), projs, p->q4, p->nx, p->ny, p->nz, p->runs, p->nruns,
                    p->dms, p->nang, vol_out);
}

int spi_pj3q_plan_destroy(spi_pj3q_plan* p) {
  if (!p) return 0;
  cudaSetDevice(p->device);
  cudaFree(p->runs);
  cudaFree(p->rows);
  cudaFree(p->dms);
  cudaFree(p->v4);
  cudaFree(p->q4);
  delete p;
  return 0;
}

}  // extern "C"

// ============================================================================
// PJ 3Q without any allocation.
//
// For callers that must not allocate device memory themselves or through a
// library: applications whose device memory is owned by a fixed arena or a
// caching allocator that must not be bypassed, and latency-critical pipelines
// that cannot absorb the implicit device synchronisation of cudaMalloc and
// cudaFree.  spi_pj3q keeps its voxel runs and rotation matrices in context
// buffers from cudaMalloc; this variant keeps them in one file-scope
// __device__ array of fixed size (kNoAllocBytes, held by every GPU that loads
// the library until the process exits) and takes all inputs and outputs as
// caller-owned device pointers.
namespace spi {

constexpr int kNoAllocMaxLines = 65536;  // ny * nz lines of voxels along x
constexpr int kNoAllocMaxAng = 16384;    // projections per call
struct NoAllocScratch {
  int2 lines[kNoAllocMaxLines];          // first/last x (1-based) of the sphere on each (y, z) line
  PjDM dms[kNoAllocMaxAng];              // rotation matrix per projection
};
constexpr size_t kNoAllocBytes = sizeof(NoAllocScratch);  // 1,114,112 bytes

static __device__ __align__(256) unsigned char g_pj3q_scratch[kNoAllocBytes];

// Device address of g_pj3q_scratch on the current device.  The host-side
// name is only a stand-in for the symbol, so the address is looked up on
// every call: the lookup allocates nothing, and a cached address would go
// stale if the device's primary context were released and the module loaded
// again at another address.
static int noalloc_scratch(NoAllocScratch** out) {
  int dev = -1;
  SPI_CUDA(cudaGetDevice(&dev));
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_pj3q_scratch);
  if (e != cudaSuccess || !p)
    return fail(kCuda, "spi_pj3q_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev, cudaGetErrorString(e));
  *out = static_cast<NoAllocScratch*>(p);
  return 0;
}

// CANG in FP64 on the device (WPRO_N's inline matrix, wpro_n.f:65-81), with
// the host's operation order and every product and sum rounded on its own
// (no fused multiply-add), as host_math.cpp evaluates it.  The matrices then
// equal spi_pj3q's unless the device's and the host's double cos/sin differ
// in a last bit that also changes the single-precision rounding.
__global__ void noalloc_dm_kernel(const float* __restrict__ angles, int nang, PjDM* __restrict__ dms) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nang) return;
  const double d2r = (double)3.14159265358979323846f / 180.0;
  const double psi = __dmul_rn((double)angles[3 * a], d2r), theta = __dmul_rn((double)angles[3 * a + 1], d2r),
               phi = __dmul_rn((double)angles[3 * a + 2], d2r);
  const double cphi = cos(phi), sphi = sin(phi), cthe = cos(theta), sthe = sin(theta), cpsi = cos(psi),
               spsi = sin(psi);
  float* d = dms[a].d;
  d[0] = (float)__dsub_rn(__dmul_rn(__dmul_rn(cphi, cthe), cpsi), __dmul_rn(sphi, spsi));
  d[1] = (float)__dadd_rn(__dmul_rn(__dmul_rn(sphi, cthe), cpsi), __dmul_rn(cphi, spsi));
  d[2] = (float)__dmul_rn(-sthe, cpsi);
  d[3] = (float)__dsub_rn(__dmul_rn(__dmul_rn(-cphi, cthe), spsi), __dmul_rn(sphi, cpsi));
  d[4] = (float)__dadd_rn(__dmul_rn(__dmul_rn(-sphi, cthe), spsi), __dmul_rn(cphi, cpsi));
  d[5] = (float)__dmul_rn(sthe, spsi);
  d[6] = (float)__dmul_rn(sthe, cphi);
  d[7] = (float)__dmul_rn(sthe, sphi);
  d[8] = (float)(cthe);
}

// PREPCUB's run of line (y, z): first and last x inside radius ri (x2 < x1 when empty)
__global__ void noalloc_lines_kernel(int nx, int ny, int nz, float ri, int ldpx, int ldpy, int ldpz,
                                     int2* __restrict__ lines) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= ny * nz) return;
  const int i2 = l % ny + 1, i1 = l / ny + 1;
  const float r = __fmul_rn(ri, ri);
  const float t = (float)(i1 - ldpz);
  const float xx = __fmul_rn(t, t);
  const float t2 = (float)(i2 - ldpy);
  const float yy = __fadd_rn(__fmul_rn(t2, t2), xx);
  int first = 0, last = -1;
  for (int i3 = 1; i3 <= nx; ++i3) {
    const float t3 = (float)(i3 - ldpx);
    const float rc = __fadd_rn(__fmul_rn(t3, t3), yy);
    if (rc <= r) {
      if (first == 0) first = i3;
      last = i3;
    }
  }
  lines[l] = make_int2(first, first ? last : -1);
}

// The WPRO_N walk of wpro_kernel, reading its runs and matrices from the
// scratch array; one thread per (projection, line).
__global__ void __launch_bounds__(128) noalloc_wpro_kernel(const float* __restrict__ cube, int nsam, int nrow,
                                                           int nslice, const NoAllocScratch* __restrict__ sc,
                                                           int nang, int ldpx, int ldpy, int ldpz,
                                                           float* __restrict__ out) {
  const int nlines = nrow * nslice;
  const long long total = (long long)nlines * nang;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t / nlines);
    const int l = (int)(t % nlines);
    const int2 run = sc->lines[l];
    if (run.y < run.x) continue;
    const PjRun r{run.x, run.y, run.x - ldpx, l % nrow + 1 - ldpy, l / nrow + 1 - ldpz};
    const PjDM dm = sc->dms[a];
    float* b = out + (size_t)a * nsam * nrow;
    const int k = r.y + ldpy;
    float xb = run_start(r, dm.d[0], dm.d[3], dm.d[6], ldpx);
    float yb = run_start(r, dm.d[1], dm.d[4], dm.d[7], ldpy);
    float zb = run_start(r, dm.d[2], dm.d[5], dm.d[8], ldpz);
    const size_t sy = (size_t)nsam, sz = (size_t)nsam * nrow;
    // the eight corner values of the current cell; a step moves the cell by
    // at most one voxel per axis, so the corners it shares are not reloaded
    int cx = -8, cy = -8, cz = -8;
    float cv[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};   // corner o = i + 2 j + 4 l
    for (int j = r.i1; j <= r.i2; ++j) {
      const int iox = __float2int_rz(xb), ioy = __float2int_rz(yb), ioz = __float2int_rz(zb);
      if (iox >= 1 && iox < nsam && ioy >= 1 && ioy < nrow && ioz >= 1 && ioz < nslice) {
        const float dx = __fsub_rn(xb, (float)iox), dy = __fsub_rn(yb, (float)ioy), dz = __fsub_rn(zb, (float)ioz);
        if (iox != cx || ioy != cy || ioz != cz) {
          const int mx = iox - cx, my = ioy - cy, mz = ioz - cz;
          const float* c0 = cube + (size_t)(ioz - 1) * sz + (size_t)(ioy - 1) * sy + (iox - 1);
          float nv[8];
#pragma unroll
          for (int o = 0; o < 8; ++o) {
            const int i = o & 1, jj = (o >> 1) & 1, l = o >> 2;
            const int oi = i + mx, oj = jj + my, ol = l + mz;
            const bool has = (unsigned)oi < 2u && (unsigned)oj < 2u && (unsigned)ol < 2u;
            nv[o] = has ? sel8(cv, oi + 2 * oj + 4 * ol) : __ldg(c0 + l * sz + jj * sy + i);
          }
#pragma unroll
          for (int o = 0; o < 8; ++o) cv[o] = nv[o];
          cx = iox; cy = ioy; cz = ioz;
        }
        const float c000 = cv[0], c100 = cv[1], c010 = cv[2], c110 = cv[3];
        const float c001 = cv[4], c101 = cv[5], c011 = cv[6], c111 = cv[7];
        const float a1 = c000;
        const float a2 = __fsub_rn(c100, a1);
        const float a3 = __fsub_rn(c010, a1);
        const float a4 = __fsub_rn(c001, a1);
        const float a5 = __fadd_rn(__fsub_rn(-a2, c010), c110);
        const float a61 = __fadd_rn(-c001, c101);
        const float a6 = __fadd_rn(-a2, a61);
        const float a7 = __fadd_rn(__fsub_rn(-a3, c001), c011);
        const float a8 = __fadd_rn(__fsub_rn(__fsub_rn(-a5, a61), c011), c111);
        const float inner = __fadd_rn(__fadd_rn(a4, __fmul_rn(a6, dx)), __fmul_rn(__fadd_rn(a7, __fmul_rn(a8, dx)), dy));
        float v = __fadd_rn(a1, __fmul_rn(dz, inner));
        v = __fadd_rn(v, __fmul_rn(a3, dy));
        v = __fadd_rn(v, __fmul_rn(dx, __fadd_rn(a2, __fmul_rn(a5, dy))));
        atomicAdd(b + (size_t)(k - 1) * nsam + (j - 1), v);
      }
      xb = __fadd_rn(xb, dm.d[0]);
      yb = __fadd_rn(yb, dm.d[1]);
      zb = __fadd_rn(zb, dm.d[2]);
    }
  }
}

}  // namespace spi

extern "C" int spi_pj3q_noalloc(const float* vol, int nx, int ny, int nz, float ri, const float* angles, int nang,
                                float* proj_out, void* stream) {
  using namespace spi;
  if (!vol || !proj_out || (nang > 0 && !angles)) return fail(kInvalid, "spi_pj3q_noalloc: NULL pointer");
  if (nx < 4 || ny < 4 || nz < 4) return fail(kInvalid, "spi_pj3q_noalloc: volume %dx%dx%d too small", nx, ny, nz);
  if ((long long)ny * nz > kNoAllocMaxLines)
    return fail(kInvalid, "spi_pj3q_noalloc: ny*nz = %lld exceeds the fixed scratch limit of %d lines",
                (long long)ny * nz, kNoAllocMaxLines);
  if (nang < 0 || nang > kNoAllocMaxAng)
    return fail(kInvalid, "spi_pj3q_noalloc: nang = %d exceeds the fixed scratch limit of %d projections", nang,
                kNoAllocMaxAng);
  if (!(ri > 0.0f)) return fail(kInvalid, "spi_pj3q_noalloc: radius %g must be positive", (double)ri);
  NoAllocScratch* sc = nullptr;
  SPI_TRY(noalloc_scratch(&sc));
  if (nang == 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int ldpx = nx / 2 + 1, ldpy = ny / 2 + 1, ldpz = nz / 2 + 1;
  noalloc_dm_kernel<<<(nang + 127) / 128, 128, 0, st>>>(angles, nang, sc->dms);
  SPI_TRY(check_kernel("noalloc_dm_kernel"));
  noalloc_lines_kernel<<<(ny * nz + 127) / 128, 128, 0, st>>>(nx, ny, nz, ri, ldpx, ldpy, ldpz, sc->lines);
  SPI_TRY(check_kernel("noalloc_lines_kernel"));
  SPI_CUDA(cudaMemsetAsync(proj_out, 0, (size_t)nang * nx * ny * sizeof(float), st));
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long total = (long long)ny * nz * nang;
  const int blocks = (int)std::min<long long>((total + 127) / 128, (long long)nsm * 16);
  noalloc_wpro_kernel<<<blocks, 128, 0, st>>>(vol, nx, ny, nz, sc, nang, ldpx, ldpy, ldpz, proj_out);
  SPI_TRY(check_kernel("noalloc_wpro_kernel"));
  return 0;
}
