// SPIDER reconstruction oracle -- TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement, in C++17 + OpenMP, of the Fortran routines of SPIDER's
// Fourier gridding back-projection (BP 3F / BP 32F), its trilinear projector
// (PJ 3Q) and its conjugate-gradient reconstruction (BP CG, linear mode).
// Every function names the reference file:line it restates.  Only the test
// suite, the smoke check and the CPU-baseline leg of the benchmark load this
// library; the product path never links, calls or falls back to it.
//
// Parity status: UNPINNED against outputs of the reference itself.  The
// reference is Fortran 77/90 + FFTW3 and neither gfortran nor libfftw3f exist
// on this machine, and the reference ships no golden volumes for this path
// (its KATs need the angle document `savangbprp`, absent from the tree).  The
// sub-functions are pinned to independent implementations instead: the
// Kaiser-Bessel table and the gridding-correction Bessel values against
// scipy.special, the FFT against numpy.fft, the Euler matrix against an
// independent rotation composition (tests/test_oracle_pins.py).
//
// Arithmetic rules (kept identical in the CUDA path so that every index,
// interpolation weight and table entry is bit-identical, and only the
// summation order of accumulations differs):
//   * coordinates, table indices and weights are IEEE float, evaluated left
//     to right without contraction (built with -ffp-contract=off);
//   * Fortran NINT = round half away from zero, IFIX = truncation;
//   * SPIDER's `QUADPI = 3.14159...` literals are default-REAL constants, so
//     pi enters the Euler-angle code rounded to single precision
//     (cang.f:62-63, wpro_n.f:62-63, hiang.f:45-46).
// The `prec` argument selects the accumulation type: 0 = REAL (FP32, the
// reference's storage types), 1 = DOUBLE (FP64 oracle).  FFTs are computed in
// double in both modes and rounded to the storage type.

#include <algorithm>
#include <cmath>
#include <climits>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

typedef std::complex<double> cd;

// pi as the reference's Euler-angle routines see it (single-precision literal)
const double QUADPI_F = (double)3.14159265358979323846f;

inline int nint_pos(float v) {            // Fortran NINT for v >= 0
  float f = std::floor(v);
  return (int)f + ((v - f) >= 0.5f ? 1 : 0);
}

inline int ifix(float v) { return (int)v; }   // truncation toward zero

// ---------------------------------------------------------------- FFT ------
// Mixed-radix recursive Cooley-Tukey in double (radices 2,3,4,5,7 and a
// generic DFT for any other prime).  sign = -1 forward (e^-i), +1 backward.
struct FFT1 {
  int n = 0;
  int sign = -1;
  std::vector<cd> w;  // w[j] = exp(sign*2*pi*i*j/n)
  std::vector<int> fac;
  FFT1() {}
  FFT1(int n_, int sign_) : n(n_), sign(sign_), w(n_) {
    for (int j = 0; j < n; ++j) {
      double a = 2.0 * M_PI * (double)j / (double)n * (double)sign;
      w[j] = cd(std::cos(a), std::sin(a));
    }
    int m = n;
    while (m > 1) {
      int p = 0;
      if (m % 4 == 0) p = 4;
      else if (m % 2 == 0) p = 2;
      else if (m % 3 == 0) p = 3;
      else if (m % 5 == 0) p = 5;
      else if (m % 7 == 0) p = 7;
      else { for (int q = 11; q <= m; q += 2) if (m % q == 0) { p = q; break; } }
      fac.push_back(p);
      m /= p;
    }
  }
  // out[k] = sum_j in[j*istride] w^(j k)
  void rec(const cd* in, int istride, cd* out, int len, int fi, int tstride, cd* tmp) const {
    if (len == 1) { out[0] = in[0]; return; }
    int p = fac[fi];
    int m = len / p;
    for (int q = 0; q < p; ++q)
      rec(in + q * istride, istride * p, out + q * m, m, fi + 1, tstride * p, tmp);
    // butterflies: X[k + r m] = sum_q w_len^{q (k + r m)} Y_q[k]
    for (int k = 0; k < m; ++k) {
      cd y[64];
      cd* yy = (p <= 64) ? y : tmp;
      for (int q = 0; q < p; ++q) {
        long e = (long)q * k * tstride % n;
        yy[q] = out[q * m + k] * w[e];
      }
      for (int r = 0; r < p; ++r) {
        cd s = 0;
        for (int q = 0; q < p; ++q) {
          long e = (long)q * r * m * tstride % n;
          s += yy[q] * w[e];
        }
        tmp[p + r] = s;   // staged to avoid clobbering yy
      }
      for (int r = 0; r < p; ++r) out[k + r * m] = tmp[p + r];
    }
  }
  void exec(const cd* in, int istride, cd* out) const {
    if ((n & (n - 1)) == 0) { pow2(in, istride, out); return; }
    std::vector<cd> tmp(2 * n + 130);
    rec(in, istride, out, n, 0, 1, tmp.data());
  }
  // iterative radix-2 decimation in time for power-of-two lengths
  void pow2(const cd* in, int istride, cd* out) const {
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int b = 0; b < lg; ++b) r |= ((i >> b) & 1) << (lg - 1 - b);
      out[r] = in[(size_t)i * istride];
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1, step = n / len;
      for (int i = 0; i < n; i += len)
        for (int k = 0; k < half; ++k) {
          cd t = out[i + k + half] * w[k * step];
          out[i + k + half] = out[i + k] - t;
          out[i + k] = out[i + k] + t;
        }
    }
  }
};

// ---------------------------------------------------- KB table (A4) -------
// FILLBESSIL, fillbessi0.f:88-125 (inline copy bp32f.f:193-214)
struct KBTable {
  float tab[5000];
  float fltb, alpha, aaaa;
  int ln2;
};

void fill_kb(int n2, KBTable& t) {
  const int ltab = 4999, ln = 5;
  t.ln2 = ln / 2;
  float v = (float)(ln - 1) / 2.0f / (float)n2;
  t.alpha = 6.5f;
  t.aaaa = 0.9f * v;
  float b0 = std::sqrt(t.alpha) * (float)std::cyl_bessel_i(1.0, (double)t.alpha);
  t.fltb = (float)ltab / (float)(t.ln2 + 1);
  for (int i = 0; i <= ltab; ++i) {
    float s = (float)i / t.fltb / (float)n2;
    if (s <= t.aaaa) {
      float q = s / t.aaaa;
      float xt = std::sqrt(1.0f - q * q);
      float ax = t.alpha * xt;
      t.tab[i] = std::sqrt(ax) * (float)std::cyl_bessel_i(1.0, (double)ax) / b0;
    } else {
      t.tab[i] = 0.0f;
    }
  }
}

// ---------------------------------------------------- Euler (A2) ----------
// CANG, cang.f:44-81
void cang(float phi, float theta, float psi, float* dm) {
  const double d2r = QUADPI_F / 180.0;
  double cphi = std::cos((double)phi * d2r), sphi = std::sin((double)phi * d2r);
  double cthe = std::cos((double)theta * d2r), sthe = std::sin((double)theta * d2r);
  double cpsi = std::cos((double)psi * d2r), spsi = std::sin((double)psi * d2r);
  dm[0] = (float)(cphi * cthe * cpsi - sphi * spsi);
  dm[1] = (float)(sphi * cthe * cpsi + cphi * spsi);
  dm[2] = (float)(-sthe * cpsi);
  dm[3] = (float)(-cphi * cthe * spsi - sphi * cpsi);
  dm[4] = (float)(-sphi * cthe * spsi + cphi * cpsi);
  dm[5] = (float)(sthe * spsi);
  dm[6] = (float)(sthe * cphi);
  dm[7] = (float)(sthe * sphi);
  dm[8] = (float)(cthe);
}

// DMS = MATMUL(SM, DM) of two column-major 3x3 REAL matrices (bp3f.f:460-466)
void matmul33(const float* sm, const float* dm, float* out) {
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      float s = sm[i] * dm[3 * j];
      s = s + sm[i + 3] * dm[1 + 3 * j];
      s = s + sm[i + 6] * dm[2 + 3 * j];
      out[i + 3 * j] = s;
    }
}

// ------------------------------------------------ Fourier grid ------------
template <class R>
struct Grid {
  int nx, n;
  std::vector<std::complex<R>> X;  // X[(k*n + j)*(nx+1) + i]
  std::vector<R> W;
  Grid(int nx_) : nx(nx_), n(2 * nx_), X((size_t)(nx_ + 1) * 4 * nx_ * nx_), W((size_t)(nx_ + 1) * 4 * nx_ * nx_) {}
  size_t idx(int i, int j, int k) const { return ((size_t)k * n + j) * (nx + 1) + i; }
};

// PADD2 + ASTA_D (bp3f.f:1307-1343, asta.f:61-92), FMRS_2 forward with the
// SPIDER sign (fftw3.f:409-419), phase (-1)^(I+J+1) (bp3f.f:453-458).
// Output bi[jrow*(nx+1) + i], jrow 0-based, i = 0..nx.
template <class R>
void stage_image(const float* proj, int nx, std::vector<std::complex<R>>& bi,
                 const FFT1& fx, const FFT1& fy, int nthreads = 1) {
  const int n = 2 * nx;
  // ASTA_D: mean of pixels outside radius L/2 (integer division, then REAL)
  float r = (float)(nx / 2);
  float rr = r * r;
  int nc = nx / 2 + 1;
  double aba = 0.0, klp = 0.0;
  for (int j = 1; j <= nx; ++j) {
    float t = (float)(j - nc);
    float xx = t * t;
    for (int i = 1; i <= nx; ++i) {
      float t2 = (float)(i - nc);
      if (xx + t2 * t2 > rr) { aba += (double)proj[(j - 1) * nx + (i - 1)]; klp += 1.0; }
    }
  }
  double qs = aba / (double)(float)klp;
  int ip = (n - nx) / 2 + nx % 2;
  std::vector<cd> img((size_t)n * n, cd(0, 0));
  for (int j = 1; j <= nx; ++j)
    for (int i = 1; i <= nx; ++i) {
      float v = (float)((double)proj[(j - 1) * nx + (i - 1)] - qs);
      img[(size_t)(ip + j - 1) * n + (ip + i - 1)] = cd(v, 0.0);
    }
  // 2D forward FFT: rows (x) then columns (y); threads as FFTW's plan uses
  bi.assign((size_t)(nx + 1) * n, std::complex<R>(0, 0));
  #pragma omp parallel num_threads(nthreads)
  {
  std::vector<cd> row(n), col(n);
  #pragma omp for schedule(static)
  for (int y = 0; y < n; ++y) {
    if (y < ip || y >= ip + nx) continue;  // zero-padding rows transform to zero
    fx.exec(&img[(size_t)y * n], 1, row.data());
    for (int x = 0; x < n; ++x) img[(size_t)y * n + x] = row[x];
  }
  #pragma omp for schedule(static)
  for (int x = 0; x <= nx; ++x) {
    fy.exec(&img[x], n, col.data());
    for (int y = 0; y < n; ++y) {
      // SPIDER sign: negate imaginary part; store in REAL or DOUBLE
      std::complex<R> v((R)col[y].real(), (R)(-col[y].imag()));
      // (-1)**(I+J+1) with J 1-based == (-1)**(i+y) with y 0-based
      if (((x + y) & 1) != 0) v = -v;
      bi[(size_t)y * (nx + 1) + x] = v;
    }
  }
  }
}

// QUADRI (quadri.f:83-150): quadratic interpolation with circular closure.
// f is FDATA(NX,NY) column-major (x fastest); x, y are 1-based.
float quadri(float xx, float yy, int nx, int ny, const float* f) {
  float x = xx, y = yy;
  if (x < 1.0f) x = x + (float)((1 - ifix(x) / nx) * nx);
  if (x > (float)nx + 0.5f) x = std::fmod(x - 1.0f, (float)nx) + 1.0f;
  if (y < 1.0f) y = y + (float)((1 - ifix(y) / ny) * ny);
  if (y > (float)ny + 0.5f) y = std::fmod(y - 1.0f, (float)ny) + 1.0f;
  const int i = ifix(x), j = ifix(y);
  const float dx0 = x - (float)i, dy0 = y - (float)j;
  int ip1 = i + 1, im1 = i - 1, jp1 = j + 1, jm1 = j - 1;
  if (ip1 > nx) ip1 -= nx;
  if (im1 < 1) im1 += nx;
  if (jp1 > ny) jp1 -= ny;
  if (jm1 < 1) jm1 += ny;
  auto F = [&](int a, int b) { return f[(size_t)(b - 1) * nx + (a - 1)]; };
  const float f0 = F(i, j);
  const float c1 = F(ip1, j) - f0;
  const float c2 = (c1 - f0 + F(im1, j)) * 0.5f;
  const float c3 = F(i, jp1) - f0;
  const float c4 = (c3 - f0 + F(i, jm1)) * 0.5f;
  const float dxb = dx0 - 1.0f, dyb = dy0 - 1.0f;
  const float hxc = (float)(int)std::copysign(1.0f, dx0);   // HXC, HYC are REAL
  const float hyc = (float)(int)std::copysign(1.0f, dy0);
  int ic = (int)((float)i + hxc), jc = (int)((float)j + hyc);
  if (ic > nx) ic -= nx; else if (ic < 1) ic += nx;
  if (jc > ny) jc -= ny; else if (jc < 1) jc += ny;
  const float c5 = ((F(ic, jc) - f0 - hxc * c1 - (hxc * (hxc - 1.0f)) * c2 - hyc * c3 - (hyc * (hyc - 1.0f)) * c4) *
                    (hxc * hyc));
  return f0 + dx0 * (c1 + dxb * c2 + dy0 * c5) + dy0 * (c3 + dyb * c4);
}

// RTSQ (rtsq.f:56-140): rotate by THETA degrees (SCLI = 1) and shift, with
// QUADRI interpolation; cod/sid are COS/SIN(THETA*DGR_TO_RAD) in REAL.
void rtsq(const float* in, float* out, int nx, int ny, float theta, float shxi, float shyi) {
  const float quadpi = 3.14159265358979323846f;
  const float dgr_to_rad = quadpi / 180.0f;
  const float shx = std::fmod(shxi, (float)nx), shy = std::fmod(shyi, (float)ny);
  const int iycen = ny / 2 + 1, ixcen = nx / 2 + 1;
  float rx1 = (float)(-nx / 2), rx2 = (float)(nx / 2), ry1 = (float)(-ny / 2), ry2 = (float)(ny / 2);
  float rxe1, rxe2, rye1, rye2;
  if (nx % 2 == 0) { rx2 = rx2 - 1.0f; rxe1 = (float)-nx; rxe2 = (float)nx; }
  else { rxe1 = (float)(-nx - 1); rxe2 = (float)(nx + 1); }
  if (ny % 2 == 0) { ry2 = ry2 - 1.0f; rye1 = (float)-ny; rye2 = (float)ny; }
  else { rye1 = (float)(-ny - 1); rye2 = (float)(ny + 1); }
  const float cod = std::cos(theta * dgr_to_rad), sid = std::sin(theta * dgr_to_rad);
  const float coddscli = cod / 1.0f, siddscli = sid / 1.0f;
  const float fixcenmshx = (float)(-ixcen) - shx, fiycenmshy = (float)(-iycen) - shy;
  for (int iy = 1; iy <= ny; ++iy) {
    float yi = (float)iy + fiycenmshy;
    if (yi < ry1) yi = std::min(yi + rye2, ry2);
    if (yi > ry2) yi = std::max(yi + rye1, ry1);
    const float ycod = yi * coddscli + (float)iycen;
    const float ysid = -yi * siddscli + (float)ixcen;
    for (int ix = 1; ix <= nx; ++ix) {
      float xi = (float)ix + fixcenmshx;
      if (xi < rx1) xi = std::min(xi + rxe2, rx2);
      if (xi > rx2) xi = std::max(xi + rxe1, rx1);
      const float yold = xi * siddscli + ycod;
      const float xold = xi * coddscli + ysid;
      out[(size_t)(iy - 1) * nx + (ix - 1)] = quadri(xold, yold, nx, ny, in);
    }
  }
}

// ONELINE, oneline.f:38-200 (called as ONELINE(J,N2,NX,...), bp3f.f:477:
// callee N = 2*NX, callee N2 = NX)
//
// zlo/zhi: only taps whose signed z index (izp for the main taps, -izp for
// the reflected ones; -NX < z < NX) lies in [zlo, zhi) are applied -- the
// owner-computes schedule of insert_images_owned.  The defaults apply all.
template <class R>
void oneline(int J, Grid<R>& g, const std::complex<R>* bi, const float* dm, const KBTable& kb,
             int zlo = INT_MIN, int zhi = INT_MAX) {
  const int N = g.n, N2 = g.nx, LN2 = kb.ln2;
  const int JP = (J >= 0) ? J : N + J;
  const float fltb = kb.fltb;
  for (int I = 0; I <= N2; ++I) {
    if (!((I * I + J * J) < (N * N / 4) && !(I == 0 && J < 0))) continue;
    float xnew = (float)I * dm[0] + (float)J * dm[3];
    float ynew = (float)I * dm[1] + (float)J * dm[4];
    float znew = (float)I * dm[2] + (float)J * dm[5];
    std::complex<R> btq;
    if (xnew < 0.0f) {
      xnew = -xnew; ynew = -ynew; znew = -znew;
      btq = std::conj(bi[(size_t)JP * (N2 + 1) + I]);
    } else {
      btq = bi[(size_t)JP * (N2 + 1) + I];
    }
    int ixn = ifix((xnew + 0.5f) + (float)N) - N;
    int iyn = ifix((ynew + 0.5f) + (float)N) - N;
    int izn = ifix((znew + 0.5f) + (float)N) - N;
    if (!(ixn <= (N2 - LN2 - 1) && iyn >= (-N2 + 2 + LN2) && iyn <= (N2 - LN2 - 1) &&
          izn >= (-N2 + 2 + LN2) && izn <= (N2 - LN2 - 1)))
      continue;
    // none of this pixel's taps lands in the owned z range
    if (!(izn + LN2 >= zlo && izn - LN2 < zhi) && !(ixn < LN2 && -izn + LN2 >= zlo && -izn - LN2 < zhi))
      continue;
    if (ixn >= 0) {
      int lb = -std::min(ixn, LN2);
      for (int lz = -LN2; lz <= LN2; ++lz) {
        int izp = izn + lz;
        if (izp < zlo || izp >= zhi) continue;
        int iza = (izp >= 0) ? izp : N + izp;
        float tz = kb.tab[nint_pos(std::fabs(znew - (float)izp) * fltb)];
        if (tz == 0.0f) continue;
        for (int ly = -LN2; ly <= LN2; ++ly) {
          int iyp = iyn + ly;
          int iya = (iyp >= 0) ? iyp : N + iyp;
          float ty = kb.tab[nint_pos(std::fabs(ynew - (float)iyp) * fltb)] * tz;
          if (ty == 0.0f) continue;
          for (int ixp = lb + ixn; ixp <= LN2 + ixn; ++ixp) {
            float wg = kb.tab[nint_pos(std::fabs(xnew - (float)ixp) * fltb)] * ty;
            if (wg != 0.0f) {
              size_t q = g.idx(ixp, iya, iza);
              g.X[q] += btq * (R)wg;
              g.W[q] += (R)wg;
            }
          }
        }
      }
    }
    if (ixn < LN2) {  // reflected points, oneline.f:118-150
      for (int lz = -LN2; lz <= LN2; ++lz) {
        int izp = izn + lz;
        if (-izp < zlo || -izp >= zhi) continue;
        int izt = (izp > 0) ? N - izp : -izp;
        float tz = kb.tab[nint_pos(std::fabs(znew - (float)izp) * fltb)];
        if (tz == 0.0f) continue;
        for (int ly = -LN2; ly <= LN2; ++ly) {
          int iyp = iyn + ly;
          int iyt = (iyp > 0) ? N - iyp : -iyp;
          float ty = kb.tab[nint_pos(std::fabs(ynew - (float)iyp) * fltb)] * tz;
          if (ty == 0.0f) continue;
          for (int ixp = ixn - LN2; ixp <= -1; ++ixp) {
            float wg = kb.tab[nint_pos(std::fabs(xnew - (float)ixp) * fltb)] * ty;
            if (wg != 0.0f) {
              size_t q = g.idx(-ixp, iyt, izt);
              g.X[q] += std::conj(btq) * (R)wg;
              g.W[q] += (R)wg;
            }
          }
        }
      }
    }
  }
}

// SYMPLANE0, bp32f.f:1051-1088 (called as SYMPLANE0(X,W,NX,N2): callee
// N2 = NX, callee N = 2*NX).  1-based IYA/IZA mapped to 0-based a-1.
template <class R>
void symplane0(Grid<R>& g) {
  const int N2 = g.nx, N = g.n;
  auto X = [&](int a, int b) -> std::complex<R>& { return g.X[g.idx(0, a - 1, b - 1)]; };
  auto W = [&](int a, int b) -> R& { return g.W[g.idx(0, a - 1, b - 1)]; };
  for (int iza = 2; iza <= N2; ++iza)
    for (int iya = 2; iya <= N2; ++iya) {
      X(iya, iza) = X(iya, iza) + std::conj(X(N - iya + 2, N - iza + 2));
      W(iya, iza) = W(iya, iza) + W(N - iya + 2, N - iza + 2);
      X(N - iya + 2, N - iza + 2) = std::conj(X(iya, iza));
      W(N - iya + 2, N - iza + 2) = W(iya, iza);
      X(N - iya + 2, iza) = X(N - iya + 2, iza) + std::conj(X(iya, N - iza + 2));
      W(N - iya + 2, iza) = W(N - iya + 2, iza) + W(iya, N - iza + 2);
      X(iya, N - iza + 2) = std::conj(X(N - iya + 2, iza));
      W(iya, N - iza + 2) = W(N - iya + 2, iza);
    }
  for (int iya = 2; iya <= N2; ++iya) {
    X(iya, 1) = X(iya, 1) + std::conj(X(N - iya + 2, 1));
    W(iya, 1) = W(iya, 1) + W(N - iya + 2, 1);
    X(N - iya + 2, 1) = std::conj(X(iya, 1));
    W(N - iya + 2, 1) = W(iya, 1);
  }
  for (int iza = 2; iza <= N2; ++iza) {
    X(1, iza) = X(1, iza) + std::conj(X(1, N - iza + 2));
    W(1, iza) = W(1, iza) + W(1, N - iza + 2);
    X(1, N - iza + 2) = std::conj(X(1, iza));
    W(1, N - iza + 2) = W(1, iza);
  }
}

// Gridding-correction radial table: WKB as a function of the integer squared
// radius LR (WINDKB2A, bp32f.f:964-1005).  nu = NNN/2 = 1.5.  I_nu(x)/x^nu and
// J_nu(x)/x^nu from their power series (exact mathematics of RIBSL/RJBSL,
// besi1.f:276-1239, at order 3/2).
double inu_over_xnu(double x, double nu) {   // I_nu(x)/x^nu
  double q = x * x / 4.0, term = 1.0 / std::tgamma(nu + 1.0), s = term;
  for (int k = 1; k < 200; ++k) { term *= q / ((double)k * (nu + k)); s += term; if (term < 1e-18 * s) break; }
  return s / std::pow(2.0, nu);
}
double jnu_over_xnu(double x, double nu) {   // J_nu(x)/x^nu
  double q = -x * x / 4.0, term = 1.0 / std::tgamma(nu + 1.0), s = term;
  for (int k = 1; k < 400; ++k) { term *= q / ((double)k * (nu + k)); s += term; if (std::fabs(term) < 1e-18 * std::fabs(s)) break; }
  return s / std::pow(2.0, nu);
}

void windkb_table(int nx, const KBTable& kb, std::vector<float>& wkb) {
  const float quadpi = 3.14159265358979323846f;
  const float twopi = 2.0f * quadpi;
  int l2 = (nx / 2) * (nx / 2);
  const double xnu = 1.5;
  const float alpha = kb.alpha;
  double wkb0 = std::pow((double)alpha, xnu) / (inu_over_xnu(alpha, xnu) * std::pow((double)alpha, xnu));
  float qrt = (twopi * kb.aaaa) * (twopi * kb.aaaa);
  wkb.assign(l2 + 1, 1.0f);
  for (int lr = 0; lr <= l2; ++lr) {
    float sigma = qrt * (float)lr - alpha * alpha;
    double w;
    if (std::fabs(sigma) < 1.0e-7f) w = 1.0;
    else if (sigma > 0.0f) w = wkb0 * jnu_over_xnu(std::sqrt((double)sigma), xnu);
    else w = wkb0 * inu_over_xnu(std::sqrt((double)std::fabs(sigma)), xnu);
    wkb[lr] = (float)std::fabs(w);
  }
}

// NRMW2 (bp3f.f:1347-1371) + FMRS_3 inverse (fftw3.f:426-449) + WINDKB2A
// (bp32f.f:945-1045).  Consumes the grid; writes vol (nx^3, x fastest).
template <class R>
void finish_volume(Grid<R>& g, const KBTable& kb, float* vol) {
  const int nx = g.nx, n = g.n, h = nx + 1;
  // NRMW2: X = X * (-1)**(I+J+K) / W  if W > 0.1 else 0   (J,K 1-based)
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i <= nx; ++i) {
        size_t q = g.idx(i, j, k);
        if (g.W[q] > (R)0.1f) {
          std::complex<R> v = g.X[q];
          if (((i + j + k) & 1) != 0) v = -v;
          g.X[q] = std::complex<R>(v.real() / g.W[q], v.imag() / g.W[q]);
        } else {
          g.X[q] = std::complex<R>(0, 0);
        }
      }
  // inverse: SPIDER sign (negate Im), c2c along z and y, c2r along x
  FFT1 fb(n, +1);
  std::vector<cd> G((size_t)h * n * n);
  #pragma omp parallel
  {
    std::vector<cd> line(n), out(n);
    #pragma omp for collapse(2)
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i <= nx; ++i) {
          std::complex<R> v = g.X[g.idx(i, j, k)];
          G[((size_t)k * n + j) * h + i] = cd((double)v.real(), -(double)v.imag());
        }
    #pragma omp for collapse(2)
    for (int k = 0; k < n; ++k)
      for (int i = 0; i <= nx; ++i) {
        for (int j = 0; j < n; ++j) line[j] = G[((size_t)k * n + j) * h + i];
        fb.exec(line.data(), 1, out.data());
        for (int j = 0; j < n; ++j) G[((size_t)k * n + j) * h + i] = out[j];
      }
    #pragma omp for collapse(2)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i <= nx; ++i) {
        for (int k = 0; k < n; ++k) line[k] = G[((size_t)k * n + j) * h + i];
        fb.exec(line.data(), 1, out.data());
        for (int k = 0; k < n; ++k) G[((size_t)k * n + j) * h + i] = out[k];
      }
  }
  // c2r along x: only the crop [ip, ip+nx) in every dimension is needed
  const int ip = (n - nx) / 2 + nx % 2;  // WINDKB2A IP (0-based start of crop)
  const R pix = (sizeof(R) == 4) ? (R)(1.0f / (float)((long)n * n * n)) : (R)(1.0 / ((double)n * n * n));
  std::vector<R> crop((size_t)nx * nx * nx);
  #pragma omp parallel
  {
    std::vector<cd> line(n), out(n);
    #pragma omp for collapse(2)
    for (int k = 0; k < nx; ++k)
      for (int j = 0; j < nx; ++j) {
        const cd* gr = &G[((size_t)(ip + k) * n + (ip + j)) * h];
        line[0] = cd(gr[0].real(), 0.0);
        line[nx] = cd(gr[nx].real(), 0.0);
        for (int i = 1; i < nx; ++i) { line[i] = gr[i]; line[n - i] = std::conj(gr[i]); }
        fb.exec(line.data(), 1, out.data());
        for (int i = 0; i < nx; ++i) {
          R v = (R)out[ip + i].real();
          crop[((size_t)k * nx + j) * nx + i] = v * pix;
        }
      }
  }
  // WINDKB2A: divide by |WKB(LR)|, shell mean, subtract, mask
  std::vector<float> wkb;
  windkb_table(nx, kb, wkb);
  const int l2 = (nx / 2) * (nx / 2), l2p = (nx / 2 - 1) * (nx / 2 - 1), c = nx / 2 + 1;
  R tnr = 0;
  long m = 0;
  for (int k = 1; k <= nx; ++k)
    for (int j = 1; j <= nx; ++j)
      for (int i = 1; i <= nx; ++i) {
        int lr = (k - c) * (k - c) + (j - c) * (j - c) + (i - c) * (i - c);
        if (lr <= l2) {
          R& v = crop[((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1)];
          v = v / (R)wkb[lr];
          if (lr >= l2p) { tnr += v; ++m; }
        }
      }
  tnr = tnr / (R)(float)m;
  for (int k = 1; k <= nx; ++k)
    for (int j = 1; j <= nx; ++j)
      for (int i = 1; i <= nx; ++i) {
        int lr = (k - c) * (k - c) + (j - c) * (j - c) + (i - c) * (i - c);
        size_t q = ((size_t)(k - 1) * nx + (j - 1)) * nx + (i - 1);
        vol[q] = (lr <= l2) ? (float)(crop[q] - tnr) : 0.0f;
      }
}

// TRIQUAD (triquad.f): triquadratic interpolation on a 3x3x3 neighbourhood.
// r, s, t are DOUBLE; the products and the 27-term sum are REAL, left to right.
float triquad(double r, double s, double t, const float* f) {
  const float c2 = 1.0f / 2.0f, c4 = 1.0f / 4.0f, c8 = 1.0f / 8.0f;
  const float rs = (float)(r * s), st = (float)(s * t), rt = (float)(r * t);
  const float rst = (float)(r * (double)st);
  const float rsq = (float)(1.0 - r * r), ssq = (float)(1.0 - s * s), tsq = (float)(1.0 - t * t);
  const float rm1 = (float)(1.0 - r), sm1 = (float)(1.0 - s), tm1 = (float)(1.0 - t);
  const float rp1 = (float)(1.0 + r), sp1 = (float)(1.0 + s), tp1 = (float)(1.0 + t);
  const float R = (float)r, S = (float)s, T = (float)t;
  float v = (-c8) * rst * rm1 * sm1 * tm1 * f[0];
  v = v + (c4) * st * rsq * sm1 * tm1 * f[1];
  v = v + (c8) * rst * rp1 * sm1 * tm1 * f[2];
  v = v + (c4) * rt * rm1 * ssq * tm1 * f[3];
  v = v + (-c2) * T * rsq * ssq * tm1 * f[4];
  v = v + (-c4) * rt * rp1 * ssq * tm1 * f[5];
  v = v + (c8) * rst * rm1 * sp1 * tm1 * f[6];
  v = v + (-c4) * st * rsq * sp1 * tm1 * f[7];
  v = v + (-c8) * rst * rp1 * sp1 * tm1 * f[8];
  v = v + (c4) * rs * rm1 * sm1 * tsq * f[9];
  v = v + (-c2) * S * rsq * sm1 * tsq * f[10];
  v = v + (-c4) * rs * rp1 * sm1 * tsq * f[11];
  v = v + (-c2) * R * rm1 * ssq * tsq * f[12];
  v = v + rsq * ssq * tsq * f[13];
  v = v + (c2) * R * rp1 * ssq * tsq * f[14];
  v = v + (-c4) * rs * rm1 * sp1 * tsq * f[15];
  v = v + (c2) * S * rsq * sp1 * tsq * f[16];
  v = v + (c4) * rs * rp1 * sp1 * tsq * f[17];
  v = v + (c8) * rst * rm1 * sm1 * tp1 * f[18];
  v = v + (-c4) * st * rsq * sm1 * tp1 * f[19];
  v = v + (-c8) * rst * rp1 * sm1 * tp1 * f[20];
  v = v + (-c4) * rt * rm1 * ssq * tp1 * f[21];
  v = v + (c2) * T * rsq * ssq * tp1 * f[22];
  v = v + (c4) * rt * rp1 * ssq * tp1 * f[23];
  v = v + (-c8) * rst * rm1 * sp1 * tp1 * f[24];
  v = v + (c4) * st * rsq * sp1 * tp1 * f[25];
  v = v + (c8) * rst * rp1 * sp1 * tp1 * f[26];
  return v;
}

// SYMVOL, SP_MP branch (symvol.f:39-180): q2 = sum over symmetries of q1
// rotated by RM (column-major 3x3 per symmetry) with TRIQDF inside radius
// sqrt(IRADI), q1 itself outside.  Volumes nx^3, x fastest; coordinates are
// centred (KLX = -nx/2 .. KNX).
void symvol(const float* q1, float* q2, int nx, const float* rm, int nsym) {
  const int klx = -nx / 2, knx = (nx % 2 == 0) ? nx / 2 - 1 : nx / 2;
  const int mn = std::min(std::abs(klx), std::abs(knx));
  const int iradi = (mn - 1) * (mn - 1);
  auto Q1 = [&](int ix, int iy, int iz) { return q1[((size_t)(iz - klx) * nx + (iy - klx)) * nx + (ix - klx)]; };
  const size_t nv = (size_t)nx * nx * nx;
  std::fill(q2, q2 + nv, 0.0f);
  for (int is = 0; is < nsym; ++is) {
    const float* R = rm + 9 * is;   // RM(i,j) = R[(i-1) + 3(j-1)]
    const bool ident = R[0] == 1.0f && R[4] == 1.0f && R[8] == 1.0f;
    for (int iz = klx; iz <= knx; ++iz)
      for (int iy = klx; iy <= knx; ++iy) {
        const double qrt0 = (double)(R[1] * (float)iy + R[2] * (float)iz);
        const double qrt1 = (double)(R[4] * (float)iy + R[5] * (float)iz);
        const double qrt2 = (double)(R[7] * (float)iy + R[8] * (float)iz);
        for (int ix = klx; ix <= knx; ++ix) {
          float& o = q2[((size_t)(iz - klx) * nx + (iy - klx)) * nx + (ix - klx)];
          if (ident) { o = o + Q1(ix, iy, iz); continue; }
          const int icrd = ix * ix + iy * iy + iz * iz;
          if (icrd <= iradi) {
            const double qr0 = qrt0 + (double)(R[0] * (float)ix);
            const double qr1 = qrt1 + (double)(R[3] * (float)ix);
            const double qr2 = qrt2 + (double)(R[6] * (float)ix);
            const int iox = (int)std::floor(qr0), ioy = (int)std::floor(qr1), ioz = (int)std::floor(qr2);
            const double dx = qr0 - iox, dy = qr1 - ioy, dz = qr2 - ioz;
            float f[27];
            for (int l = 0; l < 27; ++l) {
              const int X = l % 3 - 1, Y = (l / 3) % 3 - 1, Z = l / 9 - 1;
              f[l] = Q1(iox + X, ioy + Y, ioz + Z);
            }
            o = o + triquad(dx, dy, dz, f);
          } else {
            o = o + Q1(ix, iy, iz);
          }
        }
      }
  }
}

// BP3FQ image loop (bp3f.f:298-515) / BP32FQ (bp32f.f:433-939): every image
// is staged and inserted row by row into grid `route[img]`, rows striped by
// LN1 = 6 under OpenMP exactly like the reference's SP_MP build.
template <class R>
void insert_images(std::vector<Grid<R>*>& grids, const float* imgs, int nx, int nang,
                   const float* dm9, const float* sm9, int nsym, const uint8_t* route,
                   const KBTable& kb, int nthreads) {
  const int n = 2 * nx;
  FFT1 fx(n, -1), fy(n, -1);
  std::vector<std::complex<R>> bi;
  for (int a = 0; a < nang; ++a) {
    stage_image<R>(imgs + (size_t)a * nx * nx, nx, bi, fx, fy, nthreads);
    Grid<R>& g = *grids[route ? route[a] : 0];
    for (int is = 0; is < std::max(1, nsym); ++is) {
      float dms[9];
      if (nsym > 1) matmul33(sm9 + 9 * is, dm9 + 9 * a, dms);
      else std::memcpy(dms, dm9 + 9 * a, sizeof(dms));
      // The reference's schedule (bp3f.f:397-398, 469-471): rows J of one
      // group, LN1 = 6 apart, run in parallel.  It is not race-free: a group
      // with J = 0 or 3 (mod 6) holds rows J and -J, which write the same
      // Friedel-mirrored voxels, and oblique rows 6 apart can share taps, so
      // with more than one thread updates are lost (rel-l2 ~1e-4 at 128^3,
      // varying run to run).  The checker runs it with one thread or uses
      // insert_images_owned; the threaded form is the timed CPU baseline.
      const int ln1 = 6;
      for (int jt = 1; jt <= ln1; ++jt) {
        #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
        for (int J = -nx + jt; J <= nx; J += ln1) oneline<R>(J, g, bi.data(), dms, kb);
      }
    }
  }
}

// Race-free parallel form of the same image loop (owner computes).  Thread t
// of T owns a contiguous range of signed z planes, balanced by the expected
// tap density of central sections (proportional to NX - |z|), and walks every
// image, symmetry and row in the serial order, applying only the taps that
// land in its planes.  Each voxel therefore receives exactly the additions of
// the one-thread loop, in the same order: the grids are bit-identical to the
// serial result for any thread count.  Images are staged (PADD2 + FFT) in
// parallel batches first.
template <class R>
void insert_images_owned(std::vector<Grid<R>*>& grids, const float* imgs, int nx, int nang,
                         const float* dm9, const float* sm9, int nsym, const uint8_t* route,
                         const KBTable& kb, int nthreads) {
  const int n = 2 * nx;
  FFT1 fx(n, -1), fy(n, -1);
  const int T = std::max(1, nthreads);
  // z ranges: signed z runs over [-nx+1, nx-1]
  std::vector<int> zb(T + 1);
  {
    double tot = 0.0;
    for (int z = -nx + 1; z <= nx - 1; ++z) tot += (double)(nx - std::abs(z));
    double acc = 0.0;
    int t = 1;
    zb[0] = -nx + 1;
    for (int z = -nx + 1; z <= nx - 1 && t < T; ++z) {
      acc += (double)(nx - std::abs(z));
      while (t < T && acc >= tot * t / T) zb[t++] = z + 1;
    }
    while (t < T) zb[t++] = nx;
    zb[T] = nx;
  }
  const size_t spec = (size_t)(nx + 1) * n;
  const int batch = (int)std::max<size_t>(1, std::min<size_t>((size_t)nang,
                                                               ((size_t)512 << 20) / (spec * sizeof(std::complex<R>))));
  std::vector<std::vector<std::complex<R>>> bis(batch);
  const int ln1 = 6;
  for (int a0 = 0; a0 < nang; a0 += batch) {
    const int nb = std::min(batch, nang - a0);
    #pragma omp parallel for num_threads(T) schedule(dynamic, 1)
    for (int b = 0; b < nb; ++b) stage_image<R>(imgs + (size_t)(a0 + b) * nx * nx, nx, bis[b], fx, fy, 1);
    #pragma omp parallel num_threads(T)
    {
      const int t = omp_get_thread_num();
      const int zlo = zb[t], zhi = zb[t + 1];
      for (int b = 0; b < nb; ++b) {
        const int a = a0 + b;
        Grid<R>& g = *grids[route ? route[a] : 0];
        for (int is = 0; is < std::max(1, nsym); ++is) {
          float dms[9];
          if (nsym > 1) matmul33(sm9 + 9 * is, dm9 + 9 * a, dms);
          else std::memcpy(dms, dm9 + 9 * a, sizeof(dms));
          for (int jt = 1; jt <= ln1; ++jt)
            for (int J = -nx + jt; J <= nx; J += ln1) oneline<R>(J, g, bis[b].data(), dms, kb, zlo, zhi);
        }
      }
    }
  }
}

template <class R>
void grid_out(const Grid<R>& g, double* x_out, double* w_out) {
  size_t nv = g.W.size();
  for (size_t q = 0; q < nv; ++q) {
    if (x_out) { x_out[2 * q] = (double)g.X[q].real(); x_out[2 * q + 1] = (double)g.X[q].imag(); }
    if (w_out) w_out[q] = (double)g.W[q];
  }
}

void rtsf(const float* in, float* out, int nx, float thetat, float shxi, float shyi);

template <class R>
int bp_run(const float* imgs_in, int nx, int nang, const float* angles, const float* symang,
           int nsym, const uint8_t* half, int halt, float* vol_all, float* vol_1, float* vol_2,
           double* x_out, double* w_out, int nthreads, const float* inplane = nullptr, bool use_rtsf = false) {
  if (nx < 8) return 101;
  // RB 3F / RB 32F: every image first goes through RTSQ (RTSF with SPIDER's
  // FBS mode on) with doc registers 6-8 (in-plane angle, x shift, y shift),
  // bp3f.f:406-425
  std::vector<float> rot;
  const float* imgs = imgs_in;
  if (inplane) {
    rot.resize((size_t)nang * nx * nx);
    #pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(static)
    for (int a = 0; a < nang; ++a) {
      if (use_rtsf)
        rtsf(imgs_in + (size_t)a * nx * nx, &rot[(size_t)a * nx * nx], nx, inplane[3 * a], inplane[3 * a + 1],
             inplane[3 * a + 2]);
      else
        rtsq(imgs_in + (size_t)a * nx * nx, &rot[(size_t)a * nx * nx], nx, nx, inplane[3 * a], inplane[3 * a + 1],
             inplane[3 * a + 2]);
    }
    imgs = rot.data();
  }
  KBTable kb;
  fill_kb(2 * nx, kb);
  std::vector<float> dm((size_t)9 * nang), sm((size_t)9 * std::max(1, nsym));
  for (int a = 0; a < nang; ++a)  // BUILDM1: CANG(phi, theta, psi), bp3f.f:1287
    cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], &dm[9 * a]);
  for (int s = 0; s < nsym; ++s)  // BUILDS, builds.f:52
    cang(symang[3 * s + 2], symang[3 * s + 1], symang[3 * s + 0], &sm[9 * s]);
  Grid<R> ge(nx);
  std::vector<Grid<R>*> grids{&ge};
  Grid<R>* go = nullptr;
  if (half) { go = new Grid<R>(nx); grids.push_back(go); }
  std::vector<uint8_t> route;
  if (half) { route.resize(nang); for (int a = 0; a < nang; ++a) route[a] = half[a] ? 0 : 1; }
  // the checker never uses the reference's racy row striping: one thread
  // runs the serial loop, more threads the owner-computes schedule (same sums)
  if (nthreads > 1)
    insert_images_owned<R>(grids, imgs, nx, nang, dm.data(), sm.data(), nsym, half ? route.data() : nullptr, kb,
                           nthreads);
  else
    insert_images<R>(grids, imgs, nx, nang, dm.data(), sm.data(), nsym, half ? route.data() : nullptr, kb, 1);
  symplane0<R>(ge);
  if (go) symplane0<R>(*go);
  if (halt) {  // BP 3F P: partial X and W after SYMPLANE0
    grid_out(ge, x_out, w_out);
    delete go;
    return 0;
  }
  // real-space symmetrisation of each output with MAXSYM > 1 (bp3f.f:252-279,
  // bp32f.f:280-300,352-368,390-405)
  auto sym = [&](float* v) {
    if (nsym <= 1 || !v) return;
    std::vector<float> tmp(v, v + (size_t)nx * nx * nx);
    symvol(tmp.data(), v, nx, sm.data(), nsym);
  };
  if (!half) {
    finish_volume<R>(ge, kb, vol_all);
    sym(vol_all);
    return 0;
  }
  // BP 32F: first sample = XE, both = XE+XO (ADDADA), second = XO
  Grid<R> both(nx);
  for (size_t q = 0; q < ge.W.size(); ++q) { both.X[q] = ge.X[q] + go->X[q]; both.W[q] = ge.W[q] + go->W[q]; }
  if (vol_1) { finish_volume<R>(ge, kb, vol_1); sym(vol_1); }
  if (vol_all) { finish_volume<R>(both, kb, vol_all); sym(vol_all); }
  if (vol_2) { finish_volume<R>(*go, kb, vol_2); sym(vol_2); }
  delete go;
  return 0;
}

// ------------------------------------------------ PJ 3Q (A14) -------------
// PREPCUB (prepcub.f:54-109): runs of voxels inside the sphere, centred.
struct RunC { int i1, i2, x, y, z; };
void prepcub(int nsam, int nrow, int nslice, float ri, int ldpx, int ldpy, int ldpz, std::vector<RunC>& runs) {
  float r = ri * ri;
  runs.clear();
  for (int i1 = 1; i1 <= nslice; ++i1) {
    float t = (float)(i1 - ldpz);
    float xx = t * t;
    for (int i2 = 1; i2 <= nrow; ++i2) {
      float t2 = (float)(i2 - ldpy);
      float yy = t2 * t2 + xx;
      bool first = true;
      for (int i3 = 1; i3 <= nsam; ++i3) {
        float t3 = (float)(i3 - ldpx);
        float rc = t3 * t3 + yy;
        if (first) {
          if (rc > r) continue;
          first = false;
          runs.push_back(RunC{i3, i3, i3 - ldpx, i2 - ldpy, i1 - ldpz});
        } else if (rc <= r) {
          runs.back().i2 = i3;
        }
      }
    }
  }
}

// WPRO_N (wpro_n.f:44-150): one projection, trilinear gather along z.
template <class R>
void wpro_n(R* b, int nsam, int nrow, int nslice, const float* cube, const std::vector<RunC>& runs,
            float phi, float theta, float psi, float ri, int ldpx, int ldpy, int ldpz) {
  const double d2r = QUADPI_F / 180.0;
  double cphi = std::cos((double)phi * d2r), sphi = std::sin((double)phi * d2r);
  double cthe = std::cos((double)theta * d2r), sthe = std::sin((double)theta * d2r);
  double cpsi = std::cos((double)psi * d2r), spsi = std::sin((double)psi * d2r);
  float dm[9];
  dm[0] = (float)(cphi * cthe * cpsi - sphi * spsi);
  dm[1] = (float)(sphi * cthe * cpsi + cphi * spsi);
  dm[2] = (float)(-sthe * cpsi);
  dm[3] = (float)(-cphi * cthe * spsi - sphi * cpsi);
  dm[4] = (float)(-sphi * cthe * spsi + cphi * cpsi);
  dm[5] = (float)(sthe * spsi);
  dm[6] = (float)(sthe * cphi);
  dm[7] = (float)(sthe * sphi);
  dm[8] = (float)(cthe);
  const float dm1 = dm[0], dm2 = dm[1], dm3 = dm[2];
  std::fill(b, b + (size_t)nsam * nrow, (R)0);
  int dim = std::min(nsam, std::min(nrow, nslice));
  bool nocheck = (2.0f * (ri + 1.0f) + 1.0f) <= (float)dim;
  auto C = [&](int x, int y, int z) -> R { return (R)cube[((size_t)(z - 1) * nrow + (y - 1)) * nsam + (x - 1)]; };
  for (const RunC& rn : runs) {
    int k = rn.y + ldpy;
    float xb = (float)rn.x * dm[0] + (float)rn.y * dm[3] + (float)rn.z * dm[6] + (float)ldpx;
    float yb = (float)rn.x * dm[1] + (float)rn.y * dm[4] + (float)rn.z * dm[7] + (float)ldpy;
    float zb = (float)rn.x * dm[2] + (float)rn.y * dm[5] + (float)rn.z * dm[8] + (float)ldpz;
    for (int j = rn.i1; j <= rn.i2; ++j) {
      int iox = ifix(xb), ioy = ifix(yb), ioz = ifix(zb);
      bool ok = nocheck || (iox >= 1 && iox < nsam && ioy >= 1 && ioy < nrow && ioz >= 1 && ioz < nslice);
      if (ok) {
        R dx = (R)(xb - (float)iox), dy = (R)(yb - (float)ioy), dz = (R)(zb - (float)ioz);
        R a1 = C(iox, ioy, ioz);
        R a2 = C(iox + 1, ioy, ioz) - a1;
        R a3 = C(iox, ioy + 1, ioz) - a1;
        R a4 = C(iox, ioy, ioz + 1) - a1;
        R a5 = -a2 - C(iox, ioy + 1, ioz) + C(iox + 1, ioy + 1, ioz);
        R a61 = -C(iox, ioy, ioz + 1) + C(iox + 1, ioy, ioz + 1);
        R a6 = -a2 + a61;
        R a7 = -a3 - C(iox, ioy, ioz + 1) + C(iox, ioy + 1, ioz + 1);
        R a8 = -a5 - a61 - C(iox, ioy + 1, ioz + 1) + C(iox + 1, ioy + 1, ioz + 1);
        R& o = b[(size_t)(k - 1) * nsam + (j - 1)];
        o = o + a1 + dz * (a4 + a6 * dx + (a7 + a8 * dx) * dy) + a3 * dy + dx * (a2 + a5 * dy);
      }
      xb = xb + dm1;
      yb = yb + dm2;
      zb = zb + dm3;
    }
  }
}

// ------------------------------------------------ BP CG (A15, A16) --------
// PREPCUB_S (prepcub_s.f:54-111): runs with 1-based linear indices.
struct RunS { int l1, l2, x, y, z; };
void prepcub_s(int n, float ri, int ldp, std::vector<RunS>& runs) {
  float r = ri * ri;
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
          runs.push_back(RunS{nmat, nmat, i3, i2, i1});
        } else if (rc <= r) {
          runs.back().l2 = nmat;
        }
      }
    }
  }
}

// PROJT difference table (bpcg.f:732-742): projt[4*(I-1) + c], I 1-based.
template <class R>
void make_projt(const R* proj, int n, std::vector<R>& projt) {
  projt.assign((size_t)4 * n * n, (R)0);
  for (int I = 1; I <= n * n - n - 1; ++I) {
    R pt = proj[I - 1];
    projt[4 * (I - 1) + 0] = pt;
    projt[4 * (I - 1) + 1] = proj[I + n - 1] - pt;
    projt[4 * (I - 1) + 2] = proj[I] - pt;
    projt[4 * (I - 1) + 3] = proj[I + n] - proj[I] - projt[4 * (I - 1) + 1];
  }
}

// BCKPJ_LIN, SP_MP branch (bckpj.f:59-94): voxel gather, direct XBB formula.
template <class R>
void bckpj_lin(R* cube, const float* dm, const R* projt, int n, const std::vector<RunS>& runs, int ldp, int ldpnm, int nthreads) {
  #pragma omp parallel for num_threads(nthreads) schedule(static)
  for (long r = 0; r < (long)runs.size(); ++r) {
    const RunS& rn = runs[r];
    float xb = ((float)(rn.x - ldp) * dm[0] + (float)(rn.y - ldp) * dm[1] + (float)(rn.z - ldp) * dm[2]) + (float)ldpnm;
    float yb = ((float)(rn.x - ldp) * dm[3] + (float)(rn.y - ldp) * dm[4] + (float)(rn.z - ldp) * dm[5]) + (float)ldpnm;
    for (int j = rn.l1; j <= rn.l2; ++j) {
      int jt = j - rn.l1;
      float xbb = xb + (float)jt * dm[0];
      float ybb = yb + (float)jt * dm[3];
      int iqx = ifix(xbb), iqy = ifix(ybb);
      const R* B = &projt[4 * ((size_t)(iqy - 1) * n + (iqx - 1))];
      R dy = (R)(ybb - (float)iqy), dx = (R)(xbb - (float)iqx);
      cube[j - 1] = cube[j - 1] + B[0] + dy * B[1] + dx * (B[2] + dy * B[3]);
    }
  }
}

// PRJCQ_N (prjcq.f:48-82): voxel splat with sequential XB accumulation.
template <class R>
void prjcq_n(const R* cube, const float* dm, R* prj, int n, const std::vector<RunS>& runs, int ldp, int ldpnm) {
  for (const RunS& rn : runs) {
    float xb = (float)(rn.x - ldp) * dm[0] + (float)(rn.y - ldp) * dm[1] + (float)(rn.z - ldp) * dm[2] + (float)ldpnm;
    float yb = (float)(rn.x - ldp) * dm[3] + (float)(rn.y - ldp) * dm[4] + (float)(rn.z - ldp) * dm[5] + (float)ldpnm;
    for (int j = rn.l1; j <= rn.l2; ++j) {
      int iqx = ifix(xb), iqy = ifix(yb);
      R c = cube[j - 1];
      R dx = (R)(xb - (float)iqx);
      R dy = (R)(yb - (float)iqy) * c;
      R dx1m = (R)1 - dx;
      R dy1m = c - dy;
      R* p = &prj[(size_t)(iqy - 1) * n + (iqx - 1)];
      p[0] += dx1m * dy1m;
      p[1] += dx * dy1m;
      p[n] += dx1m * dy;
      p[n + 1] += dx * dy;
      xb = xb + dm[0];
      yb = yb + dm[3];
    }
  }
}

// HIANG (hiang.f:40-112): fold theta >= 90, truncate phi to 0.01 deg, merge
// duplicates into weights LB, psi := 0, rebuild DM in double.
// ang[3*i] = phi, ang[3*i+1] = theta, ang[3*i+2] = psi.  Returns LO.
int hiang(std::vector<float>& ang, int nang, std::vector<float>& dm, std::vector<int>& lb) {
  lb.assign(nang, 1);
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
  for (int i = 0; i < nang - 1; ++i) {
    if (lb[i] != 0) {
      for (int j = i + 1; j < nang; ++j) {
        if (lb[i] != 0) {   // the reference tests LB(I) here (hiang.f:66)
          if (ang[3 * i] == ang[3 * j] && ang[3 * i + 1] == ang[3 * j + 1]) { lb[i] += 1; lb[j] = 0; }
        }
      }
    }
  }
  int lo = 0;
  for (int i = 0; i < nang; ++i) {
    if (lb[i] != 0) {
      ang[3 * lo] = ang[3 * i];
      ang[3 * lo + 1] = ang[3 * i + 1];
      ang[3 * lo + 2] = 0.0f;
      lb[lo] = lb[i];
      ++lo;
    }
  }
  const double d2r = QUADPI_F / 180.0;
  dm.assign((size_t)9 * lo, 0.0f);
  for (int i = 0; i < lo; ++i) {
    double cphi = std::cos((double)ang[3 * i] * d2r), sphi = std::sin((double)ang[3 * i] * d2r);
    double cthe = std::cos((double)ang[3 * i + 1] * d2r), sthe = std::sin((double)ang[3 * i + 1] * d2r);
    double cpsi = 1.0, spsi = 0.0;
    float* d = &dm[9 * i];
    d[0] = (float)(cphi * cthe * cpsi - sphi * spsi);
    d[1] = (float)(sphi * cthe * cpsi + cphi * spsi);
    d[2] = (float)(-sthe * cpsi);
    d[3] = (float)(-cphi * cthe * spsi - sphi * cpsi);
    d[4] = (float)(-sphi * cthe * spsi + cphi * cpsi);
    d[5] = (float)(sthe * spsi);
    d[6] = (float)(sthe * cphi);
    d[7] = (float)(sthe * sphi);
    d[8] = (float)(cthe);
  }
  return lo;
}

// FIXEDGE1/2/3 (bpcg.f:1278-1517): zero outside the runs, then extend the
// edge values by `w` voxels along x, then y, then z.
template <class R>
void fixedge(R* p, int n, const std::vector<RunS>& runs, int mode) {
  const long nnn = (long)n * n * n;
  size_t nt = 0;
  for (long i = 1; i <= nnn; ++i) {
    if (nt >= runs.size()) p[i - 1] = 0;
    else if (i < runs[nt].l1) p[i - 1] = 0;
    else if (i == runs[nt].l2) ++nt;
  }
  auto at = [&](int i, int j, int k) -> R& { return p[((size_t)(k - 1) * n + (j - 1)) * n + (i - 1)]; };
  // axis passes; `get(line, t)` addresses element t (1-based) of a line
  for (int axis = 0; axis < 3; ++axis) {
    for (int a = 1; a <= n; ++a)
      for (int b = 1; b <= n; ++b) {
        auto L = [&](int t) -> R& {
          if (axis == 0) return at(t, b, a);      // K=a, J=b, I=t
          if (axis == 1) return at(b, t, a);      // K=a, I=b, J=t
          return at(b, a, t);                     // J=a, I=b, K=t
        };
        if (mode == 1) {
          for (int t = 1; t <= n - 1; ++t) if (L(t + 1) != (R)0) { L(t) = L(t + 1); break; }
          for (int t = n; t >= 2; --t) if (L(t - 1) != (R)0) { L(t) = L(t - 1); break; }
        } else if (mode == 2) {
          for (int t = 2; t <= n - 1; ++t) if (L(t + 1) != (R)0) { L(t) = L(t + 1); L(t - 1) = L(t + 1); break; }
          for (int t = n - 1; t >= 2; --t) if (L(t - 1) != (R)0) { L(t) = L(t - 1); L(t + 1) = L(t - 1); break; }
        } else {
          for (int t = 3; t <= n - 1; ++t) if (L(t + 1) != (R)0) { L(t) = L(t + 1); L(t - 1) = L(t + 1); L(t - 2) = L(t + 1); break; }
          for (int t = n - 2; t >= 2; --t) if (L(t - 1) != (R)0) { L(t) = L(t - 1); L(t + 1) = L(t - 1); L(t + 2) = L(t - 1); break; }
        }
      }
  }
}

// BFIRSTS / BSECOND / BTHIRD (bpcg.f:1521-1588)
template <class R>
void regularize(R* bcke, const R* p, int n, R anoise, const std::vector<RunS>& runs, int mode) {
  auto P = [&](long q) -> R { return p[q]; };
  const long sx = 1, sy = n, sz = (long)n * n;
  for (const RunS& rn : runs)
    for (int j = rn.l1; j <= rn.l2; ++j) {
      long q = j - 1;
      R v;
      if (mode == 1) {
        v = (R)6 * P(q) - (+P(q + sx) + P(q + sy) + P(q + sz) + P(q - sx) + P(q - sy) + P(q - sz));
      } else if (mode == 2) {
        v = (R)18 * P(q) - (R)4.0f * P(q + sx) + P(q + 2 * sx) - (R)4.0f * P(q - sx) + P(q - 2 * sx)
            - (R)4.0f * P(q + sy) + P(q + 2 * sy) - (R)4.0f * P(q - sy) + P(q - 2 * sy)
            - (R)4.0f * P(q + sz) + P(q + 2 * sz) - (R)4.0f * P(q - sz) + P(q - 2 * sz);
      } else {
        v = (R)60 * P(q) - (R)15.0f * P(q + sx) + (R)6.0f * P(q + 2 * sx) - P(q + 3 * sx)
            - (R)15.0f * P(q - sx) + (R)6.0f * P(q - 2 * sx) - P(q - 3 * sx)
            - (R)15.0f * P(q + sy) + (R)6.0f * P(q + 2 * sy) - P(q + 3 * sy)
            - (R)15.0f * P(q - sy) + (R)6.0f * P(q - 2 * sy) - P(q - 3 * sy)
            - (R)15.0f * P(q + sz) + (R)6.0f * P(q + 2 * sz) - P(q + 3 * sz)
            - (R)15.0f * P(q - sz) + (R)6.0f * P(q - 2 * sz) - P(q - 3 * sz);
      }
      bcke[q] = bcke[q] + anoise * v;
    }
}

// BPCG (bpcg.f:70-411) -> BPCG_2 (bpcg.f:425-814) -> HIANG -> BPCG_3_LIN
// (bpcg.f:818-1238), linear interpolation, non-MPI.  `logv` receives
// (iteration, err, chi2) triples.  Returns IRTFLG-style status.
// ------------------------------------------- BP CG, FBS interpolation -----
// SPIDER real FFTs as FMRS calls them with SPIDER_SIGN and SPIDER_SCALE
// (fmrs.f:76-132, fftw3.f:376-450): forward = r2c with the imaginary parts
// negated, no scale; inverse = imaginary parts negated, c2r, times 1/N.  The
// half spectrum is [..][n/2+1] (x fastest).  c2r semantics: complex
// transforms along the other axes, then a real transform along x that uses
// only the real parts of the x = 0 and x = n/2 bins (what FFTW's c2r does
// with them; the derivative spectra of FBS2_PREP / FBS3_PREP are not
// Hermitian in those planes, so the reference's output there is whatever
// its c2r makes of it, and both this restatement and the GPU take this form).
void spider_fwd(const double* f, int n, int dims, std::vector<cd>& F) {
  const int h = n / 2 + 1;
  const long planes = dims == 3 ? n : 1;
  F.assign((size_t)planes * n * h, cd(0, 0));
  FFT1 fx(n, -1);
  std::vector<cd> line(n), out(n);
  for (long k = 0; k < planes; ++k)
    for (int j = 0; j < n; ++j) {
      for (int i = 0; i < n; ++i) line[i] = cd(f[((size_t)k * n + j) * n + i], 0.0);
      fx.exec(line.data(), 1, out.data());
      for (int i = 0; i < h; ++i) F[((size_t)k * n + j) * h + i] = out[i];
    }
  for (long k = 0; k < planes; ++k)   // along y
    for (int i = 0; i < h; ++i) {
      for (int j = 0; j < n; ++j) line[j] = F[((size_t)k * n + j) * h + i];
      fx.exec(line.data(), 1, out.data());
      for (int j = 0; j < n; ++j) F[((size_t)k * n + j) * h + i] = out[j];
    }
  if (dims == 3)
    for (int j = 0; j < n; ++j)   // along z
      for (int i = 0; i < h; ++i) {
        for (int k = 0; k < n; ++k) line[k] = F[((size_t)k * n + j) * h + i];
        fx.exec(line.data(), 1, out.data());
        for (int k = 0; k < n; ++k) F[((size_t)k * n + j) * h + i] = out[k];
      }
  for (auto& v : F) v = std::conj(v);   // SPIDER sign
}

void spider_inv(std::vector<cd> G, int n, int dims, double* f) {
  const int h = n / 2 + 1;
  const long planes = dims == 3 ? n : 1;
  for (auto& v : G) v = std::conj(v);   // SPIDER sign
  FFT1 fb(n, +1);
  std::vector<cd> line(n), out(n);
  for (long k = 0; k < planes; ++k)
    for (int i = 0; i < h; ++i) {
      for (int j = 0; j < n; ++j) line[j] = G[((size_t)k * n + j) * h + i];
      fb.exec(line.data(), 1, out.data());
      for (int j = 0; j < n; ++j) G[((size_t)k * n + j) * h + i] = out[j];
    }
  if (dims == 3)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < h; ++i) {
        for (int k = 0; k < n; ++k) line[k] = G[((size_t)k * n + j) * h + i];
        fb.exec(line.data(), 1, out.data());
        for (int k = 0; k < n; ++k) G[((size_t)k * n + j) * h + i] = out[k];
      }
  const double scale = 1.0 / (dims == 3 ? (double)n * n * n : (double)n * n);
  for (long k = 0; k < planes; ++k)
    for (int j = 0; j < n; ++j) {
      const cd* g = &G[((size_t)k * n + j) * h];
      line[0] = cd(g[0].real(), 0.0);
      for (int i = 1; i < h; ++i) {
        line[i] = g[i];
        if (n - i != i) line[n - i] = std::conj(g[i]);
      }
      if (n % 2 == 0) line[n / 2] = cd(g[n / 2].real(), 0.0);
      fb.exec(line.data(), 1, out.data());
      for (int i = 0; i < n; ++i) f[((size_t)k * n + j) * n + i] = out[i].real() * scale;
    }
}

// -i*w*v in the interleaved form of FBS2_PREP / FBS3_PREP: (re, im) -> (im w, -re w)
static inline cd mul_mi(cd v, double w) { return cd(v.imag() * w, -v.real() * w); }

// FBS2_PREP (fbs2.f:182-247): x, y and xy derivatives of an n x n image
// through the 2D FFT.  WY(n/2) keeps the value (n/2) 2 pi / n here (FBS3_PREP
// zeroes its Nyquist frequencies, FBS2_PREP does not).
template <class R>
void fbs2_prep(const R* img, int n, std::vector<R>& x1, std::vector<R>& y1, std::vector<R>& xy2) {
  const int h = n / 2 + 1;
  std::vector<double> f((size_t)n * n);
  for (size_t i = 0; i < f.size(); ++i) f[i] = (double)img[i];
  std::vector<cd> F;
  spider_fwd(f.data(), n, 2, F);
  const float a4 = 6.28318530717958647692f / (float)n;   // A4 = PI2 / NX in REAL
  std::vector<cd> X((size_t)n * h), Y((size_t)n * h), XY((size_t)n * h);
  for (int j = 0; j < n; ++j) {
    const double wy = (double)((float)(j <= n / 2 ? j : j - n) * a4);
    for (int i = 0; i < h; ++i) {
      const double wx = (double)((float)i * a4);
      const size_t q = (size_t)j * h + i;
      X[q] = mul_mi(F[q], wx);
      Y[q] = mul_mi(F[q], wy);
      XY[q] = mul_mi(X[q], wy);
    }
  }
  std::vector<double> o((size_t)n * n);
  auto out = [&](std::vector<cd>& G, std::vector<R>& dst) {
    spider_inv(G, n, 2, o.data());
    dst.resize(o.size());
    for (size_t i = 0; i < o.size(); ++i) dst[i] = (R)o[i];
  };
  out(X, x1);
  out(Y, y1);
  out(XY, xy2);
}

// FBS3_PREP (fbs3.f:294-407): the seven derivatives of an n^3 volume.  The
// XZ2 real part takes X1's real part (fbs3.f:379: X1(2*K+1) where the
// pattern of the other lines has X1(2*K+2)); kept as the reference has it.
template <class R>
void fbs3_prep(const R* vol, int n, std::vector<R>* d /* x1 y1 z1 xy2 xz2 yz2 xyz */) {
  const int h = n / 2 + 1;
  std::vector<double> f((size_t)n * n * n);
  for (size_t i = 0; i < f.size(); ++i) f[i] = (double)vol[i];
  std::vector<cd> F;
  spider_fwd(f.data(), n, 3, F);
  const float a4 = 6.28318530717958647692f / (float)n;   // A4 = PI2 / N in REAL
  auto wsig = [&](int j) -> double {   // WY / WZ with the Nyquist entry zeroed
    if (n % 2 == 0 && j == n / 2) return 0.0;
    return (double)((float)(j <= n / 2 ? j : j - n) * a4);
  };
  std::vector<std::vector<cd>> D(7, std::vector<cd>(F.size()));
  for (int l = 0; l < n; ++l)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < h; ++i) {
        const size_t q = ((size_t)l * n + j) * h + i;
        const double wx = (double)((float)i * a4), wy = wsig(j), wz = wsig(l);
        const cd x1 = mul_mi(F[q], wx), y1 = mul_mi(F[q], wy), xy2 = mul_mi(x1, wy);
        D[0][q] = x1;
        D[1][q] = y1;
        D[2][q] = mul_mi(F[q], wz);
        D[3][q] = xy2;
        D[4][q] = cd(x1.real() * wz, -x1.real() * wz);   // fbs3.f:379-380 as written
        D[5][q] = mul_mi(y1, wz);
        D[6][q] = mul_mi(xy2, wz);
      }
  std::vector<double> o((size_t)n * n * n);
  for (int m = 0; m < 7; ++m) {
    spider_inv(D[m], n, 3, o.data());
    d[m].resize(o.size());
    for (size_t i = 0; i < o.size(); ++i) d[m][i] = (R)o[i];
  }
}

// one cubic along x (fbs2.f / fbs3.f): F(DX) from values and x derivatives at 0, 1
template <class R>
static inline R cub(R f0, R d0, R f1, R d1, R dx, R dx2, R dx3) {
  R a2 = (R)3 * (f1 - f0) - (R)2 * d0 - d1;
  R a3 = (R)2 * (-f1 + f0) + d0 + d1;
  return f0 + d0 * dx + a2 * dx2 + a3 * dx3;
}

static inline int fmodulo(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

// FBS2 (fbs2.f:94-180) with CHKBOUND: bicubic from values and derivatives,
// indices wrapped (MODULO).  Arrays are [n][n] (x fastest), 0-based.
template <class R>
R fbs2(float x, float y, int n, const R* f, const R* x1, const R* y1, const R* xy2) {
  const int i = (int)std::floor(x), j = (int)std::floor(y);
  const R dx = (R)(x - (float)i), dy = (R)(y - (float)j);
  const R dx2 = dx * dx, dx3 = dx * dx * dx;
  const int i2 = fmodulo(i - 1, n), j2 = fmodulo(j - 1, n), i3 = fmodulo(i, n), j3 = fmodulo(j, n);
  auto at = [&](const R* a, int ii, int jj) { return a[(size_t)jj * n + ii]; };
  const R adx = cub<R>(at(f, i2, j2), at(x1, i2, j2), at(f, i3, j2), at(x1, i3, j2), dx, dx2, dx3);
  const R bdx = cub<R>(at(f, i2, j3), at(x1, i2, j3), at(f, i3, j3), at(x1, i3, j3), dx, dx2, dx3);
  const R dadx = cub<R>(at(y1, i2, j2), at(xy2, i2, j2), at(y1, i3, j2), at(xy2, i3, j2), dx, dx2, dx3);
  const R dbdx = cub<R>(at(y1, i2, j3), at(xy2, i2, j3), at(y1, i3, j3), at(xy2, i3, j3), dx, dx2, dx3);
  const R a2 = (R)3 * (bdx - adx) - (R)2 * dadx - dbdx;
  const R a3 = (R)2 * (adx - bdx) + dadx + dbdx;
  return adx + dadx * dy + a2 * (dy * dy) + a3 * (dy * dy * dy);
}

// FBS3 (fbs3.f:60-290): tricubic from the volume and its seven derivatives,
// indices wrapped.  d = {x1, y1, z1, xy2, xz2, yz2, xyz}, each [n][n][n].
template <class R>
R fbs3(float x, float y, float z, int n, const R* f1, const std::vector<R>* d) {
  const int i = (int)std::floor(x), j = (int)std::floor(y), l = (int)std::floor(z);
  const int i2 = fmodulo(i - 1, n), j2 = fmodulo(j - 1, n), l2 = fmodulo(l - 1, n);
  const int i3 = (i2 + 1) % n, j3 = (j2 + 1) % n, l3 = (l2 + 1) % n;
  const R dx = (R)(x - (float)i), dy = (R)(y - (float)j), dz = (R)(z - (float)l);
  const R dx2 = dx * dx, dx3 = dx * dx * dx, dy2 = dy * dy, dy3 = dy * dy * dy;
  auto at = [&](const R* a, int ii, int jj, int ll) { return a[((size_t)ll * n + jj) * n + ii]; };
  const R *X1 = d[0].data(), *Y1 = d[1].data(), *Z1 = d[2].data(), *XY2 = d[3].data(), *XZ2 = d[4].data(),
          *YZ2 = d[5].data(), *XYZ = d[6].data();
  // value and z-derivative on plane L: bicubic in (x, y) of (F, X1, Y1, XY2) and (Z1, XZ2, YZ2, XYZ)
  auto plane = [&](const R* f, const R* fx, const R* fy, const R* fxy, int ll) {
    const R adx = cub<R>(at(f, i2, j2, ll), at(fx, i2, j2, ll), at(f, i3, j2, ll), at(fx, i3, j2, ll), dx, dx2, dx3);
    const R bdx = cub<R>(at(f, i2, j3, ll), at(fx, i2, j3, ll), at(f, i3, j3, ll), at(fx, i3, j3, ll), dx, dx2, dx3);
    const R dadx = cub<R>(at(fy, i2, j2, ll), at(fxy, i2, j2, ll), at(fy, i3, j2, ll), at(fxy, i3, j2, ll), dx, dx2, dx3);
    const R dbdx = cub<R>(at(fy, i2, j3, ll), at(fxy, i2, j3, ll), at(fy, i3, j3, ll), at(fxy, i3, j3, ll), dx, dx2, dx3);
    const R a2 = (R)3 * (bdx - adx) - (R)2 * dadx - dbdx;
    const R a3 = (R)2 * (adx - bdx) + dadx + dbdx;
    return adx + dadx * dy + a2 * dy2 + a3 * dy3;
  };
  const R c0 = plane(f1, X1, Y1, XY2, l2), dc0 = plane(Z1, XZ2, YZ2, XYZ, l2);
  const R c1 = plane(f1, X1, Y1, XY2, l3), dc1 = plane(Z1, XZ2, YZ2, XYZ, l3);
  const R a2 = (R)3 * (c1 - c0) - (R)2 * dc0 - dc1;
  const R a3 = (R)2 * (c0 - c1) + dc0 + dc1;
  return c0 + dc0 * dz + a2 * (dz * dz) + a3 * (dz * dz * dz);
}

// Fortran MODULO for REAL: A - FLOOR(A/P)*P, here as fmod with the sign of P
static inline float fmodulo_real(float a, float p) {
  float r = std::fmod(a, p);
  if (r != 0.0f && ((r < 0.0f) != (p < 0.0f))) r += p;
  return r;
}

// RTSF (rtsf.f:109-205), the SCLI = 1 branch that RB 3F / RB 32F take
// (bp3f.f:414-417 passes SCLI = 1.0): FBS2_PREP of the image, then FBS2 with
// wrapped indices at the rotated and shifted source position of every output
// pixel.  REAL arithmetic, left to right; THETA = THETAT * PI / 180.
void rtsf(const float* in, float* out, int nx, float thetat, float shxi, float shyi) {
  const int ny = nx;
  std::vector<float> x1, y1, xy2;
  fbs2_prep<float>(in, nx, x1, y1, xy2);
  const float pi = 3.14159265358979323846f;
  const float theta = thetat * pi / 180.0f;
  const float costh = std::cos(theta), sinth = std::sin(theta);
  const int cx = nx / 2 + 1, cy = ny / 2 + 1;
  const float shx = fmodulo_real(shxi, (float)nx), shy = fmodulo_real(shyi, (float)ny);
  const float fy0 = -shy - (float)cy, fy1 = -shy + (float)ny - (float)cy, fy2 = -shy - (float)ny - (float)cy;
  const float fx0 = -shx - (float)cx, fx1 = -shx + (float)nx - (float)cx, fx2 = -shx - (float)nx - (float)cx;
  const float shypny = shy + (float)ny, shxpnx = shx + (float)nx;
  for (int iy = 1; iy <= ny; ++iy) {
    float fy = (float)iy + fy0;
    if ((float)(iy - 1) < shy) fy = (float)iy + fy1;
    if ((float)(iy - 1) >= shypny) fy = (float)iy + fy2;
    const float ycod = costh * fy + (float)cy;
    const float ysid = -sinth * fy + (float)cx;
    for (int ix = 1; ix <= nx; ++ix) {
      float fx = (float)ix + fx0;
      if ((float)(ix - 1) < shx) fx = (float)ix + fx1;
      if ((float)(ix - 1) >= shxpnx) fx = (float)ix + fx2;
      const float xold = costh * fx + ysid;
      const float yold = sinth * fx + ycod;
      out[(size_t)(iy - 1) * nx + (ix - 1)] = fbs2<float>(xold, yold, nx, in, x1.data(), y1.data(), xy2.data());
    }
  }
}

// PRJCQ_FBS3 (prjcq.f:97-167): every line (J, K) of the cube, sample I
// walked with XB += DM(1), YB += DM(2), ZB += DM(3); pixel (I, J) sums over K.
template <class R>
void prjcq_fbs3(const R* cube, const float* dm, R* prj, int n, const std::vector<R>* d) {
  std::fill(prj, prj + (size_t)n * n, (R)0);
  const int h = n / 2;
  for (int k = 1; k <= n; ++k)
    for (int j = 1; j <= n; ++j) {
      // -N/2*DM(1) + (J-N/2-1)*DM(4) + (K-N/2-1)*DM(7) + N/2+1, left to right in REAL
      float xb = -((float)h * dm[0]) + (float)(j - h - 1) * dm[3] + (float)(k - h - 1) * dm[6] + (float)h + 1.0f;
      float yb = -((float)h * dm[1]) + (float)(j - h - 1) * dm[4] + (float)(k - h - 1) * dm[7] + (float)h + 1.0f;
      float zb = -((float)h * dm[2]) + (float)(j - h - 1) * dm[5] + (float)(k - h - 1) * dm[8] + (float)h + 1.0f;
      for (int i = 1; i <= n; ++i) {
        const int iox = ifix(xb), ioy = ifix(yb), ioz = ifix(zb);
        if (iox >= 1 && iox < n && ioy >= 1 && ioy < n && ioz >= 1 && ioz < n)
          prj[(size_t)(j - 1) * n + (i - 1)] += fbs3<R>(xb, yb, zb, n, cube, d);
        xb = xb + dm[0];
        yb = yb + dm[1];
        zb = zb + dm[2];
      }
    }
}

// WPRO_FBS (wpro_fbs.f:1-150): PJ 3F, WPRO_N's walk along the PREPCUB runs
// with an FBS3 sample (wrapped indices) per voxel; the bounds test, when the
// sphere does not fit, admits IFIX in 1..N (wpro_fbs.f:138-144).
template <class R>
void wpro_fbs(R* b, int n, const R* cube, const std::vector<R>* d, const std::vector<RunC>& runs, float phi,
              float theta, float psi, float ri, int ldp) {
  const double d2r = QUADPI_F / 180.0;
  double cphi = std::cos((double)phi * d2r), sphi = std::sin((double)phi * d2r);
  double cthe = std::cos((double)theta * d2r), sthe = std::sin((double)theta * d2r);
  double cpsi = std::cos((double)psi * d2r), spsi = std::sin((double)psi * d2r);
  float dm[9];
  dm[0] = (float)(cphi * cthe * cpsi - sphi * spsi);
  dm[1] = (float)(sphi * cthe * cpsi + cphi * spsi);
  dm[2] = (float)(-sthe * cpsi);
  dm[3] = (float)(-cphi * cthe * spsi - sphi * cpsi);
  dm[4] = (float)(-sphi * cthe * spsi + cphi * cpsi);
  dm[5] = (float)(sthe * spsi);
  dm[6] = (float)(sthe * cphi);
  dm[7] = (float)(sthe * sphi);
  dm[8] = (float)(cthe);
  std::fill(b, b + (size_t)n * n, (R)0);
  const bool nocheck = (2.0f * (ri + 1.0f) + 1.0f) <= (float)n;
  for (const RunC& rn : runs) {
    const int k = rn.y + ldp;
    float xb = (float)rn.x * dm[0] + (float)rn.y * dm[3] + (float)rn.z * dm[6] + (float)ldp;
    float yb = (float)rn.x * dm[1] + (float)rn.y * dm[4] + (float)rn.z * dm[7] + (float)ldp;
    float zb = (float)rn.x * dm[2] + (float)rn.y * dm[5] + (float)rn.z * dm[8] + (float)ldp;
    for (int j = rn.i1; j <= rn.i2; ++j) {
      const int iox = ifix(xb), ioy = ifix(yb), ioz = ifix(zb);
      if (nocheck || (iox > 0 && iox <= n && ioy > 0 && ioy <= n && ioz > 0 && ioz <= n)) {
        R& o = b[(size_t)(k - 1) * n + (j - 1)];
        o = o + fbs3<R>(xb, yb, zb, n, cube, d);
      }
      xb = xb + dm[0];
      yb = yb + dm[1];
      zb = zb + dm[2];
    }
  }
}

// BCKPJ_FBS (bckpj.f:123-164): voxel gather along the runs, sequential XB += DM(1), YB += DM(4).
template <class R>
void bckpj_fbs(R* cube, const float* dm, const R* proj, const R* x1, const R* y1, const R* xy2, int n,
               const std::vector<RunS>& runs, int ldp, int ldpnm, int nthreads) {
  #pragma omp parallel for num_threads(nthreads) schedule(static)
  for (long r = 0; r < (long)runs.size(); ++r) {
    const RunS& rn = runs[r];
    float xb = ((float)(rn.x - ldp) * dm[0] + (float)(rn.y - ldp) * dm[1] + (float)(rn.z - ldp) * dm[2]) + (float)ldpnm;
    float yb = ((float)(rn.x - ldp) * dm[3] + (float)(rn.y - ldp) * dm[4] + (float)(rn.z - ldp) * dm[5]) + (float)ldpnm;
    for (int j = rn.l1; j <= rn.l2; ++j) {
      cube[j - 1] = cube[j - 1] + fbs2<R>(xb, yb, n, proj, x1, y1, xy2);
      xb = xb + dm[0];
      yb = yb + dm[3];
    }
  }
}

template <class R>
int bpcg_run(const float* projs, int n, int nang, const float* angles, float ri, float errm, float chim,
             int maxit, int mode, float anoise, float* vol, float* logv, int* niter, int* nang_eff,
             double* stats, int nthreads, bool fbs = false) {
  const int ldp = n / 2 + 1, ldpnm = ldp;
  std::vector<RunS> runs;
  prepcub_s(n, ri, ldp, runs);
  const long nnn = (long)n * n * n;
  std::vector<R> cb(nnn, (R)0);
  std::vector<float> ang((size_t)3 * nang), dm((size_t)9 * nang);
  double d_aba = 0, d_sus = 0, d_ssq = 0, d_klp = 0, d_kls = 0;
  std::vector<R> proj((size_t)n * n), projt;
  for (int k = 0; k < nang; ++k) {
    ang[3 * k + 2] = angles[3 * k + 0];   // psi
    ang[3 * k + 1] = angles[3 * k + 1];   // theta
    ang[3 * k + 0] = angles[3 * k + 2];   // phi
    cang(ang[3 * k], ang[3 * k + 1], ang[3 * k + 2], &dm[9 * k]);
    const float* x = projs + (size_t)k * n * n;
    // ASTASQ (bpcg.f:1244-1274)
    float r = ri * ri;
    int nc = n / 2 + 1;
    for (int j = 1; j <= n; ++j) {
      float t = (float)(j - nc);
      float xx = t * t;
      for (int i = 1; i <= n; ++i) {
        float t2 = (float)(i - nc);
        float v = x[(j - 1) * n + (i - 1)];
        if ((xx + t2 * t2) > r) { d_aba += (double)v; d_klp += 1; }
        else { d_ssq += (double)v * (double)v; d_sus += (double)v; d_kls += 1; }
      }
    }
    for (int i = 0; i < n * n; ++i) proj[i] = (R)x[i];
    if (fbs) {   // bpcg.f:713-731
      std::vector<R> dx1, dy1, dxy2;
      fbs2_prep<R>(proj.data(), n, dx1, dy1, dxy2);
      bckpj_fbs<R>(cb.data(), &dm[9 * k], proj.data(), dx1.data(), dy1.data(), dxy2.data(), n, runs, ldp, ldpnm,
                   nthreads);
    } else {
      make_projt<R>(proj.data(), n, projt);
      bckpj_lin<R>(cb.data(), &dm[9 * k], projt.data(), n, runs, ldp, ldpnm, nthreads);
    }
  }
  d_aba = d_aba / d_klp;
  R bnorm = 0;
  R qt = (sizeof(R) == 4) ? (R)(float)(d_aba * nang) : (R)(d_aba * nang);
  for (const RunS& rn : runs)
    for (int j = rn.l1; j <= rn.l2; ++j) {
      R c = (sizeof(R) == 4) ? (R)(float)((double)cb[j - 1] - (double)qt) : cb[j - 1] - qt;
      cb[j - 1] = c;
      bnorm = bnorm + c * c;
    }
  d_ssq = d_ssq - d_aba * (2 * d_sus - d_aba * d_kls);
  R chi2 = (R)d_ssq;
  if (stats) { stats[0] = d_klp; stats[1] = d_aba; stats[2] = (double)bnorm; stats[3] = (double)chi2; }
  std::vector<int> lb;
  int lo = hiang(ang, nang, dm, lb);
  if (nang_eff) *nang_eff = lo;
  float di = (float)(n / 2);
  const float extra = fbs ? 0.0f : 1.0f;   // FBS: RI + MODE > DI (bpcg.f:269-276), linear: RI + MODE + 1
  if ((mode == 1 && (ri + 1.0f + extra) > di) || (mode == 2 && (ri + 2.0f + extra) > di) ||
      (mode == 3 && (ri + 3.0f + extra) > di))
    return 102;  // 'RADIUS TOO LARGE', bpcg.f:272-290
  // BPCG_3_LIN
  std::vector<R> bckn(nnn, (R)0), bckp(nnn, (R)0), bcke(nnn, (R)0);
  R q = 0;
  int it_done = 0;
  std::vector<std::vector<R>> pbuf(nthreads > 0 ? nthreads : 1);
  for (int iter = 1; iter <= maxit; ++iter) {
    R delsq = 0;
    for (const RunS& rn : runs)
      for (int j = rn.l1; j <= rn.l2; ++j) delsq = delsq + cb[j - 1] * cb[j - 1];
    q = q * delsq;
    for (const RunS& rn : runs)
      for (int j = rn.l1; j <= rn.l2; ++j) bckp[j - 1] = cb[j - 1] - q * bckp[j - 1];
    q = (R)-1 / delsq;
    std::fill(bcke.begin(), bcke.end(), (R)0);
    int numth = nthreads > 0 ? nthreads : 1;
    if (fbs) {   // BPCG_3_FBS (bpcg.f:1760-1822): derivatives of BCKP, full-cube projections, FBS2 back-projection
      std::vector<R> d3[7];
      fbs3_prep<R>(bckp.data(), n, d3);
      std::vector<std::vector<R>> projs_k(lo, std::vector<R>((size_t)n * n));
      #pragma omp parallel for num_threads(numth) schedule(dynamic, 1)
      for (int k = 0; k < lo; ++k) prjcq_fbs3<R>(bckp.data(), &dm[9 * k], projs_k[k].data(), n, d3);
      for (int k = 0; k < lo; ++k) {
        std::vector<R>& pj = projs_k[k];
        if (lb[k] > 1)
          for (auto& v : pj) v = v * (R)lb[k];
        std::vector<R> dx1, dy1, dxy2;
        fbs2_prep<R>(pj.data(), n, dx1, dy1, dxy2);
        bckpj_fbs<R>(bcke.data(), &dm[9 * k], pj.data(), dx1.data(), dy1.data(), dxy2.data(), n, runs, ldp, ldpnm,
                     nthreads);
      }
    }
    for (int k0 = 0; k0 < (fbs ? 0 : lo); k0 += numth) {
      int lnum = std::min(numth, lo - k0);
      std::vector<std::vector<R>> projs_k(lnum, std::vector<R>((size_t)n * n, (R)0));
      #pragma omp parallel for num_threads(numth) schedule(static)
      for (int t = 0; t < lnum; ++t) prjcq_n<R>(bckp.data(), &dm[9 * (k0 + t)], projs_k[t].data(), n, runs, ldp, ldpnm);
      for (int t = 0; t < lnum; ++t) {
        std::vector<R>& pj = projs_k[t];
        if (lb[k0 + t] > 1)
          for (auto& v : pj) v = v * (R)lb[k0 + t];
        make_projt<R>(pj.data(), n, projt);
        bckpj_lin<R>(bcke.data(), &dm[9 * (k0 + t)], projt.data(), n, runs, ldp, ldpnm, nthreads);
      }
    }
    fixedge<R>(bckp.data(), n, runs, mode);
    regularize<R>(bcke.data(), bckp.data(), n, (R)anoise, runs, mode);
    R akden = 0;
    for (const RunS& rn : runs)
      for (int j = rn.l1; j <= rn.l2; ++j) akden = akden + bckp[j - 1] * bcke[j - 1];
    R p = delsq / akden;
    for (const RunS& rn : runs)
      for (int j = rn.l1; j <= rn.l2; ++j) {
        bckn[j - 1] = bckn[j - 1] + p * bckp[j - 1];
        cb[j - 1] = cb[j - 1] - p * bcke[j - 1];
      }
    R err = delsq / bnorm;
    chi2 = chi2 - p * delsq;
    if (logv) { logv[3 * (iter - 1)] = (float)iter; logv[3 * (iter - 1) + 1] = (float)err; logv[3 * (iter - 1) + 2] = (float)chi2; }
    it_done = iter;
    if (std::fabs((double)err) <= errm || std::fabs((double)chi2) <= chim) break;
  }
  if (niter) *niter = it_done;
  for (long i = 0; i < nnn; ++i) vol[i] = (float)bckn[i];
  return 0;
}

}  // namespace

// ============================================================ C ABI =======
// ------------------------------------------- FourierSlice (P1 adjoint) ----
// The central-slice pair on ONELINE's geometry with the weights W dropped
// (no counterpart in the reference).  The slice values T are in the layout
// and sign of the staged spectra the insertion reads (cuFFT R2C of the
// padded, shifted image; ONELINE's BI = conj(T)).  Every tap -- voxel,
// table weight, Hermitian flip and reflected point -- is enumerated exactly
// as oneline() does (oneline.f:38-200), so
//   insert:  X[v] += wg * BTQ (main taps), X[v'] += wg * conj(BTQ) (reflected),
//            BTQ = BI, or conj(BI) for a pixel whose x < 0 was flipped;
//   extract: the real-linear adjoint of insert,
//            BI_adj = sum wg * X[v] + sum wg * conj(X[v']), conj'ed for a
//            flipped pixel, and T = conj(BI_adj).
// visit(I, flipped, q, wg, reflected) for every nonzero tap of row J whose
// signed z index (izp for main taps, -izp for reflected ones) lies in
// [zlo, zhi), as oneline() filters it for the owner-computes schedule.
template <class F>
void oneline_taps(int J, int nx, const float* dm, const KBTable& kb, F&& visit, int zlo = INT_MIN,
                  int zhi = INT_MAX) {
  const int N = 2 * nx, N2 = nx, LN2 = kb.ln2;
  const float fltb = kb.fltb;
  auto idx = [&](int i, int j, int k) { return ((size_t)k * N + j) * (nx + 1) + i; };
  for (int I = 0; I <= N2; ++I) {
    if (!((I * I + J * J) < (N * N / 4) && !(I == 0 && J < 0))) continue;
    float xnew = (float)I * dm[0] + (float)J * dm[3];
    float ynew = (float)I * dm[1] + (float)J * dm[4];
    float znew = (float)I * dm[2] + (float)J * dm[5];
    bool flipped = false;
    if (xnew < 0.0f) { xnew = -xnew; ynew = -ynew; znew = -znew; flipped = true; }
    int ixn = ifix((xnew + 0.5f) + (float)N) - N;
    int iyn = ifix((ynew + 0.5f) + (float)N) - N;
    int izn = ifix((znew + 0.5f) + (float)N) - N;
    if (!(ixn <= (N2 - LN2 - 1) && iyn >= (-N2 + 2 + LN2) && iyn <= (N2 - LN2 - 1) &&
          izn >= (-N2 + 2 + LN2) && izn <= (N2 - LN2 - 1)))
      continue;
    if (!(izn + LN2 >= zlo && izn - LN2 < zhi) && !(ixn < LN2 && -izn + LN2 >= zlo && -izn - LN2 < zhi))
      continue;
    if (ixn >= 0) {
      int lb = -std::min(ixn, LN2);
      for (int lz = -LN2; lz <= LN2; ++lz) {
        int izp = izn + lz, iza = (izp >= 0) ? izp : N + izp;
        if (izp < zlo || izp >= zhi) continue;
        float tz = kb.tab[nint_pos(std::fabs(znew - (float)izp) * fltb)];
        if (tz == 0.0f) continue;
        for (int ly = -LN2; ly <= LN2; ++ly) {
          int iyp = iyn + ly, iya = (iyp >= 0) ? iyp : N + iyp;
          float ty = kb.tab[nint_pos(std::fabs(ynew - (float)iyp) * fltb)] * tz;
          if (ty == 0.0f) continue;
          for (int ixp = lb + ixn; ixp <= LN2 + ixn; ++ixp) {
            float wg = kb.tab[nint_pos(std::fabs(xnew - (float)ixp) * fltb)] * ty;
            if (wg != 0.0f) visit(I, flipped, idx(ixp, iya, iza), wg, false);
          }
        }
      }
    }
    if (ixn < LN2) {
      for (int lz = -LN2; lz <= LN2; ++lz) {
        int izp = izn + lz, izt = (izp > 0) ? N - izp : -izp;
        if (-izp < zlo || -izp >= zhi) continue;
        float tz = kb.tab[nint_pos(std::fabs(znew - (float)izp) * fltb)];
        if (tz == 0.0f) continue;
        for (int ly = -LN2; ly <= LN2; ++ly) {
          int iyp = iyn + ly, iyt = (iyp > 0) ? N - iyp : -iyp;
          float ty = kb.tab[nint_pos(std::fabs(ynew - (float)iyp) * fltb)] * tz;
          if (ty == 0.0f) continue;
          for (int ixp = ixn - LN2; ixp <= -1; ++ixp) {
            float wg = kb.tab[nint_pos(std::fabs(xnew - (float)ixp) * fltb)] * ty;
            if (wg != 0.0f) visit(I, flipped, idx(-ixp, iyt, izt), wg, true);
          }
        }
      }
    }
  }
}

// T [nang][N][nx+1] -> X [N][N][nx+1], FP64, images in order, rows J = -NX+1..NX;
// threads own contiguous ranges of signed z (every voxel's sum in that order)
void fslice_insert(const cd* T, int nx, int nang, const float* dm9, const KBTable& kb, cd* X, int nthreads) {
  const int N = 2 * nx;
  const int nt = std::max(1, std::min(nthreads, 2 * nx - 1));
  #pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num(), T_ = omp_get_num_threads();
    const int zlo = -nx + 1 + (int)((long)(2 * nx - 1) * t / T_);
    const int zhi = -nx + 1 + (int)((long)(2 * nx - 1) * (t + 1) / T_);
    for (int a = 0; a < nang; ++a)
      for (int J = -nx + 1; J <= nx; ++J) {
        const int JP = (J >= 0) ? J : N + J;
        const cd* row = T + ((size_t)a * N + JP) * (nx + 1);
        oneline_taps(
            J, nx, dm9 + 9 * a, kb,
            [&](int I, bool flipped, size_t q, float wg, bool refl) {
              const cd bi = std::conj(row[I]);
              const cd btq = flipped ? std::conj(bi) : bi;
              X[q] += (double)wg * (refl ? std::conj(btq) : btq);
            },
            zlo, zhi);
      }
  }
}

void fslice_extract(const cd* X, int nx, int nang, const float* dm9, const KBTable& kb, cd* T, int nthreads) {
  const int N = 2 * nx;
  #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int a = 0; a < nang; ++a) {
    std::vector<cd> acc(nx + 1);
    std::vector<char> flip(nx + 1);
    for (int J = -nx + 1; J <= nx; ++J) {
      const int JP = (J >= 0) ? J : N + J;
      std::fill(acc.begin(), acc.end(), cd(0, 0));
      std::fill(flip.begin(), flip.end(), 0);
      oneline_taps(J, nx, dm9 + 9 * a, kb, [&](int I, bool flipped, size_t q, float wg, bool refl) {
        acc[I] += (double)wg * (refl ? std::conj(X[q]) : X[q]);
        flip[I] = flipped;
      });
      cd* row = T + ((size_t)a * N + JP) * (nx + 1);
      for (int I = 0; I <= nx; ++I) {
        const cd bi_adj = flip[I] ? std::conj(acc[I]) : acc[I];
        row[I] = std::conj(bi_adj);
      }
    }
  }
}

extern "C" {

// FourierSlice pair in FP64: angles (psi, theta, phi) per slice; complex
// arrays interleaved (re, im).
void orc_fslice_insert(const double* T, int nx, const float* angles, int nang, double* X_out, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  KBTable kb;
  fill_kb(2 * nx, kb);
  std::vector<float> dm((size_t)9 * nang);
  for (int a = 0; a < nang; ++a) cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], &dm[9 * a]);
  const size_t nv = (size_t)(nx + 1) * 4 * nx * nx;
  std::fill(X_out, X_out + 2 * nv, 0.0);
  fslice_insert(reinterpret_cast<const cd*>(T), nx, nang, dm.data(), kb, reinterpret_cast<cd*>(X_out), nthreads);
}

void orc_fslice_extract(const double* X, int nx, const float* angles, int nang, double* T_out, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  KBTable kb;
  fill_kb(2 * nx, kb);
  std::vector<float> dm((size_t)9 * nang);
  for (int a = 0; a < nang; ++a) cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], &dm[9 * a]);
  fslice_extract(reinterpret_cast<const cd*>(X), nx, nang, dm.data(), kb, reinterpret_cast<cd*>(T_out), nthreads);
}

void orc_fillbessil(int n2, float* tab, float* fltb, float* alpha, float* aaaa) {
  KBTable t;
  fill_kb(n2, t);
  std::memcpy(tab, t.tab, sizeof(t.tab));
  *fltb = t.fltb; *alpha = t.alpha; *aaaa = t.aaaa;
}

void orc_windkb_table(int nx, float* out) {
  KBTable t;
  fill_kb(2 * nx, t);
  std::vector<float> w;
  windkb_table(nx, t, w);
  std::memcpy(out, w.data(), w.size() * sizeof(float));
}

void orc_cang(float phi, float theta, float psi, float* dm) { cang(phi, theta, psi, dm); }

// forward (sign=-1) or backward (+1) complex DFT of length n, interleaved re/im
void orc_fft_c2c(const double* in, double* out, int n, int sign) {
  FFT1 f(n, sign);
  f.exec(reinterpret_cast<const cd*>(in), 1, reinterpret_cast<cd*>(out));
}

// One image through PADD2/FFT/phase: bi_out [2nx][nx+1] complex (re,im)
void orc_stage_image(const float* proj, int nx, double* bi_out) {
  FFT1 fx(2 * nx, -1), fy(2 * nx, -1);
  std::vector<std::complex<double>> bi;
  stage_image<double>(proj, nx, bi, fx, fy);
  std::memcpy(bi_out, bi.data(), bi.size() * sizeof(cd));
}

// BP 3F (halt=0: volume; halt=1: BP 3F P partial X,W) and BP 32F (half!=NULL).
// angles: 3 per image (psi, theta, phi, degrees); symang: 3 per symmetry.
int orc_bp3f(const float* imgs, int nx, int nang, const float* angles, const float* symang, int nsym,
             const uint8_t* half, int halt, int prec, float* vol_all, float* vol_1, float* vol_2,
             double* x_out, double* w_out, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (prec == 1)
    return bp_run<double>(imgs, nx, nang, angles, symang, nsym, half, halt, vol_all, vol_1, vol_2, x_out, w_out, nthreads);
  return bp_run<float>(imgs, nx, nang, angles, symang, nsym, half, halt, vol_all, vol_1, vol_2, x_out, w_out, nthreads);
}

// RB 3F (half == NULL) / RB 32F: as orc_bp3f after RTSQ of every image with
// inplane[3*i] = angle (deg), inplane[3*i+1] = x shift, inplane[3*i+2] = y shift
int orc_rb3f(const float* imgs, int nx, int nang, const float* angles, const float* inplane, const uint8_t* half,
             int prec, float* vol_all, float* vol_1, float* vol_2, int nthreads, int fbs) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (prec == 1)
    return bp_run<double>(imgs, nx, nang, angles, nullptr, 0, half, 0, vol_all, vol_1, vol_2, nullptr, nullptr,
                          nthreads, inplane, fbs != 0);
  return bp_run<float>(imgs, nx, nang, angles, nullptr, 0, half, 0, vol_all, vol_1, vol_2, nullptr, nullptr,
                       nthreads, inplane, fbs != 0);
}

// RTSF of one square image (rtsf.f:109-205, SCLI = 1)
void orc_rtsf(const float* in, float* out, int nx, float theta, float shx, float shy) {
  rtsf(in, out, nx, theta, shx, shy);
}

// SYMVOL of a volume with symmetry angle triples (psi, theta, phi)
void orc_symvol(const float* q1, float* q2, int nx, const float* symang, int nsym) {
  std::vector<float> sm((size_t)9 * nsym);
  for (int s = 0; s < nsym; ++s) cang(symang[3 * s + 2], symang[3 * s + 1], symang[3 * s], &sm[9 * s]);
  symvol(q1, q2, nx, sm.data(), nsym);
}

// RTSQ of one image (rtsq.f:56-140)
void orc_rtsq(const float* in, float* out, int nx, int ny, float theta, float shx, float shy) {
  rtsq(in, out, nx, ny, theta, shx, shy);
}

// A BP 32F insertion session: two FP32 grids allocated and zeroed once (as
// BP32FQ does before its image loop, bp32f.f:490-500), then images inserted.
struct BpSession {
  int nx;
  KBTable kb;
  Grid<float> ge, go;
  BpSession(int n) : nx(n), ge(n), go(n) { fill_kb(2 * n, kb); }
};

void* orc_bp_session_open(int nx) { return new BpSession(nx); }
void orc_bp_session_free(void* s) { delete static_cast<BpSession*>(s); }
int orc_bp_session_insert(void* sp, const float* imgs, int nang, const float* angles, const uint8_t* half,
                          int nthreads) {
  BpSession* S = static_cast<BpSession*>(sp);
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  std::vector<float> dm((size_t)9 * nang);
  for (int a = 0; a < nang; ++a) cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], &dm[9 * a]);
  std::vector<Grid<float>*> grids{&S->ge, &S->go};
  std::vector<uint8_t> route(nang);
  for (int a = 0; a < nang; ++a) route[a] = (half && !half[a]) ? 1 : 0;
  insert_images<float>(grids, imgs, S->nx, nang, dm.data(), nullptr, 0, route.data(), S->kb, nthreads);
  return 0;
}

// BP 32F insertion only (PADD2 + FFT + ONELINE into two FP32 grids), the
// timed CPU baseline: with nthreads > 1 it uses the reference's OpenMP row
// striping (LN1 = 6), race included.
int orc_bp_insert_only(const float* imgs, int nx, int nang, const float* angles, const uint8_t* half,
                       int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  KBTable kb;
  fill_kb(2 * nx, kb);
  std::vector<float> dm((size_t)9 * nang);
  for (int a = 0; a < nang; ++a) cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], &dm[9 * a]);
  Grid<float> ge(nx), go(nx);
  std::vector<Grid<float>*> grids{&ge, &go};
  std::vector<uint8_t> route(nang);
  for (int a = 0; a < nang; ++a) route[a] = (half && !half[a]) ? 1 : 0;
  insert_images<float>(grids, imgs, nx, nang, dm.data(), nullptr, 0, route.data(), kb, nthreads);
  return 0;
}

// PJ 3Q: vol (nx,ny,nz x fastest), angles 3 per projection (psi,theta,phi)
void orc_pj3q(const float* vol, int nx, int ny, int nz, float ri, const float* angles, int nang,
              int prec, float* proj_out, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  int ldpx = nx / 2 + 1, ldpy = ny / 2 + 1, ldpz = nz / 2 + 1;
  std::vector<RunC> runs;
  prepcub(nx, ny, nz, ri, ldpx, ldpy, ldpz, runs);
  #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int a = 0; a < nang; ++a) {
    float* out = proj_out + (size_t)a * nx * ny;
    if (prec == 1) {
      std::vector<double> b((size_t)nx * ny);
      wpro_n<double>(b.data(), nx, ny, nz, vol, runs, angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], ri, ldpx, ldpy, ldpz);
      for (size_t i = 0; i < b.size(); ++i) out[i] = (float)b[i];
    } else {
      wpro_n<float>(out, nx, ny, nz, vol, runs, angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], ri, ldpx, ldpy, ldpz);
    }
  }
}

// PJ 3F: PJ 3Q with FBS interpolation (PJ3Q_N(.TRUE.), vtil2.f:222-228,
// writpro_n.f:154-205): FBS3_PREP of the cubic volume, then WPRO_FBS per angle
void orc_pj3f(const float* vol, int n, float ri, const float* angles, int nang, int prec, float* proj_out,
              int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  const int ldp = n / 2 + 1;
  std::vector<RunC> runs;
  prepcub(n, n, n, ri, ldp, ldp, ldp, runs);
  auto go = [&](auto zero) {
    using R = decltype(zero);
    std::vector<R> cube((size_t)n * n * n);
    for (size_t i = 0; i < cube.size(); ++i) cube[i] = (R)vol[i];
    std::vector<R> d[7];
    fbs3_prep<R>(cube.data(), n, d);
    #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int a = 0; a < nang; ++a) {
      std::vector<R> b((size_t)n * n);
      wpro_fbs<R>(b.data(), n, cube.data(), d, runs, angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], ri, ldp);
      float* out = proj_out + (size_t)a * n * n;
      for (size_t i = 0; i < b.size(); ++i) out[i] = (float)b[i];
    }
  };
  if (prec == 1) go(0.0); else go(0.0f);
}

// Number of voxel runs PREPCUB produces (for tests of the run lists)
int orc_prepcub_count(int nx, int ny, int nz, float ri) {
  std::vector<RunC> runs;
  prepcub(nx, ny, nz, ri, nx / 2 + 1, ny / 2 + 1, nz / 2 + 1, runs);
  return (int)runs.size();
}

int orc_bpcg(const float* projs, int n, int nang, const float* angles, float ri, float errm, float chim,
             int maxit, int mode, float lambda, int prec, float* vol, float* logv, int* niter, int* nang_eff,
             double* stats, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (prec == 1)
    return bpcg_run<double>(projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol, logv, niter, nang_eff, stats, nthreads);
  return bpcg_run<float>(projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol, logv, niter, nang_eff, stats, nthreads);
}

// BP CG with FBS interpolation (the 'F' answer, BPCG_3_FBS)
int orc_bpcg_fbs(const float* projs, int n, int nang, const float* angles, float ri, float errm, float chim,
                 int maxit, int mode, float lambda, int prec, float* vol, float* logv, int* niter, int* nang_eff,
                 double* stats, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (prec == 1)
    return bpcg_run<double>(projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol, logv, niter, nang_eff,
                            stats, nthreads, true);
  return bpcg_run<float>(projs, n, nang, angles, ri, errm, chim, maxit, mode, lambda, vol, logv, niter, nang_eff,
                         stats, nthreads, true);
}

// FBS2_PREP + FBS2 at the given points of one n x n image (prec 1: FP64)
void orc_fbs2(const float* img, int n, const float* xy, int npts, int prec, double* out) {
  if (prec == 1) {
    std::vector<double> f(img, img + (size_t)n * n), a, b, c;
    fbs2_prep<double>(f.data(), n, a, b, c);
    for (int p = 0; p < npts; ++p) out[p] = fbs2<double>(xy[2 * p], xy[2 * p + 1], n, f.data(), a.data(), b.data(), c.data());
  } else {
    std::vector<float> f(img, img + (size_t)n * n), a, b, c;
    fbs2_prep<float>(f.data(), n, a, b, c);
    for (int p = 0; p < npts; ++p) out[p] = fbs2<float>(xy[2 * p], xy[2 * p + 1], n, f.data(), a.data(), b.data(), c.data());
  }
}

// FBS3_PREP + FBS3 at the given points of one n^3 volume (FP64)
void orc_fbs3(const float* vol, int n, const float* xyz, int npts, double* out) {
  std::vector<double> f(vol, vol + (size_t)n * n * n);
  std::vector<double> d[7];
  fbs3_prep<double>(f.data(), n, d);
  for (int p = 0; p < npts; ++p) out[p] = fbs3<double>(xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2], n, f.data(), d);
}

// PRJCQ_FBS3 of vol for each (psi, theta, phi) (prec 1: FP64)
void orc_prjcq_fbs3(const float* vol, int n, const float* angles, int nang, int prec, float* proj_out) {
  std::vector<double> f(vol, vol + (size_t)n * n * n);
  std::vector<double> d[7];
  fbs3_prep<double>(f.data(), n, d);
  std::vector<float> ff(vol, vol + (size_t)n * n * n);
  std::vector<float> d32[7];
  if (prec != 1) fbs3_prep<float>(ff.data(), n, d32);
  for (int k = 0; k < nang; ++k) {
    float dm[9];
    cang(angles[3 * k + 2], angles[3 * k + 1], angles[3 * k + 0], dm);
    if (prec == 1) {
      std::vector<double> p((size_t)n * n);
      prjcq_fbs3<double>(f.data(), dm, p.data(), n, d);
      for (size_t i = 0; i < p.size(); ++i) proj_out[(size_t)k * n * n + i] = (float)p[i];
    } else {
      prjcq_fbs3<float>(ff.data(), dm, proj_out + (size_t)k * n * n, n, d32);
    }
  }
}

// Single operator applications, for adjointness and parity tests.
// A (PRJCQ_N) of vol into proj for each angle triple (psi,theta,phi) with DM
// built by CANG; At (BCKPJ_LIN via PROJT) of projections into vol (summed).
void orc_prjcq(const float* vol, int n, float ri, const float* angles, int nang, int prec, float* proj_out) {
  const int ldp = n / 2 + 1;
  std::vector<RunS> runs;
  prepcub_s(n, ri, ldp, runs);
  long nnn = (long)n * n * n;
  for (int a = 0; a < nang; ++a) {
    float dm[9];
    cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], dm);
    if (prec == 1) {
      std::vector<double> c(vol, vol + nnn), p((size_t)n * n, 0.0);
      prjcq_n<double>(c.data(), dm, p.data(), n, runs, ldp, ldp);
      for (size_t i = 0; i < p.size(); ++i) proj_out[(size_t)a * n * n + i] = (float)p[i];
    } else {
      std::vector<float> p((size_t)n * n, 0.0f);
      prjcq_n<float>(vol, dm, p.data(), n, runs, ldp, ldp);
      std::memcpy(proj_out + (size_t)a * n * n, p.data(), p.size() * sizeof(float));
    }
  }
}

void orc_bckpj(const float* projs, int n, float ri, const float* angles, int nang, int prec, float* vol_out) {
  const int ldp = n / 2 + 1;
  std::vector<RunS> runs;
  prepcub_s(n, ri, ldp, runs);
  long nnn = (long)n * n * n;
  if (prec == 1) {
    std::vector<double> c(nnn, 0.0), pj((size_t)n * n), pt;
    for (int a = 0; a < nang; ++a) {
      float dm[9];
      cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], dm);
      for (int i = 0; i < n * n; ++i) pj[i] = projs[(size_t)a * n * n + i];
      make_projt<double>(pj.data(), n, pt);
      bckpj_lin<double>(c.data(), dm, pt.data(), n, runs, ldp, ldp, 1);
    }
    for (long i = 0; i < nnn; ++i) vol_out[i] = (float)c[i];
  } else {
    std::vector<float> c(nnn, 0.0f), pt;
    for (int a = 0; a < nang; ++a) {
      float dm[9];
      cang(angles[3 * a + 2], angles[3 * a + 1], angles[3 * a + 0], dm);
      make_projt<float>(projs + (size_t)a * n * n, n, pt);
      bckpj_lin<float>(c.data(), dm, pt.data(), n, runs, ldp, ldp, 1);
    }
    std::memcpy(vol_out, c.data(), nnn * sizeof(float));
  }
}

// HIANG on angle triples (psi,theta,phi) -> effective (phi,theta) list + LB
int orc_hiang(const float* angles, int nang, float* phi_theta_out, int* lb_out, float* dm_out) {
  std::vector<float> ang((size_t)3 * nang), dm;
  for (int k = 0; k < nang; ++k) { ang[3 * k] = angles[3 * k + 2]; ang[3 * k + 1] = angles[3 * k + 1]; ang[3 * k + 2] = angles[3 * k]; }
  std::vector<int> lb;
  int lo = hiang(ang, nang, dm, lb);
  for (int i = 0; i < lo; ++i) { phi_theta_out[2 * i] = ang[3 * i]; phi_theta_out[2 * i + 1] = ang[3 * i + 1]; lb_out[i] = lb[i]; }
  if (dm_out) std::memcpy(dm_out, dm.data(), dm.size() * sizeof(float));
  return lo;
}

void orc_fixedge(float* p, int n, float ri, int mode) {
  std::vector<RunS> runs;
  prepcub_s(n, ri, n / 2 + 1, runs);
  fixedge<float>(p, n, runs, mode);
}

int orc_prepcub_s_count(int n, float ri) {
  std::vector<RunS> runs;
  prepcub_s(n, ri, n / 2 + 1, runs);
  return (int)runs.size();
}

}  // extern "C"
