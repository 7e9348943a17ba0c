// Host-side constant tables and rotation matrices.  Compiled with
// -ffp-contract=off so that single-precision expressions round exactly as
// the Fortran statements they restate; the GPU kernels receive these tables
// unchanged, so every interpolation weight is bit-identical to the CPU form.
#include "common.h"

#include <cmath>
#include <cstdarg>
#include <cstring>

namespace spi {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

const char* last_error_cstr() { return g_last_error.c_str(); }

// Modified Bessel function I1 by its power series sum_k (x/2)^(2k+1)/(k!(k+1)!),
// accurate to double rounding for the arguments used here (0 <= x <= 6.5).
static double bessel_i1_series(double x) {
  double t = 0.5 * x, t2 = t * t, term = t, sum = t;
  for (int k = 1; k < 100; ++k) {
    term *= t2 / ((double)k * (double)(k + 1));
    sum += term;
    if (term < 1e-19 * sum) break;
  }
  return sum;
}

// Generalised Kaiser-Bessel table of FILLBESSIL (fillbessi0.f:88-125):
// LN = 5, LN2 = 2, V = 2/N2, ALPHA = 6.5, AAAA = 0.9 V, FLTB = 4999/3,
// TABI(i) = sqrt(alpha x) I1(alpha x) / (sqrt(alpha) I1(alpha)),
// x = sqrt(1 - (s/AAAA)^2), s = i/FLTB/N2, zero beyond AAAA.
void fill_kb(int n2, KBTab& t) {
  const int ltab = 4999, ln = 5;
  t.ln2 = ln / 2;
  float v = (float)(ln - 1) / 2.0f / (float)n2;
  t.alpha = 6.5f;
  t.aaaa = 0.9f * v;
  float b0 = std::sqrt(t.alpha) * (float)bessel_i1_series((double)t.alpha);
  t.fltb = (float)ltab / (float)(t.ln2 + 1);
  for (int i = 0; i <= ltab; ++i) {
    float s = (float)i / t.fltb / (float)n2;
    if (s <= t.aaaa) {
      float q = s / t.aaaa;
      float x = std::sqrt(1.0f - q * q);
      float ax = t.alpha * x;
      t.tab[i] = std::sqrt(ax) * (float)bessel_i1_series((double)ax) / b0;
    } else {
      t.tab[i] = 0.0f;
    }
  }
}

// I_nu(x)/x^nu and J_nu(x)/x^nu from the hypergeometric series
// 2^-nu sum_k (+-x^2/4)^k / (k! Gamma(nu+k+1)).
static double inu_scaled(double x, double nu) {
  double q = 0.25 * x * x, term = 1.0 / std::tgamma(nu + 1.0), s = term;
  for (int k = 1; k < 300; ++k) {
    term *= q / ((double)k * (nu + (double)k));
    s += term;
    if (term < 1e-19 * s) break;
  }
  return s * std::pow(2.0, -nu);
}
static double jnu_scaled(double x, double nu) {
  double q = -0.25 * x * x, term = 1.0 / std::tgamma(nu + 1.0), s = term;
  for (int k = 1; k < 400; ++k) {
    term *= q / ((double)k * (nu + (double)k));
    s += term;
    if (std::fabs(term) < 1e-19 * std::fabs(s)) break;
  }
  return s * std::pow(2.0, -nu);
}

// |WKB| of WINDKB2A (bp32f.f:964-1005) for every integer squared radius
// LR = 0..(nx/2)^2: nu = NNN/2 = 1.5, QRT = (2 pi AAAA)^2 in REAL,
// SIGMA = QRT*LR - ALPHA^2; WKB = WKB0 * (I or J)_nu(sqrt|SIGMA|)/sqrt|SIGMA|^nu
// with WKB0 = ALPHA^nu / I_nu(ALPHA); WKB = 1 when |SIGMA| < 1e-7.
void windkb_table(int nx, const KBTab& kb, std::vector<float>& wkb) {
  const float quadpi = 3.14159265358979323846f;
  const float twopi = 2.0f * quadpi;
  const int l2 = (nx / 2) * (nx / 2);
  const double nu = 1.5;
  const float alpha = kb.alpha;
  const double wkb0 = 1.0 / inu_scaled((double)alpha, nu);
  const float qrt = (twopi * kb.aaaa) * (twopi * kb.aaaa);
  wkb.assign(l2 + 1, 1.0f);
  for (int lr = 0; lr <= l2; ++lr) {
    float sigma = qrt * (float)lr - alpha * alpha;
    double w;
    if (std::fabs(sigma) < 1.0e-7f) w = 1.0;
    else if (sigma > 0.0f) w = wkb0 * jnu_scaled(std::sqrt((double)sigma), nu);
    else w = wkb0 * inu_scaled(std::sqrt((double)std::fabs(sigma)), nu);
    wkb[lr] = (float)std::fabs(w);
  }
}

// Euler angles to rotation matrix, CANG (cang.f:44-81).  The reference's
// QUADPI literal is a default-REAL constant, so pi enters rounded to single
// precision before the double-precision trigonometry.
static void euler_dm(float phi, float theta, float psi, float* dm) {
  const double quadpi = (double)3.14159265358979323846f;
  const double d2r = quadpi / 180.0;
  const double cphi = std::cos((double)phi * d2r), sphi = std::sin((double)phi * d2r);
  const double cthe = std::cos((double)theta * d2r), sthe = std::sin((double)theta * d2r);
  const double cpsi = std::cos((double)psi * d2r), spsi = std::sin((double)psi * d2r);
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

void cang(float phi, float theta, float psi, float* dm9) { euler_dm(phi, theta, psi, dm9); }

// WPRO_N builds the same matrix inline (wpro_n.f:65-81)
void cang_pj(float phi, float theta, float psi, float* dm9) { euler_dm(phi, theta, psi, dm9); }

// MATMUL(SM, DM) for column-major 3x3 REAL matrices, k summed 1..3 in order
void matmul33(const float* sm, const float* dm, float* out) {
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      float s = sm[i] * dm[3 * j];
      s = s + sm[i + 3] * dm[1 + 3 * j];
      s = s + sm[i + 6] * dm[2 + 3 * j];
      out[i + 3 * j] = s;
    }
}

}  // namespace spi
