// Host-side filter taps. Compiled with -ffp-contract=off: every f64 operation
// rounds on its own, as in VISAR's Zig (no contraction).
#include <cmath>
#include <cstdint>
#include <cstring>

#include "vb.h"

namespace vb {

namespace {

// 2^(i/64), i = 0..63, correctly rounded to f64 (the table of OpenCV's
// softfloat f64 exp that VISAR restates at src/imgproc/filter.zig:353-375).
const double kExp2Tab[64] = {
    0x1.0000000000000p+0, 0x1.02c9a3e778061p+0, 0x1.059b0d3158574p+0, 0x1.0874518759bc8p+0,
    0x1.0b5586cf9890fp+0, 0x1.0e3ec32d3d1a2p+0, 0x1.11301d0125b51p+0, 0x1.1429aaea92de0p+0,
    0x1.172b83c7d517bp+0, 0x1.1a35beb6fcb75p+0, 0x1.1d4873168b9aap+0, 0x1.2063b88628cd6p+0,
    0x1.2387a6e756238p+0, 0x1.26b4565e27cddp+0, 0x1.29e9df51fdee1p+0, 0x1.2d285a6e4030bp+0,
    0x1.306fe0a31b715p+0, 0x1.33c08b26416ffp+0, 0x1.371a7373aa9cbp+0, 0x1.3a7db34e59ff7p+0,
    0x1.3dea64c123422p+0, 0x1.4160a21f72e2ap+0, 0x1.44e086061892dp+0, 0x1.486a2b5c13cd0p+0,
    0x1.4bfdad5362a27p+0, 0x1.4f9b2769d2ca7p+0, 0x1.5342b569d4f82p+0, 0x1.56f4736b527dap+0,
    0x1.5ab07dd485429p+0, 0x1.5e76f15ad2148p+0, 0x1.6247eb03a5585p+0, 0x1.6623882552225p+0,
    0x1.6a09e667f3bcdp+0, 0x1.6dfb23c651a2fp+0, 0x1.71f75e8ec5f74p+0, 0x1.75feb564267c9p+0,
    0x1.7a11473eb0187p+0, 0x1.7e2f336cf4e62p+0, 0x1.82589994cce13p+0, 0x1.868d99b4492edp+0,
    0x1.8ace5422aa0dbp+0, 0x1.8f1ae99157736p+0, 0x1.93737b0cdc5e5p+0, 0x1.97d829fde4e50p+0,
    0x1.9c49182a3f090p+0, 0x1.a0c667b5de565p+0, 0x1.a5503b23e255dp+0, 0x1.a9e6b5579fdbfp+0,
    0x1.ae89f995ad3adp+0, 0x1.b33a2b84f15fbp+0, 0x1.b7f76f2fb5e47p+0, 0x1.bcc1e904bc1d2p+0,
    0x1.c199bdd85529cp+0, 0x1.c67f12e57d14bp+0, 0x1.cb720dcef9069p+0, 0x1.d072d4a07897cp+0,
    0x1.d5818dcfba487p+0, 0x1.da9e603db3285p+0, 0x1.dfc97337b9b5fp+0, 0x1.e502ee78b3ff6p+0,
    0x1.ea4afa2a490dap+0, 0x1.efa1bee615a27p+0, 0x1.f50765b6e4540p+0, 0x1.fa7c1819e90d8p+0,
};

// rint by the magic-number trick (src/core/saturate.zig:8-17); exact for |x| < 2^51.
inline double rint_magic(double x) {
  volatile double m = 6755399441055744.0;  // keep the add/sub pair
  return (x + m) - m;
}

// OpenCV's softfloat f64 exp as restated at src/imgproc/filter.zig:350-399:
// x * 64/ln2 split into an integer part (table index and exponent) and a
// fraction evaluated by a degree-5 polynomial, every step one IEEE f64 op.
// It is not correctly rounded, which is why std exp() cannot stand in.
double cv_exp(double x) {
  if (std::isnan(x)) return x;
  if (std::isinf(x)) return x > 0 ? x : 0.0;
  const double a0 = 0x1.3ce0f3e46f431p-7;
  const double p5 = 1.0 / a0;
  const double p4 = 0x1.62e42fefa39f1p-1 / a0;
  const double p3 = 0x1.ebfbdff82a45ap-3 / a0;
  const double p2 = 0x1.c6b08d81fec75p-5 / a0;
  const double p1 = 0x1.3b2a72b4f3cd3p-7 / a0;
  const double p0 = 0x1.5e7aa1566c2a4p-10 / a0;
  const double prescale = 0x1.71547652b82fep+0 * 64.0;
  const double max_val = 3000.0 * 64.0;
  uint64_t bits;
  std::memcpy(&bits, &x, 8);
  double x0 = (((bits >> 52) & 0x7ff) > 1023 + 10) ? (x < 0 ? -max_val : max_val) : x * prescale;
  const double r = rint_magic(x0);
  const int v = (int)r;
  long long e = (long long)(v >> 6) + 1023;
  if (e < 0) e = 0;
  if (e > 2047) e = 2047;
  const uint64_t tb = (uint64_t)e << 52;
  double buf;
  std::memcpy(&buf, &tb, 8);
  x0 = (x0 - r) * (1.0 / 64.0);
  const double poly = ((((p0 * x0 + p1) * x0 + p2) * x0 + p3) * x0 + p4) * x0 + p5;
  return buf * a0 * kExp2Tab[v & 63] * poly;
}

}  // namespace

// getGaussianKernelBitExact (src/imgproc/filter.zig:407-443): binomial tables
// for sigma <= 0 and n <= 9, else exp(-x^2/(2 sigma^2)) normalised by the
// reciprocal of the sum.
void gaussian_kernel(double *out, int n, double sigma) {
  static const double s1[] = {1.0};
  static const double s3[] = {0.25, 0.5, 0.25};
  static const double s5[] = {0.0625, 0.25, 0.375, 0.25, 0.0625};
  static const double s7[] = {0.03125, 0.109375, 0.21875, 0.28125, 0.21875, 0.109375, 0.03125};
  static const double s9[] = {4.0 / 256, 13.0 / 256, 30.0 / 256, 51.0 / 256, 60.0 / 256,
                              51.0 / 256, 30.0 / 256, 13.0 / 256, 4.0 / 256};
  static const double *small[] = {s1, s3, s5, s7, s9};
  if (n % 2 == 1 && n <= 9 && sigma <= 0) {
    std::memcpy(out, small[n / 2], sizeof(double) * n);
    return;
  }
  const double nf = (double)n;
  const double sx = sigma > 0 ? sigma : std::fma(nf, 0.15, 0.35);
  const double scale2x = -0.125 / (sx * sx);
  const int half = (n - 1) / 2;
  double sum = 0;
  long long x = 1 - (long long)n;
  for (int i = 0; i < half; i++) {
    const double t = cv_exp((double)(x * x) * scale2x);
    out[i] = t;
    sum += t;
    x += 2;
  }
  sum = sum * 2 + 1;
  if (n % 2 == 0) sum += 1;
  const double mul1 = 1.0 / sum;
  for (int i = 0; i < half; i++) {
    out[i] *= mul1;
    out[n - 1 - i] = out[i];
  }
  out[half] = mul1;
  if (n % 2 == 0) out[half + 1] = mul1;
}

// OpenCV's automatic kernel size (src/imgproc/filter.zig:447-451).
int gaussian_ksize(double sigma, bool depth_is_u8) {
  const double k = depth_is_u8 ? 3 : 4;
  const double r = std::round(sigma * k * 2 + 1);
  if (!(r >= 0) || r > 1e6) return -1;  // VISAR casts to u32; such sigmas are invalid kernels
  return (int)((unsigned)r | 1u);
}

// getGaussianKernelFixedPoint_ED (src/imgproc/filter.zig:458-476): the half
// kernel quantised to `bits` fractional bits from the edge inwards, each
// rounding error carried into the next tap; the centre takes the remainder.
void gaussian_kernel_fixed(int64_t *out, int n, double sigma, int bits) {
  double k[128];
  gaussian_kernel(k, n, sigma);
  const double m = (double)(1ULL << bits);
  double err = 0;
  uint64_t sum = 0;
  for (int i = 0; i < n / 2; i++) {
    const double a = k[i] * m + err;
    const double v = rint_magic(a);
    err = a - v;
    const uint64_t q = (uint64_t)(v > 0 ? v : 0.0);
    out[i] = (int64_t)q;
    out[n - 1 - i] = (int64_t)q;
    sum += q;
  }
  out[n / 2] = (int64_t)((1ULL << bits) - 2 * sum);
}

// getDerivKernels (src/imgproc/filter.zig:817-854).
bool deriv_kernel(int *out, int n, int order, int ksize) {
  if (ksize == -1) {
    if (n != 3 || order > 1) return false;
    if (order == 0) {
      out[0] = 3; out[1] = 10; out[2] = 3;
    } else {
      out[0] = -1; out[1] = 0; out[2] = 1;
    }
    return true;
  }
  const int want = ksize == 1 ? 3 : ksize;
  if (n != want) return false;
  if (ksize == 1 && order == 0) {
    out[0] = 0; out[1] = 1; out[2] = 0;
    return true;
  }
  if (order >= n) return false;
  int a[33] = {0};
  a[0] = 1;
  int len = 1;
  for (int it = 0; it < n - order - 1; it++) {
    int b[33] = {0};
    for (int j = 0; j < len; j++) {
      b[j] += a[j];
      b[j + 1] += a[j];
    }
    std::memcpy(a, b, sizeof(a));
    len++;
  }
  for (int it = 0; it < order; it++) {
    int b[33] = {0};
    for (int j = 0; j < len; j++) {
      b[j] -= a[j];
      b[j + 1] += a[j];
    }
    std::memcpy(a, b, sizeof(a));
    len++;
  }
  std::memcpy(out, a, sizeof(int) * n);
  return true;
}

}  // namespace vb
