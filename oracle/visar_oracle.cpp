// ORACLE -- test infrastructure only. A CPU restatement of VISAR's imgproc
// stencil-and-warp path (the Zig sources under src/core and src/imgproc of
// VISAR), used by tests/, the smoke check and bench.py's CPU baseline to
// check and time the CUDA library. Nothing in the product links or calls it.
//
// It follows the Zig code path by path, including VISAR's dispatch between
// specialised and generic kernels, its accumulator types, its operation
// order for f32 (16-lane vector bodies vs scalar row tails) and its
// finishing/rounding steps. Where VISAR's own unit tests prove a SIMD fast
// path equal to a scalar definition (color.zig:596-681 HSV/gray/YCrCb,
// resize.zig:654-743 resize fast paths, morph.zig:595-670 run decomposition,
// filter.zig:960-986 box windows), the scalar definition is restated.
//
// Rows are spread over std::thread workers like Exec.parallelFor
// (src/core/pool.zig:31-39).
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off: no fused multiply-adds
// except where VISAR writes @mulAdd, which is std::fma here).
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <thread>
#include <type_traits>
#include <vector>

#include "../include/visar.h"

namespace {

// ------------------------------------------------------------ threading

int g_threads = 0;

int nthreads() {
  if (g_threads > 0) return g_threads;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// Exec.parallelFor: chunks of at least `grain` rows, up to 4 x threads chunks,
// claimed dynamically.
void parallel_for(size_t n, size_t grain, const std::function<void(size_t, size_t)> &f) {
  if (n == 0) return;
  const int t = nthreads();
  const size_t max_chunks = std::max<size_t>(1, n / std::max<size_t>(1, grain));
  const size_t chunks = std::min<size_t>(max_chunks, (size_t)t * 4);
  if (chunks <= 1 || t <= 1) {
    f(0, n);
    return;
  }
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (;;) {
      const size_t c = next.fetch_add(1);
      if (c >= chunks) return;
      f(n * c / chunks, n * (c + 1) / chunks);
    }
  };
  std::vector<std::thread> ws;
  const int nw = (int)std::min<size_t>((size_t)t - 1, chunks - 1);
  for (int i = 0; i < nw; i++) ws.emplace_back(work);
  work();
  for (auto &w : ws) w.join();
}

// ----------------------------------------------------------- saturation

// sat.rint (src/core/saturate.zig:8-17): (x + m) - m.
inline double rint_d(double x) {
  volatile double m = 6755399441055744.0;
  return (x + m) - m;
}
inline float rint_f(float x) {
  volatile float m = 12582912.0f;
  return (x + m) - m;
}

template <class T> struct Lim {
  static constexpr double lo = (double)std::numeric_limits<T>::lowest();
  static constexpr double hi = (double)std::numeric_limits<T>::max();
};

template <class D> constexpr bool is_float() { return std::is_floating_point<D>::value; }

// sat.cast(D, x) (saturate.zig:20-49).
template <class D, class S>
D cast(S x) {
  if constexpr (std::is_same<S, D>::value) {
    return x;
  } else if constexpr (is_float<D>()) {
    return (D)x;
  } else if constexpr (is_float<S>()) {
    if (std::isnan(x)) return 0;
    const double r = rint_d((double)x);
    if (r <= Lim<D>::lo) return (D)Lim<D>::lo;
    if (r >= Lim<D>::hi) return (D)Lim<D>::hi;
    return (D)(long long)r;
  } else {
    const long long v = (long long)x;
    if (v < (long long)Lim<D>::lo) return (D)Lim<D>::lo;
    if (v > (long long)Lim<D>::hi) return (D)Lim<D>::hi;
    return (D)v;
  }
}

// satV (src/imgproc/filter.zig:44-58).
template <class D, class S>
D satv(S v) {
  if constexpr (std::is_same<S, D>::value) {
    return v;
  } else if constexpr (is_float<D>()) {
    return (D)v;
  } else if constexpr (is_float<S>()) {
    float r = rint_f((float)v);
    // @min(@max(r, lo), hi): a NaN takes the low bound.
    float c = std::isnan(r) ? (float)Lim<D>::lo : std::min(std::max(r, (float)Lim<D>::lo), (float)Lim<D>::hi);
    return (D)(long long)c;
  } else {
    long long w = (long long)v;
    return (D)std::min(std::max(w, (long long)Lim<D>::lo), (long long)Lim<D>::hi);
  }
}

// ---------------------------------------------------------------- images

template <class T>
struct Img {
  int w, h, cn;
  size_t stride;  // elements
  T *data;
  T *row(size_t y) const { return data + y * stride; }
  size_t row_len() const { return (size_t)w * cn; }
};

struct Error {
  int status;
  const char *name;
};

[[noreturn]] void fail(int st, const char *n) { throw Error{st, n}; }

template <class T>
Img<T> typed(const visar_image *c, int depth) {
  if (!c || !c->data) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  if ((int)c->depth != depth) fail(VISAR_UNSUPPORTED, "Unsupported");
  if (c->channels == 0 || c->channels > 512) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  if (c->stride % sizeof(T) != 0) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  if (c->width == 0 || c->height == 0) fail(VISAR_INVALID_ARGUMENT, "InvalidSize");
  const size_t stride = c->stride / sizeof(T);
  if (stride < (size_t)c->width * c->channels) fail(VISAR_INVALID_ARGUMENT, "InvalidSize");
  return Img<T>{(int)c->width, (int)c->height, (int)c->channels, stride, static_cast<T *>(c->data)};
}

template <class T>
Img<T> alloc_like(std::vector<T> &buf, int w, int h, int cn) {
  buf.assign((size_t)w * h * cn, T(0));
  return Img<T>{w, h, cn, (size_t)w * cn, buf.data()};
}

template <class T>
void copy_img(const Img<T> &s, const Img<T> &d) {
  for (int y = 0; y < s.h; y++) std::memcpy(d.row(y), s.row(y), s.row_len() * sizeof(T));
}

// --------------------------------------------------------------- border

// border.map (src/imgproc/border.zig:22-37), with VISAR's reflection loop.
long long border_map(long long p, long long n, int border) {
  if (p >= 0 && p < n) return p;
  switch (border) {
    case 0: return -1;
    case 1: return p < 0 ? 0 : n - 1;
    case 2:
    case 4: {
      if (n == 1) return 0;
      const long long delta = border == 4 ? 1 : 0;
      long long q = p;
      while (q < 0 || q >= n) {
        if (q < 0) q = -q - 1 + delta;
        else q = n - 1 - (q - n) - delta;
      }
      return q;
    }
    case 3: {
      long long q = p % n;
      if (q < 0) q += n;
      return q;
    }
  }
  return -1;
}

// =============================================================== cvtColor

constexpr int kGrayShift = 15, R2G = 9798, G2G = 19235, B2G = 3735;
constexpr int kShift = 14, R2Y = 4899, G2Y = 9617, B2Y = 1868;
constexpr int kHsvShift = 12;

struct HsvTables {
  int sdiv[256], hdiv[256];
  HsvTables() {
    sdiv[0] = hdiv[0] = 0;
    for (int i = 1; i < 256; i++) {
      sdiv[i] = (int)std::round((double)(255 << kHsvShift) / (double)i);
      hdiv[i] = (int)std::round((double)(180 << kHsvShift) / (6.0 * (double)i));
    }
  }
};
const HsvTables &hsv_tables() {
  static HsvTables t;
  return t;
}

enum Kind { kReorder, kGray, kFromGray, kHsv, kFromHsv, kYcrcb, kFromYcrcb };
struct CInfo {
  int scn, dcn, sb, db;
  Kind kind;
};

bool color_info(int code, CInfo &ci) {
  switch (code) {
    case 0: ci = {3, 4, 0, 0, kReorder}; return true;
    case 1: ci = {4, 3, 0, 0, kReorder}; return true;
    case 2: ci = {3, 4, 0, 2, kReorder}; return true;
    case 3: ci = {4, 3, 0, 2, kReorder}; return true;
    case 4: ci = {3, 3, 0, 2, kReorder}; return true;
    case 5: ci = {4, 4, 0, 2, kReorder}; return true;
    case 6: ci = {3, 1, 0, 0, kGray}; return true;
    case 7: ci = {3, 1, 2, 0, kGray}; return true;
    case 8: ci = {1, 3, 0, 0, kFromGray}; return true;
    case 9: ci = {1, 4, 0, 0, kFromGray}; return true;
    case 10: ci = {4, 1, 0, 0, kGray}; return true;
    case 11: ci = {4, 1, 2, 0, kGray}; return true;
    case 36: ci = {3, 3, 0, 0, kYcrcb}; return true;
    case 37: ci = {3, 3, 2, 0, kYcrcb}; return true;
    case 38: ci = {3, 3, 0, 0, kFromYcrcb}; return true;
    case 39: ci = {3, 3, 0, 2, kFromYcrcb}; return true;
    case 40: ci = {3, 3, 0, 0, kHsv}; return true;
    case 41: ci = {3, 3, 2, 0, kHsv}; return true;
    case 54: ci = {3, 3, 0, 0, kFromHsv}; return true;
    case 55: ci = {3, 3, 0, 2, kFromHsv}; return true;
  }
  return false;
}

// hsv2rgbF32 (color.zig:550-569).
void hsv2rgb(float h_in, float hscale, float s, float v, float out[3]) {
  if (s == 0) {
    out[0] = out[1] = out[2] = v;
    return;
  }
  float h = h_in * hscale;
  while (h < 0) h += 6;
  while (h >= 6) h -= 6;
  int sector = (int)std::floor(h);
  h -= (float)sector;
  if (sector < 0 || sector >= 6) {
    sector = 0;
    h = 0;
  }
  const float tab[4] = {v, v * (1 - s), v * std::fma(-s, h, 1.0f), v * std::fma(-s, 1 - h, 1.0f)};
  static const unsigned char sd[6][3] = {{1, 3, 0}, {1, 0, 2}, {3, 0, 1}, {0, 2, 1}, {0, 1, 3}, {2, 1, 0}};
  out[0] = tab[sd[sector][2]];
  out[1] = tab[sd[sector][1]];
  out[2] = tab[sd[sector][0]];
}

template <class T>
void convert_px(const CInfo &inf, const T *p, T *o) {
  const T alpha = is_float<T>() ? T(1) : T(std::numeric_limits<T>::max());
  switch (inf.kind) {
    case kReorder: {
      const bool swap = inf.sb != inf.db;
      if (swap) {
        o[0] = p[2]; o[1] = p[1]; o[2] = p[0];
      } else {
        o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
      }
      if (inf.dcn == 4) o[3] = inf.scn == 4 ? p[3] : alpha;
      break;
    }
    case kGray: {
      const int bi = inf.sb, ri = 2 - inf.sb;
      if constexpr (is_float<T>()) {
        o[0] = (float)p[bi] * 0.114f + (float)p[1] * 0.587f + (float)p[ri] * 0.299f;
      } else {
        const uint32_t y = ((uint32_t)p[bi] * B2G + (uint32_t)p[1] * G2G + (uint32_t)p[ri] * R2G + (1u << (kGrayShift - 1))) >> kGrayShift;
        o[0] = (T)y;
      }
      break;
    }
    case kFromGray: {
      o[0] = o[1] = o[2] = p[0];
      if (inf.dcn == 4) o[3] = alpha;
      break;
    }
    case kYcrcb: {
      if constexpr (is_float<T>()) {
        const float b = p[inf.sb], g = p[1], r = p[2 - inf.sb];
        const float y = b * 0.114f + g * 0.587f + r * 0.299f;
        o[0] = y;
        o[1] = (r - y) * 0.713f + 0.5f;
        o[2] = (b - y) * 0.564f + 0.5f;
      } else {
        const int b = p[inf.sb], g = p[1], r = p[2 - inf.sb];
        const int y = (b * B2Y + g * G2Y + r * R2Y + (1 << (kShift - 1))) >> kShift;
        const int delta = 128 << kShift;
        o[0] = cast<T>(y);
        o[1] = cast<T>(((r - y) * 11682 + delta + (1 << (kShift - 1))) >> kShift);
        o[2] = cast<T>(((b - y) * 9241 + delta + (1 << (kShift - 1))) >> kShift);
      }
      break;
    }
    case kFromYcrcb: {
      if constexpr (is_float<T>()) {
        const float y = p[0], cr = p[1] - 0.5f, cb = p[2] - 0.5f;
        o[inf.db] = y + cb * 1.773f;
        o[1] = y + cb * -0.344f + cr * -0.714f;
        o[2 - inf.db] = y + cr * 1.403f;
      } else {
        const int y = p[0], cr = (int)p[1] - 128, cb = (int)p[2] - 128;
        const int half = 1 << (kShift - 1);
        o[inf.db] = cast<T>(y + ((cb * 29049 + half) >> kShift));
        o[1] = cast<T>(y + ((cb * -5636 + cr * -11698 + half) >> kShift));
        o[2 - inf.db] = cast<T>(y + ((cr * 22987 + half) >> kShift));
      }
      break;
    }
    case kHsv: {
      if constexpr (is_float<T>()) {
        // rgb2hsvF32 (color.zig:534-546)
        const float b = p[inf.sb], g = p[1], r = p[2 - inf.sb];
        const float eps = std::numeric_limits<float>::epsilon();
        const float v = std::max(std::max(r, g), b);
        const float vmin = std::min(std::min(r, g), b);
        float diff = v - vmin;
        const float s = diff / (std::fabs(v) + eps);
        diff = 60.0f / (diff + eps);
        float h = v == r ? (g - b) * diff : v == g ? (b - r) * diff + 120.0f : (r - g) * diff + 240.0f;
        if (h < 0) h += 360.0f;
        o[0] = h; o[1] = s; o[2] = v;
      } else {
        // rgb2hsvU8 (color.zig:515-532)
        const HsvTables &t = hsv_tables();
        const int b = p[inf.sb], g = p[1], r = p[2 - inf.sb];
        const int v = std::max(std::max(r, g), b);
        const int vmin = std::min(std::min(r, g), b);
        const int diff = v - vmin;
        const int vr = v == r ? -1 : 0, vg = v == g ? -1 : 0;
        const int half = 1 << (kHsvShift - 1);
        const int s = (diff * t.sdiv[v] + half) >> kHsvShift;
        int h = (vr & (g - b)) + (~vr & ((vg & (b - r + 2 * diff)) + ((~vg) & (r - g + 4 * diff))));
        h = (h * t.hdiv[diff] + half) >> kHsvShift;
        if (h < 0) h += 180;
        o[0] = cast<T>(h);
        o[1] = (T)s;
        o[2] = (T)v;
      }
      break;
    }
    case kFromHsv: {
      float rgb[3];
      if constexpr (is_float<T>()) {
        hsv2rgb(p[0], (float)(6.0 / 360.0), p[1], p[2], rgb);
        o[inf.db] = rgb[2]; o[1] = rgb[1]; o[2 - inf.db] = rgb[0];
      } else {
        hsv2rgb((float)p[0], (float)(6.0 / 180.0), (float)p[1] * (float)(1.0 / 255.0), (float)p[2] * (float)(1.0 / 255.0), rgb);
        auto tr = [](float x) -> T { return (T)std::min(std::max(std::trunc(x), 0.0f), 255.0f); };
        o[inf.db] = tr(rgb[2] * 255.0f);
        o[1] = tr(rgb[1] * 255.0f);
        o[2 - inf.db] = tr(rgb[0] * 255.0f);
      }
      break;
    }
  }
}

bool color_supported(int depth, Kind k) {
  switch (k) {
    case kReorder: case kFromGray: return true;
    case kGray: return depth == 0 || depth == 2 || depth == 5;
    default: return depth == 0 || depth == 5;
  }
}

template <class T>
void cvt_color_t(const visar_image *src, const visar_image *dst, const CInfo &ci, int depth) {
  Img<T> s = typed<T>(src, depth);
  Img<T> d = typed<T>(dst, depth);
  if (s.w != d.w || s.h != d.h) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  if (s.cn != ci.scn || d.cn != ci.dcn) fail(VISAR_UNSUPPORTED, "UnsupportedChannels");
  if (!color_supported(depth, ci.kind)) fail(VISAR_UNSUPPORTED, "Unsupported");
  parallel_for(s.h, std::max(1, (1 << 15) / s.w), [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++)
      for (int x = 0; x < s.w; x++) convert_px<T>(ci, s.row(y) + (size_t)x * ci.scn, d.row(y) + (size_t)x * ci.dcn);
  });
}

// ============================================================== filtering

// cvExp (filter.zig:350-399): OpenCV's softfloat f64 exp. The 2^(i/64) table
// is the correctly rounded one; the polynomial constants are softfloat's.
double cv_exp(double x) {
  static double tab[64];
  static bool init = [] {
    // 2^(i/64) correctly rounded: computed in long double and checked
    // against its neighbours would still risk a misrounding, so the exact
    // values are listed (hex floats).
    static const double t[64] = {
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
    std::memcpy(tab, t, sizeof(t));
    return true;
  }();
  (void)init;
  if (std::isnan(x)) return x;
  if (std::isinf(x)) return x > 0 ? x : 0;
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
  double x0 = ((bits >> 52) & 0x7ff) > 1023 + 10 ? (x < 0 ? -max_val : max_val) : x * prescale;
  const double r = rint_d(x0);
  const int v = (int)r;
  const long long e = std::min<long long>(std::max<long long>((long long)(v >> 6) + 1023, 0), 2047);
  const uint64_t tb = (uint64_t)e << 52;
  double buf;
  std::memcpy(&buf, &tb, 8);
  x0 = (x0 - r) * (1.0 / 64.0);
  const double poly = ((((p0 * x0 + p1) * x0 + p2) * x0 + p3) * x0 + p4) * x0 + p5;
  return buf * a0 * tab[v & 63] * poly;
}

// gaussianKernel (filter.zig:407-443).
void gaussian_kernel(double *out, int n, double sigma) {
  static const std::vector<std::vector<double>> small = {
      {1.0},
      {0.25, 0.5, 0.25},
      {0.0625, 0.25, 0.375, 0.25, 0.0625},
      {0.03125, 0.109375, 0.21875, 0.28125, 0.21875, 0.109375, 0.03125},
      {4.0 / 256.0, 13.0 / 256.0, 30.0 / 256.0, 51.0 / 256.0, 60.0 / 256.0, 51.0 / 256.0, 30.0 / 256.0, 13.0 / 256.0, 4.0 / 256.0},
  };
  if (n % 2 == 1 && n <= 9 && sigma <= 0) {
    for (int i = 0; i < n; i++) out[i] = small[n / 2][i];
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

int gaussian_ksize(double sigma, bool u8) {
  const double k = u8 ? 3 : 4;
  const double r = std::round(sigma * k * 2 + 1);
  if (!(r >= 0) || r > 1e6) return -1;
  return (int)((uint32_t)r | 1u);
}

// gaussianKernelFixed (filter.zig:458-476).
template <class K>
void gaussian_kernel_fixed(K *out, int n, double sigma, int bits) {
  double tmp[128];
  gaussian_kernel(tmp, n, sigma);
  const double m = (double)(1ULL << bits);
  double err = 0;
  uint64_t sum = 0;
  for (int i = 0; i < n / 2; i++) {
    const double a = tmp[i] * m + err;
    const double v = rint_d(a);
    err = a - v;
    const uint64_t q = (uint64_t)std::max(v, 0.0);
    out[i] = (K)q;
    out[n - 1 - i] = (K)q;
    sum += q;
  }
  out[n / 2] = (K)((1ULL << bits) - 2 * sum);
}

// reduce (filter.zig:96-109).
template <class K>
void reduce(std::vector<K> &k, int &shift, uint64_t &sum) {
  int tz = (int)sizeof(K) * 8 - 1;
  for (K v : k)
    if (v != 0) tz = std::min(tz, __builtin_ctzll((unsigned long long)v));
  sum = 0;
  for (K &v : k) {
    v >>= tz;
    sum += v;
  }
  shift = tz;
}

// derivKernel (filter.zig:817-854).
bool deriv_kernel(int *out, int n, int order, int ksize) {
  if (ksize == -1) {
    if (n != 3 || order > 1) return false;
    if (order == 0) { out[0] = 3; out[1] = 10; out[2] = 3; }
    else { out[0] = -1; out[1] = 0; out[2] = 1; }
    return true;
  }
  if (ksize < -1 || ksize == 0) return false;
  const int want = ksize == 1 ? 3 : ksize;
  if (n != want) return false;
  if (ksize == 1 && order == 0) {
    out[0] = 0; out[1] = 1; out[2] = 0;
    return true;
  }
  if (order >= n) return false;
  int a[32] = {0};
  a[0] = 1;
  int len = 1;
  for (int it = 0; it < n - order - 1; it++) {
    int b[32] = {0};
    for (int j = 0; j < len; j++) { b[j] += a[j]; b[j + 1] += a[j]; }
    std::memcpy(a, b, sizeof(a));
    len++;
  }
  for (int it = 0; it < order; it++) {
    int b[32] = {0};
    for (int j = 0; j < len; j++) { b[j] -= a[j]; b[j + 1] += a[j]; }
    std::memcpy(a, b, sizeof(a));
    len++;
  }
  std::memcpy(out, a, sizeof(int) * n);
  return true;
}

// Finish kinds (filter.zig:60-116, 478-483).
enum Fin { FinCast, FinScaled, FinShift, FinU8Fixed, FinU16Fixed };

// Separable filter spec: S source, D destination; A is the accumulator:
// int64 stands for VISAR's exact integer accumulators (u16/u32/u64/i16/i32;
// none of them wraps or saturates at VISAR's kernel bounds), float for f32.
template <class S, class A, class D, class K>
struct Spec {
  Fin fin;
  double scale;
  bool const_kernel;  // SpecK: compile-time kernels (vfirstConst / hsecondConst)
};

template <class A, class K>
A mul(K k, A v) {
  return (A)k * v;
}

enum Sym { kNone, kEven, kOdd };

template <class K>
Sym symmetry(const K *k, int n) {
  bool even = true, odd = true;
  for (int i = 0; i < n / 2; i++) {
    const K a = k[i], b = k[n - 1 - i];
    if (a != b) even = false;
    if (std::is_unsigned<K>::value) odd = false;
    else if (a != -b) odd = false;
  }
  if (n % 2 == 1 && k[n / 2] != 0) odd = false;
  return even ? kEven : odd ? kOdd : kNone;
}

// tapsV (vector body; filter.zig:232-252) on one sample position.
template <class A, class K, class F>
A taps_v(F ld, const K *k, int nk, Sym sym) {
  const int r = nk / 2;
  if (sym == kNone) {
    A a = 0;
    for (int j = 0; j < nk; j++) a = a + ld(j) * (A)k[j];
    return a;
  }
  A a = sym == kEven ? ld(r) * (A)k[r] : (A)0;
  for (int i = 0; i < r; i++) {
    const A pair = sym == kEven ? ld(i) + ld(nk - 1 - i) : ld(nk - 1 - i) - ld(i);
    a = a + pair * (A)(sym == kEven ? k[i] : k[nk - 1 - i]);
  }
  return a;
}

// tapsS (scalar tail; filter.zig:254-258).
template <class A, class K, class F>
A taps_s(F ld, const K *k, int nk) {
  A a = mul<A>(k[0], ld(0));
  for (int j = 1; j < nk; j++) a = a + mul<A>(k[j], ld(j));
  return a;
}

// constTaps (filter.zig:316-328) and the const scalar tail (0 + k*v ...).
template <class A, class K, class F>
A taps_const_v(F ld, const K *k, int nk) {
  const int r = nk / 2;
  A a = ld(r) * (A)k[r];
  for (int i = 0; i < r; i++) {
    const A pair = ld(i) + ld(nk - 1 - i);
    a += k[i] == 1 ? pair : pair * (A)k[i];
  }
  return a;
}
template <class A, class K, class F>
A taps_const_s(F ld, const K *k, int nk) {
  A a = 0;
  for (int j = 0; j < nk; j++) a += (A)k[j] * ld(j);
  return a;
}

template <class D, class A>
D finish(A v, Fin fin, double scale) {
  switch (fin) {
    case FinCast: return satv<D>(v);
    case FinScaled: return satv<D>((float)v * (float)scale);
    case FinShift: {
      // (v +| 2^(s-1)) >> s, min maxInt(D); s passed in `scale`.
      const int s = (int)scale;
      const uint64_t half = (1ULL << s) >> 1;
      const uint64_t r = ((uint64_t)v + half) >> s;
      return (D)std::min<uint64_t>(r, (uint64_t)std::numeric_limits<D>::max());
    }
    case FinU8Fixed: return (D)std::min<uint64_t>(((uint64_t)v + (1ULL << 15)) >> 16, 255);
    case FinU16Fixed: return (D)std::min<uint64_t>(((uint64_t)v + (1ULL << 31)) >> 32, 65535);
  }
  return D(0);
}

constexpr int kLanesF32 = 16;  // filter.zig:139-142 lanes(f32)

// separable + chunk (filter.zig:120-205): vertical taps into a padded row,
// horizontal border by replicating filtered columns, horizontal taps.
template <class S, class A, class D, class K>
void separable(const Img<S> &s, const Img<D> &d, const std::vector<K> &kx, const std::vector<K> &ky, int border, Fin fin,
               double scale, bool const_kernel) {
  if (s.w != d.w || s.h != d.h || s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  if (kx.empty() || ky.empty() || kx.size() % 2 == 0 || ky.size() % 2 == 0) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
  const int cn = s.cn;
  const size_t n = s.row_len();
  const int nkx = (int)kx.size(), nky = (int)ky.size();
  const int rx = nkx / 2, ry = nky / 2;
  const size_t n16 = is_float<A>() ? n - n % kLanesF32 : n;  // order split only matters for f32
  const Sym vsym = symmetry(ky.data(), nky), hsym = symmetry(kx.data(), nkx);
  const size_t grain = std::max<size_t>(8, (1 << 16) / std::max<size_t>(1, n));
  parallel_for(s.h, grain, [&](size_t y0, size_t y1) {
    std::vector<A> vrow(n + 2 * (size_t)rx * cn);
    std::vector<S> const_row(border == 0 ? n : 0, S(0));
    A const_v = 0;
    for (int j = 0; j < nky; j++) const_v = const_v + mul<A>(ky[j], (A)0);
    std::vector<const S *> rows(nky);
    for (size_t y = y0; y < y1; y++) {
      for (int j = 0; j < nky; j++) {
        const long long sy = border_map((long long)y + j - ry, s.h, border);
        rows[j] = sy >= 0 ? s.row(sy) : const_row.data();
      }
      A *mid = vrow.data() + (size_t)rx * cn;
      for (size_t x = 0; x < n; x++) {
        auto ld = [&](int j) -> A { return (A)rows[j][x]; };
        const bool tail = x >= n16;
        A v;
        if (const_kernel) v = tail ? taps_const_s<A>(ld, ky.data(), nky) : taps_const_v<A>(ld, ky.data(), nky);
        else v = tail ? taps_s<A>(ld, ky.data(), nky) : taps_v<A>(ld, ky.data(), nky, vsym);
        mid[x] = v;
      }
      for (int i = 0; i < rx; i++) {
        A *lp = vrow.data() + (size_t)i * cn;
        A *rp = vrow.data() + (size_t)(rx + s.w + i) * cn;
        const long long lx = border_map((long long)i - rx, s.w, border);
        const long long rxx = border_map((long long)s.w + i, s.w, border);
        for (int c = 0; c < cn; c++) {
          lp[c] = lx >= 0 ? mid[lx * cn + c] : const_v;
          rp[c] = rxx >= 0 ? mid[rxx * cn + c] : const_v;
        }
      }
      D *out = d.row(y);
      for (size_t x = 0; x < n; x++) {
        auto ld = [&](int i) -> A { return vrow[x + (size_t)i * cn]; };
        const bool tail = x >= n16;
        A v;
        if (const_kernel) v = tail ? taps_const_s<A>(ld, kx.data(), nkx) : taps_const_v<A>(ld, kx.data(), nkx);
        else v = tail ? taps_s<A>(ld, kx.data(), nkx) : taps_v<A>(ld, kx.data(), nkx, hsym);
        out[x] = finish<D, A>(v, fin, scale);
      }
    }
  });
}

template <class T>
void gaussian_t(const visar_image *src, const visar_image *dst, int depth, int kw, int kh, double sx, double sy_arg, int border) {
  Img<T> s = typed<T>(src, depth);
  Img<T> d = typed<T>(dst, depth);
  const double sy = sy_arg > 0 ? sy_arg : sx;
  if (kw == 0) kw = gaussian_ksize(sx, depth == 0);
  if (kh == 0) kh = gaussian_ksize(sy, depth == 0);
  if (kw <= 0 || kh <= 0 || kw % 2 == 0 || kh % 2 == 0 || kw > 127 || kh > 127) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
  if (s.w != d.w || s.h != d.h || s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  if (border != 0) {
    if (s.w == 1) kw = 1;
    if (s.h == 1) kh = 1;
  }
  if constexpr (std::is_same<T, uint8_t>::value) {
    std::vector<uint16_t> kx(kw), ky(kh);
    gaussian_kernel_fixed(kx.data(), kw, sx, 8);
    gaussian_kernel_fixed(ky.data(), kh, sy, 8);
    std::vector<uint16_t> kxr = kx, kyr = ky;
    int shx, shy;
    uint64_t sumx, sumy;
    reduce(kxr, shx, sumx);
    reduce(kyr, shy, sumy);
    if (255 * sumx * sumy <= 65535) {
      const int shift = 16 - (shx + shy);
      const bool same = kw == kh && kxr == kyr;
      const bool k3 = same && kw == 3 && shift == 4 && kxr == std::vector<uint16_t>{1, 2, 1};
      const bool k5 = same && kw == 5 && shift == 8 && kxr == std::vector<uint16_t>{1, 4, 6, 4, 1};
      separable<uint8_t, long long, uint8_t, uint16_t>(s, d, kxr, kyr, border, FinShift, (double)shift, k3 || k5);
      return;
    }
    separable<uint8_t, long long, uint8_t, uint16_t>(s, d, kx, ky, border, FinU8Fixed, 1, false);
  } else if constexpr (std::is_same<T, uint16_t>::value) {
    std::vector<uint32_t> kx(kw), ky(kh);
    gaussian_kernel_fixed(kx.data(), kw, sx, 16);
    gaussian_kernel_fixed(ky.data(), kh, sy, 16);
    std::vector<uint32_t> kxr = kx, kyr = ky;
    int shx, shy;
    uint64_t sumx, sumy;
    reduce(kxr, shx, sumx);
    reduce(kyr, shy, sumy);
    if (65535ULL * sumx * sumy <= 0xffffffffULL) {
      const int shift = 32 - (shx + shy);
      const bool same = kw == kh && kxr == kyr;
      const bool k3 = same && kw == 3 && shift == 4 && kxr == std::vector<uint32_t>{1, 2, 1};
      const bool k5 = same && kw == 5 && shift == 8 && kxr == std::vector<uint32_t>{1, 4, 6, 4, 1};
      separable<uint16_t, long long, uint16_t, uint32_t>(s, d, kxr, kyr, border, FinShift, (double)shift, k3 || k5);
      return;
    }
    separable<uint16_t, long long, uint16_t, uint32_t>(s, d, kx, ky, border, FinU16Fixed, 1, false);
  } else {
    std::vector<double> kxd(kw), kyd(kh);
    gaussian_kernel(kxd.data(), kw, sx);
    gaussian_kernel(kyd.data(), kh, sy);
    std::vector<float> kx(kw), ky(kh);
    for (int i = 0; i < kw; i++) kx[i] = (float)kxd[i];
    for (int i = 0; i < kh; i++) ky[i] = (float)kyd[i];
    bool ck = false;
    if (std::is_same<T, float>::value && kw == kh && kx == ky) {
      ck = (kw == 3 && kx == std::vector<float>{0.25f, 0.5f, 0.25f}) ||
           (kw == 5 && kx == std::vector<float>{0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f});
    }
    separable<T, float, T, float>(s, d, kx, ky, border, FinCast, 1, ck);
  }
}

// boxU8 (filter.zig:638-771): running column sums, window sums, then
// round(f32(sum) * f32(scale)) half to even. (The integer-multiply and
// prefix-sum variants are used only where they give exactly this.)
void box_u8(const Img<uint8_t> &s, const Img<uint8_t> &d, int kw, int kh, int border, double scale) {
  if (s.w != d.w || s.h != d.h || s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  const int cn = s.cn;
  const size_t n = s.row_len();
  const int rx = kw / 2, ry = kh / 2;
  const float scs = (float)scale;
  const size_t grain = std::max<size_t>(16, (1 << 17) / std::max<size_t>(1, n));
  parallel_for(s.h, grain, [&](size_t y0, size_t y1) {
    std::vector<uint32_t> col_buf(n + 2 * (size_t)rx * cn);
    uint32_t *col = col_buf.data() + (size_t)rx * cn;
    std::fill(col, col + n, 0u);
    const long long top = (long long)y0 - ry;
    for (int j = 0; j < kh; j++) {
      const uint8_t *r = s.row(border_map(top + j, s.h, border));
      for (size_t x = 0; x < n; x++) col[x] += r[x];
    }
    for (size_t y = y0; y < y1; y++) {
      if (y > y0) {
        const uint8_t *add = s.row(border_map((long long)y + ry, s.h, border));
        const uint8_t *sub = s.row(border_map((long long)y - ry - 1, s.h, border));
        for (size_t x = 0; x < n; x++) col[x] = col[x] + add[x] - sub[x];
      }
      for (int i = 0; i < rx; i++) {
        const long long lx = border_map((long long)i - rx, s.w, border);
        const long long rxx = border_map((long long)s.w + i, s.w, border);
        for (int c = 0; c < cn; c++) {
          col_buf[(size_t)i * cn + c] = col[lx * cn + c];
          col_buf[(size_t)(rx + s.w + i) * cn + c] = col[rxx * cn + c];
        }
      }
      uint8_t *out = d.row(y);
      for (size_t x = 0; x < n; x++) {
        uint32_t sum = col_buf[x];
        for (int i = 1; i < kw; i++) sum += col_buf[x + (size_t)i * cn];
        out[x] = cast<uint8_t>((float)sum * scs);
      }
    }
  });
}

template <class T>
void box_t(const visar_image *src, const visar_image *dst, int depth, int kw, int kh, bool normalize, int border) {
  Img<T> s = typed<T>(src, depth);
  Img<T> d = typed<T>(dst, depth);
  if (kw > 255 || kh > 255 || kw % 2 == 0 || kh % 2 == 0) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
  const double scale = normalize ? 1.0 / (double)(kw * kh) : 1.0;
  if constexpr (is_float<T>()) {
    separable<T, float, T, float>(s, d, std::vector<float>(kw, 1.0f), std::vector<float>(kh, 1.0f), border, FinScaled, scale, false);
  } else {
    if constexpr (std::is_same<T, uint8_t>::value) {
      if (border != 0) {
        box_u8(s, d, kw, kh, border, scale);
        return;
      }
    }
    separable<T, long long, T, uint8_t>(s, d, std::vector<uint8_t>(kw, 1), std::vector<uint8_t>(kh, 1), border, FinScaled, scale, false);
  }
}

// sobel (filter.zig:867-906).
template <class S, class D>
void sobel_t(const Img<S> &s, const Img<D> &d, int dx, int dy, int ksize, double scale, int border) {
  if (ksize > 31 || ksize < -1) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
  const int n = ksize <= 1 ? 3 : ksize;
  const int nx = (ksize == 1 && dx > 0) ? 3 : n, ny = (ksize == 1 && dy > 0) ? 3 : n;
  std::vector<int> kx(nx), ky(ny);
  if (!deriv_kernel(kx.data(), nx, dx, (ksize == 1 && dx == 0) ? 1 : ksize == 1 ? 3 : ksize)) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
  if (!deriv_kernel(ky.data(), ny, dy, (ksize == 1 && dy == 0) ? 1 : ksize == 1 ? 3 : ksize)) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
  if constexpr (is_float<D>() || is_float<S>()) {
    std::vector<float> fx(kx.begin(), kx.end()), fy(ky.begin(), ky.end());
    separable<S, float, D, float>(s, d, fx, fy, border, FinScaled, scale, false);
  } else {
    // i16 (bound fits), i32 cast, or i32 scaled: all exact sums.
    separable<S, long long, D, int>(s, d, kx, ky, border, scale == 1 ? FinCast : FinScaled, scale, false);
  }
}

// ================================================================= resize

struct Tap2 {
  int o[2];
  int w[2];
};
struct Tap4 {
  int o[4];
  int w[4];
};

// linearTapU8 (resize.zig:181-214).
Tap2 linear_tap_u8(size_t d, uint32_t ssize, uint32_t dsize, bool area, bool pin) {
  const double inv = (double)dsize / (double)ssize;
  const double scale = 1.0 / inv;
  const double df = (double)d;
  long long sx;
  float fx;
  if (area) {
    sx = (long long)std::floor(df * scale);
    fx = (float)((df + 1) - (double)(sx + 1) * inv);
    fx = fx <= 0 ? 0 : fx - std::floor(fx);
  } else {
    fx = (float)((df + 0.5) * scale - 0.5);
    const float fl = std::floor(fx);
    sx = (long long)fl;
    fx -= fl;
  }
  const long long last = (long long)ssize - 1;
  if (pin && sx < 0) { sx = 0; fx = 0; }
  if (pin && sx >= last) { sx = last; fx = 0; }
  Tap2 t;
  t.w[0] = cast<int16_t>((1.0f - fx) * 2048.0f);
  t.w[1] = cast<int16_t>(fx * 2048.0f);
  t.o[0] = (int)std::min(std::max(sx, 0LL), last);
  t.o[1] = (int)std::min(std::max(sx + 1, 0LL), last);
  return t;
}

// linearU8 through ru8.separable: hrowPixels keeps (acc >> 4) as i16,
// vlinear rounds (resize_u8.zig:651-711).
void linear_u8(const Img<uint8_t> &s, const Img<uint8_t> &d, bool area) {
  const int cn = s.cn;
  std::vector<Tap2> xt(d.w), yt(d.h);
  for (int x = 0; x < d.w; x++) xt[x] = linear_tap_u8(x, s.w, d.w, area, true);
  for (int y = 0; y < d.h; y++) yt[y] = linear_tap_u8(y, s.h, d.h, area, false);
  parallel_for(d.h, 8, [&](size_t y0, size_t y1) {
    std::vector<int16_t> h0(d.row_len()), h1(d.row_len());
    for (size_t y = y0; y < y1; y++) {
      const Tap2 ty = yt[y];
      for (int k = 0; k < 2; k++) {
        const uint8_t *r = s.row(ty.o[k]);
        int16_t *h = k == 0 ? h0.data() : h1.data();
        for (int x = 0; x < d.w; x++)
          for (int c = 0; c < cn; c++) {
            const int acc = (int)r[(size_t)xt[x].o[0] * cn + c] * xt[x].w[0] + (int)r[(size_t)xt[x].o[1] * cn + c] * xt[x].w[1];
            h[(size_t)x * cn + c] = (int16_t)(acc >> 4);
          }
      }
      uint8_t *o = d.row(y);
      for (size_t i = 0; i < d.row_len(); i++) {
        const int t = (((int)h0[i] * ty.w[0]) >> 16) + (((int)h1[i] * ty.w[1]) >> 16);
        o[i] = cast<uint8_t>((t + 2) >> 2);
      }
    }
  });
}

// Generic `linear` (resize.zig:284-423) for u8: the definition VISAR tests its
// u8 fast paths against (resize.zig:654-682). x taps from linearTapU8 (first
// index and both weights); hrow sums s[xi]*a0 + s[xi+cn]*a1 in i32 (the second
// tap is the first when xi is the row's last pixel); vrow rounds
// ((r0 >> 4) * b0 >> 16) + ((r1 >> 4) * b1 >> 16), then (+2) >> 2, saturated.
void linear_generic_u8(const Img<uint8_t> &s, const Img<uint8_t> &d, bool area) {
  const int cn = s.cn;
  const size_t n = d.row_len();
  std::vector<uint32_t> xofs(n);
  std::vector<std::array<int, 2>> alpha(n);
  for (int x = 0; x < d.w; x++) {
    const Tap2 t = linear_tap_u8(x, s.w, d.w, area, true);
    for (int c = 0; c < cn; c++) {
      xofs[(size_t)x * cn + c] = (uint32_t)t.o[0] * cn + c;
      alpha[(size_t)x * cn + c] = {t.w[0], t.w[1]};
    }
  }
  const size_t last_x = s.row_len() - cn;
  std::vector<int32_t> r0(n), r1(n);
  auto hrow = [&](const uint8_t *row, int32_t *out) {
    for (size_t i = 0; i < n; i++) {
      const size_t xi = xofs[i];
      const size_t x1 = xi >= last_x ? xi : xi + cn;
      out[i] = (int32_t)row[xi] * alpha[i][0] + (int32_t)row[x1] * alpha[i][1];
    }
  };
  for (int y = 0; y < d.h; y++) {
    const Tap2 t = linear_tap_u8(y, s.h, d.h, area, false);
    hrow(s.row(t.o[0]), r0.data());
    hrow(s.row(t.o[1]), r1.data());
    uint8_t *o = d.row(y);
    for (size_t i = 0; i < n; i++) {
      const int32_t v = (((r0[i] >> 4) * t.w[0]) >> 16) + (((r1[i] >> 4) * t.w[1]) >> 16);
      o[i] = cast<uint8_t>((v + 2) >> 2);
    }
  }
}

// ru8.half (resize_u8.zig:384-447).
void half_u8(const Img<uint8_t> &s, const Img<uint8_t> &d) {
  const int cn = s.cn;
  parallel_for(d.h, 16, [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++) {
      const uint8_t *a = s.row(2 * y), *b = s.row(2 * y + 1);
      uint8_t *o = d.row(y);
      for (int x = 0; x < d.w; x++)
        for (int c = 0; c < cn; c++) {
          const size_t i = (size_t)2 * x * cn + c;
          o[(size_t)x * cn + c] = (uint8_t)(((uint32_t)a[i] + a[i + cn] + b[i] + b[i + cn] + 2) >> 2);
        }
    }
  });
}

void cubic_coeffs(float x, float c[4]) {
  const float A = -0.75f;
  c[0] = ((A * (x + 1) - 5 * A) * (x + 1) + 8 * A) * (x + 1) - 4 * A;
  c[1] = ((A + 2) * x - (A + 3)) * x * x + 1;
  c[2] = ((A + 2) * (1 - x) - (A + 3)) * (1 - x) * (1 - x) + 1;
  c[3] = 1 - c[0] - c[1] - c[2];
}

// cubicU8 (resize.zig:246-282) with vcubic (resize_u8.zig:742-763).
void cubic_u8(const Img<uint8_t> &s, const Img<uint8_t> &d) {
  const int cn = s.cn;
  auto tab = [](uint32_t ssize, uint32_t dsize) {
    std::vector<Tap4> t(dsize);
    const double scale = 1.0 / ((double)dsize / (double)ssize);
    for (uint32_t i = 0; i < dsize; i++) {
      float fx = (float)(((double)i + 0.5) * scale - 0.5);
      const float sx = std::floor(fx);
      fx -= sx;
      const long long isx = (long long)sx;
      float cf[4];
      cubic_coeffs(fx, cf);
      for (int k = 0; k < 4; k++) {
        t[i].w[k] = cast<int16_t>(cf[k] * 2048.0f);
        t[i].o[k] = (int)std::min(std::max(isx - 1 + k, 0LL), (long long)ssize - 1);
      }
    }
    return t;
  };
  const std::vector<Tap4> xt = tab(s.w, d.w), yt = tab(s.h, d.h);
  const float scale = 1.0f / (float)(2048 * 2048);
  parallel_for(d.h, 8, [&](size_t y0, size_t y1) {
    std::vector<int32_t> h(4 * d.row_len());
    for (size_t y = y0; y < y1; y++) {
      const Tap4 ty = yt[y];
      for (int k = 0; k < 4; k++) {
        const uint8_t *r = s.row(ty.o[k]);
        for (int x = 0; x < d.w; x++)
          for (int c = 0; c < cn; c++) {
            int acc = 0;
            for (int j = 0; j < 4; j++) acc += (int)r[(size_t)xt[x].o[j] * cn + c] * xt[x].w[j];
            h[k * d.row_len() + (size_t)x * cn + c] = acc;
          }
      }
      float bs[4];
      for (int k = 0; k < 4; k++) bs[k] = (float)ty.w[k] * scale;
      uint8_t *o = d.row(y);
      const size_t n = d.row_len();
      for (size_t i = 0; i < n; i++) {
        const float v = std::fma((float)h[i], bs[0], std::fma((float)h[n + i], bs[1], std::fma((float)h[2 * n + i], bs[2], (float)h[3 * n + i] * bs[3])));
        o[i] = cast<uint8_t>(v);
      }
    }
  });
}

// ru8.areaInt (resize_u8.zig:1213-1277): u32 block sum * f32(1/area), half to even.
void area_int_u8(const Img<uint8_t> &s, const Img<uint8_t> &d, int ix, int iy) {
  const int cn = s.cn;
  const float scale = 1.0f / (float)(ix * iy);
  parallel_for(d.h, 4, [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++) {
      uint8_t *o = d.row(y);
      for (int x = 0; x < d.w; x++)
        for (int c = 0; c < cn; c++) {
          uint32_t sum = 0;
          for (int dy = 0; dy < iy; dy++) {
            const uint8_t *r = s.row(y * iy + dy);
            for (int dx = 0; dx < ix; dx++) sum += r[((size_t)x * ix + dx) * cn + c];
          }
          o[(size_t)x * cn + c] = cast<uint8_t>((float)sum * scale);
        }
    }
  });
}

// Generic areaInt (resize.zig:425-464).
template <class T>
void area_int_generic(const Img<T> &s, const Img<T> &d, int ix, int iy) {
  const int cn = s.cn;
  const uint32_t area = (uint32_t)(ix * iy);
  parallel_for(d.h, 8, [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++) {
      T *dr = d.row(y);
      if constexpr (std::is_same<T, uint8_t>::value) {
        if (ix == 2 && iy == 2) {
          const T *a = s.row(2 * y), *b = s.row(2 * y + 1);
          for (int x = 0; x < d.w; x++)
            for (int c = 0; c < cn; c++) {
              const size_t i = (size_t)2 * x * cn + c;
              dr[(size_t)x * cn + c] = (T)(((uint32_t)a[i] + a[i + cn] + b[i] + b[i + cn] + 2) >> 2);
            }
          continue;
        }
      }
      for (int x = 0; x < d.w; x++)
        for (int c = 0; c < cn; c++) {
          if constexpr (is_float<T>() || std::is_signed<T>::value) {
            double sum = 0;
            for (int dy = 0; dy < iy; dy++) {
              const T *r = s.row(y * iy + dy);
              for (int dx = 0; dx < ix; dx++) sum += (double)(float)r[((size_t)x * ix + dx) * cn + c];
            }
            dr[(size_t)x * cn + c] = cast<T>(sum / (double)area);
          } else {
            uint64_t sum = 0;
            for (int dy = 0; dy < iy; dy++) {
              const T *r = s.row(y * iy + dy);
              for (int dx = 0; dx < ix; dx++) sum += r[((size_t)x * ix + dx) * cn + c];
            }
            dr[(size_t)x * cn + c] = (T)((sum + area / 2) / area);
          }
        }
    }
  });
}

struct AreaTab {
  uint32_t di, si;
  float alpha;
};

// areaTab (resize.zig:470-493).
std::vector<AreaTab> area_tab(uint32_t ssize, uint32_t dsize, double scale) {
  std::vector<AreaTab> list;
  for (uint32_t dx = 0; dx < dsize; dx++) {
    const double fsx1 = (double)dx * scale;
    const double fsx2 = fsx1 + scale;
    const double cellw = std::min(scale, (double)ssize - fsx1);
    long long sx1 = (long long)std::ceil(fsx1);
    const long long sx2 = (long long)std::floor(fsx2);
    const long long sx2c = std::min(sx2, (long long)ssize - 1);
    sx1 = std::min(sx1, (long long)ssize - 1);
    if ((double)sx1 - fsx1 > 1e-3) list.push_back({dx, (uint32_t)(sx1 - 1), (float)(((double)sx1 - fsx1) / cellw)});
    for (long long sx = sx1; sx < sx2; sx++) list.push_back({dx, (uint32_t)sx, (float)(1.0 / cellw)});
    if (fsx2 - (double)sx2 > 1e-3) list.push_back({dx, (uint32_t)sx2c, (float)(std::min(std::min(fsx2 - (double)sx2, 1.0), cellw) / cellw)});
  }
  return list;
}

// areaGeneric (resize.zig:534-565): OpenCV's ResizeArea_Invoker with f32
// accumulation; ru8.area is bit-exact with it (resize.zig:703-743).
template <class T>
void area_generic(const Img<T> &s, const Img<T> &d) {
  const std::vector<AreaTab> xtab = area_tab(s.w, d.w, (double)s.w / (double)d.w);
  const std::vector<AreaTab> ytab = area_tab(s.h, d.h, (double)s.h / (double)d.h);
  std::vector<uint32_t> ystart(d.h + 1);
  {
    uint32_t k = 0;
    for (int dy = 0; dy < d.h; dy++) {
      ystart[dy] = k;
      while (k < ytab.size() && ytab[k].di == (uint32_t)dy) k++;
    }
    ystart[d.h] = k;
  }
  const int cn = s.cn;
  parallel_for(d.h, 4, [&](size_t y0, size_t y1) {
    const size_t n = d.row_len();
    std::vector<float> hbuf(n), sum(n);
    for (size_t dy = y0; dy < y1; dy++) {
      std::fill(sum.begin(), sum.end(), 0.0f);
      for (uint32_t e = ystart[dy]; e < ystart[dy + 1]; e++) {
        const AreaTab yt = ytab[e];
        std::fill(hbuf.begin(), hbuf.end(), 0.0f);
        const T *sr = s.row(yt.si);
        for (const AreaTab &xt : xtab)
          for (int c = 0; c < cn; c++) hbuf[(size_t)xt.di * cn + c] += (float)sr[(size_t)xt.si * cn + c] * xt.alpha;
        for (size_t i = 0; i < n; i++) sum[i] += hbuf[i] * yt.alpha;
      }
      T *o = d.row(dy);
      for (size_t i = 0; i < n; i++) o[i] = cast<T>(sum[i]);
    }
  });
}

// Generic linear (resize.zig:284-423) for non-u8 samples.
template <class T>
void linear_generic(const Img<T> &s, const Img<T> &d, bool area) {
  const int cn = s.cn;
  const double scale_x = (double)s.w / (double)d.w, scale_y = (double)s.h / (double)d.h;
  auto coord = [&](size_t dd, double scale, uint32_t len, long long &i, double &f) {
    long long sx;
    double ff;
    if (area) {
      const double df = (double)dd;
      sx = (long long)std::floor(df * scale);
      ff = (df + 1) - (double)(sx + 1) / scale;
      ff = ff <= 0 ? 0 : ff - std::floor(ff);
    } else {
      const double fx = ((double)dd + 0.5) * scale - 0.5;
      sx = (long long)std::floor(fx);
      ff = fx - (double)sx;
    }
    if (sx < 0) { sx = 0; ff = 0; }
    if (sx >= (long long)len - 1) { sx = (long long)len - 1; ff = 0; }
    i = sx;
    f = ff;
  };
  std::vector<uint32_t> xofs(d.row_len());
  std::vector<float> a0(d.row_len()), a1(d.row_len());
  for (int x = 0; x < d.w; x++) {
    long long i;
    double f;
    coord(x, scale_x, s.w, i, f);
    for (int c = 0; c < cn; c++) {
      xofs[(size_t)x * cn + c] = (uint32_t)(i * cn + c);
      a0[(size_t)x * cn + c] = (float)(1.0 - f);
      a1[(size_t)x * cn + c] = (float)f;
    }
  }
  const size_t last = s.row_len() - cn;
  parallel_for(d.h, 8, [&](size_t y0, size_t y1) {
    std::vector<float> r0(d.row_len()), r1(d.row_len());
    for (size_t y = y0; y < y1; y++) {
      long long i;
      double f;
      coord(y, scale_y, s.h, i, f);
      const size_t sy0 = (size_t)i, sy1 = (size_t)std::min<long long>(i + 1, s.h - 1);
      const float b0 = (float)(1.0 - f), b1 = (float)f;
      for (int k = 0; k < 2; k++) {
        const T *sr = s.row(k == 0 ? sy0 : sy1);
        float *out = k == 0 ? r0.data() : r1.data();
        for (size_t j = 0; j < d.row_len(); j++) {
          const size_t xi = xofs[j];
          const size_t x1 = xi >= last ? xi : xi + cn;
          out[j] = (float)sr[xi] * a0[j] + (float)sr[x1] * a1[j];
        }
      }
      T *o = d.row(y);
      for (size_t j = 0; j < d.row_len(); j++) o[j] = cast<T>(r0[j] * b0 + r1[j] * b1);
    }
  });
}

// Generic cubic in f32 (resize.zig:577-640).
template <class T>
void cubic_generic(const Img<T> &s, const Img<T> &d) {
  const int cn = s.cn;
  struct Tap { long long o[4]; float w[4]; };
  auto fill = [](uint32_t dsize, double scale, uint32_t len) {
    std::vector<Tap> t(dsize);
    for (uint32_t i = 0; i < dsize; i++) {
      const double fx = ((double)i + 0.5) * scale - 0.5;
      const long long sx = (long long)std::floor(fx);
      cubic_coeffs((float)(fx - (double)sx), t[i].w);
      for (int k = 0; k < 4; k++) t[i].o[k] = std::min(std::max(sx - 1 + k, 0LL), (long long)len - 1);
    }
    return t;
  };
  const std::vector<Tap> xt = fill(d.w, (double)s.w / (double)d.w, s.w), yt = fill(d.h, (double)s.h / (double)d.h, s.h);
  parallel_for(d.h, 4, [&](size_t y0, size_t y1) {
    const size_t n = d.row_len();
    std::vector<float> h(4 * n);
    for (size_t y = y0; y < y1; y++) {
      const Tap t = yt[y];
      for (int k = 0; k < 4; k++) {
        const T *sr = s.row(t.o[k]);
        for (int x = 0; x < d.w; x++)
          for (int c = 0; c < cn; c++) {
            float acc = 0;
            for (int j = 0; j < 4; j++) acc += (float)sr[xt[x].o[j] * cn + c] * xt[x].w[j];
            h[k * n + (size_t)x * cn + c] = acc;
          }
      }
      T *o = d.row(y);
      for (size_t i = 0; i < n; i++) o[i] = cast<T>(h[i] * t.w[0] + h[n + i] * t.w[1] + h[2 * n + i] * t.w[2] + h[3 * n + i] * t.w[3]);
    }
  });
}

// nearest (resize.zig:64-105).
template <class T>
void nearest(const Img<T> &s, const Img<T> &d) {
  const int cn = s.cn;
  const double ifx = (double)s.w / (double)d.w, ify = (double)s.h / (double)d.h;
  std::vector<uint32_t> xofs(d.w);
  for (int x = 0; x < d.w; x++) xofs[x] = std::min((uint32_t)std::floor((double)x * ifx), (uint32_t)s.w - 1) * cn;
  parallel_for(d.h, 16, [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++) {
      const uint32_t sy = std::min((uint32_t)std::floor((double)y * ify), (uint32_t)s.h - 1);
      const T *sr = s.row(sy);
      T *dr = d.row(y);
      for (int x = 0; x < d.w; x++) std::memcpy(dr + (size_t)x * cn, sr + xofs[x], sizeof(T) * cn);
    }
  });
}

template <class T>
void resize_t(const visar_image *src, const visar_image *dst, int depth, int interp) {
  Img<T> s = typed<T>(src, depth);
  Img<T> d = typed<T>(dst, depth);
  if (s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  if (s.w == d.w && s.h == d.h) {
    copy_img(s, d);
    return;
  }
  if constexpr (std::is_same<T, uint8_t>::value) {
    if (s.cn <= 4) {
      const bool exact_half = s.w == 2 * d.w && s.h == 2 * d.h;
      switch (interp) {
        case 1:
          if (exact_half) half_u8(s, d);
          else linear_u8(s, d, false);
          return;
        case 3: {
          if (d.w > s.w || d.h > s.h) return linear_u8(s, d, true);
          if (exact_half) return half_u8(s, d);
          const int ix = s.w / d.w, iy = s.h / d.h;
          if (ix * d.w == s.w && iy * d.h == s.h) return area_int_u8(s, d, ix, iy);
          return area_generic(s, d);
        }
        case 2: return cubic_u8(s, d);
        default: break;
      }
    }
  }
  switch (interp) {
    case 0: return nearest(s, d);
    case 1:
      if constexpr (std::is_same<T, uint8_t>::value) return linear_u8(s, d, false);
      else return linear_generic(s, d, false);
    case 3: {
      if (d.w > s.w || d.h > s.h) {
        if constexpr (std::is_same<T, uint8_t>::value) return linear_u8(s, d, true);
        else return linear_generic(s, d, true);
      }
      const int ix = s.w / d.w, iy = s.h / d.h;
      if (ix * d.w == s.w && iy * d.h == s.h) return area_int_generic(s, d, ix, iy);
      return area_generic(s, d);
    }
    case 2: return cubic_generic(s, d);
  }
  fail(VISAR_UNSUPPORTED, "Unsupported");
}

// ================================================================= warps

long long to_idx(float f) { return (long long)std::min(std::max(f, -1.0e9f), 1.0e9f); }

// warpAffine (geometry.zig:410-533): per pixel nearestPixel / linearPixel.
// The 16-pixel u8 fast path (warpLinear16) computes the same fmas and
// rounding for blocks whose taps are all inside.
template <class T>
void warp_affine_t(const Img<T> &s, const Img<T> &d, const double m[6], int interp, int border, double value) {
  const double det = m[0] * m[4] - m[1] * m[3];
  if (det == 0) fail(VISAR_UNSUPPORTED, "Unsupported");
  if (s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  const double dd = 1.0 / det;
  const double a11 = m[4] * dd, a22 = m[0] * dd, a12 = -m[1] * dd, a21 = -m[3] * dd;
  const double b1 = -a11 * m[2] - a12 * m[5];
  const double b2 = -a21 * m[2] - a22 * m[5];
  const float mf[6] = {(float)a11, (float)a12, (float)b1, (float)a21, (float)a22, (float)b2};
  const T cval = cast<T>(value);
  const float cv = (float)cval;
  const int cn = s.cn;
  parallel_for(d.h, 4, [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++) {
      const float yf = (float)y;
      const float bx = mf[1] * yf + mf[2];
      const float by = mf[4] * yf + mf[5];
      T *dr = d.row(y);
      for (int x = 0; x < d.w; x++) {
        const float xf = (float)x;
        const float sx = std::fma(mf[0], xf, bx);
        const float sy = std::fma(mf[3], xf, by);
        T *o = dr + (size_t)x * cn;
        if (interp == 0) {
          const long long ix = to_idx(rint_f(std::min(std::max(sx, -4.0e6f), 4.0e6f)));
          const long long iy = to_idx(rint_f(std::min(std::max(sy, -4.0e6f), 4.0e6f)));
          const long long mx = border_map(ix, s.w, border), my = border_map(iy, s.h, border);
          if (mx >= 0 && my >= 0) std::memcpy(o, s.row(my) + mx * cn, sizeof(T) * cn);
          else for (int c = 0; c < cn; c++) o[c] = cval;
          continue;
        }
        const float fx = std::floor(sx), fy = std::floor(sy);
        const float ax = sx - fx, ay = sy - fy;
        const long long ix = to_idx(fx), iy = to_idx(fy);
        if (border == 0 && (ix < -1 || iy < -1 || ix >= s.w || iy >= s.h)) {
          for (int c = 0; c < cn; c++) o[c] = cval;
          continue;
        }
        const long long xs[2] = {border_map(ix, s.w, border), border_map(ix + 1, s.w, border)};
        const long long ys[2] = {border_map(iy, s.h, border), border_map(iy + 1, s.h, border)};
        for (int c = 0; c < cn; c++) {
          float p[4];
          for (int k = 0; k < 4; k++) {
            const long long px = xs[k & 1], py = ys[k >> 1];
            p[k] = (px >= 0 && py >= 0) ? (float)s.row(py)[px * cn + c] : cv;
          }
          const float v0 = std::fma(ax, p[1] - p[0], p[0]);
          const float v1 = std::fma(ax, p[3] - p[2], p[2]);
          const float v = std::fma(ay, v1 - v0, v0);
          o[c] = is_float<T>() ? (T)v : cast<T>(v);
        }
      }
    }
  });
}

double clamp_e9(double v) { return std::isnan(v) ? 1.0e9 : std::max(-1.0e9, std::min(v, 1.0e9)); }

// warpPerspective -> warpGeneric (geometry.zig:586-672).
template <class T>
void warp_persp_t(const Img<T> &s, const Img<T> &d, const double m[9], int interp, int border, double value) {
  const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
  if (det == 0) fail(VISAR_UNSUPPORTED, "Unsupported");
  if (s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  const double r = 1.0 / det;
  const double inv[9] = {
      (m[4] * m[8] - m[5] * m[7]) * r, (m[2] * m[7] - m[1] * m[8]) * r, (m[1] * m[5] - m[2] * m[4]) * r,
      (m[5] * m[6] - m[3] * m[8]) * r, (m[0] * m[8] - m[2] * m[6]) * r, (m[2] * m[3] - m[0] * m[5]) * r,
      (m[3] * m[7] - m[4] * m[6]) * r, (m[1] * m[6] - m[0] * m[7]) * r, (m[0] * m[4] - m[1] * m[3]) * r,
  };
  const T cval = cast<T>(value);
  const float cv = (float)cval;
  const int cn = s.cn;
  parallel_for(d.h, 8, [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++) {
      T *dr = d.row(y);
      const double fy = (double)y;
      for (int x = 0; x < d.w; x++) {
        const double fx = (double)x;
        double sx = inv[0] * fx + inv[1] * fy + inv[2];
        double sy = inv[3] * fx + inv[4] * fy + inv[5];
        const double w = inv[6] * fx + inv[7] * fy + inv[8];
        const double iw = w != 0 ? 1.0 / w : 0;
        sx *= iw;
        sy *= iw;
        T *o = dr + (size_t)x * cn;
        if (interp == 0) {
          const long long ix = (long long)std::round(clamp_e9(sx));
          const long long iy = (long long)std::round(clamp_e9(sy));
          const long long mx = border_map(ix, s.w, border), my = border_map(iy, s.h, border);
          if (mx >= 0 && my >= 0) std::memcpy(o, s.row(my) + mx * cn, sizeof(T) * cn);
          else for (int c = 0; c < cn; c++) o[c] = cval;
          continue;
        }
        const double x0f = std::floor(clamp_e9(sx)), y0f = std::floor(clamp_e9(sy));
        const float ax = (float)(sx - x0f), ay = (float)(sy - y0f);
        const long long ix = (long long)x0f, iy = (long long)y0f;
        if (border == 0 && (ix < -1 || iy < -1 || ix >= s.w || iy >= s.h)) {
          for (int c = 0; c < cn; c++) o[c] = cval;
          continue;
        }
        const long long xs[2] = {border_map(ix, s.w, border), border_map(ix + 1, s.w, border)};
        const long long ys[2] = {border_map(iy, s.h, border), border_map(iy + 1, s.h, border)};
        const float wt[4] = {(1 - ax) * (1 - ay), ax * (1 - ay), (1 - ax) * ay, ax * ay};
        for (int c = 0; c < cn; c++) {
          float acc = 0;
          for (int k = 0; k < 4; k++) {
            const long long px = xs[k & 1], py = ys[k >> 1];
            const float v = (px >= 0 && py >= 0) ? (float)s.row(py)[px * cn + c] : cv;
            acc += v * wt[k];
          }
          o[c] = cast<T>(acc);
        }
      }
    }
  });
}

// ============================================================= threshold

double otsu(const uint32_t *hist, size_t total) {
  const double scale = 1.0 / (double)total;
  double mu = 0;
  for (int i = 0; i < 256; i++) mu += (double)i * (double)hist[i];
  mu *= scale;
  double mu1 = 0, q1 = 0, max_sigma = 0, max_val = 0;
  const double eps = std::numeric_limits<double>::epsilon();
  for (int i = 0; i < 256; i++) {
    const double p_i = (double)hist[i] * scale;
    mu1 *= q1;
    q1 += p_i;
    const double q2 = 1.0 - q1;
    if (std::min(q1, q2) < eps || std::max(q1, q2) > 1.0 - eps) continue;
    mu1 = (mu1 + (double)i * p_i) / q1;
    const double mu2 = (mu - q1 * mu1) / q2;
    const double sigma = q1 * q2 * (mu1 - mu2) * (mu1 - mu2);
    if (sigma > max_sigma) {
      max_sigma = sigma;
      max_val = (double)i;
    }
  }
  return max_val;
}

double triangle(const uint32_t *hist) {
  int left = 0, right = 0, max_ind = 0;
  uint32_t mx = 0;
  for (int i = 0; i < 256; i++)
    if (hist[i] > 0) { left = i; break; }
  if (left > 0) left -= 1;
  for (int i = 255; i > 0; i--)
    if (hist[i] > 0) { right = i; break; }
  if (right < 255) right += 1;
  for (int j = 0; j < 256; j++)
    if (hist[j] > mx) { mx = hist[j]; max_ind = j; }
  bool flip = false;
  uint32_t h[256];
  std::memcpy(h, hist, sizeof(h));
  if (max_ind - left < right - max_ind) {
    flip = true;
    std::reverse(h, h + 256);
    left = 255 - right;
    max_ind = 255 - max_ind;
  }
  int thresh = left;
  const double a = (double)mx, b = (double)(left - max_ind);
  double dist = 0;
  for (int j = left + 1; j <= max_ind; j++) {
    const double td = a * (double)j + b * (double)h[j];
    if (td > dist) { dist = td; thresh = j; }
  }
  thresh -= 1;
  if (flip) thresh = 255 - thresh;
  return (double)thresh;
}

template <class T>
double threshold_t(const Img<T> &s, const Img<T> &d, double thresh, double maxval, int kind, int automode) {
  if (s.w != d.w || s.h != d.h || s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  if (automode != 0) {
    if (!std::is_same<T, uint8_t>::value || s.cn != 1) fail(VISAR_UNSUPPORTED, "Unsupported");
    uint32_t hist[256] = {0};
    for (int y = 0; y < s.h; y++)
      for (int x = 0; x < s.w; x++) hist[(uint8_t)s.row(y)[x]]++;
    thresh = automode == 1 ? otsu(hist, (size_t)s.w * s.h) : triangle(hist);
  }
  auto sel = [&](T v, T t, T m) -> T {
    const bool gt = v > t;
    switch (kind) {
      case 0: return gt ? m : T(0);
      case 1: return gt ? T(0) : m;
      case 2: return gt ? t : v;
      case 3: return gt ? v : T(0);
      default: return gt ? T(0) : v;
    }
  };
  const T m = cast<T>(maxval);
  if constexpr (std::is_same<T, uint8_t>::value) {
    const double fl = std::floor(thresh);
    const int ti = std::isnan(fl) ? 0 : (int)std::min(std::max(fl, -1e9), 1e9);
    if (ti < 0 || ti >= 255) {
      uint8_t lut[256];
      for (int i = 0; i < 256; i++) {
        const bool gt = i > ti;
        const uint8_t v = (uint8_t)i;
        switch (kind) {
          case 0: lut[i] = gt ? m : 0; break;
          case 1: lut[i] = gt ? 0 : m; break;
          case 2: lut[i] = gt ? cast<uint8_t>(ti) : v; break;
          case 3: lut[i] = gt ? v : 0; break;
          default: lut[i] = gt ? 0 : v; break;
        }
      }
      for (int y = 0; y < s.h; y++)
        for (size_t i = 0; i < s.row_len(); i++) d.row(y)[i] = lut[s.row(y)[i]];
      return thresh;
    }
    const T t = (T)ti;
    for (int y = 0; y < s.h; y++)
      for (size_t i = 0; i < s.row_len(); i++) d.row(y)[i] = sel(s.row(y)[i], t, m);
    return thresh;
  } else {
    if constexpr (!is_float<T>()) {
      if (std::floor(thresh) < Lim<T>::lo) {
        for (int y = 0; y < s.h; y++)
          for (size_t i = 0; i < s.row_len(); i++) {
            T o = 0;
            if (kind == 3) o = s.row(y)[i];
            else if (kind == 0) o = m;
            d.row(y)[i] = o;
          }
        return thresh;
      }
    }
    const T t = is_float<T>() ? (T)thresh : cast<T>(std::floor(thresh));
    parallel_for(s.h, std::max<size_t>(1, (1 << 15) / s.row_len()), [&](size_t y0, size_t y1) {
      for (size_t y = y0; y < y1; y++)
        for (size_t i = 0; i < s.row_len(); i++) d.row(y)[i] = sel(s.row(y)[i], t, m);
    });
    return thresh;
  }
}

// ============================================================ morphology

// structuringElement (morph.zig:32-59).
std::vector<uint8_t> structuring_element(int shape, int w, int h) {
  std::vector<uint8_t> buf((size_t)w * h, 0);
  const int ax = w / 2, ay = h / 2;
  const uint32_t r = ay, c = ax;
  const double inv_r2 = r > 0 ? 1.0 / (double)(r * r) : 0;
  for (int i = 0; i < h; i++) {
    int j1 = 0, j2 = 0;
    if (shape == 0 || (shape == 1 && i == ay)) {
      j2 = w;
    } else if (shape == 1) {
      j1 = ax;
      j2 = j1 + 1;
    } else {
      const long long dy = (long long)i - r;
      if (std::llabs(dy) <= (long long)r) {
        const double dxf = (double)c * std::sqrt((double)((uint64_t)(r * r) - (uint64_t)(dy * dy)) * inv_r2);
        const long long dx = (long long)std::round(dxf);
        j1 = (int)std::max((long long)c - dx, 0LL);
        j2 = (int)std::min((long long)c + dx + 1, (long long)w);
      }
    }
    for (int j = j1; j < j2; j++) buf[(size_t)i * w + j] = 1;
  }
  return buf;
}

template <class T>
T max_of() { return is_float<T>() ? std::numeric_limits<T>::infinity() : std::numeric_limits<T>::max(); }
template <class T>
T min_of() { return is_float<T>() ? -std::numeric_limits<T>::infinity() : std::numeric_limits<T>::lowest(); }

// generalPass (morph.zig:489-519): the per-tap definition that VISAR's run
// decomposition is tested against.
template <class T>
void general_pass(bool is_max, const Img<T> &s, const Img<T> &d, const std::vector<uint8_t> &mask, int kw, int kh, int ax, int ay) {
  const int cn = s.cn;
  parallel_for(s.h, 8, [&](size_t y0, size_t y1) {
    for (size_t y = y0; y < y1; y++) {
      T *dr = d.row(y);
      const T init = is_max ? min_of<T>() : max_of<T>();
      for (size_t i = 0; i < d.row_len(); i++) dr[i] = init;
      for (int ky = 0; ky < kh; ky++) {
        const long long sy = (long long)y + ky - ay;
        if (sy < 0 || sy >= s.h) continue;
        const T *sr = s.row(sy);
        for (int kx = 0; kx < kw; kx++) {
          if (!mask[(size_t)ky * kw + kx]) continue;
          const long long off = (long long)kx - ax;
          const long long x0 = std::max(0LL, -off), x1 = std::min((long long)s.w, (long long)s.w - off);
          if (x1 <= x0) continue;
          for (long long i = x0 * cn; i < x1 * cn; i++) {
            const T v = sr[i + off * cn];
            T &o = dr[i];
            o = is_max ? (v > o ? v : o) : (v < o ? v : o);
          }
        }
      }
    }
  });
}

template <class T>
void morph_iter(bool is_max, const Img<T> &src, const Img<T> &dst, const std::vector<uint8_t> &mask, int kw, int kh, int iterations) {
  if (iterations == 0) return copy_img(src, dst);
  std::vector<T> a, b;
  Img<T> cur = src;
  Img<T> tmp = alloc_like(a, src.w, src.h, src.cn);
  for (int it = 0; it < iterations; it++) {
    const Img<T> out = ((iterations - 1 - it) % 2 == 0) ? dst : tmp;
    Img<T> in = cur;
    std::vector<T> copy;
    if (in.data == out.data) {  // never in place
      in = alloc_like(copy, src.w, src.h, src.cn);
      copy_img(cur, in);
    }
    general_pass(is_max, in, out, mask, kw, kh, kw / 2, kh / 2);
    cur = out;
  }
}

template <class T>
void sub_sat(const Img<T> &a, const Img<T> &b, const Img<T> &d) {
  for (int y = 0; y < d.h; y++)
    for (size_t i = 0; i < d.row_len(); i++) {
      const T x = a.row(y)[i], z = b.row(y)[i];
      if constexpr (is_float<T>()) d.row(y)[i] = x - z;
      else d.row(y)[i] = x > z ? cast<T>((long long)x - (long long)z) : T(0);
    }
}

template <class T>
void morphology_t(const visar_image *src, const visar_image *dst, int depth, int op, const std::vector<uint8_t> &mask, int kw, int kh, int it) {
  Img<T> s0 = typed<T>(src, depth);
  Img<T> d = typed<T>(dst, depth);
  if (s0.w != d.w || s0.h != d.h || s0.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
  std::vector<T> sc;
  Img<T> s = alloc_like(sc, s0.w, s0.h, s0.cn);  // a private copy: dst may alias src
  copy_img(s0, s);
  std::vector<T> tb, t2b;
  Img<T> t = alloc_like(tb, s.w, s.h, s.cn);
  Img<T> t2 = alloc_like(t2b, s.w, s.h, s.cn);
  switch (op) {
    case 0: morph_iter(false, s, d, mask, kw, kh, it); break;
    case 1: morph_iter(true, s, d, mask, kw, kh, it); break;
    case 2: morph_iter(false, s, t, mask, kw, kh, it); morph_iter(true, t, d, mask, kw, kh, it); break;
    case 3: morph_iter(true, s, t, mask, kw, kh, it); morph_iter(false, t, d, mask, kw, kh, it); break;
    case 4: morph_iter(false, s, t, mask, kw, kh, it); morph_iter(true, s, d, mask, kw, kh, it); sub_sat(d, t, d); break;
    case 5: morph_iter(false, s, t, mask, kw, kh, it); morph_iter(true, t, t2, mask, kw, kh, it); sub_sat(s, t2, d); break;
    case 6: morph_iter(true, s, t, mask, kw, kh, it); morph_iter(false, t, t2, mask, kw, kh, it); sub_sat(t2, s, d); break;
  }
}

// ================================================================ pyramids

// Exact accumulators of pyramid.zig:25-33 (u8 -> u16, u16 -> u32, i16 -> i32,
// f32 -> f32); int64 / float here.
template <class T> struct PAcc { using A = int64_t; };
template <> struct PAcc<float> { using A = float; };

template <class T, class A>
T pfinish(A v, int s) {
  if constexpr (std::is_same<A, float>::value) return v * (1.0f / (float)(1 << s));
  else return (T)((v + (1 << (s - 1))) >> s);
}

// pyrDown downChunk (pyramid.zig:99-127): vert5 of the five mapped rows into a
// row padded with two mapped pixels each side, then h5s at every even pixel.
template <class T>
void pyr_down_t(const Img<T> &s, const Img<T> &d, int border) {
  using A = typename PAcc<T>::A;
  const int cn = s.cn, w = s.w;
  const size_t n = (size_t)w * cn, pad = 2 * (size_t)cn;
  int lmap[2], rmap[2];
  for (int i = 0; i < 2; i++) {
    lmap[i] = (int)border_map(i - 2, w, border);
    rmap[i] = (int)border_map(w + i, w, border);
  }
  parallel_for(d.h, 2, [&](size_t y0, size_t y1) {
    std::vector<A> p(n + 2 * pad);
    for (size_t y = y0; y < y1; y++) {
      const T *r[5];
      for (int k = 0; k < 5; k++) r[k] = s.row(border_map((long long)(2 * y + k) - 2, s.h, border));
      A *mid = p.data() + pad;
      for (size_t x = 0; x < n; x++) {
        const A a = r[0][x], b = r[1][x], c = r[2][x], e = r[3][x], f = r[4][x];
        mid[x] = (a + f) + (b + e) * (A)4 + c * (A)6;
      }
      for (int i = 0; i < 2; i++)
        for (int ch = 0; ch < cn; ch++) {
          p[(size_t)i * cn + ch] = mid[(size_t)lmap[i] * cn + ch];
          p[pad + n + (size_t)i * cn + ch] = mid[(size_t)rmap[i] * cn + ch];
        }
      T *out = d.row(y);
      for (size_t x = 0; x < d.row_len(); x++) {
        const size_t e = 2 * x - x % cn;  // padded element of the first tap
        const A v = (p[e] + p[e + 4 * cn]) + (p[e + cn] + p[e + 3 * cn]) * (A)4 + p[e + 2 * cn] * (A)6;
        out[x] = pfinish<T, A>(v, 8);
      }
    }
  });
}

// pyrUp upChunk (pyramid.zig:428-518): vert3 into even / odd rows padded by
// one pixel each side (pixel -1 is pixel 1, pixel w is pixel w-1), then the
// even / odd horizontal sums.
template <class T>
void pyr_up_t(const Img<T> &s, const Img<T> &d) {
  using A = typename PAcc<T>::A;
  const int cn = s.cn, w = s.w, h = s.h;
  const size_t n = (size_t)w * cn;
  const int left = w > 1 ? 1 : 0;
  parallel_for(h, 1, [&](size_t y0, size_t y1) {
    std::vector<A> qe(n + 2 * cn), qo(n + 2 * cn);
    for (size_t y = y0; y < y1; y++) {
      const T *a = s.row(y > 0 ? y - 1 : (h > 1 ? 1 : 0));
      const T *b = s.row(y);
      const T *c = s.row(y + 1 < (size_t)h ? y + 1 : y);
      for (size_t x = 0; x < n; x++) {
        const A va = a[x], vb = b[x], vc = c[x];
        qe[cn + x] = (va + vc) + vb * (A)6;
        qo[cn + x] = (vb + vc) * (A)4;
      }
      for (std::vector<A> *q : {&qe, &qo})
        for (int ch = 0; ch < cn; ch++) {
          (*q)[ch] = (*q)[(size_t)cn + (size_t)left * cn + ch];
          (*q)[cn + n + ch] = (*q)[n + ch];
        }
      for (int k = 0; k < 2; k++) {
        const std::vector<A> &q = k == 0 ? qe : qo;
        T *out = d.row(2 * y + k);
        for (size_t x = 0; x < n; x++) {
          const size_t o = 2 * x - x % cn;
          out[o] = pfinish<T, A>((q[x] + q[x + 2 * cn]) + q[x + cn] * (A)6, 6);
          out[o + cn] = pfinish<T, A>((q[x + cn] + q[x + 2 * cn]) * (A)4, 6);
        }
      }
    }
  });
}

template <class T>
void pyr_d(const visar_image *src, const visar_image *dst, int depth, int border, bool up) {
  Img<T> s = typed<T>(src, depth);
  Img<T> d = typed<T>(dst, depth);
  if (up) {
    if (border != 4) fail(VISAR_UNSUPPORTED, "Unsupported");
    if (d.cn != s.cn || d.w != 2 * s.w || d.h != 2 * s.h) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    pyr_up_t(s, d);
  } else {
    if (border == 0) fail(VISAR_UNSUPPORTED, "Unsupported");
    if (d.cn != s.cn || d.w != (s.w + 1) / 2 || d.h != (s.h + 1) / 2) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    pyr_down_t(s, d, border);
  }
}

// ======================================================= undistort / remap

// linalg.inv3 / mul3 (src/calib3d/linalg.zig:417-438).
bool inv3(const double a[9], double out[9]) {
  const double det = a[0] * (a[4] * a[8] - a[7] * a[5]) - a[1] * (a[3] * a[8] - a[6] * a[5]) + a[2] * (a[3] * a[7] - a[6] * a[4]);
  if (det == 0) return false;
  const double d = 1 / det;
  const double r[9] = {(a[4] * a[8] - a[5] * a[7]) * d, (a[2] * a[7] - a[1] * a[8]) * d, (a[1] * a[5] - a[2] * a[4]) * d,
                       (a[5] * a[6] - a[3] * a[8]) * d, (a[0] * a[8] - a[2] * a[6]) * d, (a[2] * a[3] - a[0] * a[5]) * d,
                       (a[3] * a[7] - a[4] * a[6]) * d, (a[1] * a[6] - a[0] * a[7]) * d, (a[0] * a[4] - a[1] * a[3]) * d};
  std::memcpy(out, r, sizeof(r));
  return true;
}

void mul3(const double a[9], const double b[9], double r[9]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
}

// MapParams (undistort.zig:26-81).
struct MapP {
  double ir[9], fx, fy, u0, v0, k[8];
  void map(double i, double j, double &u, double &v) const {
    double x = (i * ir[1] + ir[2]) + j * ir[0];
    double y = (i * ir[4] + ir[5]) + j * ir[3];
    if (!(ir[6] == 0 && ir[7] == 0 && ir[8] == 1)) {
      const double w = 1.0 / ((i * ir[7] + ir[8]) + j * ir[6]);
      x = x * w;
      y = y * w;
    }
    const double x2 = x * x, y2 = y * y, r2 = x2 + y2, xy2 = 2 * x * y;
    double kr = 1 + ((k[4] * r2 + k[1]) * r2 + k[0]) * r2;
    if (k[5] != 0 || k[6] != 0 || k[7] != 0) kr /= 1 + ((k[7] * r2 + k[6]) * r2 + k[5]) * r2;
    const double xd = x * kr + k[2] * xy2 + k[3] * (r2 + 2 * x2);
    const double yd = y * kr + k[2] * (r2 + 2 * y2) + k[3] * xy2;
    u = fx * xd + u0;
    v = fy * yd + v0;
  }
};

MapP map_params(const double ir[9], const double K[9], const double k8[8]) {
  MapP p;
  std::memcpy(p.ir, ir, sizeof(p.ir));
  p.fx = K[0];
  p.fy = K[4];
  p.u0 = K[2];
  p.v0 = K[5];
  std::memcpy(p.k, k8, sizeof(p.k));
  return p;
}

// fix (undistort.zig:114-122): round(v * 32) half to even, clamped.
int fix32(double v) {
  const double c = std::min(std::max(v * 32, -2147483647.0), 2147483647.0);
  return (int)std::nearbyint(c);
}

// sample (undistort.zig:124-172): 15-bit fixed-point bilinear, border 0.
void sample_fixed(const Img<uint8_t> &s, int iu, int iv, uint8_t *o) {
  const int cn = s.cn, W = s.w, H = s.h;
  const int sx = iu >> 5, sy = iv >> 5, a = iu & 31, b = iv & 31;
  const int w[4] = {(32 - a) * (32 - b), a * (32 - b), (32 - a) * b, a * b};
  if (sx >= W || sx + 1 < 0 || sy >= H || sy + 1 < 0) {
    for (int c = 0; c < cn; c++) o[c] = 0;
    return;
  }
  for (int c = 0; c < cn; c++) {
    int sum = 0;
    for (int q = 0; q < 4; q++) {
      const int px = sx + (q & 1), py = sy + (q >> 1);
      const int v = (px >= 0 && px < W && py >= 0 && py < H) ? s.row(py)[(size_t)px * cn + c] : 0;
      sum += v * w[q];
    }
    o[c] = (uint8_t)((sum + 512) >> 10);
  }
}

// ================================================== tracker tail (f4)

// equalizeHist (src/imgproc/hist.zig:20-45): LUT from the cumulative
// histogram without the first occupied bin, f32 scale, sat.cast.
void equalize_lut(const uint32_t hist[256], uint64_t total, uint8_t lut[256], bool &fill, int &fill_value) {
  int i = 0;
  while (hist[i] == 0) i++;
  fill = hist[i] == total;
  fill_value = i;
  for (int k = 0; k < 256; k++) lut[k] = 0;
  if (fill) return;
  const float scale = 255.0f / (float)(total - hist[i]);
  uint32_t acc = 0;
  lut[i] = 0;
  for (int k = i + 1; k < 256; k++) {
    acc += hist[k];
    lut[k] = cast<uint8_t>((float)acc * scale);
  }
}

// connectedComponentsWithStats (src/imgproc/components.zig) by flood fill
// with OpenCV's numbering, as VISAR's own test reference (components.zig:562-
// 613): components in raster order of their first pixel (4-connectivity) or
// of their first 2x2 block (8-connectivity); statistics from integer sums.
struct CcStat {
  long long x0, y0, x1, y1, area, sx2, sy;
};

int cc_label(const Img<uint8_t> &s, std::vector<int32_t> &out, int conn, std::vector<CcStat> &st) {
  const int w = s.w, h = s.h;
  out.assign((size_t)w * h, 0);
  std::vector<std::pair<int, int>> stack;
  int next = 1;
  auto flood = [&](int x, int y, int l) {
    out[(size_t)y * w + x] = l;
    stack.push_back({x, y});
    while (!stack.empty()) {
      const auto p = stack.back();
      stack.pop_back();
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          if ((dx == 0 && dy == 0) || (conn == 4 && dx != 0 && dy != 0)) continue;
          const int nx = p.first + dx, ny = p.second + dy;
          if (nx < 0 || ny < 0 || nx >= w || ny >= h) continue;
          if (s.row(ny)[nx] == 0 || out[(size_t)ny * w + nx] != 0) continue;
          out[(size_t)ny * w + nx] = l;
          stack.push_back({nx, ny});
        }
    }
  };
  if (conn == 4) {
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++)
        if (s.row(y)[x] != 0 && out[(size_t)y * w + x] == 0) flood(x, y, next++);
  } else {
    for (int by = 0; by < (h + 1) / 2; by++)
      for (int bx = 0; bx < (w + 1) / 2; bx++)
        for (int dy = 0; dy < 2; dy++)
          for (int dx = 0; dx < 2; dx++) {
            const int x = bx * 2 + dx, y = by * 2 + dy;
            if (x >= w || y >= h || s.row(y)[x] == 0 || out[(size_t)y * w + x] != 0) continue;
            flood(x, y, next++);
          }
  }
  const long long big = std::numeric_limits<long long>::max();
  st.assign(next, CcStat{big, big, 0, 0, 0, 0, 0});
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      CcStat &a = st[out[(size_t)y * w + x]];
      a.x0 = std::min<long long>(a.x0, x);
      a.y0 = std::min<long long>(a.y0, y);
      a.x1 = std::max<long long>(a.x1, x);
      a.y1 = std::max<long long>(a.y1, y);
      a.area++;
      a.sx2 += 2LL * x;
      a.sy += y;
    }
  return next;
}

// ============================================================== dispatch

int src_depth(const visar_image *c) {
  if (!c) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  switch (c->depth) {
    case 0: case 2: case 3: case 5: return (int)c->depth;
  }
  fail(VISAR_UNSUPPORTED, "Unsupported");
}

thread_local char t_err[128];

template <class F>
int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const Error &e) {
    std::snprintf(t_err, sizeof(t_err), "%s", e.name);
    return e.status;
  }
}

#define ORACLE_DISPATCH(depth, FN, ...)                      \
  switch (depth) {                                           \
    case 0: FN<uint8_t>(__VA_ARGS__); break;                 \
    case 2: FN<uint16_t>(__VA_ARGS__); break;                \
    case 3: FN<int16_t>(__VA_ARGS__); break;                 \
    case 5: FN<float>(__VA_ARGS__); break;                   \
  }

int check_border(int b) {
  if (b < 0 || b > 4) fail(VISAR_UNSUPPORTED, "Unsupported");
  return b;
}

template <class S>
void sep2d_s(const visar_image *src, const visar_image *dst, int depth, const std::vector<float> &kx, const std::vector<float> &ky, int border) {
  Img<S> s = typed<S>(src, depth);
  const int dd = src_depth(dst);
  switch (dd) {
    case 0: separable<S, float, uint8_t, float>(s, typed<uint8_t>(dst, 0), kx, ky, border, FinCast, 1, false); break;
    case 2: separable<S, float, uint16_t, float>(s, typed<uint16_t>(dst, 2), kx, ky, border, FinCast, 1, false); break;
    case 3: separable<S, float, int16_t, float>(s, typed<int16_t>(dst, 3), kx, ky, border, FinCast, 1, false); break;
    case 5: separable<S, float, float, float>(s, typed<float>(dst, 5), kx, ky, border, FinCast, 1, false); break;
  }
}

template <class S>
void sobel_s(const visar_image *src, const visar_image *dst, int depth, int dx, int dy, int ksize, double scale, int border) {
  Img<S> s = typed<S>(src, depth);
  if (!dst) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  if (dst->depth == 3) {
    if (!std::is_same<S, uint8_t>::value) fail(VISAR_UNSUPPORTED, "Unsupported");
    sobel_t<S, int16_t>(s, typed<int16_t>(dst, 3), dx, dy, ksize, scale, border);
  } else if (dst->depth == 5) {
    sobel_t<S, float>(s, typed<float>(dst, 5), dx, dy, ksize, scale, border);
  } else {
    fail(VISAR_UNSUPPORTED, "Unsupported");
  }
}

template <class T>
void resize_d(const visar_image *src, const visar_image *dst, int depth, int interp) { resize_t<T>(src, dst, depth, interp); }

template <class T>
void warp_affine_d(const visar_image *src, const visar_image *dst, int depth, const double *m, int interp, int border, double value) {
  warp_affine_t<T>(typed<T>(src, depth), typed<T>(dst, depth), m, interp, border, value);
}

template <class T>
void warp_persp_d(const visar_image *src, const visar_image *dst, int depth, const double *m, int interp, int border, double value) {
  warp_persp_t<T>(typed<T>(src, depth), typed<T>(dst, depth), m, interp, border, value);
}

template <class T>
void threshold_d(const visar_image *src, const visar_image *dst, int depth, double thresh, double maxval, int kind, int automode, double *out) {
  *out = threshold_t<T>(typed<T>(src, depth), typed<T>(dst, depth), thresh, maxval, kind, automode);
}

template <class T>
void gaussian_d(const visar_image *src, const visar_image *dst, int depth, int kw, int kh, double sx, double sy, int border) {
  gaussian_t<T>(src, dst, depth, kw, kh, sx, sy, border);
}

template <class T>
void box_d(const visar_image *src, const visar_image *dst, int depth, int kw, int kh, bool norm, int border) {
  box_t<T>(src, dst, depth, kw, kh, norm, border);
}

template <class T>
void cvt_d(const visar_image *src, const visar_image *dst, int depth, const CInfo &ci) { cvt_color_t<T>(src, dst, ci, depth); }

template <class T>
void morph_d(const visar_image *src, const visar_image *dst, int depth, int op, const std::vector<uint8_t> &mask, int kw, int kh, int it) {
  morphology_t<T>(src, dst, depth, op, mask, kw, kh, it);
}

}  // namespace

extern "C" {

const char *oracle_last_error(void) { return t_err; }
void oracle_set_num_threads(int n) { g_threads = n; }
int oracle_get_num_threads(void) { return nthreads(); }

int oracle_cvt_color(const visar_image *src, const visar_image *dst, int code) {
  return guarded([&] {
    CInfo ci;
    if (code < 0 || code >= 56 || !color_info(code, ci)) fail(VISAR_UNSUPPORTED, "Unsupported");
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, cvt_d, src, dst, depth, ci);
  });
}

int oracle_resize(const visar_image *src, const visar_image *dst, int interp) {
  return guarded([&] {
    if (interp < 0 || interp > 4) fail(VISAR_UNSUPPORTED, "Unsupported");
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, resize_d, src, dst, depth, interp);
  });
}

// grayDownsample (src/videoio/frame.zig:169-335): per output pixel the k x k
// block sums of B, G and R (alpha ignored), l = sb*1868 + sg*9617 + sr*4899
// (u32); k == 2 rounds (l + 2^15) >> 16 (`pairs`), every other k truncates
// min(255, f32(l) * f32(1 / (k*k*2^14)) + 0.5) (`blocks`, f32 steps unfused).
int oracle_gray_downsample(const visar_image *src, const visar_image *dst, int k) {
  return guarded([&] {
    if (k <= 0) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    Img<uint8_t> s = typed<uint8_t>(src, 0);
    Img<uint8_t> d = typed<uint8_t>(dst, 0);
    if (k > 16 || d.cn != 1 || (s.cn != 3 && s.cn != 4)) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    if (d.w != s.w / k || d.h != s.h / k) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    const int cn = s.cn;
    const float inv = 1.0f / (float)(k * k * (1 << 14));
    parallel_for(d.h, 8, [&](size_t y0, size_t y1) {
      for (size_t oy = y0; oy < y1; oy++) {
        uint8_t *o = d.row(oy);
        for (int ox = 0; ox < d.w; ox++) {
          uint32_t sb = 0, sg = 0, sr = 0;
          for (int dy = 0; dy < k; dy++) {
            const uint8_t *r = s.row(oy * k + dy) + (size_t)ox * k * cn;
            for (int dx = 0; dx < k; dx++) {
              sb += r[dx * cn];
              sg += r[dx * cn + 1];
              sr += r[dx * cn + 2];
            }
          }
          const uint32_t l = sb * 1868u + sg * 9617u + sr * 4899u;
          if (k == 2) {
            o[ox] = (uint8_t)((l + (1u << 15)) >> 16);
          } else {
            const float f = std::min(255.0f, (float)l * inv + 0.5f);
            o[ox] = (uint8_t)(uint32_t)f;
          }
        }
      }
    });
  });
}

// The generic kernels VISAR's resize tests compare its dispatch against
// (resize.zig:654-682 `linear`, :701-743 `areaGeneric`); u8 only.
int oracle_resize_generic_u8(const visar_image *src, const visar_image *dst, int interp) {
  return guarded([&] {
    Img<uint8_t> s = typed<uint8_t>(src, 0);
    Img<uint8_t> d = typed<uint8_t>(dst, 0);
    if (s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    if (interp == 1) linear_generic_u8(s, d, false);
    else if (interp == 3) area_generic(s, d);
    else fail(VISAR_UNSUPPORTED, "Unsupported");
  });
}

int oracle_pyr_down(const visar_image *src, const visar_image *dst, int border) {
  return guarded([&] {
    check_border(border);
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, pyr_d, src, dst, depth, border, false);
  });
}

int oracle_pyr_up(const visar_image *src, const visar_image *dst, int border) {
  return guarded([&] {
    check_border(border);
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, pyr_d, src, dst, depth, border, true);
  });
}

void expand_dist(const double *dist, size_t nd, double k8[8]) {
  for (int i = 0; i < 8; i++) k8[i] = 0;
  if (!dist) return;
  if (nd != 0 && nd != 4 && nd != 5 && nd != 8) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  for (size_t i = 0; i < nd; i++) k8[i] = dist[i];
}

// undistort (undistort.zig:204-281): stripes of min(max(1, 4096 / w), h) rows,
// the new camera's v0 moved up by the stripe's first row.
int oracle_undistort(const visar_image *src, const visar_image *dst, const double K[9], const double *dist, size_t nd,
                     const double *new_k) {
  return guarded([&] {
    Img<uint8_t> s = typed<uint8_t>(src, 0);
    Img<uint8_t> d = typed<uint8_t>(dst, 0);
    if (!K) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    if (s.w != d.w || s.h != d.h || s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    if (s.cn < 1 || s.cn > 4) fail(VISAR_UNSUPPORTED, "Unsupported");
    double k8[8];
    expand_dist(dist, nd, k8);
    const double *ar0 = new_k ? new_k : K;
    const int stripe = std::min(std::max(1, 4096 / std::max(s.w, 1)), s.h);
    const int nstripes = (s.h + stripe - 1) / stripe;
    parallel_for(nstripes, 1, [&](size_t s0, size_t s1) {
      for (size_t st = s0; st < s1; st++) {
        const int y0 = (int)st * stripe, y1 = std::min(y0 + stripe, s.h);
        double ar[9], ir[9];
        std::memcpy(ar, ar0, sizeof(ar));
        ar[5] = ar0[5] - (double)y0;
        if (!inv3(ar, ir)) continue;  // the stripe is left as it is
        const MapP p = map_params(ir, K, k8);
        for (int y = y0; y < y1; y++) {
          uint8_t *o = d.row(y);
          for (int x = 0; x < d.w; x++) {
            double u, v;
            p.map((double)(y - y0), (double)x, u, v);
            sample_fixed(s, fix32(u), fix32(v), o + (size_t)x * s.cn);
          }
        }
      }
    });
  });
}

int oracle_init_undistort_rectify_map(const double K[9], const double *dist, size_t nd, const double *R, const double *new_k,
                                      const visar_image *mapx, const visar_image *mapy) {
  return guarded([&] {
    Img<float> mx = typed<float>(mapx, 5);
    Img<float> my = typed<float>(mapy, 5);
    if (!K) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    double k8[8];
    expand_dist(dist, nd, k8);
    const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double m[9], ir[9];
    mul3(new_k ? new_k : K, R ? R : eye, m);
    if (!inv3(m, ir)) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    if (mx.w != my.w || mx.h != my.h || mx.cn != my.cn || mx.cn != 1) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    const MapP p = map_params(ir, K, k8);
    parallel_for(mx.h, 16, [&](size_t y0, size_t y1) {
      for (size_t y = y0; y < y1; y++)
        for (int x = 0; x < mx.w; x++) {
          double u, v;
          p.map((double)y, (double)x, u, v);
          mx.row(y)[x] = (float)u;
          my.row(y)[x] = (float)v;
        }
    });
  });
}

// remap -> linearF32 (undistort.zig:288-392).
int oracle_remap(const visar_image *src, const visar_image *dst, const visar_image *mapx, const visar_image *mapy, double value) {
  return guarded([&] {
    Img<uint8_t> s = typed<uint8_t>(src, 0);
    Img<uint8_t> d = typed<uint8_t>(dst, 0);
    Img<float> mx = typed<float>(mapx, 5);
    Img<float> my = typed<float>(mapy, 5);
    const double rv = std::round(value);
    const uint8_t bv = (uint8_t)(rv != rv ? 0 : std::min(255.0, std::max(0.0, rv)));
    if (d.w != mx.w || d.h != mx.h || mx.w != my.w || mx.h != my.h || mx.cn != my.cn || mx.cn != 1)
      fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    if (s.cn != d.cn || s.cn < 1 || s.cn > 4) fail(VISAR_UNSUPPORTED, "Unsupported");
    const int cn = s.cn;
    parallel_for(d.h, 8, [&](size_t y0, size_t y1) {
      for (size_t y = y0; y < y1; y++) {
        uint8_t *o = d.row(y);
        for (int x = 0; x < d.w; x++) {
          const float sx = mx.row(y)[x], sy = my.row(y)[x];
          const float fx = std::floor(sx), fy = std::floor(sy);
          uint8_t *op = o + (size_t)x * cn;
          if (!(fx >= -1 && fy >= -1 && fx < (float)s.w && fy < (float)s.h)) {
            for (int c = 0; c < cn; c++) op[c] = bv;
            continue;
          }
          const float ax = sx - fx, ay = sy - fy;
          const int ix = (int)fx, iy = (int)fy;
          for (int c = 0; c < cn; c++) {
            float p[4];
            for (int q = 0; q < 4; q++) {
              const int px = ix + (q & 1), py = iy + (q >> 1);
              p[q] = (px >= 0 && px < s.w && py >= 0 && py < s.h) ? (float)s.row(py)[(size_t)px * cn + c] : (float)bv;
            }
            const float v0 = std::fma(ax, p[1] - p[0], p[0]);
            const float v1 = std::fma(ax, p[3] - p[2], p[2]);
            const float v = std::fma(ay, v1 - v0, v0);
            op[c] = (uint8_t)std::min(std::max(std::nearbyint(v), 0.0f), 255.0f);
          }
        }
      }
    });
  });
}

int oracle_equalize_hist(const visar_image *src, const visar_image *dst) {
  return guarded([&] {
    Img<uint8_t> s = typed<uint8_t>(src, 0);
    Img<uint8_t> d = typed<uint8_t>(dst, 0);
    if (s.cn != 1 || s.w != d.w || s.h != d.h || s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    uint32_t hist[256] = {0};
    for (int y = 0; y < s.h; y++)
      for (int x = 0; x < s.w; x++) hist[s.row(y)[x]]++;
    uint8_t lut[256];
    bool fill;
    int fv;
    equalize_lut(hist, (uint64_t)s.w * s.h, lut, fill, fv);
    for (int y = 0; y < s.h; y++)
      for (int x = 0; x < s.w; x++) d.row(y)[x] = fill ? (uint8_t)fv : lut[s.row(y)[x]];
  });
}

// adaptiveThreshold (src/imgproc/threshold.zig:307-360, C ABI capi.zig:326-337).
int oracle_adaptive_threshold(const visar_image *src, const visar_image *dst, double maxval, int method, int type, int block,
                              double delta) {
  return guarded([&] {
    if (method != 0 && method != 1) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    if (type != 0 && type != 1) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    if (block < 3) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    Img<uint8_t> s = typed<uint8_t>(src, 0);
    Img<uint8_t> d = typed<uint8_t>(dst, 0);
    if (s.w != d.w || s.h != d.h || s.cn != d.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    if (s.cn != 1) fail(VISAR_UNSUPPORTED, "UnsupportedChannels");
    if (block % 2 != 1) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
    std::vector<uint8_t> mbuf((size_t)s.w * s.h);
    visar_image mi{(uint32_t)s.w, (uint32_t)s.h, 1, 0, (size_t)s.w, mbuf.data()};
    if (method == 0) {
      box_t<uint8_t>(src, &mi, 0, block, block, true, 1);
    } else {
      std::vector<float> f((size_t)s.w * s.h), fb((size_t)s.w * s.h);
      for (int y = 0; y < s.h; y++)
        for (int x = 0; x < s.w; x++) f[(size_t)y * s.w + x] = (float)s.row(y)[x];
      visar_image fi{(uint32_t)s.w, (uint32_t)s.h, 1, 5, (size_t)s.w * 4, f.data()};
      visar_image fo{(uint32_t)s.w, (uint32_t)s.h, 1, 5, (size_t)s.w * 4, fb.data()};
      gaussian_t<float>(&fi, &fo, 5, block, block, 0.0, 0.0, 1);
      for (size_t i = 0; i < fb.size(); i++) mbuf[i] = cast<uint8_t>(fb[i]);
    }
    const int imax = cast<uint8_t>(maxval);
    double dl = type == 0 ? std::ceil(delta) : std::floor(delta);
    dl = std::min(std::max(dl, -1024.0), 1024.0);
    const int idelta = (int)dl;
    for (int y = 0; y < s.h; y++)
      for (int x = 0; x < s.w; x++) {
        const int sv = s.row(y)[x], mv = mbuf[(size_t)y * s.w + x];
        const bool gt = sv + idelta > mv;
        d.row(y)[x] = (uint8_t)((type == 0 ? gt : !gt) ? imax : 0);
      }
  });
}

// Background.apply (src/video/track.zig:30-81) on an explicit u16 model.
int oracle_background_apply(uint16_t *model, int *primed, int shift, const visar_image *frame, const visar_image *mask,
                            int threshold) {
  return guarded([&] {
    Img<uint8_t> f = typed<uint8_t>(frame, 0);
    Img<uint8_t> m = typed<uint8_t>(mask, 0);
    if (f.cn != 1 || f.w != m.w || f.h != m.h || f.cn != m.cn) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    const int t = std::min(std::max(threshold, 0), 255);
    for (int y = 0; y < f.h; y++)
      for (int x = 0; x < f.w; x++) {
        uint16_t &b = model[(size_t)y * f.w + x];
        const int fv = f.row(y)[x];
        if (!*primed) {
          b = (uint16_t)(fv << 8);
          m.row(y)[x] = 0;
          continue;
        }
        const int bv = b;
        const bool fg = std::abs(fv - (bv >> 8)) > t;
        m.row(y)[x] = fg ? 255 : 0;
        const int sh = shift + (fg ? 2 : 0);
        b = (uint16_t)(bv + (((fv << 8) - bv) >> sh));
      }
    *primed = 1;
  });
}

// visar_connected_components (capi.zig:529-551): labels, count, stats rows
// (left, top, width, height, area), centroids (cx, cy).
int oracle_connected_components(const visar_image *src, const visar_image *labels, int connectivity, int32_t *stats,
                                double *centroids, size_t max, size_t *count) {
  return guarded([&] {
    Img<uint8_t> s = typed<uint8_t>(src, 0);
    Img<int32_t> l = typed<int32_t>(labels, 4);
    if (s.cn != 1 || l.cn != 1 || s.w != l.w || s.h != l.h) fail(VISAR_SIZE_MISMATCH, "SizeMismatch");
    std::vector<int32_t> out;
    std::vector<CcStat> st;
    const int n = cc_label(s, out, connectivity == 4 ? 4 : 8, st);
    for (int y = 0; y < s.h; y++)
      for (int x = 0; x < s.w; x++) l.row(y)[x] = out[(size_t)y * s.w + x];
    *count = (size_t)n;
    for (size_t i = 0; i < std::min<size_t>(max, (size_t)n); i++) {
      const CcStat &a = st[i];
      if (stats) {
        int32_t *o = stats + i * 5;
        if (a.area == 0) {
          o[0] = -1; o[1] = std::numeric_limits<int32_t>::max(); o[2] = 0; o[3] = 0; o[4] = 0;
        } else {
          o[0] = (int32_t)a.x0; o[1] = (int32_t)a.y0; o[2] = (int32_t)(a.x1 - a.x0 + 1); o[3] = (int32_t)(a.y1 - a.y0 + 1);
          o[4] = (int32_t)a.area;
        }
      }
      if (centroids) {
        const double ar = (double)std::max<long long>(a.area, 1);
        centroids[2 * i] = a.area == 0 ? std::nan("") : (double)a.sx2 / 2.0 / ar;
        centroids[2 * i + 1] = a.area == 0 ? std::nan("") : (double)a.sy / ar;
      }
    }
  });
}

int oracle_gaussian_blur(const visar_image *src, const visar_image *dst, int kw, int kh, double sx, double sy, int border) {
  return guarded([&] {
    check_border(border);
    if (kw < 0 || kh < 0) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, gaussian_d, src, dst, depth, kw, kh, sx, sy, border);
  });
}

int oracle_box_filter(const visar_image *src, const visar_image *dst, int kw, int kh, int normalize, int border) {
  return guarded([&] {
    check_border(border);
    if (kw <= 0 || kh <= 0) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, box_d, src, dst, depth, kw, kh, normalize != 0, border);
  });
}

int oracle_sobel(const visar_image *src, const visar_image *dst, int dx, int dy, int ksize, double scale, int border) {
  return guarded([&] {
    check_border(border);
    if (dx < 0 || dy < 0) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, sobel_s, src, dst, depth, dx, dy, ksize, scale, border);
  });
}

int oracle_sep_filter_2d(const visar_image *src, const visar_image *dst, const float *kx, int nkx, const float *ky, int nky, int border) {
  return guarded([&] {
    check_border(border);
    if (!kx || !ky || nkx < 0 || nky < 0) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    if (nkx > 255 || nky > 255) fail(VISAR_INVALID_ARGUMENT, "InvalidKernel");
    const int depth = src_depth(src);
    std::vector<float> vx(kx, kx + nkx), vy(ky, ky + nky);
    ORACLE_DISPATCH(depth, sep2d_s, src, dst, depth, vx, vy, border);
  });
}

int oracle_threshold(const visar_image *src, const visar_image *dst, double thresh, double maxval, int type, double *used) {
  double t = thresh;
  const int rc = guarded([&] {
    const int kind = type & 7;
    if (kind > 4) fail(VISAR_UNSUPPORTED, "Unsupported");
    const int automode = (type & 8) ? 1 : (type & 16) ? 2 : 0;
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, threshold_d, src, dst, depth, thresh, maxval, kind, automode, &t);
  });
  if (used) *used = t;
  return rc;
}

int oracle_morphology(const visar_image *src, const visar_image *dst, int op, int shape, int kw, int kh, int iterations) {
  return guarded([&] {
    if (op < 0 || op > 6 || shape < 0 || shape > 2) fail(VISAR_UNSUPPORTED, "Unsupported");
    if (kw <= 0 || kh <= 0 || kw > 255 || kh > 255 || iterations < 0) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    const std::vector<uint8_t> mask = structuring_element(shape, kw, kh);
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, morph_d, src, dst, depth, op, mask, kw, kh, iterations);
  });
}

int oracle_warp_affine(const visar_image *src, const visar_image *dst, const double m[6], int interp, int border, double value) {
  return guarded([&] {
    check_border(border);
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, warp_affine_d, src, dst, depth, m, interp == 0 ? 0 : 1, border, value);
  });
}

int oracle_warp_perspective(const visar_image *src, const visar_image *dst, const double m[9], int interp, int border, double value) {
  return guarded([&] {
    check_border(border);
    const int depth = src_depth(src);
    ORACLE_DISPATCH(depth, warp_persp_d, src, dst, depth, m, interp == 0 ? 0 : 1, border, value);
  });
}

// Known-answer hooks for the pinning tests.
void oracle_gaussian_kernel(double *out, int n, double sigma) { gaussian_kernel(out, n, sigma); }
void oracle_gaussian_kernel_fixed_u16(uint16_t *out, int n, double sigma) { gaussian_kernel_fixed(out, n, sigma, 8); }
void oracle_gaussian_kernel_fixed_u32(uint32_t *out, int n, double sigma) { gaussian_kernel_fixed(out, n, sigma, 16); }
int oracle_deriv_kernel(int *out, int n, int order, int ksize) { return deriv_kernel(out, n, order, ksize) ? 0 : -1; }
long long oracle_border_map(long long p, long long len, int border) { return border_map(p, len, border); }
int oracle_sat_u8_f32(float x) { return cast<uint8_t>(x); }
int oracle_sat_i16_f32(float x) { return cast<int16_t>(x); }
int oracle_satv_u8_f32(float x) { return satv<uint8_t>(x); }
int oracle_satv_i16_f32(float x) { return satv<int16_t>(x); }
double oracle_cv_exp(double x) { return cv_exp(x); }
void oracle_structuring_element(int shape, int w, int h, uint8_t *out) {
  const std::vector<uint8_t> m = structuring_element(shape, w, h);
  std::memcpy(out, m.data(), m.size());
}

}  // extern "C"
