// Host-side tables shared by the per-call C ABI and the batch engine.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "vb.h"

namespace vb {

// sat.cast(i16, f32) on the host.
int sat_i16(float x) {
  if (x != x) return 0;
  const double r = std::nearbyint((double)x);
  if (r <= -32768.0) return -32768;
  if (r >= 32767.0) return 32767;
  return (int)r;
}

// linearCoord + Weights(T).coef (resize.zig:156-179, 410-415).
FLinTap lin_tap_f(long long d, uint32_t ssize, uint32_t dsize, bool area, bool is_x) {
  const double scale = (double)ssize / (double)dsize;
  long long sx;
  double f;
  if (area) {
    const double df = (double)d;
    sx = (long long)std::floor(df * scale);
    f = (df + 1) - (double)(sx + 1) / scale;
    f = f <= 0 ? 0 : f - std::floor(f);
  } else {
    const double fx = ((double)d + 0.5) * scale - 0.5;
    sx = (long long)std::floor(fx);
    f = fx - (double)sx;
  }
  if (sx < 0) {
    sx = 0;
    f = 0;
  }
  if (sx >= (long long)ssize - 1) {
    sx = (long long)ssize - 1;
    f = 0;
  }
  FLinTap t;
  t.o0 = (int)sx;
  t.o1 = is_x ? ((sx >= (long long)ssize - 1) ? (int)sx : (int)sx + 1) : (int)std::min(sx + 1, (long long)ssize - 1);
  t.a0 = (float)(1.0 - f);
  t.a1 = (float)f;
  return t;
}

// linearTapU8 (src/imgproc/resize.zig:181-214): OpenCV's 8-bit bilinear taps, the
// source coordinate in f32 and each weight rounded to 11 bits on its own.
LinTap lin_tap_u8(long long d, uint32_t ssize, uint32_t dsize, bool area, bool pin) {
  const double inv = (double)dsize / (double)ssize;
  const double scale = 1.0 / inv;
  const double df = (double)d;
  long long sx;
  float fx;
  if (area) {
    sx = (long long)std::floor(df * scale);
    fx = (float)((df + 1) - (double)(sx + 1) * inv);
    fx = fx <= 0 ? 0.0f : fx - std::floor(fx);
  } else {
    fx = (float)((df + 0.5) * scale - 0.5);
    const float fl = std::floor(fx);
    sx = (long long)fl;
    fx -= fl;
  }
  const long long last = (long long)ssize - 1;
  if (pin && sx < 0) {
    sx = 0;
    fx = 0;
  }
  if (pin && sx >= last) {
    sx = last;
    fx = 0;
  }
  LinTap t;
  t.w0 = sat_i16((1.0f - fx) * 2048.0f);
  t.w1 = sat_i16(fx * 2048.0f);
  t.o0 = (int)std::min(std::max(sx, 0LL), last);
  t.o1 = (int)std::min(std::max(sx + 1, 0LL), last);
  return t;
}

// getStructuringElement (src/imgproc/morph.zig:32-59).
std::vector<uint8_t> structuring_element(int shape, int w, int h) {
  std::vector<uint8_t> m((size_t)w * h, 0);
  const int ax = w / 2, ay = h / 2;
  const long long r = ay, c = ax;
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
      if (std::llabs(dy) <= r) {
        const double dxf = (double)c * std::sqrt((double)(unsigned long long)(r * r - dy * dy) * inv_r2);
        const long long dx = (long long)std::round(dxf);
        j1 = (int)std::max(c - dx, 0LL);
        j2 = (int)std::min(c + dx + 1, (long long)w);
      }
    }
    for (int j = j1; j < j2; j++) m[(size_t)i * w + j] = 1;
  }
  return m;
}

// invertAffine (src/imgproc/geometry.zig:591-602) in f64, rounded to f32 as
// warpAffine uses it (geometry.zig:412-415). False for a singular matrix.
bool affine_inverse_f32(const double m[6], float out[6]) {
  const double det = m[0] * m[4] - m[1] * m[3];
  if (det == 0) return false;
  const double dd = 1.0 / det;
  const double a11 = m[4] * dd, a22 = m[0] * dd, a12 = -m[1] * dd, a21 = -m[3] * dd;
  const double b1 = -a11 * m[2] - a12 * m[5];
  const double b2 = -a21 * m[2] - a22 * m[5];
  out[0] = (float)a11;
  out[1] = (float)a12;
  out[2] = (float)b1;
  out[3] = (float)a21;
  out[4] = (float)a22;
  out[5] = (float)b2;
  return true;
}

// invert3 (src/imgproc/geometry.zig:604-613): adjugate over the determinant.
bool perspective_inverse(const double m[9], double out[9]) {
  const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                     m[2] * (m[3] * m[7] - m[4] * m[6]);
  if (det == 0) return false;
  const double r = 1.0 / det;
  out[0] = (m[4] * m[8] - m[5] * m[7]) * r;
  out[1] = (m[2] * m[7] - m[1] * m[8]) * r;
  out[2] = (m[1] * m[5] - m[2] * m[4]) * r;
  out[3] = (m[5] * m[6] - m[3] * m[8]) * r;
  out[4] = (m[0] * m[8] - m[2] * m[6]) * r;
  out[5] = (m[2] * m[3] - m[0] * m[5]) * r;
  out[6] = (m[3] * m[7] - m[4] * m[6]) * r;
  out[7] = (m[1] * m[6] - m[0] * m[7]) * r;
  out[8] = (m[0] * m[4] - m[1] * m[3]) * r;
  return true;
}

}  // namespace vb
