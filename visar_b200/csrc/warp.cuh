// Per-pixel warpAffine / warpPerspective with the channel count known at
// compile time (src/imgproc/geometry.zig:403-672), shared by the per-call
// kernels (warp.cu) and the batched tile kernels (batch.cu). The caller
// guarantees 0 <= x < d.w and 0 <= y < d.h.
//
// warpAffine follows OpenCV 5's float kernel as VISAR does: the inverse
// matrix (f64 on the host) is rounded to f32; per row bx = m1*y + m2 and
// by = m4*y + m5 (unfused); per pixel sx = fma(m0, x, bx), sy = fma(m3, x, by);
// bilinear blending is fma(ax, p1 - p0, p0), fma(ax, p3 - p2, p2), then
// fma(ay, v1 - v0, v0), rounded half to even. warpPerspective works per
// pixel in f64 with a reciprocal of w, and blends with four f32 weights.
#pragma once
#include <cmath>

#include "vb.h"

namespace vb {
namespace wp {

struct AffArgs {
  float m[6];
  int interp, border;
  float cv;  // border value as f32 (after saturation to T)
};

struct PerArgs {
  double m[9];
  int interp, border;
  float cv;
};

__device__ __forceinline__ long long to_idx(float f) {
  return (long long)fminf(fmaxf(f, -1.0e9f), 1.0e9f);
}

template <class T>
__device__ __forceinline__ T round_to(float v) {
  if constexpr (IsFloat<T>::v) return v;
  else return cast_sat<T>(v);
}

// Byte k of w as an exact f32 (2^23 + b, minus 2^23): two integer/float ops
// instead of an int-to-float conversion.
__device__ __forceinline__ float bytef(uint32_t w, int k) {
  return __fsub_rn(__uint_as_float(0x4B000000u | ((w >> (8 * k)) & 0xFFu)), 8388608.0f);
}

// sat.cast(u8, v): round half to even and saturate (NaN -> 0). Clamping to
// [-1, 256] first keeps that result and brings v below 2^22, where adding
// 1.5 * 2^23 rounds it to an integer held in the low mantissa bits.
__device__ __forceinline__ uint8_t round_u8(float v) {
  const float c = fminf(fmaxf(v, -1.0f), 256.0f);
  const int q = (int)(__float_as_uint(__fadd_rn(c, 12582912.0f)) - 0x4B400000u);
  return (uint8_t)min(max(q, 0), 255);
}

template <class T>
__device__ __forceinline__ T round_fast(float v) {
  if constexpr (sizeof(T) == 1) return round_u8(v);
  else return round_to<T>(v);
}

// Loads the two horizontally adjacent source pixels (ix, ix + 1) of row rp,
// all CN channels, as f32. 3-channel u8 rows use two aligned 8-byte loads
// when the 16-byte window stays inside the row (`wide`).
template <class T, int CN>
__device__ __forceinline__ void load_pair(const T *rp, int ix, bool wide, int row_bytes, float *p, float *q) {
  if constexpr (sizeof(T) == 1 && CN == 3) {
    const int b = ix * 3;
    const int a8 = b & ~7;
    if (wide && a8 + 16 <= row_bytes) {
      const uint2 lo = *reinterpret_cast<const uint2 *>(rp + a8);
      const uint2 hi = *reinterpret_cast<const uint2 *>(rp + a8 + 8);
      const int off = b - a8;  // 0..7
      const uint32_t wa = off >= 4 ? lo.y : lo.x;
      const uint32_t wb = off >= 4 ? hi.x : lo.y;
      const uint32_t wc = off >= 4 ? hi.y : hi.x;
      const unsigned sel = 0x3210u + 0x1111u * (unsigned)(off & 3);
      const uint32_t b0 = __byte_perm(wa, wb, sel);  // bytes off .. off+3
      const uint32_t b1 = __byte_perm(wb, wc, sel);  // bytes off+4 .. off+7
      p[0] = bytef(b0, 0); p[1] = bytef(b0, 1); p[2] = bytef(b0, 2);
      q[0] = bytef(b0, 3); q[1] = bytef(b1, 0); q[2] = bytef(b1, 1);
      return;
    }
  }
  if constexpr (sizeof(T) == 1 && CN == 4) {
    const uint32_t u = *reinterpret_cast<const uint32_t *>(rp + ix * 4);
    const uint32_t v = *reinterpret_cast<const uint32_t *>(rp + ix * 4 + 4);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      p[c] = bytef(u, c);
      q[c] = bytef(v, c);
    }
    return;
  }
#pragma unroll
  for (int c = 0; c < CN; c++) {
    p[c] = to_f(rp[ix * CN + c]);
    q[c] = to_f(rp[ix * CN + CN + c]);
  }
}

__device__ __forceinline__ double clamp_e9(double v) {
  // std.math.clamp(v, -1e9, 1e9) = @max(-1e9, @min(v, 1e9)); a NaN gives 1e9.
  return fmax(-1.0e9, fmin(v, 1.0e9));
}

// warpAffine with the channel count known at compile time. Same arithmetic
// as k_warp_affine; pixels whose four taps are inside the source skip the
// border logic (VISAR's warpLinear16 fast path computes the same values).
template <class T, int CN>
__device__ __forceinline__ void affine_px(const DImg &s, const DImg &d, const AffArgs &a, int wide, int x, int y) {
  const float yf = (float)y;
  const float bx = __fadd_rn(__fmul_rn(a.m[1], yf), a.m[2]);
  const float by = __fadd_rn(__fmul_rn(a.m[4], yf), a.m[5]);
  const float xf = (float)x;
  const float sx = fmaf(a.m[0], xf, bx);
  const float sy = fmaf(a.m[3], xf, by);
  T *o = row_ptr<T>(d, y) + x * CN;
  if (a.interp == 0) {
    const long long ix = to_idx(rintf(fminf(fmaxf(sx, -4.0e6f), 4.0e6f)));
    const long long iy = to_idx(rintf(fminf(fmaxf(sy, -4.0e6f), 4.0e6f)));
    const int mx = border_map(ix, s.w, a.border);
    const int my = border_map(iy, s.h, a.border);
    if (mx >= 0 && my >= 0) {
      const T *p = row_ptr<const T>(s, my) + mx * CN;
#pragma unroll
      for (int c = 0; c < CN; c++) o[c] = p[c];
    } else {
      const T cvT = round_to<T>(a.cv);
#pragma unroll
      for (int c = 0; c < CN; c++) o[c] = cvT;
    }
    return;
  }
  const float fx = floorf(sx), fy = floorf(sy);
  const float ax = __fsub_rn(sx, fx), ay = __fsub_rn(sy, fy);
  float p0[CN], p1[CN], p2[CN], p3[CN];
  if (fx >= 0.0f && fy >= 0.0f && fx < (float)(s.w - 1) && fy < (float)(s.h - 1)) {
    const int ix = (int)fx, iy = (int)fy;
    const int rb = s.w * CN * (int)sizeof(T);
    load_pair<T, CN>(row_ptr<const T>(s, iy), ix, wide, rb, p0, p1);
    load_pair<T, CN>(row_ptr<const T>(s, iy + 1), ix, wide, rb, p2, p3);
  } else {
    const long long ix = to_idx(fx), iy = to_idx(fy);
    if (a.border == kConstant && (ix < -1 || iy < -1 || ix >= s.w || iy >= s.h)) {
      const T cvT = round_to<T>(a.cv);
#pragma unroll
      for (int c = 0; c < CN; c++) o[c] = cvT;
      return;
    }
    const int x0 = border_map(ix, s.w, a.border), x1 = border_map(ix + 1, s.w, a.border);
    const int y0 = border_map(iy, s.h, a.border), y1 = border_map(iy + 1, s.h, a.border);
    const T *r0 = y0 >= 0 ? row_ptr<const T>(s, y0) : nullptr;
    const T *r1 = y1 >= 0 ? row_ptr<const T>(s, y1) : nullptr;
#pragma unroll
    for (int c = 0; c < CN; c++) {
      p0[c] = (r0 && x0 >= 0) ? to_f(r0[x0 * CN + c]) : a.cv;
      p1[c] = (r0 && x1 >= 0) ? to_f(r0[x1 * CN + c]) : a.cv;
      p2[c] = (r1 && x0 >= 0) ? to_f(r1[x0 * CN + c]) : a.cv;
      p3[c] = (r1 && x1 >= 0) ? to_f(r1[x1 * CN + c]) : a.cv;
    }
  }
#pragma unroll
  for (int c = 0; c < CN; c++) {
    const float v0 = fmaf(ax, __fsub_rn(p1[c], p0[c]), p0[c]);
    const float v1 = fmaf(ax, __fsub_rn(p3[c], p2[c]), p2[c]);
    o[c] = round_fast<T>(fmaf(ay, __fsub_rn(v1, v0), v0));
  }
}

// warpPerspective with the channel count known at compile time and an
// interior fast path (same arithmetic as k_warp_persp).
template <class T, int CN>
__device__ __forceinline__ void persp_px(const DImg &s, const DImg &d, const PerArgs &a, int wide, int x, int y) {
  const double fx = (double)x, fy = (double)y;
  double sx = __dadd_rn(__dadd_rn(__dmul_rn(a.m[0], fx), __dmul_rn(a.m[1], fy)), a.m[2]);
  double sy = __dadd_rn(__dadd_rn(__dmul_rn(a.m[3], fx), __dmul_rn(a.m[4], fy)), a.m[5]);
  const double w = __dadd_rn(__dadd_rn(__dmul_rn(a.m[6], fx), __dmul_rn(a.m[7], fy)), a.m[8]);
  const double iw = w != 0.0 ? __drcp_rn(w) : 0.0;  // correctly rounded: equals 1.0 / w
  sx = __dmul_rn(sx, iw);
  sy = __dmul_rn(sy, iw);
  T *o = row_ptr<T>(d, y) + x * CN;
  if (a.interp == 0) {
    const long long ix = (long long)round(clamp_e9(sx));
    const long long iy = (long long)round(clamp_e9(sy));
    const int mx = border_map(ix, s.w, a.border);
    const int my = border_map(iy, s.h, a.border);
    if (mx >= 0 && my >= 0) {
      const T *p = row_ptr<const T>(s, my) + mx * CN;
#pragma unroll
      for (int c = 0; c < CN; c++) o[c] = p[c];
    } else {
      const T cvT = round_to<T>(a.cv);
#pragma unroll
      for (int c = 0; c < CN; c++) o[c] = cvT;
    }
    return;
  }
  const double x0f = floor(clamp_e9(sx));
  const double y0f = floor(clamp_e9(sy));
  const float ax = (float)__dsub_rn(sx, x0f);
  const float ay = (float)__dsub_rn(sy, y0f);
  const float one_ax = __fsub_rn(1.0f, ax), one_ay = __fsub_rn(1.0f, ay);
  const float wt0 = __fmul_rn(one_ax, one_ay), wt1 = __fmul_rn(ax, one_ay), wt2 = __fmul_rn(one_ax, ay),
              wt3 = __fmul_rn(ax, ay);
  float v0[CN], v1[CN], v2[CN], v3[CN];
  if (x0f >= 0.0 && y0f >= 0.0 && x0f < (double)(s.w - 1) && y0f < (double)(s.h - 1)) {
    const int ix = (int)x0f, iy = (int)y0f;
    const int rb = s.w * CN * (int)sizeof(T);
    load_pair<T, CN>(row_ptr<const T>(s, iy), ix, wide, rb, v0, v1);
    load_pair<T, CN>(row_ptr<const T>(s, iy + 1), ix, wide, rb, v2, v3);
  } else {
    const long long ix = (long long)x0f, iy = (long long)y0f;
    if (a.border == kConstant && (ix < -1 || iy < -1 || ix >= s.w || iy >= s.h)) {
      const T cvT = round_to<T>(a.cv);
#pragma unroll
      for (int c = 0; c < CN; c++) o[c] = cvT;
      return;
    }
    const int x0 = border_map(ix, s.w, a.border), x1 = border_map(ix + 1, s.w, a.border);
    const int y0 = border_map(iy, s.h, a.border), y1 = border_map(iy + 1, s.h, a.border);
    const T *r0 = y0 >= 0 ? row_ptr<const T>(s, y0) : nullptr;
    const T *r1 = y1 >= 0 ? row_ptr<const T>(s, y1) : nullptr;
#pragma unroll
    for (int c = 0; c < CN; c++) {
      v0[c] = (r0 && x0 >= 0) ? to_f(r0[x0 * CN + c]) : a.cv;
      v1[c] = (r0 && x1 >= 0) ? to_f(r0[x1 * CN + c]) : a.cv;
      v2[c] = (r1 && x0 >= 0) ? to_f(r1[x0 * CN + c]) : a.cv;
      v3[c] = (r1 && x1 >= 0) ? to_f(r1[x1 * CN + c]) : a.cv;
    }
  }
#pragma unroll
  for (int c = 0; c < CN; c++) {
    float acc = 0.0f;
    acc = __fadd_rn(acc, __fmul_rn(v0[c], wt0));
    acc = __fadd_rn(acc, __fmul_rn(v1[c], wt1));
    acc = __fadd_rn(acc, __fmul_rn(v2[c], wt2));
    acc = __fadd_rn(acc, __fmul_rn(v3[c], wt3));
    o[c] = round_fast<T>(acc);
  }
}

template <class T>
inline float sat_value_host(double v) {
  // sat.cast(T, value) on the host, returned as f32 (geometry.zig:417, 674-676).
  if constexpr (IsFloat<T>::v) {
    return (float)v;
  } else {
    if (v != v) return 0.0f;
    double r = std::nearbyint(v);
    if (r <= (double)Lim<T>::lo) return (float)Lim<T>::lo;
    if (r >= (double)Lim<T>::hi) return (float)Lim<T>::hi;
    return (float)(int)r;
  }
}

// Four consecutive pixels x0 .. x0 + 3 of row y of a one-channel u8 image,
// INTER_LINEAR (the arithmetic of affine_px / persp_px): the coordinates of
// all four first, then every tap load, then the blends, so that the four
// pixels' loads are in flight together, and one 4-byte store (the
// destination row at x0 is 4-byte aligned). Pixels whose taps leave the
// source, or that lie past the row, take the per-pixel path.
//
// The fast path keeps conversions off the transcendental unit, with the
// same values: a pixel's taps are inside exactly when 0 <= sx < w - 1 and
// 0 <= sy < h - 1 (floor and the +-1e9 clamp change nothing there, and NaN
// fails the test); floor(sx) is then sx + 2^52 rounded toward zero, less
// 2^52 (2^23 in f32), exact below 2^52 (2^23), its low word the integer;
// tap bytes become f32 as 2^23 + b - 2^23; x steps by exact adds.
template <bool PERSP>
__device__ __forceinline__ void warp4_u8(const DImg &s, const DImg &d, const PerArgs &pa, const AffArgs &aa, int wide,
                                         int x0, int y) {
  constexpr double kTwo52 = 4503599627370496.0;
  constexpr float kTwo23 = 8388608.0f;
  float ax[4], ay[4];
  long long off[4];  // source offset of tap (ix, iy); -1: per-pixel path
  float bx = 0.0f, by = 0.0f, xf0 = 0.0f;
  double fx0 = 0.0, fy = 0.0;
  if constexpr (PERSP) {
    fx0 = (double)x0;
    fy = (double)y;
  } else {
    const float yf = (float)y;
    bx = __fadd_rn(__fmul_rn(aa.m[1], yf), aa.m[2]);
    by = __fadd_rn(__fmul_rn(aa.m[4], yf), aa.m[5]);
    xf0 = (float)x0;
  }
  // Inner bounds: below w - 1 (h - 1), and below the clamp (and 2^23 in f32).
  const double limx = fmin((double)(s.w - 1), 1.0e9), limy = fmin((double)(s.h - 1), 1.0e9);
  const float flimx = fminf((float)(s.w - 1), kTwo23), flimy = fminf((float)(s.h - 1), kTwo23);
#pragma unroll
  for (int p = 0; p < 4; p++) {
    bool inner;
    int ix, iy;
    if constexpr (PERSP) {
      const double fx = __dadd_rn(fx0, (double)p);
      double sx = __dadd_rn(__dadd_rn(__dmul_rn(pa.m[0], fx), __dmul_rn(pa.m[1], fy)), pa.m[2]);
      double sy = __dadd_rn(__dadd_rn(__dmul_rn(pa.m[3], fx), __dmul_rn(pa.m[4], fy)), pa.m[5]);
      const double w = __dadd_rn(__dadd_rn(__dmul_rn(pa.m[6], fx), __dmul_rn(pa.m[7], fy)), pa.m[8]);
      const double iw = w != 0.0 ? __drcp_rn(w) : 0.0;
      sx = __dmul_rn(sx, iw);
      sy = __dmul_rn(sy, iw);
      inner = sx >= 0.0 && sy >= 0.0 && sx < limx && sy < limy;
      const double tx = __dadd_rz(inner ? sx : 0.0, kTwo52), ty = __dadd_rz(inner ? sy : 0.0, kTwo52);
      ix = (int)__double2loint(tx);
      iy = (int)__double2loint(ty);
      ax[p] = (float)__dsub_rn(sx, __dsub_rn(tx, kTwo52));
      ay[p] = (float)__dsub_rn(sy, __dsub_rn(ty, kTwo52));
    } else {
      const float xf = __fadd_rn(xf0, (float)p);
      const float sx = fmaf(aa.m[0], xf, bx), sy = fmaf(aa.m[3], xf, by);
      inner = sx >= 0.0f && sy >= 0.0f && sx < flimx && sy < flimy;
      const float tx = __fadd_rz(inner ? sx : 0.0f, kTwo23), ty = __fadd_rz(inner ? sy : 0.0f, kTwo23);
      ix = (int)(__float_as_uint(tx) & 0x7FFFFFu);
      iy = (int)(__float_as_uint(ty) & 0x7FFFFFu);
      ax[p] = __fsub_rn(sx, __fsub_rn(tx, kTwo23));
      ay[p] = __fsub_rn(sy, __fsub_rn(ty, kTwo23));
    }
    off[p] = inner && x0 + p < d.w ? (long long)iy * s.stride + ix : -1;
  }
  float v[4][4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const uint8_t *r = s.p + (off[p] < 0 ? 0 : off[p]);  // in bounds either way
    v[p][0] = __fsub_rn(__uint_as_float(0x4B000000u | __ldg(r)), kTwo23);
    v[p][1] = __fsub_rn(__uint_as_float(0x4B000000u | __ldg(r + 1)), kTwo23);
    v[p][2] = __fsub_rn(__uint_as_float(0x4B000000u | __ldg(r + s.stride)), kTwo23);
    v[p][3] = __fsub_rn(__uint_as_float(0x4B000000u | __ldg(r + s.stride + 1)), kTwo23);
  }
  uint32_t out = 0;
#pragma unroll
  for (int p = 0; p < 4; p++) {
    float val;
    if constexpr (PERSP) {
      const float one_ax = __fsub_rn(1.0f, ax[p]), one_ay = __fsub_rn(1.0f, ay[p]);
      float acc = 0.0f;
      acc = __fadd_rn(acc, __fmul_rn(v[p][0], __fmul_rn(one_ax, one_ay)));
      acc = __fadd_rn(acc, __fmul_rn(v[p][1], __fmul_rn(ax[p], one_ay)));
      acc = __fadd_rn(acc, __fmul_rn(v[p][2], __fmul_rn(one_ax, ay[p])));
      acc = __fadd_rn(acc, __fmul_rn(v[p][3], __fmul_rn(ax[p], ay[p])));
      val = acc;
    } else {
      const float v0 = fmaf(ax[p], __fsub_rn(v[p][1], v[p][0]), v[p][0]);
      const float v1 = fmaf(ax[p], __fsub_rn(v[p][3], v[p][2]), v[p][2]);
      val = fmaf(ay[p], __fsub_rn(v1, v0), v0);
    }
    out |= (uint32_t)round_u8(val) << (8 * p);
  }
  uint8_t *o = row_ptr<uint8_t>(d, y) + x0;
  const unsigned fast = (off[0] >= 0 ? 1u : 0u) | (off[1] >= 0 ? 2u : 0u) | (off[2] >= 0 ? 4u : 0u) | (off[3] >= 0 ? 8u : 0u);
  if (fast == 15u) {
    *reinterpret_cast<uint32_t *>(o) = out;
    return;
  }
  const int np = min(4, d.w - x0);
#pragma unroll 1
  for (int p = 0; p < np; p++) {
    if ((fast >> p) & 1u) {
      o[p] = (uint8_t)(out >> (8 * p));
    } else if constexpr (PERSP) {
      persp_px<uint8_t, 1>(s, d, pa, wide, x0 + p, y);
    } else {
      affine_px<uint8_t, 1>(s, d, aa, wide, x0 + p, y);
    }
  }
}

}  // namespace wp
}  // namespace vb
