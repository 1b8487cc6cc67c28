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
  const double iw = w != 0.0 ? __ddiv_rn(1.0, w) : 0.0;
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

}  // namespace wp
}  // namespace vb
