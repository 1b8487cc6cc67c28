// warpAffine / warpPerspective (src/imgproc/geometry.zig:403-672).
//
// warpAffine follows OpenCV 5's float kernel as VISAR does: the inverse
// matrix (f64 on the host) is rounded to f32; per row bx = m1*y + m2 and
// by = m4*y + m5 (unfused); per pixel sx = fma(m0, x, bx), sy = fma(m3, x, by);
// bilinear blending is fma(ax, p1 - p0, p0), fma(ax, p3 - p2, p2), then
// fma(ay, v1 - v0, v0), rounded half to even. warpPerspective works per
// pixel in f64 with a reciprocal of w, and blends with four f32 weights.
#include "vb.h"

namespace vb {

namespace {

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

template <class T>
__global__ void __launch_bounds__(256) k_warp_affine(DImg s, DImg d, AffArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= d.w) return;
  const int cn = d.cn;
  const float yf = (float)y;
  const float bx = __fadd_rn(__fmul_rn(a.m[1], yf), a.m[2]);
  const float by = __fadd_rn(__fmul_rn(a.m[4], yf), a.m[5]);
  const float xf = (float)x;
  const float sx = fmaf(a.m[0], xf, bx);
  const float sy = fmaf(a.m[3], xf, by);
  T *o = row_ptr<T>(d, y) + (long long)x * cn;
  const T cvT = round_to<T>(a.cv);
  if (a.interp == 0) {
    // nearestPixel (geometry.zig:496-502)
    const long long ix = to_idx(rintf(fminf(fmaxf(sx, -4.0e6f), 4.0e6f)));
    const long long iy = to_idx(rintf(fminf(fmaxf(sy, -4.0e6f), 4.0e6f)));
    const int mx = border_map(ix, s.w, a.border);
    const int my = border_map(iy, s.h, a.border);
    if (mx >= 0 && my >= 0) {
      const T *p = row_ptr<const T>(s, my) + (long long)mx * cn;
      for (int c = 0; c < cn; c++) o[c] = p[c];
    } else {
      for (int c = 0; c < cn; c++) o[c] = cvT;
    }
    return;
  }
  // linearPixel (geometry.zig:508-533)
  const float fx = floorf(sx), fy = floorf(sy);
  const float ax = __fsub_rn(sx, fx), ay = __fsub_rn(sy, fy);
  const long long ix = to_idx(fx), iy = to_idx(fy);
  if (a.border == kConstant && (ix < -1 || iy < -1 || ix >= s.w || iy >= s.h)) {
    for (int c = 0; c < cn; c++) o[c] = cvT;
    return;
  }
  const int x0 = border_map(ix, s.w, a.border), x1 = border_map(ix + 1, s.w, a.border);
  const int y0 = border_map(iy, s.h, a.border), y1 = border_map(iy + 1, s.h, a.border);
  const T *r0 = y0 >= 0 ? row_ptr<const T>(s, y0) : nullptr;
  const T *r1 = y1 >= 0 ? row_ptr<const T>(s, y1) : nullptr;
  for (int c = 0; c < cn; c++) {
    const float p0 = (r0 && x0 >= 0) ? to_f(r0[(long long)x0 * cn + c]) : a.cv;
    const float p1 = (r0 && x1 >= 0) ? to_f(r0[(long long)x1 * cn + c]) : a.cv;
    const float p2 = (r1 && x0 >= 0) ? to_f(r1[(long long)x0 * cn + c]) : a.cv;
    const float p3 = (r1 && x1 >= 0) ? to_f(r1[(long long)x1 * cn + c]) : a.cv;
    const float v0 = fmaf(ax, __fsub_rn(p1, p0), p0);
    const float v1 = fmaf(ax, __fsub_rn(p3, p2), p2);
    o[c] = round_to<T>(fmaf(ay, __fsub_rn(v1, v0), v0));
  }
}

__device__ __forceinline__ double clamp_e9(double v) {
  // std.math.clamp(v, -1e9, 1e9) = @max(-1e9, @min(v, 1e9)); a NaN gives 1e9.
  return fmax(-1.0e9, fmin(v, 1.0e9));
}

template <class T>
__global__ void __launch_bounds__(256) k_warp_persp(DImg s, DImg d, PerArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= d.w) return;
  const int cn = d.cn;
  const double fx = (double)x, fy = (double)y;
  double sx = __dadd_rn(__dadd_rn(__dmul_rn(a.m[0], fx), __dmul_rn(a.m[1], fy)), a.m[2]);
  double sy = __dadd_rn(__dadd_rn(__dmul_rn(a.m[3], fx), __dmul_rn(a.m[4], fy)), a.m[5]);
  const double w = __dadd_rn(__dadd_rn(__dmul_rn(a.m[6], fx), __dmul_rn(a.m[7], fy)), a.m[8]);
  const double iw = w != 0.0 ? __ddiv_rn(1.0, w) : 0.0;
  sx = __dmul_rn(sx, iw);
  sy = __dmul_rn(sy, iw);
  T *o = row_ptr<T>(d, y) + (long long)x * cn;
  const T cvT = round_to<T>(a.cv);
  if (a.interp == 0) {
    const long long ix = (long long)round(clamp_e9(sx));
    const long long iy = (long long)round(clamp_e9(sy));
    const int mx = border_map(ix, s.w, a.border);
    const int my = border_map(iy, s.h, a.border);
    if (mx >= 0 && my >= 0) {
      const T *p = row_ptr<const T>(s, my) + (long long)mx * cn;
      for (int c = 0; c < cn; c++) o[c] = p[c];
    } else {
      for (int c = 0; c < cn; c++) o[c] = cvT;
    }
    return;
  }
  const double x0f = floor(clamp_e9(sx));
  const double y0f = floor(clamp_e9(sy));
  const float ax = (float)__dsub_rn(sx, x0f);
  const float ay = (float)__dsub_rn(sy, y0f);
  const long long ix = (long long)x0f, iy = (long long)y0f;
  if (a.border == kConstant && (ix < -1 || iy < -1 || ix >= s.w || iy >= s.h)) {
    for (int c = 0; c < cn; c++) o[c] = cvT;
    return;
  }
  const int x0 = border_map(ix, s.w, a.border), x1 = border_map(ix + 1, s.w, a.border);
  const int y0 = border_map(iy, s.h, a.border), y1 = border_map(iy + 1, s.h, a.border);
  const float one_ax = __fsub_rn(1.0f, ax), one_ay = __fsub_rn(1.0f, ay);
  const float wt[4] = {__fmul_rn(one_ax, one_ay), __fmul_rn(ax, one_ay), __fmul_rn(one_ax, ay), __fmul_rn(ax, ay)};
  const T *r0 = y0 >= 0 ? row_ptr<const T>(s, y0) : nullptr;
  const T *r1 = y1 >= 0 ? row_ptr<const T>(s, y1) : nullptr;
  for (int c = 0; c < cn; c++) {
    const float v0 = (r0 && x0 >= 0) ? to_f(r0[(long long)x0 * cn + c]) : a.cv;
    const float v1 = (r0 && x1 >= 0) ? to_f(r0[(long long)x1 * cn + c]) : a.cv;
    const float v2 = (r1 && x0 >= 0) ? to_f(r1[(long long)x0 * cn + c]) : a.cv;
    const float v3 = (r1 && x1 >= 0) ? to_f(r1[(long long)x1 * cn + c]) : a.cv;
    float acc = 0.0f;
    acc = __fadd_rn(acc, __fmul_rn(v0, wt[0]));
    acc = __fadd_rn(acc, __fmul_rn(v1, wt[1]));
    acc = __fadd_rn(acc, __fmul_rn(v2, wt[2]));
    acc = __fadd_rn(acc, __fmul_rn(v3, wt[3]));
    o[c] = cast_sat<T>(acc);
  }
}

template <class T>
float sat_value_host(double v) {
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

template <class T>
cudaError_t run_affine(const DImg &s, const DImg &d, const float m[6], int interp, int border, double value, cudaStream_t st) {
  AffArgs a;
  for (int i = 0; i < 6; i++) a.m[i] = m[i];
  a.interp = interp;
  a.border = border;
  a.cv = sat_value_host<T>(value);
  k_warp_affine<T><<<dim3(ceil_div(d.w, 256), d.h), 256, 0, st>>>(s, d, a);
  note_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t run_persp(const DImg &s, const DImg &d, const double m[9], int interp, int border, double value, cudaStream_t st) {
  PerArgs a;
  for (int i = 0; i < 9; i++) a.m[i] = m[i];
  a.interp = interp;
  a.border = border;
  a.cv = sat_value_host<T>(value);
  k_warp_persp<T><<<dim3(ceil_div(d.w, 256), d.h), 256, 0, st>>>(s, d, a);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_warp_affine(const DImg &s, const DImg &d, int depth, const float m[6], int interp, int border, double value,
                               cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  switch (depth) {
    case k8U: return run_affine<uint8_t>(s, d, m, interp, border, value, st);
    case k16U: return run_affine<uint16_t>(s, d, m, interp, border, value, st);
    case k16S: return run_affine<int16_t>(s, d, m, interp, border, value, st);
    case k32F: return run_affine<float>(s, d, m, interp, border, value, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_warp_perspective(const DImg &s, const DImg &d, int depth, const double m[9], int interp, int border,
                                    double value, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  switch (depth) {
    case k8U: return run_persp<uint8_t>(s, d, m, interp, border, value, st);
    case k16U: return run_persp<uint16_t>(s, d, m, interp, border, value, st);
    case k16S: return run_persp<int16_t>(s, d, m, interp, border, value, st);
    case k32F: return run_persp<float>(s, d, m, interp, border, value, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace vb
