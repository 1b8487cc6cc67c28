// warpAffine / warpPerspective (src/imgproc/geometry.zig:403-672).
//
// warpAffine follows OpenCV 5's float kernel as VISAR does: the inverse
// matrix (f64 on the host) is rounded to f32; per row bx = m1*y + m2 and
// by = m4*y + m5 (unfused); per pixel sx = fma(m0, x, bx), sy = fma(m3, x, by);
// bilinear blending is fma(ax, p1 - p0, p0), fma(ax, p3 - p2, p2), then
// fma(ay, v1 - v0, v0), rounded half to even. warpPerspective works per
// pixel in f64 with a reciprocal of w, and blends with four f32 weights.
#include "warp.cuh"

namespace vb {

namespace {

using namespace wp;


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
  const double iw = w != 0.0 ? __drcp_rn(w) : 0.0;  // correctly rounded: equals 1.0 / w
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

template <class T, int CN>
__global__ void __launch_bounds__(256) k_warp_affine_c(DImg s, DImg d, AffArgs a, int wide) {
  // 8 x 32 thread blocks: each warp covers 8 x 4 output pixels, a compact
  // source footprint for rotated sampling.
  const int x = blockIdx.x * 8 + threadIdx.x;
  const int y = blockIdx.y * 32 + threadIdx.y;
  if (x < d.w && y < d.h) affine_px<T, CN>(s, d, a, wide, x, y);
}

template <class T, int CN>
__global__ void __launch_bounds__(256) k_warp_persp_c(DImg s, DImg d, PerArgs a, int wide) {
  const int x = blockIdx.x * 8 + threadIdx.x;
  const int y = blockIdx.y * 32 + threadIdx.y;
  if (x < d.w && y < d.h) persp_px<T, CN>(s, d, a, wide, x, y);
}

// One-channel u8 INTER_LINEAR: 8 x 32 threads of 4 consecutive pixels each
// (a block covers 32 x 32 output pixels, a warp 32 x 4).
template <bool PERSP>
__global__ void __launch_bounds__(256) k_warp4_u8(DImg s, DImg d, PerArgs pa, AffArgs aa, int wide) {
  const int x0 = (blockIdx.x * 8 + threadIdx.x) * 4;
  const int y = blockIdx.y * 32 + threadIdx.y;
  if (x0 < d.w && y < d.h) warp4_u8<PERSP>(s, d, pa, aa, wide, x0, y);
}

// k_warp4_u8 applies: one-channel u8, INTER_LINEAR, 4-byte aligned destination rows.
inline bool warp4_ok(const DImg &d, int interp, int cn, size_t tsize) {
  return tsize == 1 && cn == 1 && interp != 0 && (uintptr_t)d.p % 4 == 0 && d.stride % 4 == 0;
}

template <class T>
cudaError_t run_affine(const DImg &s, const DImg &d, const float m[6], int interp, int border, double value, cudaStream_t st) {
  AffArgs a;
  for (int i = 0; i < 6; i++) a.m[i] = m[i];
  a.interp = interp;
  a.border = border;
  a.cv = sat_value_host<T>(value);
  const dim3 g2(ceil_div(d.w, 8), ceil_div(d.h, 32)), b2(8, 32);
  const int wide = ((uintptr_t)s.p % 8 == 0) && (s.stride % 8 == 0);
  const bool al4 = ((uintptr_t)s.p % 4 == 0) && (s.stride % 4 == 0);
  if (warp4_ok(d, interp, d.cn, sizeof(T))) {
    k_warp4_u8<false><<<dim3(ceil_div(d.w, 32), ceil_div(d.h, 32)), b2, 0, st>>>(s, d, PerArgs{}, a, wide);
    note_launch();
    return cudaGetLastError();
  }
  switch (d.cn) {
    case 1: k_warp_affine_c<T, 1><<<g2, b2, 0, st>>>(s, d, a, wide); break;
    case 3: k_warp_affine_c<T, 3><<<g2, b2, 0, st>>>(s, d, a, wide); break;
    case 4:
      if (sizeof(T) != 1 || al4) {
        k_warp_affine_c<T, 4><<<g2, b2, 0, st>>>(s, d, a, wide);
        break;
      }
      [[fallthrough]];
    default: k_warp_affine<T><<<dim3(ceil_div(d.w, 256), d.h), 256, 0, st>>>(s, d, a);
  }
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
  const dim3 g2(ceil_div(d.w, 8), ceil_div(d.h, 32)), b2(8, 32);
  const int wide = ((uintptr_t)s.p % 8 == 0) && (s.stride % 8 == 0);
  const bool al4 = ((uintptr_t)s.p % 4 == 0) && (s.stride % 4 == 0);
  if (warp4_ok(d, interp, d.cn, sizeof(T))) {
    k_warp4_u8<true><<<dim3(ceil_div(d.w, 32), ceil_div(d.h, 32)), b2, 0, st>>>(s, d, a, AffArgs{}, wide);
    note_launch();
    return cudaGetLastError();
  }
  switch (d.cn) {
    case 1: k_warp_persp_c<T, 1><<<g2, b2, 0, st>>>(s, d, a, wide); break;
    case 3: k_warp_persp_c<T, 3><<<g2, b2, 0, st>>>(s, d, a, wide); break;
    case 4:
      if (sizeof(T) != 1 || al4) {
        k_warp_persp_c<T, 4><<<g2, b2, 0, st>>>(s, d, a, wide);
        break;
      }
      [[fallthrough]];
    default: k_warp_persp<T><<<dim3(ceil_div(d.w, 256), d.h), 256, 0, st>>>(s, d, a);
  }
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
