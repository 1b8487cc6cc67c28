// resize (src/imgproc/resize.zig, src/imgproc/resize_u8.zig). Coordinate and
// weight tables are built on the host (capi.cu) exactly as VISAR builds them;
// the kernels evaluate one output sample per thread with VISAR's arithmetic.
#include "vb.h"

namespace vb {

namespace {

// Nearest: output pixel (x, y) copies source pixel (xofs[x], yofs[y]).
template <class T>
__global__ void __launch_bounds__(256) k_nearest(DImg s, DImg d, const int *xofs, const int *yofs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const long long n = (long long)d.w * d.cn;
  if (i >= n) return;
  const int x = (int)(i / d.cn), ch = (int)(i - (long long)x * d.cn);
  row_ptr<T>(d, y)[i] = row_ptr<const T>(s, yofs[y])[(long long)xofs[x] * s.cn + ch];
}

// OpenCV's fixed-point bilinear for u8 (resize_u8.zig:651-711): each source
// row is resampled horizontally into (s0*w0 + s1*w1) >> 4, then
// ((h0*b0) >> 16) + ((h1*b1) >> 16) is rounded with (+2) >> 2 and clamped.
__global__ void __launch_bounds__(256) k_u8_linear(DImg s, DImg d, const LinTap *xt, const LinTap *yt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int cn = d.cn;
  const long long n = (long long)d.w * cn;
  if (i >= n) return;
  const int x = (int)(i / cn), ch = (int)(i - (long long)x * cn);
  const LinTap tx = xt[x], ty = yt[y];
  const uint8_t *r0 = row_ptr<const uint8_t>(s, ty.o0);
  const uint8_t *r1 = row_ptr<const uint8_t>(s, ty.o1);
  const long long a0 = (long long)tx.o0 * cn + ch, a1 = (long long)tx.o1 * cn + ch;
  const int h0 = ((int)r0[a0] * tx.w0 + (int)r0[a1] * tx.w1) >> 4;
  const int h1 = ((int)r1[a0] * tx.w0 + (int)r1[a1] * tx.w1) >> 4;
  const int t = ((h0 * ty.w0) >> 16) + ((h1 * ty.w1) >> 16);
  row_ptr<uint8_t>(d, y)[i] = (uint8_t)min(max((t + 2) >> 2, 0), 255);
}

// The same per output pixel with the channel count known at compile time:
// one 16-byte tap load, 32-bit offsets, the row taps uniform per CTA row.
template <int CN>
__global__ void __launch_bounds__(256) k_u8_linear_c(DImg s, DImg d, const LinTap *xt, const LinTap *yt) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= d.w) return;
  const int4 tx = *reinterpret_cast<const int4 *>(xt + x);
  const LinTap ty = yt[y];
  const uint8_t *r0 = row_ptr<const uint8_t>(s, ty.o0);
  const uint8_t *r1 = row_ptr<const uint8_t>(s, ty.o1);
  const int a0 = tx.x * CN, a1 = tx.y * CN;
  uint8_t *o = row_ptr<uint8_t>(d, y) + x * CN;
#pragma unroll
  for (int c = 0; c < CN; c++) {
    const int h0 = ((int)r0[a0 + c] * tx.z + (int)r0[a1 + c] * tx.w) >> 4;
    const int h1 = ((int)r1[a0 + c] * tx.z + (int)r1[a1 + c] * tx.w) >> 4;
    const int t = ((h0 * ty.w0) >> 16) + ((h1 * ty.w1) >> 16);
    o[c] = (uint8_t)min(max((t + 2) >> 2, 0), 255);
  }
}

// Exact halving, 4 output pixels per thread through 8-byte loads and 4-byte
// stores (rows 8-byte aligned; checked by the launcher).
template <int CN>
__global__ void __launch_bounds__(256) k_u8_half_v(DImg s, DImg d) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;  // group of 4 output pixels
  const int y = blockIdx.y;
  const int x0 = g * 4;
  if (x0 >= d.w) return;
  const uint8_t *a = row_ptr<const uint8_t>(s, 2 * y);
  const uint8_t *b = row_ptr<const uint8_t>(s, 2 * y + 1);
  uint8_t *o = row_ptr<uint8_t>(d, y);
  if (x0 + 4 <= d.w) {
    uint64_t ra[CN], rb[CN];
#pragma unroll
    for (int k = 0; k < CN; k++) {
      ra[k] = reinterpret_cast<const uint64_t *>(a + (size_t)x0 * 2 * CN)[k];
      rb[k] = reinterpret_cast<const uint64_t *>(b + (size_t)x0 * 2 * CN)[k];
    }
    const uint8_t *ba = reinterpret_cast<const uint8_t *>(ra);
    const uint8_t *bb = reinterpret_cast<const uint8_t *>(rb);
    uint32_t out[CN];
    uint8_t *ob = reinterpret_cast<uint8_t *>(out);
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
      for (int c = 0; c < CN; c++) {
        const int i = 2 * p * CN + c;
        ob[p * CN + c] = (uint8_t)(((unsigned)ba[i] + ba[i + CN] + bb[i] + bb[i + CN] + 2) >> 2);
      }
#pragma unroll
    for (int k = 0; k < CN; k++) reinterpret_cast<uint32_t *>(o + (size_t)x0 * CN)[k] = out[k];
  } else {
    for (int x = x0; x < d.w; x++)
      for (int c = 0; c < CN; c++) {
        const int i = 2 * x * CN + c;
        o[x * CN + c] = (uint8_t)(((unsigned)a[i] + a[i + CN] + b[i] + b[i + CN] + 2) >> 2);
      }
  }
}

// Exact halving (resize_u8.zig:381-447): (a + b + c + d + 2) >> 2.
__global__ void __launch_bounds__(256) k_u8_half(DImg s, DImg d) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int cn = d.cn;
  const long long n = (long long)d.w * cn;
  if (i >= n) return;
  const long long x = i / cn;
  const int ch = (int)(i - x * cn);
  const uint8_t *a = row_ptr<const uint8_t>(s, 2LL * y);
  const uint8_t *b = row_ptr<const uint8_t>(s, 2LL * y + 1);
  const long long j = 2 * x * cn + ch;
  row_ptr<uint8_t>(d, y)[i] = (uint8_t)(((unsigned)a[j] + a[j + cn] + b[j] + b[j + cn] + 2) >> 2);
}

// OpenCV's fixed-point bicubic for u8 (resize.zig:246-282, resize_u8.zig:742-763):
// integer horizontal sums, then an fma chain with weights b * 2^-22.
__global__ void __launch_bounds__(256) k_u8_cubic(DImg s, DImg d, const CubTap *xt, const CubTap *yt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int cn = d.cn;
  const long long n = (long long)d.w * cn;
  if (i >= n) return;
  const int x = (int)(i / cn), ch = (int)(i - (long long)x * cn);
  const CubTap tx = xt[x], ty = yt[y];
  float h[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint8_t *r = row_ptr<const uint8_t>(s, ty.o[k]);
    int acc = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) acc += (int)r[(long long)tx.o[j] * cn + ch] * tx.w[j];
    h[k] = (float)acc;
  }
  const float sc = 1.0f / (2048.0f * 2048.0f);
  float b[4];
#pragma unroll
  for (int k = 0; k < 4; k++) b[k] = __fmul_rn((float)ty.w[k], sc);
  const float v = fmaf(h[0], b[0], fmaf(h[1], b[1], fmaf(h[2], b[2], __fmul_rn(h[3], b[3]))));
  row_ptr<uint8_t>(d, y)[i] = cast_sat<uint8_t>(v);
}

// Integer-factor INTER_AREA. u8 with <= 4 channels (resize_u8.zig:1210-1277):
// the block sum times the f32 reciprocal of the block area, rounded half to
// even. Other cases follow the generic areaInt (resize.zig:425-464).
template <class T>
__global__ void __launch_bounds__(256) k_area_int(DImg s, DImg d, int ix, int iy, int mode) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int cn = d.cn;
  const long long n = (long long)d.w * cn;
  if (i >= n) return;
  const long long x = i / cn;
  const int ch = (int)(i - x * cn);
  const int area = ix * iy;
  T *o = row_ptr<T>(d, y) + i;
  if constexpr (!IsFloat<T>::v) {
  if (mode == 0) {  // u8 fast: f32 reciprocal
    unsigned sum = 0;
    for (int dy = 0; dy < iy; dy++) {
      const T *r = row_ptr<const T>(s, (long long)y * iy + dy);
      for (int dx = 0; dx < ix; dx++) sum += (unsigned)r[(x * ix + dx) * cn + ch];
    }
    const float scale = __fdiv_rn(1.0f, (float)area);
    *o = cast_sat<T>(__fmul_rn((float)sum, scale));
    return;
  } else if (mode == 1) {  // u8 2x2 on the generic path: round half up
    const T *a = row_ptr<const T>(s, 2LL * y);
    const T *b = row_ptr<const T>(s, 2LL * y + 1);
    const long long j = 2 * x * cn + ch;
    *o = (T)(((unsigned)a[j] + a[j + cn] + b[j] + b[j + cn] + 2) >> 2);
    return;
  } else if (mode == 2) {  // unsigned: (sum + area/2) / area
    unsigned long long sum = 0;
    for (int dy = 0; dy < iy; dy++) {
      const T *r = row_ptr<const T>(s, (long long)y * iy + dy);
      for (int dx = 0; dx < ix; dx++) sum += (unsigned long long)r[(x * ix + dx) * cn + ch];
    }
    *o = (T)((sum + (unsigned long long)(area / 2)) / (unsigned long long)area);
    return;
  }
  }
  {  // signed / float: f64 sum / area
    double sum = 0;
    for (int dy = 0; dy < iy; dy++) {
      const T *r = row_ptr<const T>(s, (long long)y * iy + dy);
      for (int dx = 0; dx < ix; dx++) sum = __dadd_rn(sum, (double)to_f(r[(x * ix + dx) * cn + ch]));
    }
    *o = cast_sat_d<T>(__ddiv_rn(sum, (double)area));
  }
}

// Fractional INTER_AREA (OpenCV's ResizeArea_Invoker; resize.zig:466-565,
// resize_u8.zig:1049-1208): per source row of the destination cell, the
// horizontal sum of s * alpha in table order, then sum(h * beta) in table
// order, all unfused f32.
template <class T>
__global__ void __launch_bounds__(256) k_area_frac(DImg s, DImg d, const AreaEnt *xtab, const int *xstart,
                                                   const AreaEnt *ytab, const int *ystart) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int cn = d.cn;
  const long long n = (long long)d.w * cn;
  if (i >= n) return;
  const int x = (int)(i / cn), ch = (int)(i - (long long)x * cn);
  const int xa = xstart[x], xb = xstart[x + 1];
  float acc = 0.0f;
  for (int e = ystart[y]; e < ystart[y + 1]; e++) {
    const AreaEnt ye = ytab[e];
    const T *r = row_ptr<const T>(s, ye.si);
    float h = __fmul_rn(to_f(r[(long long)xtab[xa].si * cn + ch]), xtab[xa].alpha);
    for (int k = xa + 1; k < xb; k++) h = __fadd_rn(h, __fmul_rn(to_f(r[(long long)xtab[k].si * cn + ch]), xtab[k].alpha));
    const float p = __fmul_rn(h, ye.alpha);
    acc = (e == ystart[y]) ? p : __fadd_rn(acc, p);
  }
  row_ptr<T>(d, y)[i] = cast_sat<T>(acc);
}

// Generic bilinear for u16 / i16 / f32 (resize.zig:284-423): f32 weights,
// h = s0*a0 + s1*a1, out = sat(h0*b0 + h1*b1), unfused.
template <class T>
__global__ void __launch_bounds__(256) k_linear_generic(DImg s, DImg d, const FLinTap *xt, const FLinTap *yt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int cn = d.cn;
  const long long n = (long long)d.w * cn;
  if (i >= n) return;
  const int x = (int)(i / cn), ch = (int)(i - (long long)x * cn);
  const FLinTap tx = xt[x], ty = yt[y];
  const T *r0 = row_ptr<const T>(s, ty.o0);
  const T *r1 = row_ptr<const T>(s, ty.o1);
  const long long a0 = (long long)tx.o0 * cn + ch, a1 = (long long)tx.o1 * cn + ch;
  const float h0 = __fadd_rn(__fmul_rn(to_f(r0[a0]), tx.a0), __fmul_rn(to_f(r0[a1]), tx.a1));
  const float h1 = __fadd_rn(__fmul_rn(to_f(r1[a0]), tx.a0), __fmul_rn(to_f(r1[a1]), tx.a1));
  row_ptr<T>(d, y)[i] = cast_sat<T>(__fadd_rn(__fmul_rn(h0, ty.a0), __fmul_rn(h1, ty.a1)));
}

// Generic bicubic in f32 (resize.zig:577-640).
template <class T>
__global__ void __launch_bounds__(256) k_cubic_generic(DImg s, DImg d, const FCubTap *xt, const FCubTap *yt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int cn = d.cn;
  const long long n = (long long)d.w * cn;
  if (i >= n) return;
  const int x = (int)(i / cn), ch = (int)(i - (long long)x * cn);
  const FCubTap tx = xt[x], ty = yt[y];
  float h[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const T *r = row_ptr<const T>(s, ty.o[k]);
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; j++) acc = __fadd_rn(acc, __fmul_rn(to_f(r[(long long)tx.o[j] * cn + ch]), tx.w[j]));
    h[k] = acc;
  }
  const float v = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(h[0], ty.w[0]), __fmul_rn(h[1], ty.w[1])), __fmul_rn(h[2], ty.w[2])),
                            __fmul_rn(h[3], ty.w[3]));
  row_ptr<T>(d, y)[i] = cast_sat<T>(v);
}

// Same-size resize: a copy (resize.zig:30).
__global__ void __launch_bounds__(256) k_copy_rows(DImg s, DImg d, long long row_bytes) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (i >= row_bytes) return;
  row_ptr<uint8_t>(d, y)[i] = row_ptr<const uint8_t>(s, y)[i];
}

inline dim3 grid_for(const DImg &d) { return dim3(ceil_div((long long)d.w * d.cn, 256), d.h); }

}  // namespace

#define VB_LAUNCH(kern, ...)                         \
  do {                                               \
    kern<<<grid_for(d), 256, 0, st>>>(__VA_ARGS__);  \
    note_launch();                                   \
    return cudaGetLastError();                       \
  } while (0)

cudaError_t launch_resize_nearest(const DImg &s, const DImg &d, int depth, const int *xofs, const int *yofs, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  switch (depth_size(depth)) {
    case 1: VB_LAUNCH(k_nearest<uint8_t>, s, d, xofs, yofs);
    case 2: VB_LAUNCH(k_nearest<uint16_t>, s, d, xofs, yofs);
    case 4: VB_LAUNCH(k_nearest<uint32_t>, s, d, xofs, yofs);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_resize_u8_linear(const DImg &s, const DImg &d, const LinTap *xt, const LinTap *yt, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  const dim3 g(ceil_div(d.w, 256), d.h);
  switch (d.cn) {
    case 1: k_u8_linear_c<1><<<g, 256, 0, st>>>(s, d, xt, yt); break;
    case 3: k_u8_linear_c<3><<<g, 256, 0, st>>>(s, d, xt, yt); break;
    case 4: k_u8_linear_c<4><<<g, 256, 0, st>>>(s, d, xt, yt); break;
    default: VB_LAUNCH(k_u8_linear, s, d, xt, yt);
  }
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_resize_u8_half(const DImg &s, const DImg &d, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  const bool al = ((uintptr_t)s.p % 8 == 0) && (s.stride % 8 == 0) && ((uintptr_t)d.p % 4 == 0) && (d.stride % 4 == 0);
  const dim3 g(ceil_div(ceil_div(d.w, 4), 256), d.h);
  if (al) {
    switch (d.cn) {
      case 1: k_u8_half_v<1><<<g, 256, 0, st>>>(s, d); note_launch(); return cudaGetLastError();
      case 2: k_u8_half_v<2><<<g, 256, 0, st>>>(s, d); note_launch(); return cudaGetLastError();
      case 3: k_u8_half_v<3><<<g, 256, 0, st>>>(s, d); note_launch(); return cudaGetLastError();
      case 4: k_u8_half_v<4><<<g, 256, 0, st>>>(s, d); note_launch(); return cudaGetLastError();
    }
  }
  VB_LAUNCH(k_u8_half, s, d);
}

cudaError_t launch_resize_u8_cubic(const DImg &s, const DImg &d, const CubTap *xt, const CubTap *yt, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  VB_LAUNCH(k_u8_cubic, s, d, xt, yt);
}

// u8fast: the u8 <= 4-channel kernel (f32 reciprocal); otherwise the generic areaInt.
cudaError_t launch_resize_area_int(const DImg &s, const DImg &d, int depth, int ix, int iy, bool u8fast, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  switch (depth) {
    case k8U: {
      const int mode = u8fast ? 0 : (ix == 2 && iy == 2) ? 1 : 2;
      VB_LAUNCH(k_area_int<uint8_t>, s, d, ix, iy, mode);
    }
    case k16U: VB_LAUNCH(k_area_int<uint16_t>, s, d, ix, iy, 2);
    case k16S: VB_LAUNCH(k_area_int<int16_t>, s, d, ix, iy, 3);
    case k32F: VB_LAUNCH(k_area_int<float>, s, d, ix, iy, 3);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_resize_area_frac(const DImg &s, const DImg &d, int depth, const AreaEnt *xtab, int nx, const int *xstart,
                                    const AreaEnt *ytab, const int *ystart, cudaStream_t st) {
  (void)nx;
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  switch (depth) {
    case k8U: VB_LAUNCH(k_area_frac<uint8_t>, s, d, xtab, xstart, ytab, ystart);
    case k16U: VB_LAUNCH(k_area_frac<uint16_t>, s, d, xtab, xstart, ytab, ystart);
    case k16S: VB_LAUNCH(k_area_frac<int16_t>, s, d, xtab, xstart, ytab, ystart);
    case k32F: VB_LAUNCH(k_area_frac<float>, s, d, xtab, xstart, ytab, ystart);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_resize_linear_generic(const DImg &s, const DImg &d, int depth, const FLinTap *xt, const FLinTap *yt, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  switch (depth) {
    case k16U: VB_LAUNCH(k_linear_generic<uint16_t>, s, d, xt, yt);
    case k16S: VB_LAUNCH(k_linear_generic<int16_t>, s, d, xt, yt);
    case k32F: VB_LAUNCH(k_linear_generic<float>, s, d, xt, yt);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_resize_cubic_generic(const DImg &s, const DImg &d, int depth, const FCubTap *xt, const FCubTap *yt, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  switch (depth) {
    case k8U: VB_LAUNCH(k_cubic_generic<uint8_t>, s, d, xt, yt);
    case k16U: VB_LAUNCH(k_cubic_generic<uint16_t>, s, d, xt, yt);
    case k16S: VB_LAUNCH(k_cubic_generic<int16_t>, s, d, xt, yt);
    case k32F: VB_LAUNCH(k_cubic_generic<float>, s, d, xt, yt);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_copy_image(const DImg &s, const DImg &d, int depth, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  const long long rb = (long long)d.w * d.cn * depth_size(depth);
  k_copy_rows<<<dim3(ceil_div(rb, 256), d.h), 256, 0, st>>>(s, d, rb);
  note_launch();
  return cudaGetLastError();
}

}  // namespace vb
