// Shared device/host helpers for the visar-b200 kernels.
//
// Arithmetic conventions (they make integer outputs bit-exact to VISAR and
// keep f32 outputs in VISAR's operation order):
//  * the library is compiled with --fmad=false, so a*b+c is never contracted;
//    fmaf/fma appear exactly where VISAR calls @mulAdd;
//  * float -> integer conversions round half to even and saturate
//    (src/core/saturate.zig:8-49, src/core/simd.zig:153-189).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vb {

// OpenCV BORDER_* numbering (src/imgproc/border.zig:5-17).
enum Border : int { kConstant = 0, kReplicate = 1, kReflect = 2, kWrap = 3, kReflect101 = 4 };

// A 2-D image in device memory: HWC samples, `stride` bytes between rows.
struct DImg {
  uint8_t *p;
  long long stride;
  int w, h, cn;
};

template <class T>
__host__ __device__ __forceinline__ T *row_ptr(const DImg &im, long long y) {
  return reinterpret_cast<T *>(im.p + y * im.stride);
}

// Index extrapolation of src/imgproc/border.zig:22-37. VISAR loops until the
// reflected index lands inside; the loop is periodic (period 2n for reflect,
// 2n-2 for reflect101), so one modulo gives the same index. Returns -1 for
// a constant border outside the range.
__host__ __device__ __forceinline__ int border_map(long long p, int len, int border) {
  if (p >= 0 && p < len) return (int)p;
  // Coordinates just outside the image (the common case): no division.
  if (p >= -(long long)len && p < 2LL * len && len > 1) {
    const int q = (int)p;
    switch (border) {
      case kReplicate: return q < 0 ? 0 : len - 1;
      case kReflect: return q < 0 ? -q - 1 : 2 * len - 1 - q;
      case kReflect101:
        if (q < 0 && q > -len) return -q;
        if (q >= len && q < 2 * len - 1) return 2 * len - 2 - q;
        break;
      case kWrap: return q < 0 ? q + len : q - len;
      default: break;
    }
  }
  switch (border) {
    case kConstant:
      return -1;
    case kReplicate:
      return p < 0 ? 0 : len - 1;
    case kReflect: {
      if (len == 1) return 0;
      long long per = 2LL * len;
      long long q = p % per;
      if (q < 0) q += per;
      return (int)(q < len ? q : per - 1 - q);
    }
    case kReflect101: {
      if (len == 1) return 0;
      long long per = 2LL * len - 2;
      long long q = p % per;
      if (q < 0) q += per;
      return (int)(q < len ? q : per - q);
    }
    case kWrap: {
      long long q = p % len;
      if (q < 0) q += len;
      return (int)q;
    }
  }
  return -1;
}

template <class T> struct Lim;
template <> struct Lim<uint8_t> { static constexpr int lo = 0, hi = 255; };
template <> struct Lim<uint16_t> { static constexpr int lo = 0, hi = 65535; };
template <> struct Lim<int16_t> { static constexpr int lo = -32768, hi = 32767; };
template <> struct Lim<int32_t> { static constexpr int lo = INT32_MIN, hi = INT32_MAX; };

template <class T> struct IsFloat { static constexpr bool v = false; };
template <> struct IsFloat<float> { static constexpr bool v = true; };

// sat.cast(D, f32) (src/core/saturate.zig:20-49): NaN -> 0, round half to even
// (the f32 value is exact in f64, so rintf is the same rounding), clamp.
template <class D>
__device__ __forceinline__ D cast_sat(float x) {
  if constexpr (IsFloat<D>::v) {
    return x;
  } else {
    if (x != x) return D(0);
    float r = rintf(x);
    if (r <= (float)Lim<D>::lo) return D(Lim<D>::lo);
    if (r >= (float)Lim<D>::hi) return D(Lim<D>::hi);
    return D((int)r);
  }
}

// sat.cast(D, f64).
template <class D>
__device__ __forceinline__ D cast_sat_d(double x) {
  if constexpr (IsFloat<D>::v) {
    return (float)x;
  } else {
    if (x != x) return D(0);
    double r = rint(x);
    if (r <= (double)Lim<D>::lo) return D(Lim<D>::lo);
    if (r >= (double)Lim<D>::hi) return D(Lim<D>::hi);
    return D((int)r);
  }
}

// satV (src/imgproc/filter.zig:44-58) for an f32 source: clamp first (a NaN
// clamps to the low bound), then round half to even.
template <class D>
__device__ __forceinline__ D satv_f(float x) {
  if constexpr (IsFloat<D>::v) {
    return x;
  } else {
    float c = fminf(fmaxf(x, (float)Lim<D>::lo), (float)Lim<D>::hi);
    return D((int)rintf(c));
  }
}

// satV for an integer source: clamp.
template <class D>
__device__ __forceinline__ D satv_i(long long x) {
  if constexpr (IsFloat<D>::v) {
    return (float)x;
  } else {
    if (x < Lim<D>::lo) return D(Lim<D>::lo);
    if (x > Lim<D>::hi) return D(Lim<D>::hi);
    return D(x);
  }
}

template <class T>
__device__ __forceinline__ float to_f(T v) {
  return (float)v;
}

__host__ __device__ __forceinline__ unsigned ceil_div(unsigned long long a, unsigned b) {
  return (unsigned)((a + b - 1) / b);
}

}  // namespace vb
