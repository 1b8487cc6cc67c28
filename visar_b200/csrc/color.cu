// cvtColor (src/imgproc/color.zig). Integer paths use OpenCV's fixed point:
// gray = (b*3735 + g*19235 + r*9798 + 2^14) >> 15 (color.zig:120-129, 394),
// YCrCb at 14 bits (color.zig:166-207), HSV with the sdiv/hdiv tables at 12
// bits (color.zig:405-532). Float paths keep VISAR's unfused operation order.
#include "vb.h"

namespace vb {

namespace {

constexpr int kYShift = 14, kR2Y = 4899, kG2Y = 9617, kB2Y = 1868;
constexpr int kHsvShift = 12;

// OpenCV's RGB2HSV_b tables: sdiv[i] = round(255*2^12 / i), hdiv[i] =
// round(180*2^12 / (6 i)), round half away from zero (color.zig:408-419).
struct HsvTabs {
  int sdiv[256];
  int hdiv[256];
};
__constant__ HsvTabs c_hsv;
bool g_hsv_ready[64] = {};

template <class T>
__device__ __forceinline__ T max_alpha() {
  if constexpr (IsFloat<T>::v) return T(1.0f);
  else return T(Lim<T>::hi);
}

// One pixel of a conversion; T is the sample type.
template <class T, int KIND, int SCN, int DCN, int SB, int DB>
__device__ __forceinline__ void convert_px(const T *p, T *o) {
  if constexpr (KIND == kReorder) {
    const bool swap = SB != DB;
    if (swap) {
      o[0] = p[2]; o[1] = p[1]; o[2] = p[0];
    } else {
      o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
    }
    if constexpr (DCN == 4) o[3] = SCN == 4 ? p[3] : max_alpha<T>();
  } else if constexpr (KIND == kGray) {
    constexpr int bi = SB, ri = 2 - SB;
    if constexpr (IsFloat<T>::v) {
      o[0] = __fadd_rn(__fadd_rn(__fmul_rn(p[bi], 0.114f), __fmul_rn(p[1], 0.587f)), __fmul_rn(p[ri], 0.299f));
    } else {
      const uint32_t y = ((uint32_t)p[bi] * kB2G + (uint32_t)p[1] * kG2G + (uint32_t)p[ri] * kR2G + (1u << (kGrayShift - 1))) >> kGrayShift;
      o[0] = (T)y;
    }
  } else if constexpr (KIND == kFromGray) {
    const T v = p[0];
    o[0] = v; o[1] = v; o[2] = v;
    if constexpr (DCN == 4) o[3] = max_alpha<T>();
  } else if constexpr (KIND == kYcrcb) {
    if constexpr (IsFloat<T>::v) {
      const float b = p[SB], g = p[1], r = p[2 - SB];
      const float y = __fadd_rn(__fadd_rn(__fmul_rn(b, 0.114f), __fmul_rn(g, 0.587f)), __fmul_rn(r, 0.299f));
      o[0] = y;
      o[1] = __fadd_rn(__fmul_rn(__fsub_rn(r, y), 0.713f), 0.5f);
      o[2] = __fadd_rn(__fmul_rn(__fsub_rn(b, y), 0.564f), 0.5f);
    } else {
      const int b = p[SB], g = p[1], r = p[2 - SB];
      const int half = 1 << (kYShift - 1);
      const int y = (b * kB2Y + g * kG2Y + r * kR2Y + half) >> kYShift;
      const int delta = 128 << kYShift;
      o[0] = (T)min(max(y, 0), 255);
      o[1] = (T)min(max(((r - y) * 11682 + delta + half) >> kYShift, 0), 255);
      o[2] = (T)min(max(((b - y) * 9241 + delta + half) >> kYShift, 0), 255);
    }
  } else if constexpr (KIND == kFromYcrcb) {
    if constexpr (IsFloat<T>::v) {
      const float y = p[0], cr = __fsub_rn(p[1], 0.5f), cb = __fsub_rn(p[2], 0.5f);
      o[DB] = __fadd_rn(y, __fmul_rn(cb, 1.773f));
      o[1] = __fadd_rn(__fadd_rn(y, __fmul_rn(cb, -0.344f)), __fmul_rn(cr, -0.714f));
      o[2 - DB] = __fadd_rn(y, __fmul_rn(cr, 1.403f));
    } else {
      const int y = p[0], cr = (int)p[1] - 128, cb = (int)p[2] - 128;
      const int half = 1 << (kYShift - 1);
      o[DB] = (T)min(max(y + ((cb * 29049 + half) >> kYShift), 0), 255);
      o[1] = (T)min(max(y + ((cb * -5636 + cr * -11698 + half) >> kYShift), 0), 255);
      o[2 - DB] = (T)min(max(y + ((cr * 22987 + half) >> kYShift), 0), 255);
    }
  } else if constexpr (KIND == kHsv) {
    if constexpr (IsFloat<T>::v) {
      // rgb2hsvF32 (color.zig:534-546)
      const float b = p[SB], g = p[1], r = p[2 - SB];
      const float eps = 1.1920928955078125e-07f;
      const float v = fmaxf(fmaxf(r, g), b);
      const float vmin = fminf(fminf(r, g), b);
      float diff = __fsub_rn(v, vmin);
      const float s = __fdiv_rn(diff, __fadd_rn(fabsf(v), eps));
      diff = __fdiv_rn(60.0f, __fadd_rn(diff, eps));
      float h;
      if (v == r) h = __fmul_rn(__fsub_rn(g, b), diff);
      else if (v == g) h = __fadd_rn(__fmul_rn(__fsub_rn(b, r), diff), 120.0f);
      else h = __fadd_rn(__fmul_rn(__fsub_rn(r, g), diff), 240.0f);
      if (h < 0) h = __fadd_rn(h, 360.0f);
      o[0] = h; o[1] = s; o[2] = v;
    } else {
      // rgb2hsvU8 (color.zig:515-532)
      const int b = p[SB], g = p[1], r = p[2 - SB];
      const int v = max(max(r, g), b);
      const int vmin = min(min(r, g), b);
      const int diff = v - vmin;
      const int vr = v == r ? -1 : 0;
      const int vg = v == g ? -1 : 0;
      const int half = 1 << (kHsvShift - 1);
      const int s = (diff * c_hsv.sdiv[v] + half) >> kHsvShift;
      int h = (vr & (g - b)) + (~vr & ((vg & (b - r + 2 * diff)) + ((~vg) & (r - g + 4 * diff))));
      h = (h * c_hsv.hdiv[diff] + half) >> kHsvShift;
      if (h < 0) h += 180;
      o[0] = (T)min(max(h, 0), 255);
      o[1] = (T)s;
      o[2] = (T)v;
    }
  } else if constexpr (KIND == kFromHsv) {
    // hsv2rgbF32 (color.zig:550-569); `1 - s*h` is one fma as in VISAR.
    float hh, hs, s, v;
    if constexpr (IsFloat<T>::v) {
      hh = p[0]; hs = 6.0f / 360.0f; s = p[1]; v = p[2];
    } else {
      hh = (float)p[0]; hs = 6.0f / 180.0f;
      s = __fmul_rn((float)p[1], 1.0f / 255.0f);
      v = __fmul_rn((float)p[2], 1.0f / 255.0f);
    }
    float rgb[3];
    if (s == 0) {
      rgb[0] = v; rgb[1] = v; rgb[2] = v;
    } else {
      float h = __fmul_rn(hh, hs);
      while (h < 0) h = __fadd_rn(h, 6.0f);
      while (h >= 6) h = __fsub_rn(h, 6.0f);
      int sector = (int)floorf(h);
      h = __fsub_rn(h, (float)sector);
      if (sector < 0 || sector >= 6) {
        sector = 0;
        h = 0;
      }
      const float tab[4] = {v, __fmul_rn(v, __fsub_rn(1.0f, s)), __fmul_rn(v, fmaf(-s, h, 1.0f)),
                            __fmul_rn(v, fmaf(-s, __fsub_rn(1.0f, h), 1.0f))};
      const unsigned char sd[6][3] = {{1, 3, 0}, {1, 0, 2}, {3, 0, 1}, {0, 2, 1}, {0, 1, 3}, {2, 1, 0}};
      rgb[0] = tab[sd[sector][2]];
      rgb[1] = tab[sd[sector][1]];
      rgb[2] = tab[sd[sector][0]];
    }
    if constexpr (IsFloat<T>::v) {
      o[DB] = rgb[2]; o[1] = rgb[1]; o[2 - DB] = rgb[0];
    } else {
      auto tr = [](float x) -> T { return (T)fminf(fmaxf(truncf(x), 0.0f), 255.0f); };
      o[DB] = tr(__fmul_rn(rgb[2], 255.0f));
      o[1] = tr(__fmul_rn(rgb[1], 255.0f));
      o[2 - DB] = tr(__fmul_rn(rgb[0], 255.0f));
    }
  }
}

// Generic kernel: one thread per pixel, 2-D grid over (pixels, rows).
template <class T, int KIND, int SCN, int DCN, int SB, int DB>
__global__ void __launch_bounds__(256) k_cvt(DImg s, DImg d) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= s.w) return;
  const T *sp = row_ptr<T>(s, y) + (long long)x * SCN;
  T *dp = row_ptr<T>(d, y) + (long long)x * DCN;
  T in[SCN];
#pragma unroll
  for (int c = 0; c < SCN; c++) in[c] = sp[c];
  T out[DCN];
  convert_px<T, KIND, SCN, DCN, SB, DB>(in, out);
#pragma unroll
  for (int c = 0; c < DCN; c++) dp[c] = out[c];
}

// u8 3- or 4-channel -> gray, 16 pixels per thread through 16-byte loads and
// one 16-byte store. Needs 16-byte aligned rows (checked by the launcher).
template <int SCN, int SB>
__global__ void __launch_bounds__(256) k_gray_u8_v16(DImg s, DImg d, int groups) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (gx >= groups) return;
  const int x0 = gx * 16;
  const uint8_t *sp = row_ptr<uint8_t>(s, y) + (long long)x0 * SCN;
  uint8_t *dp = row_ptr<uint8_t>(d, y) + x0;
  if (x0 + 16 <= s.w) {
    uint4 v[SCN];
#pragma unroll
    for (int k = 0; k < SCN; k++) v[k] = reinterpret_cast<const uint4 *>(sp)[k];
    const uint8_t *b = reinterpret_cast<const uint8_t *>(v);
    uint8_t o[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const uint32_t bb = b[i * SCN + SB], gg = b[i * SCN + 1], rr = b[i * SCN + 2 - SB];
      o[i] = (uint8_t)((bb * kB2G + gg * kG2G + rr * kR2G + (1u << (kGrayShift - 1))) >> kGrayShift);
    }
    *reinterpret_cast<uint4 *>(dp) = *reinterpret_cast<const uint4 *>(o);
  } else {
    for (int i = 0; x0 + i < s.w; i++) {
      const uint32_t bb = sp[i * SCN + SB], gg = sp[i * SCN + 1], rr = sp[i * SCN + 2 - SB];
      dp[i] = (uint8_t)((bb * kB2G + gg * kG2G + rr * kR2G + (1u << (kGrayShift - 1))) >> kGrayShift);
    }
  }
}

void ensure_hsv_tables() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || g_hsv_ready[dev]) return;
  HsvTabs t;
  t.sdiv[0] = 0;
  t.hdiv[0] = 0;
  for (int i = 1; i < 256; i++) {
    t.sdiv[i] = (int)std::round((double)(255 << kHsvShift) / (double)i);
    t.hdiv[i] = (int)std::round((double)(180 << kHsvShift) / (6.0 * (double)i));
  }
  cudaMemcpyToSymbol(c_hsv, &t, sizeof(t));
  g_hsv_ready[dev] = true;
}

template <class T, int KIND, int SCN, int DCN, int SB, int DB>
cudaError_t run(const DImg &s, const DImg &d, cudaStream_t st) {
  if constexpr (KIND == kGray && sizeof(T) == 1 && (SCN == 3 || SCN == 4)) {
    const bool aligned = ((uintptr_t)s.p % 16 == 0) && ((uintptr_t)d.p % 16 == 0) && (s.stride % 16 == 0) &&
                         (d.stride % 16 == 0);
    if (aligned) {
      const int groups = (s.w + 15) / 16;
      dim3 grid(ceil_div(groups, 256), s.h);
      k_gray_u8_v16<SCN, SB><<<grid, 256, 0, st>>>(s, d, groups);
      note_launch();
      return cudaGetLastError();
    }
  }
  dim3 grid(ceil_div(s.w, 256), s.h);
  k_cvt<T, KIND, SCN, DCN, SB, DB><<<grid, 256, 0, st>>>(s, d);
  note_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t dispatch(const DImg &s, const DImg &d, const ColorInfo &ci, cudaStream_t st) {
  switch (ci.kind) {
    case kReorder:
      if (ci.scn == 3 && ci.dcn == 3) return ci.sb != ci.db ? run<T, kReorder, 3, 3, 0, 2>(s, d, st) : run<T, kReorder, 3, 3, 0, 0>(s, d, st);
      if (ci.scn == 3 && ci.dcn == 4) return ci.sb != ci.db ? run<T, kReorder, 3, 4, 0, 2>(s, d, st) : run<T, kReorder, 3, 4, 0, 0>(s, d, st);
      if (ci.scn == 4 && ci.dcn == 3) return ci.sb != ci.db ? run<T, kReorder, 4, 3, 0, 2>(s, d, st) : run<T, kReorder, 4, 3, 0, 0>(s, d, st);
      if (ci.scn == 4 && ci.dcn == 4) return ci.sb != ci.db ? run<T, kReorder, 4, 4, 0, 2>(s, d, st) : run<T, kReorder, 4, 4, 0, 0>(s, d, st);
      break;
    case kGray:
      if (ci.scn == 3) return ci.sb == 0 ? run<T, kGray, 3, 1, 0, 0>(s, d, st) : run<T, kGray, 3, 1, 2, 0>(s, d, st);
      if (ci.scn == 4) return ci.sb == 0 ? run<T, kGray, 4, 1, 0, 0>(s, d, st) : run<T, kGray, 4, 1, 2, 0>(s, d, st);
      break;
    case kFromGray:
      return ci.dcn == 3 ? run<T, kFromGray, 1, 3, 0, 0>(s, d, st) : run<T, kFromGray, 1, 4, 0, 0>(s, d, st);
    case kHsv:
      if constexpr (sizeof(T) == 1) ensure_hsv_tables();
      return ci.sb == 0 ? run<T, kHsv, 3, 3, 0, 0>(s, d, st) : run<T, kHsv, 3, 3, 2, 0>(s, d, st);
    case kFromHsv:
      return ci.db == 0 ? run<T, kFromHsv, 3, 3, 0, 0>(s, d, st) : run<T, kFromHsv, 3, 3, 0, 2>(s, d, st);
    case kYcrcb:
      return ci.sb == 0 ? run<T, kYcrcb, 3, 3, 0, 0>(s, d, st) : run<T, kYcrcb, 3, 3, 2, 0>(s, d, st);
    case kFromYcrcb:
      return ci.db == 0 ? run<T, kFromYcrcb, 3, 3, 0, 0>(s, d, st) : run<T, kFromYcrcb, 3, 3, 0, 2>(s, d, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

// The caller has checked depth support per kind (color.zig:107-114).
cudaError_t launch_cvt_color(const DImg &s, const DImg &d, int depth, const ColorInfo &ci, cudaStream_t st) {
  if (s.w == 0 || s.h == 0) return cudaSuccess;
  switch (depth) {
    case k8U: return dispatch<uint8_t>(s, d, ci, st);
    case k16U:
      if (ci.kind == kHsv || ci.kind == kFromHsv || ci.kind == kYcrcb || ci.kind == kFromYcrcb) return cudaErrorInvalidValue;
      return dispatch<uint16_t>(s, d, ci, st);
    case k16S:
      if (ci.kind != kReorder && ci.kind != kFromGray) return cudaErrorInvalidValue;
      return dispatch<int16_t>(s, d, ci, st);
    case k32F: return dispatch<float>(s, d, ci, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace vb
