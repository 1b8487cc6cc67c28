// Fast separable filter for the common shapes: 3x3 / 5x5 / 7x7 kernels on
// 1-, 3- or 4-channel u8 (fixed-point Gaussian) and f32 (Gaussian) images.
//
// Thread layout: see k_sep_fast. The input band is staged in shared memory
// with cp.async (every row of the band in flight at once), and both passes
// are short rolled loops over the rows, so the code stays resident in the
// instruction cache.
//
// Arithmetic. u8: the fixed-point taps are 8-bit integers summing to 256, so
// every vertical sum is <= 255*256 and every 2-D sum <= 256*65280 < 2^24:
// f32 fma evaluates them exactly, in any order, and the result is rounded
// once as (v + 2^15) >> 16 -- VISAR's u8 Gaussian (filter.zig:511-547).
// f32: the vector-body / scalar-tail operation orders of VISAR's engine are
// reproduced per sample (see sepfilter.cu), so results are bit-exact.
#pragma once
#include <algorithm>
#include <type_traits>

#include "vb.h"

namespace vb {
namespace fast {

struct FastArgs {
  float kx[7], ky[7];
  int border, n16, symx, symy, shift;
  long long n;  // samples per row
};

__device__ __forceinline__ long long fdiv(long long a, int b) {
  long long q = a / b;
  if ((a % b) != 0 && (a < 0)) q--;
  return q;
}

__device__ __forceinline__ float u8f(uint32_t w, int k) {
  // byte k of w as an exact f32 (2^23 + b, minus 2^23)
  return __fsub_rn(__uint_as_float(0x4B000000u | ((w >> (8 * k)) & 0xFFu)), 8388608.0f);
}

// Vertical or horizontal tap sum of one sample. EXACT: integer-valued sums
// below 2^24 (any order). Otherwise VISAR's f32 order: the vector body folds
// mirrored taps by the kernel's symmetry SYM (filter.zig:232-252), the
// scalar tail sums left to right (filter.zig:254-258).
template <int K, bool EXACT, int SYM>
__device__ __forceinline__ float tsum_body(const float *v, const float *k) {
  constexpr int R = K / 2;
  if constexpr (EXACT) {
    float a = __fmul_rn(v[R], k[R]);
#pragma unroll
    for (int i = 0; i < R; i++) a = fmaf(__fadd_rn(v[i], v[K - 1 - i]), k[i], a);
    return a;
  } else if constexpr (SYM == 1) {
    float a = __fmul_rn(v[R], k[R]);
#pragma unroll
    for (int i = 0; i < R; i++) a = __fadd_rn(a, __fmul_rn(__fadd_rn(v[i], v[K - 1 - i]), k[i]));
    return a;
  } else if constexpr (SYM == 2) {
    float a = 0.0f;
#pragma unroll
    for (int i = 0; i < R; i++) a = __fadd_rn(a, __fmul_rn(__fsub_rn(v[K - 1 - i], v[i]), k[K - 1 - i]));
    return a;
  } else {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < K; j++) a = __fadd_rn(a, __fmul_rn(v[j], k[j]));
    return a;
  }
}

template <int K>
__device__ __forceinline__ float tsum_tail(const float *v, const float *k) {
  float a = __fmul_rn(k[0], v[0]);
#pragma unroll
  for (int j = 1; j < K; j++) a = __fadd_rn(a, __fmul_rn(k[j], v[j]));
  return a;
}

__device__ __forceinline__ void cp_async(void *smem, const void *gmem, int bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem));
}

template <class S>
struct Word;  // 4 samples as stored in shared memory
template <>
struct Word<uint8_t> {
  using T = uint32_t;
};
template <>
struct Word<float> {
  using T = float4;
};

template <class S>
__device__ __forceinline__ void unpack(const typename Word<S>::T &w, float *o) {
  if constexpr (sizeof(S) == 1) {
#pragma unroll
    for (int k = 0; k < 4; k++) o[k] = u8f(w, k);
  } else {
    o[0] = w.x; o[1] = w.y; o[2] = w.z; o[3] = w.w;
  }
}

template <class S>
__device__ __forceinline__ typename Word<S>::T pack_in(const float *v) {
  if constexpr (sizeof(S) == 1) {
    uint32_t w = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) w |= (uint32_t)v[k] << (8 * k);
    return w;
  } else {
    return make_float4(v[0], v[1], v[2], v[3]);
  }
}

// Vertical pass of one word column: a KY-row register window walks down the
// band. SEL: some column of the word uses VISAR's scalar-tail order.
template <class S, int KY, int NT, int RH, bool EXACT, int SYM, bool SEL>
__device__ __forceinline__ void vpass(typename Word<S>::T (*sin)[NT], float4 (*sv)[NT], const float *ky, const bool *vtail,
                                      int t) {
  float win[KY][4];
#pragma unroll
  for (int j = 0; j < KY - 1; j++) unpack<S>(sin[j][t], win[j]);
#pragma unroll 1
  for (int r = 0; r < RH; r++) {
    unpack<S>(sin[r + KY - 1][t], win[KY - 1]);
    float vs[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float col[KY];
#pragma unroll
      for (int j = 0; j < KY; j++) col[j] = win[j][k];
      if constexpr (SEL) vs[k] = vtail[k] ? tsum_tail<KY>(col, ky) : tsum_body<KY, EXACT, SYM>(col, ky);
      else vs[k] = tsum_body<KY, EXACT, SYM>(col, ky);
    }
    sv[r][t] = make_float4(vs[0], vs[1], vs[2], vs[3]);
#pragma unroll
    for (int j = 0; j < KY - 1; j++)
#pragma unroll
      for (int k = 0; k < 4; k++) win[j][k] = win[j + 1][k];
  }
}

// u8 result of an exact f32 sum v < 2^24: (v + 2^(s-1)) >> s.
__device__ __forceinline__ unsigned fin_u8(float v, int shift) {
  const unsigned u = __float2uint_rz(v);
  const unsigned q = (u + (1u << (shift - 1))) >> shift;
  return q > 255u ? 255u : q;
}

// Horizontal pass of one output word for all rows of the band.
template <class S, int KX, int CN, int NT, int RH, int HW, bool EXACT, int SYM, bool SEL>
__device__ __forceinline__ void hpass(float4 (*sv)[NT], const DImg &d, const FastArgs &a, int t, long long gs, int y0,
                                      const bool *otail) {
  constexpr int RX = KX / 2;
  const long long n = a.n;
  const bool full = gs + 4 <= n;
#pragma unroll 1
  for (int r = 0; r < RH; r++) {
    const int y = y0 + r;
    if (y >= d.h) break;
    float rr[(2 * HW + 1) * 4];
#pragma unroll
    for (int q = 0; q < 2 * HW + 1; q++) {
      const float4 v = sv[r][t - HW + q];
      rr[q * 4 + 0] = v.x; rr[q * 4 + 1] = v.y; rr[q * 4 + 2] = v.z; rr[q * 4 + 3] = v.w;
    }
    float o[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float tap[KX];
#pragma unroll
      for (int i = 0; i < KX; i++) tap[i] = rr[HW * 4 + k + (i - RX) * CN];
      if constexpr (SEL) o[k] = otail[k] ? tsum_tail<KX>(tap, a.kx) : tsum_body<KX, EXACT, SYM>(tap, a.kx);
      else o[k] = tsum_body<KX, EXACT, SYM>(tap, a.kx);
    }
    S *dp = row_ptr<S>(d, y);
    if constexpr (sizeof(S) == 1) {
      uint32_t packed = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) packed |= fin_u8(o[k], a.shift) << (8 * k);
      if (full) *reinterpret_cast<uint32_t *>(dp + gs) = packed;
      else
        for (int k = 0; k < 4 && gs + k < n; k++) dp[gs + k] = (uint8_t)(packed >> (8 * k));
    } else {
      if (full) *reinterpret_cast<float4 *>(dp + gs) = make_float4(o[0], o[1], o[2], o[3]);
      else
        for (int k = 0; k < 4 && gs + k < n; k++) dp[gs + k] = o[k];
    }
  }
}

// A CTA filters a band of RH output rows x NT 4-sample words.
//  1. Every source row of the band (RH + KY - 1 rows) is copied into shared
//     memory with cp.async, all requests in flight at once (words that reach
//     outside the row go through the border map instead).
//  2. Vertical pass: each thread walks its word's column down the band with
//     a KY-row register window (a small rolled loop), writing the vertical
//     sums to shared memory.
//  3. Horizontal pass: each output thread reads its word and the halo words
//     (aligned 16-byte loads) per row and writes the output word.
// The first and last HW words of a CTA are halo words (not output).
template <class S, int KX, int KY, int CN, int NT, int RH, bool EXACT, int SYMX, int SYMY>
__device__ __forceinline__ void sep_band(const DImg &s, const DImg &d, const FastArgs &a, int bx, int by,
                                         unsigned char *smem_raw) {
  using WT = typename Word<S>::T;
  constexpr int RX = KX / 2, RY = KY / 2;
  constexpr int HW = (RX * CN + 3) / 4;
  constexpr int OW = NT - 2 * HW;
  constexpr int NR = RH + KY - 1;
  WT(*sin)[NT] = reinterpret_cast<WT(*)[NT]>(smem_raw);
  // Vertical sums: for f32 row r of the sums overwrites input row r, which
  // the thread writing it (the only reader of that column) has consumed.
  float4(*sv)[NT] = sizeof(WT) == sizeof(float4) ? reinterpret_cast<float4(*)[NT]>(smem_raw)
                                                  : reinterpret_cast<float4(*)[NT]>(smem_raw + sizeof(WT) * NR * NT);

  const int t = threadIdx.x;
  const long long gw = (long long)bx * OW + t - HW;
  const long long gs = gw * 4;
  const int W = s.w, H = s.h;
  const long long n = a.n;
  const int y0 = by * RH;
  const bool inside = gs >= 0 && gs + 4 <= n;

  // Words reaching outside the row: their columns' border-mapped sample
  // indices (the same for every row), -1 for a constant-border column.
  int msi[4] = {0, 0, 0, 0};
  if (!inside) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int g = (int)gs + k;
      const int px = g >= 0 ? g / CN : -((-g + CN - 1) / CN);
      const int mx = border_map(px, W, a.border);
      msi[k] = mx < 0 ? -1 : mx * CN + (g - px * CN);
    }
  }
#pragma unroll 1
  for (int j = 0; j < NR; j++) {
    const int my = border_map(y0 - RY + j, H, a.border);
    if (my < 0) {
      float z[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      sin[j][t] = pack_in<S>(z);
    } else if (inside) {
      cp_async(&sin[j][t], row_ptr<const S>(s, my) + gs, (int)sizeof(WT));
    } else {
      const S *rp = row_ptr<const S>(s, my);
      float v[4];
#pragma unroll
      for (int k = 0; k < 4; k++) v[k] = msi[k] < 0 ? 0.0f : (float)rp[msi[k]];
      sin[j][t] = pack_in<S>(v);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();

  // VISAR's scalar tail can only be reached by the CTAs at the right end of
  // a row (and, on narrow images, by reflected halo columns of CTA 0).
  const long long end_sample = ((long long)bx * OW - HW + NT) * 4;
  const bool tail_cta = !EXACT && (end_sample > a.n16 || (bx == 0 && a.n16 < 8LL * NT));
  bool vtail[4] = {false, false, false, false};
  bool any_vtail = false;
  if (tail_cta) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int g = (int)gs + k;
      const int px = g >= 0 ? g / CN : -((-g + CN - 1) / CN);
      const int ch = g - px * CN;
      const int mx = border_map(px, W, a.border);
      vtail[k] = mx >= 0 && (mx * CN + ch) >= a.n16;  // the column's own sample index
      any_vtail = any_vtail || vtail[k];
    }
  }
  if (any_vtail) vpass<S, KY, NT, RH, EXACT, SYMY, true>(sin, sv, a.ky, vtail, t);
  else vpass<S, KY, NT, RH, EXACT, SYMY, false>(sin, sv, a.ky, vtail, t);
  __syncthreads();
  if (t >= HW && t < NT - HW && gs < n) {
    bool otail[4];
    bool any_otail = false;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      otail[k] = tail_cta && (gs + k) >= a.n16;
      any_otail = any_otail || otail[k];
    }
    if (any_otail) hpass<S, KX, CN, NT, RH, HW, EXACT, SYMX, true>(sv, d, a, t, gs, y0, otail);
    else hpass<S, KX, CN, NT, RH, HW, EXACT, SYMX, false>(sv, d, a, t, gs, y0, otail);
  }
}

template <class S, int KX, int KY, int CN, int NT, int RH, bool EXACT, int SYMX, int SYMY>
__global__ void __launch_bounds__(NT) k_sep_fast(DImg s, DImg d, FastArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  sep_band<S, KX, KY, CN, NT, RH, EXACT, SYMX, SYMY>(s, d, a, blockIdx.x, blockIdx.y, smem_raw);
}

}  // namespace fast
}  // namespace vb
