// Fast erode / dilate pass for u8 images whose structuring element rows are
// runs centred on the anchor (rect, cross and ellipse of odd size, which is
// what getStructuringElement builds, src/imgproc/morph.zig:32-59), with a
// horizontal reach of at most 4 samples (half-width * channels <= 4).
//
// Output (x, y) = min (or max) over element rows ky of the horizontal min
// over [x - d_ky, x + d_ky] of source row y + ky - ay, pixels outside the
// image ignored (they hold the identity). A CTA of NT threads owns NT
// 4-sample words of a band of RH output rows; every thread loads all RH+KH-1
// source rows of its word (identity-padded) into registers and shared
// memory, then after one barrier computes the horizontal run minima of each
// row with byte permutes and 4-lane SIMD minima (__vminu4 / __vmaxu4), and
// the vertical combination in registers. min/max are exact, so the result
// equals VISAR's per-tap definition (morph.zig:489-519).
#pragma once
#include <vector>

#include "vb.h"

namespace vb {
namespace fast {

struct MFArgs {
  int d[16];      // half-width of element row ky (-1: empty row)
  int dv[3];      // the distinct half-widths, dv[0] <= dv[1] <= dv[2]
  int ndv;
  int ay;
  long long n;    // samples per row
};

// Builds the kernel arguments for a structuring element (kh x kw mask,
// anchor at the centre); false when the fast pass does not cover it.
inline bool morph_fast_args(const std::vector<uint8_t> &mask, int kw, int kh, int cn, int width, MFArgs &a) {
  if (!(cn == 1 || cn == 3 || cn == 4)) return false;
  if (kw % 2 == 0 || kh % 2 == 0 || kh > 9) return false;
  a = MFArgs{};
  a.ay = kh / 2;
  a.n = (long long)width * cn;
  const int ax = kw / 2;
  int ndv = 0;
  for (int ky = 0; ky < kh; ky++) {
    int j1 = -1, j2 = -1;
    for (int x = 0; x < kw; x++)
      if (mask[(size_t)ky * kw + x]) {
        if (j1 < 0) j1 = x;
        j2 = x;
      }
    if (j1 < 0) {
      a.d[ky] = -1;
      continue;
    }
    for (int x = j1; x <= j2; x++)
      if (!mask[(size_t)ky * kw + x]) return false;  // not a single run
    if (ax - j1 != j2 - ax) return false;            // not centred
    const int dh = ax - j1;
    if (dh * cn > 4) return false;
    a.d[ky] = dh;
    bool seen = false;
    for (int i = 0; i < ndv; i++) seen = seen || a.dv[i] == dh;
    if (!seen) {
      if (ndv == 3) return false;
      a.dv[ndv++] = dh;
    }
  }
  if (ndv == 0) return false;
  for (int i = ndv; i < 3; i++) a.dv[i] = a.dv[ndv - 1];
  a.ndv = ndv;
  return true;
}

template <bool MAX>
__device__ __forceinline__ uint32_t vop(uint32_t a, uint32_t b) {
  return MAX ? __vmaxu4(a, b) : __vminu4(a, b);
}

// Samples gs-4..gs+7 are (prev, cur, next); returns the word shifted by s
// samples (s in [-4, 4]).
__device__ __forceinline__ uint32_t shifted(uint32_t prev, uint32_t cur, uint32_t next, int s) {
  if (s >= 0) return __byte_perm(cur, next, 0x3210 + 0x1111 * s);
  return __byte_perm(prev, cur, 0x3210 + 0x1111 * (4 + s));
}

template <int CN, bool MAX>
__device__ __forceinline__ uint32_t hrun(uint32_t prev, uint32_t cur, uint32_t next, int dh) {
  uint32_t v = cur;
  for (int k = 1; k <= dh; k++) {
    v = vop<MAX>(v, shifted(prev, cur, next, k * CN));
    v = vop<MAX>(v, shifted(prev, cur, next, -k * CN));
  }
  return v;
}

template <int CN, int KH, int NT, int RH, bool MAX>
__device__ __forceinline__ void morph_band(const DImg &s, const DImg &d, const MFArgs &a, int bx, int by,
                                           uint32_t (*buf)[NT]) {
  constexpr int NR = RH + KH - 1;
  constexpr int OW = NT - 2;  // one halo word on each side
  const uint32_t ident = MAX ? 0u : 0xFFFFFFFFu;
  const int t = threadIdx.x;
  const long long gw = (long long)bx * OW + t - 1;
  const long long gs = gw * 4;
  const long long n = a.n;
  const int y0 = by * RH;
  const int H = s.h;

#pragma unroll
  for (int j = 0; j < NR; j++) {
    const int sy = y0 - a.ay + j;
    uint32_t w = ident;
    if (sy >= 0 && sy < H) {
      const uint8_t *rp = row_ptr<const uint8_t>(s, sy);
      if (gs >= 0 && gs + 4 <= n) {
        w = *reinterpret_cast<const uint32_t *>(rp + gs);
      } else {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const long long g = gs + k;
          if (g >= 0 && g < n) w = (w & ~(0xFFu << (8 * k))) | ((uint32_t)rp[g] << (8 * k));
        }
      }
    }
    buf[j][t] = w;
  }
  __syncthreads();
  if (t == 0 || t == NT - 1 || gs >= n) return;  // no barrier follows in this function

  // Horizontal run minima of every source row, for each distinct half-width.
  uint32_t h0[NR], h1[NR], h2[NR];
#pragma unroll
  for (int j = 0; j < NR; j++) {
    const uint32_t p = buf[j][t - 1], c = buf[j][t], x = buf[j][t + 1];
    h0[j] = hrun<CN, MAX>(p, c, x, a.dv[0]);
    h1[j] = a.ndv > 1 ? hrun<CN, MAX>(p, c, x, a.dv[1]) : h0[j];
    h2[j] = a.ndv > 2 ? hrun<CN, MAX>(p, c, x, a.dv[2]) : h1[j];
  }
  const bool full = gs + 4 <= n;
#pragma unroll
  for (int r = 0; r < RH; r++) {
    const int y = y0 + r;
    if (y >= H) break;
    uint32_t v = ident;
#pragma unroll
    for (int ky = 0; ky < KH; ky++) {
      const int dk = a.d[ky];
      if (dk < 0) continue;
      const uint32_t hv = dk == a.dv[0] ? h0[r + ky] : dk == a.dv[1] ? h1[r + ky] : h2[r + ky];
      v = vop<MAX>(v, hv);
    }
    uint8_t *dp = row_ptr<uint8_t>(d, y);
    if (full) *reinterpret_cast<uint32_t *>(dp + gs) = v;
    else
      for (int k = 0; k < 4 && gs + k < n; k++) dp[gs + k] = (uint8_t)(v >> (8 * k));
  }
}

template <int CN, int KH, int NT, int RH, bool MAX>
__global__ void __launch_bounds__(NT) k_morph_fast(DImg s, DImg d, MFArgs a) {
  __shared__ uint32_t buf[RH + KH - 1][NT];
  morph_band<CN, KH, NT, RH, MAX>(s, d, a, blockIdx.x, blockIdx.y, buf);
}

}  // namespace fast
}  // namespace vb
