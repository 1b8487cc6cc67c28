// Warp-strip stencils for u8 images: a warp owns a strip of 32 four-sample
// words across RH output rows and walks down it, keeping the vertical window
// in registers; horizontal neighbours come from the adjacent lanes by warp
// shuffles. The outer lanes of a strip are halo (loaded, not written), so a
// strip writes 32 - 2*halo words. No shared memory and no block barriers:
// each warp streams its own rows, with kBatch row loads in flight.
//
// Two operations:
//  * gauss_strip: u8 Gaussian whose fixed-point taps are g * binomial(K)
//    with g a power of two (the 3x3 and 5x5 sigma <= 0 kernels: [64,128,64]
//    and [16,64,96,64,16], filter.zig:363-390). Then the exact result
//    (sum kx*ky*v + 2^15) >> 16 equals (H + 2^(15-2e)) >> (16-2e) with
//    g = 2^e and H = sum bx*by*v <= 255 * (2^(K-1))^2 < 2^16, so both passes
//    run on two samples per 32-bit register (16-bit lanes that never carry).
//  * morph_strip: erode / dilate with a centred-run element whose per-row
//    half-widths are a compile-time profile (rect, cross, ellipse 3-9), one
//    pass or two fused (erode then dilate = OPEN, dilate then erode = CLOSE).
//    Samples are held two per register in 16-bit lanes, where min/max are
//    native instructions (byte-lane min/max are not). Out-of-image pixels hold
//    the identity (morph.zig:489-519).
//
// Rows stream through a double buffer: the loads of the next kBatch rows are
// issued before the current kBatch rows are computed.
#pragma once
#include "morphfast.cuh"
#include "vb.h"

namespace vb {
namespace strip {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kBatch = 8;  // row loads in flight per lane

// Column description of one lane's word.
struct Cols {
  long long gs;  // first sample of the word
  bool inside;   // all four samples inside the row
  int msi[4];    // sample index each byte reads (-1: fill value)
};

// Gaussian rows: samples outside the row go through the border map (constant
// border: fill). Morphology (ident): outside samples take the fill value.
template <int CN>
__device__ __forceinline__ Cols make_cols(long long gs, long long n, int W, int border, bool ident) {
  Cols c;
  c.gs = gs;
  c.inside = gs >= 0 && gs + 4 <= n;
#pragma unroll
  for (int k = 0; k < 4; k++) c.msi[k] = -1;
  if (!c.inside) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const long long g = gs + k;
      if (ident) {
        c.msi[k] = (g >= 0 && g < n) ? (int)g : -1;
      } else {
        const long long px = g >= 0 ? g / CN : -((-g + CN - 1) / CN);
        const int mx = border_map(px, W, border);
        c.msi[k] = mx < 0 ? -1 : (int)(mx * CN + (g - px * CN));
      }
    }
  }
  return c;
}

__device__ __forceinline__ uint32_t load_word(const uint8_t *row, const Cols &c, uint32_t fill) {
  if (c.inside) return __ldg(reinterpret_cast<const uint32_t *>(row + c.gs));
  uint32_t w = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t b = c.msi[k] < 0 ? ((fill >> (8 * k)) & 0xFFu) : (uint32_t)__ldg(row + c.msi[k]);
    w |= b << (8 * k);
  }
  return w;
}

__device__ __forceinline__ void store_word(uint8_t *row, long long gs, long long n, uint32_t w) {
  if (gs + 4 <= n) {
    *reinterpret_cast<uint32_t *>(row + gs) = w;
  } else {
    for (int k = 0; k < 4 && gs + k < n; k++) row[gs + k] = (uint8_t)(w >> (8 * k));
  }
}

// ------------------------------------------------------------ Gaussian

template <int K>
struct Binom;
template <>
struct Binom<3> {
  static constexpr int e = 6;  // g = 64
};
template <>
struct Binom<5> {
  static constexpr int e = 4;  // g = 16
};

// Pair (V[s], V[s+1]) in 16-bit lanes, s relative to the lane's word start,
// from the pairs of words -NW..NW (pq[2*(w+NW)] = samples 0,1 of word w).
template <int NW>
__device__ __forceinline__ uint32_t pair_at(const uint32_t *pq, int s) {
  const int t = s + 4 * NW;
  return (t & 1) ? __byte_perm(pq[t >> 1], pq[(t >> 1) + 1], 0x5432) : pq[t >> 1];
}

// Horizontal binomial sums of the two output pairs of this lane's word, from
// the vertical sums (lo = samples 0,1; hi = samples 2,3) of every lane.
template <int K, int CN>
__device__ __forceinline__ void hsum(uint32_t lo, uint32_t hi, uint32_t &h0, uint32_t &h1) {
  constexpr int R = K / 2;
  constexpr int NW = (R * CN + 3) / 4;
  uint32_t pq[2 * (2 * NW + 1) + 1];
  pq[2 * NW] = lo;
  pq[2 * NW + 1] = hi;
#pragma unroll
  for (int k = 1; k <= NW; k++) {
    pq[2 * (NW - k)] = __shfl_up_sync(kFull, lo, k);
    pq[2 * (NW - k) + 1] = __shfl_up_sync(kFull, hi, k);
    pq[2 * (NW + k)] = __shfl_down_sync(kFull, lo, k);
    pq[2 * (NW + k) + 1] = __shfl_down_sync(kFull, hi, k);
  }
  pq[2 * (2 * NW + 1)] = 0;
  uint32_t h[2];
#pragma unroll
  for (int o = 0; o < 2; o++) {
    const int c = 2 * o;
    if constexpr (K == 3) {
      h[o] = pair_at<NW>(pq, c - CN) + pair_at<NW>(pq, c + CN) + (pair_at<NW>(pq, c) << 1);
    } else {
      const uint32_t a = pair_at<NW>(pq, c - 2 * CN) + pair_at<NW>(pq, c + 2 * CN);
      const uint32_t b = pair_at<NW>(pq, c - CN) + pair_at<NW>(pq, c + CN);
      h[o] = a + (b << 2) + pair_at<NW>(pq, c) * 6u;
    }
  }
  h0 = h[0];
  h1 = h[1];
}

struct GaussArgs {
  int border;
};

// One strip tile: words [tx*OW - NW, tx*OW - NW + 32) of rows
// [ty*RH, ty*RH + RH); `lane` is this thread's lane.
template <int K, int CN, int RH>
__device__ __forceinline__ void gauss_strip(const DImg &s, const DImg &d, int border, int tx, int ty, int lane) {
  constexpr int R = K / 2;
  constexpr int NW = (R * CN + 3) / 4;
  constexpr int OW = 32 - 2 * NW;
  constexpr int NR = RH + K - 1;
  constexpr int E = Binom<K>::e;
  constexpr int SH = 16 - 2 * E;
  constexpr uint32_t RND = (1u << (SH - 1)) * 0x00010001u;
  const long long n = (long long)s.w * CN;
  const long long gw = (long long)tx * OW - NW + lane;
  const Cols c = make_cols<CN>(gw * 4, n, s.w, border, false);
  const int y0 = ty * RH;
  const bool out_lane = lane >= NW && lane < 32 - NW && c.gs < n;
  // Binomial cascade of pairwise sums; after row j the last stage holds the
  // binomial sum of rows j-K+1..j.
  uint32_t pl[K - 1], ph[K - 1];
#pragma unroll
  for (int k = 0; k < K - 1; k++) pl[k] = ph[k] = 0;
  auto load_batch = [&](int jb, uint32_t (&w)[kBatch]) {
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      w[k] = 0;
      if (jb + k < NR) {
        const int my = border_map(y0 - R + jb + k, s.h, border);
        if (my >= 0) w[k] = load_word(row_ptr<const uint8_t>(s, my), c, 0u);
      }
    }
  };
  uint32_t w[kBatch], wn[kBatch];
  load_batch(0, w);
#pragma unroll 1
  for (int jb = 0; jb < NR; jb += kBatch) {
    if (jb + kBatch < NR) load_batch(jb + kBatch, wn);
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      const int j = jb + k;
      if (j >= NR) break;
      uint32_t cl = __byte_perm(w[k], 0, 0x4140), ch = __byte_perm(w[k], 0, 0x4342);
#pragma unroll
      for (int q = 0; q < K - 1; q++) {
        const uint32_t nl = cl + pl[q], nh = ch + ph[q];
        pl[q] = cl;
        ph[q] = ch;
        cl = nl;
        ch = nh;
      }
      if (j < K - 1) continue;  // window not full yet (warp-uniform)
      uint32_t h0, h1;
      hsum<K, CN>(cl, ch, h0, h1);
      const int y = y0 + j - (K - 1);
      if (out_lane && y < d.h) {
        const uint32_t t0 = (h0 + RND) >> SH, t1 = (h1 + RND) >> SH;
        store_word(row_ptr<uint8_t>(d, y), c.gs, n, __byte_perm(t0, t1, 0x6420));
      }
    }
#pragma unroll
    for (int k = 0; k < kBatch; k++) w[k] = wn[k];
  }
}

// ---------------------------------------------------------- morphology

// A structuring element as per-row half-widths of centred runs (-1: empty
// row), e.g. Prof<0, 2, 2, 2, 0> for the 5x5 ellipse.
template <int... D>
struct Prof {
  static constexpr int KH = sizeof...(D);
  __host__ __device__ static constexpr int at(int i) {
    constexpr int a[KH] = {D...};
    return a[i];
  }
  __host__ __device__ static constexpr int maxd() {
    int m = 0;
    for (int i = 0; i < KH; i++) m = at(i) > m ? at(i) : m;
    return m;
  }
};

template <bool MAX>
__device__ __forceinline__ uint32_t pop(uint32_t a, uint32_t b) {
  return MAX ? __vmaxu2(a, b) : __vminu2(a, b);
}

// Runs of every half-width 0..M of the two sample pairs of this lane's word
// (r[w][0]: samples 0,1; r[w][1]: samples 2,3), from every lane's pairs.
template <int M, int CN, bool MAX>
__device__ __forceinline__ void pair_runs(uint32_t lo, uint32_t hi, uint32_t (&r)[M + 1][2]) {
  constexpr int NW = (M * CN + 3) / 4;
  uint32_t pq[2 * (2 * NW + 1) + 1];
  pq[2 * NW] = lo;
  pq[2 * NW + 1] = hi;
#pragma unroll
  for (int k = 1; k <= NW; k++) {
    pq[2 * (NW - k)] = __shfl_up_sync(kFull, lo, k);
    pq[2 * (NW - k) + 1] = __shfl_up_sync(kFull, hi, k);
    pq[2 * (NW + k)] = __shfl_down_sync(kFull, lo, k);
    pq[2 * (NW + k) + 1] = __shfl_down_sync(kFull, hi, k);
  }
  pq[2 * (2 * NW + 1)] = 0;
#pragma unroll
  for (int p = 0; p < 2; p++) {
    const int o = 2 * p;
    r[0][p] = pair_at<NW>(pq, o);
#pragma unroll
    for (int w = 1; w <= M; w++) r[w][p] = pop<MAX>(r[w - 1][p], pop<MAX>(pair_at<NW>(pq, o - w * CN), pair_at<NW>(pq, o + w * CN)));
  }
}

// Running vertical combination: acc[j] collects output row (r - j + ay)
// while source row r arrives, from element row j.
template <class PR, bool MAX>
struct Acc {
  static constexpr int KH = PR::KH;
  static constexpr uint32_t I = MAX ? 0u : 0x00FF00FFu;
  uint32_t a[KH][2];
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int j = 0; j < KH; j++) a[j][0] = a[j][1] = I;
  }
  // Adds a row of runs; returns the completed output pairs (of row r - (KH-1) + ay).
  template <int M>
  __device__ __forceinline__ void add(const uint32_t (&r)[M + 1][2], uint32_t &o0, uint32_t &o1) {
#pragma unroll
    for (int j = 0; j < KH; j++) {
      const int dj = PR::at(j);
      if (dj < 0) continue;
      a[j][0] = pop<MAX>(a[j][0], r[dj][0]);
      a[j][1] = pop<MAX>(a[j][1], r[dj][1]);
    }
    o0 = a[KH - 1][0];
    o1 = a[KH - 1][1];
#pragma unroll
    for (int j = KH - 1; j > 0; j--) {
      a[j][0] = a[j - 1][0];
      a[j][1] = a[j - 1][1];
    }
    a[0][0] = a[0][1] = I;
  }
};

// Pairs of the samples outside the row set to the identity.
__device__ __forceinline__ void mask_pairs(uint32_t &lo, uint32_t &hi, const Cols &c, uint32_t ident) {
  if (c.inside) return;
  if (c.msi[0] < 0) lo = (lo & 0xFFFF0000u) | (ident & 0xFFFFu);
  if (c.msi[1] < 0) lo = (lo & 0x0000FFFFu) | (ident & 0xFFFF0000u);
  if (c.msi[2] < 0) hi = (hi & 0xFFFF0000u) | (ident & 0xFFFFu);
  if (c.msi[3] < 0) hi = (hi & 0x0000FFFFu) | (ident & 0xFFFF0000u);
}

// One pass (FUSED = false: extremum MAX1 with element P1) or two fused
// passes (MAX1 with P1, then !MAX1 with P2) over a strip whose outer HALO
// lanes are not written. A lane's first-pass value at sample k of its word
// is exact once the lanes within its reach exist, so HALO words of
// (M1 + M2) * CN samples suffice.
template <class P1, class P2, int CN, int RH, bool MAX1, bool FUSED>
struct MorphStrip {
  static constexpr int M1 = P1::maxd(), M2 = FUSED ? P2::maxd() : 0;
  static constexpr int KH1 = P1::KH, KH2 = FUSED ? P2::KH : 1;
  static constexpr int HALO = ((M1 + M2) * CN + 3) / 4 > 0 ? ((M1 + M2) * CN + 3) / 4 : 1;
  static constexpr int OW = 32 - 2 * HALO;
  static constexpr int AY1 = KH1 / 2, AY2 = FUSED ? KH2 / 2 : 0;
  static constexpr int NSRC = RH + (KH1 - 1) + (FUSED ? KH2 - 1 : 0);

  static __device__ __forceinline__ void run(const DImg &s, const DImg &d, int tx, int ty, int lane) {
    constexpr bool MAX2 = !MAX1;
    constexpr uint32_t I1 = MAX1 ? 0u : 0xFFFFFFFFu;
    constexpr uint32_t I2p = MAX2 ? 0u : 0x00FF00FFu;
    const long long n = (long long)s.w * CN;
    const long long gw = (long long)tx * OW - HALO + lane;
    const Cols c = make_cols<CN>(gw * 4, n, s.w, 0, true);
    const int H = s.h;
    const int y0 = ty * RH;
    const int first = y0 - AY2 - AY1;
    const bool out_lane = lane >= HALO && lane < 32 - HALO && c.gs < n;
    Acc<P1, MAX1> acc1;
    Acc<P2, MAX2> acc2;
    acc1.init();
    acc2.init();
    auto load_batch = [&](int jb, uint32_t (&w)[kBatch]) {
#pragma unroll
      for (int k = 0; k < kBatch; k++) {
        const int sy = first + jb + k;
        w[k] = I1;
        if (jb + k < NSRC && sy >= 0 && sy < H) w[k] = load_word(row_ptr<const uint8_t>(s, sy), c, I1);
      }
    };
    uint32_t w[kBatch], wn[kBatch];
    load_batch(0, w);
#pragma unroll 1
    for (int jb = 0; jb < NSRC; jb += kBatch) {
      if (jb + kBatch < NSRC) load_batch(jb + kBatch, wn);
#pragma unroll
      for (int k = 0; k < kBatch; k++) {
        const int j = jb + k;
        if (j >= NSRC) break;
        uint32_t r1[M1 + 1][2];
        pair_runs<M1, CN, MAX1>(__byte_perm(w[k], 0, 0x4140), __byte_perm(w[k], 0, 0x4342), r1);
        uint32_t v0, v1;
        acc1.template add<M1>(r1, v0, v1);
        if (j < KH1 - 1) continue;
        const int y1 = first + j - (KH1 - 1) + AY1;  // first-pass row completed
        if constexpr (!FUSED) {
          if (out_lane && y1 < d.h) store_word(row_ptr<uint8_t>(d, y1), c.gs, n, __byte_perm(v0, v1, 0x6420));
        } else {
          // First-pass values outside the image are the second pass's identity.
          if (y1 < 0 || y1 >= H) {
            v0 = v1 = I2p;
          } else {
            mask_pairs(v0, v1, c, I2p);
          }
          uint32_t r2[M2 + 1][2];
          pair_runs<M2, CN, MAX2>(v0, v1, r2);
          uint32_t u0, u1;
          acc2.template add<M2>(r2, u0, u1);
          if (j < (KH1 - 1) + (KH2 - 1)) continue;
          const int y2 = y1 - (KH2 - 1) + AY2;
          if (out_lane && y2 < d.h) store_word(row_ptr<uint8_t>(d, y2), c.gs, n, __byte_perm(u0, u1, 0x6420));
        }
      }
#pragma unroll
      for (int k = 0; k < kBatch; k++) w[k] = wn[k];
    }
  }
};

// The element profiles with compiled kernels (getStructuringElement of
// morph.zig:32-59 for these shapes and sizes); kProfileCount = none.
using ProfRect3 = Prof<1, 1, 1>;
using ProfRect5 = Prof<2, 2, 2, 2, 2>;
using ProfRect7 = Prof<3, 3, 3, 3, 3, 3, 3>;
using ProfCross3 = Prof<0, 1, 0>;
using ProfCross5 = Prof<0, 0, 2, 0, 0>;
using ProfEll5 = Prof<0, 2, 2, 2, 0>;
using ProfEll7 = Prof<0, 2, 3, 3, 3, 2, 0>;
enum ProfileId { kRect3, kRect5, kRect7, kCross3, kCross5, kEll5, kEll7, kProfileCount };

template <class PR>
inline bool prof_matches(const int *d, int kh) {
  if (kh != PR::KH) return false;
  for (int i = 0; i < kh; i++)
    if (d[i] != PR::at(i)) return false;
  return true;
}

// The compiled profile equal to the element's half-widths, else kProfileCount.
inline int profile_of(const int *d, int kh) {
  if (prof_matches<ProfRect3>(d, kh)) return kRect3;
  if (prof_matches<ProfRect5>(d, kh)) return kRect5;
  if (prof_matches<ProfRect7>(d, kh)) return kRect7;
  if (prof_matches<ProfCross3>(d, kh)) return kCross3;
  if (prof_matches<ProfCross5>(d, kh)) return kCross5;
  if (prof_matches<ProfEll5>(d, kh)) return kEll5;
  if (prof_matches<ProfEll7>(d, kh)) return kEll7;
  return kProfileCount;
}

inline int profile_maxd(int id) {
  static const int m[kProfileCount] = {1, 2, 3, 1, 2, 2, 3};
  return id >= 0 && id < kProfileCount ? m[id] : 99;
}

}  // namespace strip
}  // namespace vb
