// Warp-strip stencils for u8 images: a warp owns a strip of 32 lanes x 8
// samples across RH output rows and walks down it, keeping the vertical
// window in registers; horizontal neighbours come from the adjacent lanes by
// warp shuffles. The outer lanes of a strip are halo (loaded, not written).
// No block barriers: each warp streams its own rows through its own slots of
// shared memory.
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
// Rows stream through a per-lane queue in shared memory: the copy of a row
// a queue depth ahead (cp.async) is issued when row j is computed, so that
// many rows per lane are in flight (the Gaussian: 15 of 16 slots; the
// morphology: a multiple of the element height, at least 8). State that moves down with the rows (the Gaussian
// cascade, the morphology row windows) alternates between register sets or
// rotates through compile-time ring slots across an unrolled row loop
// instead of being moved.
#pragma once
#include <utility>
#include "morphfast.cuh"
#include "vb.h"

namespace vb {
namespace strip {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kSPL = 8;  // samples per lane (one 8-byte word)

// Warps per block of the strip kernels (per-warp shared-memory slots).
constexpr int kWarpsPerBlock = 4;

// The four sample pairs (16-bit lanes) of 8 bytes: pairs (0,1) (2,3) (4,5) (6,7).
__device__ __forceinline__ void unpack_pairs(uint2 v, uint32_t (&p)[4]) {
  p[0] = __byte_perm(v.x, 0, 0x4140);
  p[1] = __byte_perm(v.x, 0, 0x4342);
  p[2] = __byte_perm(v.y, 0, 0x4140);
  p[3] = __byte_perm(v.y, 0, 0x4342);
}

// The low bytes of four pair registers as 8 bytes.
__device__ __forceinline__ uint2 pack_pairs(const uint32_t (&p)[4]) {
  return make_uint2(__byte_perm(p[0], p[1], 0x6420), __byte_perm(p[2], p[3], 0x6420));
}

// Sample pairs of this lane and NL neighbour lanes each side, gathered by
// shuffles: q[4*(l+NL) + i] = pair i of lane (self + l). Only the pairs that
// samples [S0, S1] (relative to this lane's first sample) touch are fetched.
template <int NL, int S0, int S1>
struct Window {
  static constexpr int NQ = 4 * (2 * NL + 1) + 1;
  uint32_t q[NQ];
  __device__ __forceinline__ void gather(const uint32_t (&own)[4]) {
    constexpr int T0 = S0 + kSPL * NL, T1 = S1 + kSPL * NL;  // sample range in q's frame
    constexpr int PMIN = T0 >> 1, PMAX = (T1 + 1) >> 1;      // pairs at() can touch
#pragma unroll
    for (int i = 0; i < NQ; i++) q[i] = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) q[4 * NL + i] = own[i];
#pragma unroll
    for (int l = 1; l <= NL; l++)
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int il = 4 * (NL - l) + i, ir = 4 * (NL + l) + i;
        if (il >= PMIN && il <= PMAX) q[il] = __shfl_up_sync(kFull, own[i], l);
        if (ir >= PMIN && ir <= PMAX) q[ir] = __shfl_down_sync(kFull, own[i], l);
      }
  }
  // (V[s], V[s+1]) for s relative to this lane's first sample.
  __device__ __forceinline__ uint32_t at(int s) const {
    const int t = s + kSPL * NL;
    return (t & 1) ? __byte_perm(q[t >> 1], q[(t >> 1) + 1], 0x5432) : q[t >> 1];
  }
};

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

struct GaussArgs {
  int border;
};

template <int K, int CN>
struct GaussGeom {
  static constexpr int R = K / 2;
  static constexpr int REACH = R * CN;
  static constexpr int HALO = (REACH + kSPL - 1) / kSPL;  // halo lanes each side
  static constexpr int OL = 32 - 2 * HALO;                // output lanes
};

// Row queue of the morphology strips in shared memory. Each lane copies its 8
// samples of source row j + QD into slot (j + QD) % QD with cp.async while
// row j is computed, so QD rows per lane are in flight without a register
// queue to rotate. Lanes outside the row store the fill into the slot
// directly. Slots are lane-private: no barriers. kQD: the least depth.
constexpr int kQD = 8;

__device__ __forceinline__ void cp_async8(uint32_t saddr, const void *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(g));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void st_shared8(uint32_t saddr, uint2 v) {
  asm volatile("st.shared.v2.u32 [%0], {%1, %2};\n" ::"r"(saddr), "r"(v.x), "r"(v.y));
}
__device__ __forceinline__ uint2 ld_shared8(uint32_t saddr) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];\n" : "=r"(v.x), "=r"(v.y) : "r"(saddr));
  return v;
}

// A predicated copy of the lane's 8 samples at g, or the fill stored into
// the slot when !p (g is then not read). No branches.
__device__ __forceinline__ void fetch8_inside(uint32_t saddr, const uint8_t *g, bool p, uint32_t fill) {
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.b32 q, %2, 0;\n"
      " @q cp.async.ca.shared.global [%0], [%1], 8;\n"
      " @!q st.shared.v2.u32 [%0], {%3, %3};\n}\n" ::"r"(saddr),
      "l"(g), "r"((int)p), "r"(fill));
}

// 8 bytes to global memory when p (no branch).
__device__ __forceinline__ void st_global8_if(uint8_t *g, uint2 v, bool p) {
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.b32 q, %3, 0;\n"
      " @q st.global.v2.u32 [%0], {%1, %2};\n}\n" ::"l"(g),
      "r"(v.x), "r"(v.y), "r"((int)p));
}

// One strip tile: lanes cover samples [(tx*OL - HALO + lane) * 8, +8) of
// rows [ty*RH, ty*RH + RH). The vertical binomial runs as a cascade of
// pairwise sums over the incoming rows (its state alternates between two
// register sets, ca and cb, so consecutive rows need no moves); the
// horizontal one on the pairs of this lane and its neighbours, scaled so that
// the result is each 16-bit lane's high byte: (F*H + 2^7) >> 8 with
// F = 2^(8-SH) equals (H + 2^(SH-1)) >> SH.
//
// Lanes that start inside the row copy 8 bytes of it into their slot of the
// row queue (source rows are readable up to their length rounded up to 8
// samples: rows of 8-sample multiples, or padded images, which the plan
// guarantees) and the others fill theirs; each lane then takes its samples
// from a 16-byte window of the warp's slot, byte k from window byte u_k,
// three byte permutes per 4-byte word (in a row's inner strips the window
// holds the lane's own bytes, unpermuted). Samples outside
// the row within the stencil's reach are thereby border-mapped (the sample of
// the mapped pixel, same channel; the window always covers them for the
// constant, replicate, reflect and reflect-101 borders), and constant-border
// ones are masked to zero. A slot is refilled only after every lane has read
// it: row j + kGQ - 1 goes into row j - 1's slot once a warp barrier has
// seen every lane past row j - 1 (so kGQ - 1 rows are in flight). Every
// tile takes this one path: a separate one for inner strips doubles the
// loop's code and its registers. The selectors live in shared memory and are
// read per row, which keeps them out of the loop's registers.
constexpr int kGQ = 16;  // row queue depth of the Gaussian strips

struct GaussQueue {
  uint32_t base;  // shared address of this lane's bytes in slot 0
  uint32_t par;   // shared address of this lane's window selectors
  __device__ __forceinline__ uint32_t slot(int j) const { return base + (uint32_t)((j & (kGQ - 1)) * 32 * kSPL); }
};

__device__ __forceinline__ GaussQueue gauss_queue(int lane) {
  __shared__ __align__(16) uint2 s_gq[kWarpsPerBlock][kGQ][32];
  __shared__ __align__(16) uint4 s_gp[kWarpsPerBlock][32][2];
  const int w = (threadIdx.x >> 5) % kWarpsPerBlock;
  return GaussQueue{(uint32_t)__cvta_generic_to_shared(&s_gq[w][0][lane]),
                    (uint32_t)__cvta_generic_to_shared(&s_gp[w][lane][0])};
}

__device__ __forceinline__ uint4 ld_shared16(uint32_t saddr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(saddr));
  return v;
}
__device__ __forceinline__ void st_shared16(uint32_t saddr, uint4 v) {
  asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};\n" ::"r"(saddr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w));
}

template <int K, int CN, int RH>
struct GaussStrip {
  using G = GaussGeom<K, CN>;
  static constexpr int R = G::R, HALO = G::HALO;
  static constexpr int E = Binom<K>::e;
  static constexpr int SH = 16 - 2 * E;
  static_assert(SH <= 8, "the scaled sum must fit a 16-bit lane");
  static constexpr uint32_t F = 1u << (8 - SH);
  static constexpr uint32_t RND = 0x00800080u;
  static constexpr int QD = kGQ - 1;  // rows in flight

  const DImg s, d;  // copies (kept in registers across the row loop)
  int border, H, first, nr, ylim, yout;
  int bA, bS;  // rows sy >= H map to bA - bS * sy (-1: constant fill)
  long long n, gs;
  bool out_lane, from;
  GaussQueue q;
  // The next source row to fetch and the next output row, at this lane's
  // samples (advanced by a stride per row).
  const uint8_t *fp;
  uint8_t *op;
  uint32_t ca[K - 1][4], cb[K - 1][4];
  int woff;  // window offset from this lane's slot

  __device__ __forceinline__ GaussStrip(const DImg &s_, const DImg &d_, int border_, int tx, int ty, int lane)
      : s(s_), d(d_), border(border_) {
    n = (long long)s.w * CN;
    gs = ((long long)tx * G::OL - HALO + lane) * kSPL;
    out_lane = lane >= HALO && lane < 32 - HALO && gs < n;
    from = gs >= 0 && gs < n;
    q = gauss_queue(lane);
    H = s.h;
    // border.map just below the image (rows H .. H + R - 1 where it matters):
    // replicate H - 1, reflect 2H - 1 - sy, reflect-101 2H - 2 - sy, wrap
    // sy - H, constant the fill (images are taller than R).
    bA = border == kReplicate ? H - 1 : border == kReflect ? 2 * H - 1 : border == kReflect101 ? 2 * H - 2
         : border == kWrap ? -H : -1;
    bS = border == kReflect || border == kReflect101 ? 1 : border == kWrap ? -1 : 0;
    const int y0 = ty * RH;
    first = y0 - R;
    // Only the rows the tile's outputs (y < h) need: at most R past the image.
    ylim = min(y0 + RH, d.h);
    nr = min(RH + K - 1, ylim - y0 + K - 1);
    fp = s.p + (long long)first * s.stride + gs;
    op = d.p + (long long)y0 * d.stride + gs;
    yout = y0;
  }

  // The window and selectors of this lane (see above), stored at q.par:
  // {a0, b0, m0, a1}, {b1, m1, keep0, keep1} for the first-level permutes of
  // window bytes 0-7 (a) and 8-15 (b), the merge (m) and the
  // constant-border masks of words 0 and 1.
  // Where byte k of this lane comes from: 0 = not needed (outside the
  // stencil's reach), 1 = strip byte t, 2 = zero (constant border).
  __device__ __forceinline__ int byte_src(int k, long long base, long long need_lo, long long need_hi, int &t) const {
    const long long g = gs + k;
    if (g < need_lo || g >= need_hi) return 0;
    if (g >= 0 && g < n) {
      t = (int)(g - base);
      return 1;
    }
    const long long px = g >= 0 ? g / CN : -((-g + CN - 1) / CN);
    const int mx = border_map(px, s.w, border);
    if (mx < 0) return 2;
    t = (int)((long long)mx * CN + (g - px * CN) - base);
    return 1;
  }

  __device__ __forceinline__ void edge_setup(int lane) {
    if (__all_sync(kFull, gs >= 0 && gs + kSPL <= n)) {
      // Inner strip: the lane's own bytes (lane 31's window starts a word
      // earlier).
      const bool last = lane * kSPL > 256 - 16;
      woff = last ? -kSPL : 0;
      const uint32_t a0 = last ? 0u : 0x3210u, b0 = last ? 0x3210u : 0u, m0 = last ? 0x7654u : 0x3210u;
      const uint32_t a1 = last ? 0u : 0x7654u, b1 = last ? 0x7654u : 0u;
      st_shared16(q.par, make_uint4(a0, b0, m0, a1));
      st_shared16(q.par + 16, make_uint4(b1, m0, ~0u, ~0u));
      return;
    }
    const long long base = gs - (long long)lane * kSPL;  // the strip's first sample
    const long long need_lo = base + kSPL * HALO - G::REACH;
    const long long need_hi = min(base + kSPL * (32 - HALO), n) + G::REACH;
    int lo = 1 << 30;
    unsigned long long keep = ~0ull;
#pragma unroll 1
    for (int k = 0; k < kSPL; k++) {
      int t = 0;
      const int r = byte_src(k, base, need_lo, need_hi, t);
      if (r == 1) lo = min(lo, t);
      if (r == 2) keep &= ~(0xFFull << (8 * k));
    }
    const int W = min(lo == (1 << 30) ? lane * kSPL : lo & ~7, 256 - 16);
    woff = W - lane * kSPL;
    uint32_t sa[2] = {0, 0}, sb[2] = {0, 0}, sm[2] = {0, 0};
#pragma unroll 1
    for (int k = 0; k < kSPL; k++) {
      int t = W;
      const int r = byte_src(k, base, need_lo, need_hi, t);
      const int u = r == 1 ? (t - W) & 15 : 0;
      const int sh = 4 * (k & 3);
      const uint32_t a = u < 8 ? (uint32_t)u << sh : 0u, b = u < 8 ? 0u : (uint32_t)(u - 8) << sh;
      const uint32_t m = (uint32_t)((u < 8 ? 0 : 4) + (k & 3)) << sh;
      if (k < 4) {
        sa[0] |= a, sb[0] |= b, sm[0] |= m;
      } else {
        sa[1] |= a, sb[1] |= b, sm[1] |= m;
      }
    }
    st_shared16(q.par, make_uint4(sa[0], sb[0], sm[0], sa[1]));
    st_shared16(q.par + 16, make_uint4(sb[1], sm[1], (uint32_t)keep, (uint32_t)(keep >> 32)));
  }

  // Source row j into its slot (rows j >= nr: nothing is read). Rows are
  // fetched in order, one per call. PRO: the first rows of the queue, which
  // hold every row above the image (R < kGQ - 1), border-mapped in full; the
  // later ones can only pass the bottom, by less than R rows where it
  // matters (j < nr), mapped in closed form (bA, bS) without branches.
  template <bool PRO>
  __device__ __forceinline__ void fetch(int j) {
    const int sy = first + j;
    int my;
    if constexpr (PRO) my = (unsigned)sy < (unsigned)H ? sy : border_map(sy, H, border);
    else my = sy < H ? sy : bA - bS * sy;
    const bool ok = j < nr && (unsigned)my < (unsigned)H && from;
    fetch8_inside(q.slot(j), fp + (long long)(my - sy) * s.stride, ok, 0u);
    fp += s.stride;
  }

  // This lane's 8 samples of row j from its window of the slot.
  __device__ __forceinline__ uint2 window(int j) const {
    const uint32_t a = q.slot(j) + woff;
    const uint4 p0 = ld_shared16(q.par), p1 = ld_shared16(q.par + 16);
    const uint2 w0 = ld_shared8(a), w1 = ld_shared8(a + 8);
    const uint32_t x0 = __byte_perm(__byte_perm(w0.x, w0.y, p0.x), __byte_perm(w1.x, w1.y, p0.y), p0.z);
    const uint32_t x1 = __byte_perm(__byte_perm(w0.x, w0.y, p0.w), __byte_perm(w1.x, w1.y, p1.x), p1.y);
    return make_uint2(x0 & p1.z, x1 & p1.w);
  }

  // The next output row (rows past the tile or the image are not written;
  // lanes write 8 bytes, into the destination's row padding at the end).
  __device__ __forceinline__ void put(const uint32_t (&h)[4]) {
    const uint2 o8 = make_uint2(__byte_perm(h[0], h[1], 0x7531), __byte_perm(h[2], h[3], 0x7531));
    st_global8_if(op, o8, out_lane && yout < ylim);
    op += d.stride;
    yout++;
  }

  // Source row j; OUT: the cascade is full (j >= K - 1) and output row
  // j - (K - 1) is computed.
  template <bool ODD, bool OUT>
  __device__ __forceinline__ void step(int j) {
    const uint32_t(&in)[K - 1][4] = ODD ? cb : ca;
    uint32_t(&out)[K - 1][4] = ODD ? ca : cb;
    cp_wait<QD - 1>();  // row j has landed
    __syncwarp();  // every lane's row j has landed; every read of row j - 1's slot is done
    fetch<false>(j + QD);
    const uint2 cur = window(j);
    cp_commit();
    // Cascade of pairwise sums: after row j the last stage holds the
    // binomial sum of rows j-K+1..j.
    uint32_t v[4];
    unpack_pairs(cur, v);
#pragma unroll
    for (int a = 0; a < K - 1; a++)
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const uint32_t t = v[i] + in[a][i];
        out[a][i] = v[i];
        v[i] = t;
      }
    if constexpr (!OUT) return;
    Window<HALO, -G::REACH, kSPL - 1 + G::REACH> win;
    win.gather(v);
    uint32_t h[4];
#pragma unroll
    for (int o = 0; o < 4; o++) {
      const int c0 = 2 * o;
      const uint32_t x = win.at(c0);
      uint32_t sum;
      if constexpr (K == 3) {
        sum = win.at(c0 - CN) + win.at(c0 + CN) + (x << 1);
      } else {
        // a + 4 b + 6 x
        const uint32_t a = win.at(c0 - 2 * CN) + win.at(c0 + 2 * CN);
        const uint32_t b = win.at(c0 - CN) + win.at(c0 + CN);
        sum = a + (b << 2) + x * 6u;
      }
      h[o] = sum * F + RND;
    }
    put(h);
  }

  __device__ __forceinline__ void rows(int lane) {
    edge_setup(lane);
#pragma unroll 1
    for (int j = 0; j < QD; j++) {
      fetch<true>(j);
      cp_commit();
    }
#pragma unroll
    for (int a = 0; a < K - 1; a++)
#pragma unroll
      for (int i = 0; i < 4; i++) ca[a][i] = 0;
    static_assert((K - 1) % 2 == 0, "the cascade fills in pairs of rows");
#pragma unroll 1
    for (int j = 0; j < K - 1; j += 2) {
      step<false, false>(j);
      step<true, false>(j + 1);
    }
    // Pairs of rows; rows past nr are neither read nor stored.
#pragma unroll 1
    for (int j = K - 1; j < nr; j += 2) {
      step<false, true>(j);
      step<true, true>(j + 1);
    }
  }
};

// The plan hands the strip source and destination rows that are readable
// and writable up to their length rounded up to 8 samples.
template <int K, int CN, int RH>
__device__ __forceinline__ void gauss_strip(const DImg &s, const DImg &d, int border, int tx, int ty, int lane) {
  GaussStrip<K, CN, RH> g(s, d, border, tx, ty, lane);
  g.rows(lane);
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
// Three-input min / max on 16-bit lanes: one instruction, the cost of pop.
template <bool MAX>
__device__ __forceinline__ uint32_t pop3(uint32_t a, uint32_t b, uint32_t c) {
  return MAX ? __vimax3_u16x2(a, b, c) : __vimin3_u16x2(a, b, c);
}

// Band decomposition of an element whose rows are centred runs, symmetric
// about the centre row, with half-widths that never grow away from it
// (every rect / cross / ellipse of getStructuringElement). With d(a) the
// half-width of the rows at distance a from the centre, the element is the
// union over a of the centred rectangles (2 d(a) + 1) x (2 a + 1), so
//   extremum over the element = extremum over a of H_d(a)(V_a)
// where V_a is the vertical extremum over the rows within distance a and H_d
// the horizontal run of half-width d. Only the a where the half-width drops
// next (or a = AY) are needed; rows whose half-width is 0 fold into the
// result directly.
template <class PR>
struct Bands {
  static constexpr int KH = PR::KH, AY = KH / 2;
  __host__ __device__ static constexpr int d(int a) { return PR::at(AY + a); }
  __host__ __device__ static constexpr bool part(int a) { return a == AY || d(a) > d(a + 1); }
  // The last part with a horizontal run (d > 0), -1 if none.
  __host__ __device__ static constexpr int last_wide() {
    int l = -1;
    for (int a = 0; a <= AY; a++)
      if (part(a) && d(a) > 0) l = a;
    return l;
  }
  __host__ __device__ static constexpr bool valid() {
    if (KH % 2 == 0) return false;
    for (int i = 0; i < KH; i++)
      if (PR::at(i) != PR::at(KH - 1 - i) || PR::at(i) < 0) return false;
    for (int a = 1; a <= AY; a++)
      if (d(a) > d(a - 1)) return false;
    return true;
  }
};

// Horizontal run of half-width D over the four pairs v of every lane.
template <int D, int CN, bool MAX>
__device__ __forceinline__ void hrun(const uint32_t (&v)[4], uint32_t (&r)[4]) {
  constexpr int REACH = D * CN;
  constexpr int NL = (REACH + kSPL - 1) / kSPL;
  Window<NL, -REACH, kSPL - 1 + REACH> win;
  win.gather(v);
#pragma unroll
  for (int p = 0; p < 4; p++) {
    r[p] = v[p];
#pragma unroll
    for (int w = 1; w <= D; w++) r[p] = pop3<MAX>(r[p], win.at(2 * p - w * CN), win.at(2 * p + w * CN));
  }
}

// Band a of the decomposition (ascending): V grows to the rows within
// distance A, and a part with a horizontal run adds H_d(A)(V) to out (HAVE:
// out already holds a part).
template <class PR, int CN, bool MAX, int ROT, int A, bool HAVE>
struct BandStep {
  static __device__ __forceinline__ void run(const uint32_t (&h)[PR::KH][4], uint32_t (&V)[4], uint32_t (&out)[4]) {
    using B = Bands<PR>;
    constexpr int KH = B::KH, AY = B::AY, LW = B::last_wide();
    if constexpr (A > 0) {
#pragma unroll
      for (int p = 0; p < 4; p++) V[p] = pop3<MAX>(V[p], h[(ROT + AY - A) % KH][p], h[(ROT + AY + A) % KH][p]);
    }
    constexpr bool PART = B::part(A) && B::d(A) > 0;
    if constexpr (PART) {
      uint32_t P[4];
      hrun<B::d(A), CN, MAX>(V, P);
#pragma unroll
      for (int p = 0; p < 4; p++) out[p] = HAVE ? pop<MAX>(out[p], P[p]) : P[p];
    }
    if constexpr (A < LW) BandStep<PR, CN, MAX, ROT, A + 1, HAVE || PART>::run(h, V, out);
  }
};

// The extremum over element PR of the KH rows in h, row i (of the window
// centred on the output row) in slot (ROT + i) % KH.
template <class PR, int CN, bool MAX, int ROT>
__device__ __forceinline__ void band_apply(const uint32_t (&h)[PR::KH][4], uint32_t (&out)[4]) {
  using B = Bands<PR>;
  static_assert(B::valid(), "band decomposition needs a symmetric element narrowing away from its centre");
  constexpr int KH = B::KH, AY = B::AY, LW = B::last_wide();
  uint32_t V[4];
#pragma unroll
  for (int p = 0; p < 4; p++) V[p] = h[(ROT + AY) % KH][p];
  if constexpr (LW >= 0) {
    BandStep<PR, CN, MAX, ROT, 0, false>::run(h, V, out);
  } else {
#pragma unroll
    for (int p = 0; p < 4; p++) out[p] = V[p];
  }
  // Rows beyond the last run have half-width 0: their centre samples.
#pragma unroll
  for (int a = (LW < 0 ? 1 : LW + 1); a <= AY; a++)
#pragma unroll
    for (int p = 0; p < 4; p++) out[p] = pop3<MAX>(out[p], h[(ROT + AY - a) % KH][p], h[(ROT + AY + a) % KH][p]);
}

// One pass (FUSED = false: extremum MAX1 with element P1) or two fused
// passes (MAX1 with P1, then !MAX1 with P2, which has P1's height) over a
// strip whose outer HALO lanes are not written. A lane's first-pass value at
// a sample is exact once the samples within its reach exist in the strip, so
// HALO lanes covering (M1 + M2) * CN samples suffice. Source rows come
// through the shared-memory row queue. The last KH rows of each pass's input
// stay in a register ring (row t in slot t mod KH; the row loop is unrolled
// by KH, so every slot index is a compile-time constant and nothing moves),
// and each output row is the band decomposition of its KH input rows. The
// row queue is QD = KH1 * m slots deep (at least 8), so a group of KH1 rows
// never wraps inside it and every slot address in the unrolled group is a
// constant offset from the group's first slot.
template <class P1, class P2, int CN, int RH, bool MAX1, bool FUSED>
struct MorphStrip {
  static constexpr int M1 = P1::maxd(), M2 = FUSED ? P2::maxd() : 0;
  static constexpr int KH1 = P1::KH, KH2 = FUSED ? P2::KH : 1;
  static_assert(!FUSED || KH1 == KH2, "fused passes use elements of one height");
  static constexpr int HALO = ((M1 + M2) * CN + kSPL - 1) / kSPL > 0 ? ((M1 + M2) * CN + kSPL - 1) / kSPL : 1;
  static constexpr int OL = 32 - 2 * HALO;
  static constexpr int AY1 = KH1 / 2, AY2 = FUSED ? KH2 / 2 : 0;
  static constexpr int NSRC = RH + (KH1 - 1) + (FUSED ? KH2 - 1 : 0);
  static constexpr bool MAX2 = !MAX1;
  static constexpr uint32_t I1 = MAX1 ? 0u : 0xFFFFFFFFu;
  static constexpr uint32_t I1p = MAX1 ? 0u : 0x00FF00FFu;
  static constexpr uint32_t I2p = MAX2 ? 0u : 0x00FF00FFu;
  static constexpr int QD = KH1 * ((kQD + KH1 - 1) / KH1);
  static constexpr uint32_t kSlot = 32 * kSPL;  // bytes of one queue slot
  // Source rows that only fill the rings before the first output row, and
  // the rows of the first steady group that compute an output before it
  // (their stores are predicated off).
  static constexpr int W = (KH1 - 1) + (FUSED ? KH2 - 1 : 0);
  static constexpr int G = W > KH1 ? W - KH1 : 0;
  // Tile modes: every lane inside the row; or lanes inside, entirely
  // outside (predicated fills) or straddling the row's end with an 8-byte
  // copy into the row padding (masked per pair: the plan hands the strips
  // rows readable and writable up to their length rounded up to 8 samples).
  enum Mode { kInside, kEdge };

  const DImg s, d;  // copies (kept in registers across the row loop)
  long long n, gs;
  int H, first, nsrc, ylim;
  bool out_lane, live, inside;
  uint32_t q0, qs;  // shared address of this lane's slot 0; of the current group's first slot
  // The next source row to fetch and the next output row, as running
  // pointers at this lane's samples (advanced by a stride per row; rows
  // outside [jlo, jhi) are fills and their pointers are not read). oc counts
  // output rows from y0 (negative for the predicated-off rows before it),
  // stored while oc < olim (0 for halo lanes and lanes past the row).
  const uint8_t *fp;
  uint8_t *op;
  int jlo, jhi, oc;
  unsigned olim;
  uint32_t keep[4];     // kEdge: 16-bit lanes of samples inside the row
  uint32_t h1[KH1][4];  // the first pass's input rows
  uint32_t h2[KH2][4];  // the second pass's input rows (first-pass results)

  __device__ __forceinline__ MorphStrip(const DImg &s_, const DImg &d_, int tx, int ty, int lane) : s(s_), d(d_) {
    n = (long long)s.w * CN;
    gs = ((long long)tx * OL - HALO + lane) * kSPL;
    inside = gs >= 0 && gs + kSPL <= n;
    H = s.h;
    const int y0 = ty * RH;
    first = y0 - AY2 - AY1;
    // Only the source rows the tile's outputs (y < h) need.
    ylim = min(y0 + RH, d.h);
    nsrc = min(NSRC, ylim - y0 + KH1 + KH2 - 2);
    out_lane = lane >= HALO && lane < 32 - HALO && gs < n;
    live = gs < n && gs + kSPL > 0;
    __shared__ __align__(16) uint2 s_q[kWarpsPerBlock][QD][32];
    q0 = (uint32_t)__cvta_generic_to_shared(&s_q[(threadIdx.x >> 5) % kWarpsPerBlock][0][lane]);
    jlo = max(0, -first);
    jhi = max(jlo, min(nsrc, H - first));
    if (!live) jhi = jlo;  // kEdge: lanes without samples in the row only fill
    fp = s.p + (long long)first * s.stride + gs;
    oc = -G;
    olim = out_lane ? (unsigned)(ylim - y0) : 0u;
    op = reinterpret_cast<uint8_t *>(reinterpret_cast<uintptr_t>(d.p) +
                                     (uintptr_t)((long long)(y0 - G) * d.stride + gs));
#pragma unroll
    for (int r = 0; r < KH2; r++)
#pragma unroll
      for (int p = 0; p < 4; p++) h2[r][p] = I2p;
  }

  // Source row j into the slot at address a (rows outside [jlo, jhi): the
  // fill). Rows are fetched in order, one per call.
  __device__ __forceinline__ void fetch(uint32_t a, int j) {
    fetch8_inside(a, fp, (unsigned)(j - jlo) < (unsigned)(jhi - jlo), I1);
    fp += s.stride;
  }

  // The next output row (rows y0 - G, y0 - G + 1, ... in order, one per
  // call), written when it belongs to the tile and the image.
  __device__ __forceinline__ void put(const uint32_t (&o)[4]) {
    st_global8_if(op, pack_pairs(o), (unsigned)oc < olim);
    op += d.stride;
    oc++;
  }

  // Source row j = (group start) + PH, PH = j mod KH1. Rows past nsrc (the
  // last group of KH1) compute values that are not stored. WARM: the first
  // group (j = PH), whose rows only fill the rings up to row W.
  template <int MODE, bool WARM, int PH>
  __device__ __forceinline__ void step(int j) {
    const uint32_t slot = qs + PH * kSlot;
    cp_wait<QD - 1>();  // row j has landed
    const uint2 cur = ld_shared8(slot);
    fetch(slot, j + QD);
    cp_commit();
    unpack_pairs(cur, h1[PH]);
    if constexpr (MODE == kEdge) {
#pragma unroll
      for (int p = 0; p < 4; p++) h1[PH][p] = (h1[PH][p] & keep[p]) | (I1p & ~keep[p]);
    }
    if constexpr (WARM && PH < KH1 - 1) return;
    uint32_t o1[4];
    band_apply<P1, CN, MAX1, (PH + 1) % KH1>(h1, o1);
    const int y1 = first + j - (KH1 - 1) + AY1;  // first-pass row completed
    if constexpr (!FUSED) {
      put(o1);
    } else {
      // First-pass row t2 = j - (KH1 - 1) goes to slot t2 mod KH2; values
      // outside the image are the second pass's identity.
      constexpr int S2 = (PH + 1) % KH2;
      const bool rin = y1 >= 0 && y1 < H;
#pragma unroll
      for (int p = 0; p < 4; p++) {
        const uint32_t v = rin ? o1[p] : I2p;
        h2[S2][p] = MODE == kEdge ? (v & keep[p]) | (I2p & ~keep[p]) : v;
      }
      if constexpr (WARM && PH < W) return;
      uint32_t o2[4];
      band_apply<P2, CN, MAX2, (PH + 2) % KH2>(h2, o2);
      put(o2);
    }
  }

  template <int MODE, bool WARM, int... PH>
  __device__ __forceinline__ void steps(int j, std::integer_sequence<int, PH...>) {
    (step<MODE, WARM, PH>(j + PH), ...);
  }

  template <int MODE>
  __device__ __forceinline__ void rows() {
    if constexpr (MODE == kEdge) {
#pragma unroll
      for (int p = 0; p < 4; p++) {
        const long long k = gs + 2 * p;
        keep[p] = (k >= 0 && k < n ? 0x0000FFFFu : 0u) | (k + 1 >= 0 && k + 1 < n ? 0xFFFF0000u : 0u);
      }
    }
#pragma unroll 1
    for (int j = 0; j < QD; j++) {
      fetch(q0 + j * kSlot, j);
      cp_commit();
    }
    // The first group (every tile has at least KH1 source rows), then the
    // steady groups; the group's first slot wraps to slot 0 after QD rows.
    qs = q0;
    steps<MODE, true>(0, std::make_integer_sequence<int, KH1>{});
#pragma unroll 1
    for (int j = KH1; j < nsrc; j += KH1) {
      qs = qs == q0 + (QD - KH1) * kSlot ? q0 : qs + KH1 * kSlot;
      steps<MODE, false>(j, std::make_integer_sequence<int, KH1>{});
    }
  }

  static __device__ __forceinline__ void run(const DImg &s, const DImg &d, int tx, int ty, int lane) {
    MorphStrip m(s, d, tx, ty, lane);
    if (__all_sync(kFull, m.inside)) m.template rows<kInside>();
    else m.template rows<kEdge>();
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
