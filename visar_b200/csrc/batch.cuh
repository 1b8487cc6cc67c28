// Device side of the batched form: the tile-queue persistent kernel and the
// per-tile operations it runs.
//
// A launch covers one shape class of one stage: n images, each cut into
// tiles_x x tiles_y tiles, numbered consecutively image after image. Every
// CTA loops: claim the next tile number from a global atomic counter, find
// its image by binary search over the tile prefix sums (cached in shared
// memory), run the operation on that tile. Thread 0 claims the following
// tile while the current one is processed, so the atomic's latency overlaps
// the work.
#pragma once
#include <algorithm>
#include <type_traits>

#include "morphfast.cuh"
#include "sepfast.cuh"
#include "strip.cuh"
#include "vb.h"
#include "warp.cuh"

namespace vb {
namespace bt {

// One image of a launch: source and destination views, tiling, and the
// per-image data some operations need.
struct BImg {
  DImg s, d;
  int tiles_x, tiles_y;
  const void *t0, *t1;  // tables (linear resize taps)
  double md[9];         // warpPerspective inverse map
  float mf[6];          // warpAffine inverse map
  float cv;             // border value as f32
  int wide;             // source rows allow 8-byte loads
  int lanes;            // row-tiled operations: log2 of the threads per row
};

struct TileQ {
  const BImg *imgs;
  const int *start;  // n + 1 tile prefix sums
  int n, total;
  int *counter;      // zero before the launch
};

constexpr int kStartCap = 1024;  // prefix sums kept in shared memory up to this many images

__device__ __forceinline__ int find_image(const int *start, int n, int t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Resident CTAs per SM an operation asks the register allocator for
// (Op::kMinBlocks when it declares one).
template <class Op, class = void>
struct MinBlocks : std::integral_constant<int, 1> {};
template <class Op>
struct MinBlocks<Op, std::void_t<decltype(Op::kMinBlocks)>> : std::integral_constant<int, Op::kMinBlocks> {};

template <class Op>
__global__ void __launch_bounds__(Op::kThreads, MinBlocks<Op>::value) k_batch(TileQ q, typename Op::Args a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_start[kStartCap + 1];
  __shared__ int s_tile[2];
  const int tid = threadIdx.x;
  const bool cached = q.n <= kStartCap;
  if (cached)
    for (int i = tid; i <= q.n; i += Op::kThreads) s_start[i] = q.start[i];
  if (tid == 0) s_tile[0] = atomicAdd(q.counter, 1);
  __syncthreads();
  const int *start = cached ? s_start : q.start;
  int buf = 0;
  int cur = s_tile[0];
  while (cur < q.total) {
    int next = 0;
    if (tid == 0) next = atomicAdd(q.counter, 1);
    const int img = find_image(start, q.n, cur);
    const BImg im = q.imgs[img];  // a copy: stores through byte pointers cannot alias it
    const int local = cur - start[img];
    const int txn = im.tiles_x;
    Op::tile(im, a, local % txn, local / txn, smem);
    // Publish the next tile; the barrier also ends every use of this tile's
    // shared memory before the next tile's loads.
    if (tid == 0) s_tile[buf ^ 1] = next;
    __syncthreads();
    buf ^= 1;
    cur = s_tile[buf];
  }
}

// Warp-granular queue: every warp claims its own tiles (lane 0 takes the
// ticket, the warp broadcasts it); no block barrier after the prefix cache.
template <class Op>
__global__ void __launch_bounds__(Op::kThreads, Op::kMinBlocks) k_batch_warp(TileQ q, typename Op::Args a) {
  __shared__ int s_start[kStartCap + 1];
  const bool cached = q.n <= kStartCap;
  if (cached)
    for (int i = threadIdx.x; i <= q.n; i += Op::kThreads) s_start[i] = q.start[i];
  __syncthreads();
  const int *start = cached ? s_start : q.start;
  const int lane = threadIdx.x & 31;
  int t = 0;
  if (lane == 0) t = atomicAdd(q.counter, 1);
  int cur = __shfl_sync(0xFFFFFFFFu, t, 0);
  while (cur < q.total) {
    if (lane == 0) t = atomicAdd(q.counter, 1);
    const int img = find_image(start, q.n, cur);
    const BImg im = q.imgs[img];  // a copy: stores through byte pointers cannot alias it
    const int local = cur - start[img];
    const int txn = im.tiles_x;
    Op::tile(im, a, local % txn, local / txn, lane);
    cur = __shfl_sync(0xFFFFFFFFu, t, 0);
  }
}

// Operations with kWarpTiles = true run under k_batch_warp (a tile per warp).
template <class Op, class = void>
struct WarpTiles : std::false_type {};
template <class Op>
struct WarpTiles<Op, std::void_t<decltype(Op::kWarpTiles)>> : std::bool_constant<Op::kWarpTiles> {};

// ------------------------------------------------------------ operations
// Each operation: kThreads, Args, host smem(Args) / tiles(w, h, Args), and
// the device tile(). tile() may return early in some threads but must not
// skip a barrier it contains for only part of the CTA.

// Gaussian through the separable band (sepfast.cuh): u8 fixed point (exact
// f32 sums) or f32 in VISAR's order. RH output rows per tile.
template <class S, int K, int CN, int RH>
struct OpGauss {
  static constexpr int kThreads = 128;
  static constexpr bool kExact = sizeof(S) == 1;
  static constexpr int HW = ((K / 2) * CN + 3) / 4;
  static constexpr int OW = kThreads - 2 * HW;
  using Args = fast::FastArgs;
  static size_t smem(const Args &) {
    constexpr int NR = RH + K - 1;
    return kExact ? (size_t)NR * kThreads * 4 + (size_t)RH * kThreads * 16 : (size_t)NR * kThreads * 16;
  }
  static int tiles_x(int w) { return (int)ceil_div(((long long)w * CN + 3) / 4, OW); }
  static int tiles_y(int h) { return (int)ceil_div(h, RH); }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &base, int tx, int ty, unsigned char *smem) {
    Args a = base;
    a.n = (long long)im.s.w * CN;
    a.n16 = (int)(a.n - a.n % 16);
    fast::sep_band<S, K, K, CN, kThreads, RH, kExact, 1, 1>(im.s, im.d, a, tx, ty, smem);
  }
};

// One erode (MAX = false) or dilate pass through the SIMD band (morphfast.cuh).
template <int CN, int KH, bool MAX>
struct OpMorph {
  static constexpr int kThreads = 128;
  static constexpr int RH = 8;
  using Args = fast::MFArgs;
  static size_t smem(const Args &) { return sizeof(uint32_t) * (RH + KH - 1) * kThreads; }
  static int tiles_x(int w) { return (int)ceil_div(((long long)w * CN + 3) / 4, kThreads - 2); }
  static int tiles_y(int h) { return (int)ceil_div(h, RH); }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &base, int tx, int ty, unsigned char *smem) {
    Args a = base;
    a.n = (long long)im.s.w * CN;
    fast::morph_band<CN, KH, kThreads, RH, MAX>(im.s, im.d, a, tx, ty, reinterpret_cast<uint32_t(*)[kThreads]>(smem));
  }
};

// Row-tiled elementwise operations. A thread owns P consecutive samples of a
// row. An image's rows are shared out to 2^lanes threads per row (per image:
// the smallest power of two covering the row, at most the CTA), so a CTA
// works on kThreads >> lanes rows at once and narrow images do not leave most
// of its threads idle. A tile is rows * (kThreads >> lanes) image rows by
// P << lanes samples. Threads walk their rows two at a time, issuing both
// rows' loads before using either (more bytes in flight per thread).
struct RowArgs {
  int rows;
};

struct RowSpan {
  int x0;    // the thread's first sample in the row
  int y;     // its first row
  int yend;  // one past the tile's last row
  int step;  // rows between the thread's rows
};

template <int kThreads, int P>
__device__ __forceinline__ RowSpan row_span(const BImg &im, int rows, int tx, int ty, int h) {
  const int lg = im.lanes;
  const int rpp = kThreads >> lg;
  const int t0 = ty * rows * rpp;
  RowSpan r;
  r.x0 = ((tx << lg) + (int)(threadIdx.x & ((1u << lg) - 1))) * P;
  r.y = t0 + (int)(threadIdx.x >> lg);
  r.yend = min(h, t0 + rows * rpp);
  r.step = rpp;
  return r;
}

template <int N>
struct VecOf;
template <>
struct VecOf<4> {
  using T = uint32_t;
};
template <>
struct VecOf<8> {
  using T = uint2;
};
template <>
struct VecOf<16> {
  using T = uint4;
};

// K vectors of N bytes held in registers; byte() and word() take constant
// indices (after unrolling).
template <int N, int K>
struct Vb {
  using T = typename VecOf<N>::T;
  T v[K];
  __device__ __forceinline__ void load(const uint8_t *p) {
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = __ldg(reinterpret_cast<const T *>(p) + k);
  }
  __device__ __forceinline__ void store(uint8_t *p) const {
#pragma unroll
    for (int k = 0; k < K; k++) reinterpret_cast<T *>(p)[k] = v[k];
  }
  __device__ __forceinline__ uint32_t byte(int i) const { return reinterpret_cast<const uint8_t *>(v)[i]; }
  __device__ __forceinline__ uint32_t &word(int i) { return reinterpret_cast<uint32_t *>(v)[i]; }
};

__device__ __forceinline__ uint32_t gray_px(uint32_t b, uint32_t g, uint32_t r) {
  return (b * kB2G + g * kG2G + r * kR2G + (1u << (kGrayShift - 1))) >> kGrayShift;
}

// BGR / BGRA -> gray (color.zig:324-403 arithmetic), P = 8 or 16 pixels per
// thread.
template <int SCN, int P>
struct OpGray {
  static constexpr int kThreads = 256, kMinBlocks = P == 16 || SCN == 4 ? 4 : 5;  // <= 64 / 48 registers
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void px(const Vb<P, SCN> &in, Vb<P, 1> &out) {
#pragma unroll
    for (int q = 0; q < P / 4; q++) {
      uint32_t w = 0;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int p = q * 4 + i;
        w |= gray_px(in.byte(p * SCN), in.byte(p * SCN + 1), in.byte(p * SCN + 2)) << (8 * i);
      }
      out.word(q) = w;
    }
  }
  // U rows per thread in flight (their loads issued together): 4 with 8
  // pixels per thread, 2 with 16.
  static constexpr int U = P == 8 ? 4 : 2;
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const RowSpan r = row_span<kThreads, P>(im, a.rows, tx, ty, im.s.h);
    const int w = im.s.w;
    if (r.x0 >= w) return;
    const bool full = r.x0 + P <= w;
    for (int y = r.y; y < r.yend; y += U * r.step) {
      const uint8_t *sp[U];
      uint8_t *dp[U];
      bool ok[U];
      uintptr_t al = 0;
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int yy = y + u * r.step;
        ok[u] = yy < r.yend;
        const int ys = ok[u] ? yy : y;  // rows past the tile repeat row y (not stored)
        sp[u] = row_ptr<const uint8_t>(im.s, ys) + (long long)r.x0 * SCN;
        dp[u] = row_ptr<uint8_t>(im.d, ys) + r.x0;
        al |= (uintptr_t)sp[u] | (uintptr_t)dp[u];
      }
      if (full && (al % P) == 0) {
        Vb<P, SCN> in[U];
#pragma unroll
        for (int u = 0; u < U; u++) in[u].load(sp[u]);
#pragma unroll
        for (int u = 0; u < U; u++) {
          Vb<P, 1> o;
          px(in[u], o);
          if (ok[u]) o.store(dp[u]);
        }
      } else {
#pragma unroll
        for (int u = 0; u < U; u++) {
          if (!ok[u]) break;
          for (int i = 0; i < P && r.x0 + i < w; i++)
            dp[u][i] = (uint8_t)gray_px(sp[u][i * SCN], sp[u][i * SCN + 1], sp[u][i * SCN + 2]);
        }
      }
    }
  }
};

// Exact halving (resize_u8.zig:381-447), P = 4 or 8 output pixels per thread.
template <int CN, int P>
struct OpHalf {
  static constexpr int kThreads = 256, kMinBlocks = P * CN >= 24 ? 3 : P * CN > 8 ? 4 : 5;  // <= 80 / 64 / 48 registers
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  // Output samples of one output row from its two source rows.
  static __device__ __forceinline__ void px(const Vb<2 * P, CN> &ra, const Vb<2 * P, CN> &rb, Vb<P, CN> &o) {
#pragma unroll
    for (int k = 0; k < P * CN / 4; k++) {
      uint32_t w = 0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int oi = k * 4 + j;  // output sample index within the P pixels
        const int p = oi / CN, c = oi % CN;
        const int i = 2 * p * CN + c;
        w |= ((ra.byte(i) + ra.byte(i + CN) + rb.byte(i) + rb.byte(i + CN) + 2u) >> 2) << (8 * j);
      }
      o.word(k) = w;
    }
  }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const RowSpan r = row_span<kThreads, P>(im, a.rows, tx, ty, im.d.h);
    const int dw = im.d.w;
    if (r.x0 >= dw) return;
    const bool full = r.x0 + P <= dw;
    const size_t xs = (size_t)r.x0 * 2 * CN;
    for (int y = r.y; y < r.yend; y += 2 * r.step) {
      const int y2 = y + r.step;
      const bool two = y2 < r.yend;
      const int yb = two ? y2 : y;
      const uint8_t *a0 = row_ptr<const uint8_t>(im.s, 2LL * y) + xs;
      const uint8_t *b0 = row_ptr<const uint8_t>(im.s, 2LL * y + 1) + xs;
      const uint8_t *a1 = row_ptr<const uint8_t>(im.s, 2LL * yb) + xs;
      const uint8_t *b1 = row_ptr<const uint8_t>(im.s, 2LL * yb + 1) + xs;
      uint8_t *o0 = row_ptr<uint8_t>(im.d, y) + (size_t)r.x0 * CN;
      uint8_t *o1 = row_ptr<uint8_t>(im.d, yb) + (size_t)r.x0 * CN;
      if (full && (((uintptr_t)a0 | (uintptr_t)b0 | (uintptr_t)a1 | (uintptr_t)b1) % (2 * P)) == 0 &&
          (((uintptr_t)o0 | (uintptr_t)o1) % P) == 0) {
        Vb<2 * P, CN> va0, vb0, va1, vb1;
        va0.load(a0);
        vb0.load(b0);
        va1.load(a1);
        vb1.load(b1);
        Vb<P, CN> w0, w1;
        px(va0, vb0, w0);
        px(va1, vb1, w1);
        w0.store(o0);
        if (two) w1.store(o1);
      } else {
        for (int p = 0; p < P && r.x0 + p < dw; p++)
          for (int c = 0; c < CN; c++) {
            const int i = 2 * p * CN + c;
            o0[p * CN + c] = (uint8_t)(((uint32_t)a0[i] + a0[i + CN] + b0[i] + b0[i + CN] + 2u) >> 2);
            if (two) o1[p * CN + c] = (uint8_t)(((uint32_t)a1[i] + a1[i + CN] + b1[i] + b1[i + CN] + 2u) >> 2);
          }
      }
    }
  }
};

// OpenCV's fixed-point bilinear for u8 (resize_u8.zig:651-711) from the
// image's tap tables (t0: x taps in pixels, t1: y taps in rows); one output
// pixel per thread, two output rows (four source rows) in flight.
template <int CN>
struct OpLinear {
  static constexpr int kThreads = 256, kMinBlocks = CN == 1 ? 5 : CN == 4 ? 3 : 4;  // <= 48 / 64 / 80 registers
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const RowSpan r = row_span<kThreads, 1>(im, a.rows, tx, ty, im.d.h);
    const int x = r.x0;
    if (x >= im.d.w) return;
    const int4 tq = reinterpret_cast<const int4 *>(im.t0)[x];
    const LinTap *yt = static_cast<const LinTap *>(im.t1);
    const int a0 = tq.x * CN, a1 = tq.y * CN;
    for (int y = r.y; y < r.yend; y += 2 * r.step) {
      const int y2 = y + r.step;
      const bool two = y2 < r.yend;
      const LinTap t0 = yt[y], t1 = yt[two ? y2 : y];
      const uint8_t *r00 = row_ptr<const uint8_t>(im.s, t0.o0), *r01 = row_ptr<const uint8_t>(im.s, t0.o1);
      const uint8_t *r10 = row_ptr<const uint8_t>(im.s, t1.o0), *r11 = row_ptr<const uint8_t>(im.s, t1.o1);
      uint32_t v[4][2][CN];
#pragma unroll
      for (int c = 0; c < CN; c++) {
        v[0][0][c] = __ldg(r00 + a0 + c);
        v[0][1][c] = __ldg(r00 + a1 + c);
        v[1][0][c] = __ldg(r01 + a0 + c);
        v[1][1][c] = __ldg(r01 + a1 + c);
        v[2][0][c] = __ldg(r10 + a0 + c);
        v[2][1][c] = __ldg(r10 + a1 + c);
        v[3][0][c] = __ldg(r11 + a0 + c);
        v[3][1][c] = __ldg(r11 + a1 + c);
      }
      uint8_t *o0 = row_ptr<uint8_t>(im.d, y) + (size_t)x * CN;
      uint8_t *o1 = row_ptr<uint8_t>(im.d, two ? y2 : y) + (size_t)x * CN;
#pragma unroll
      for (int c = 0; c < CN; c++) {
        const int h00 = ((int)v[0][0][c] * tq.z + (int)v[0][1][c] * tq.w) >> 4;
        const int h01 = ((int)v[1][0][c] * tq.z + (int)v[1][1][c] * tq.w) >> 4;
        const int u0 = ((h00 * t0.w0) >> 16) + ((h01 * t0.w1) >> 16);
        o0[c] = (uint8_t)min(max((u0 + 2) >> 2, 0), 255);
        if (two) {
          const int h10 = ((int)v[2][0][c] * tq.z + (int)v[2][1][c] * tq.w) >> 4;
          const int h11 = ((int)v[3][0][c] * tq.z + (int)v[3][1][c] * tq.w) >> 4;
          const int u1 = ((h10 * t1.w0) >> 16) + ((h11 * t1.w1) >> 16);
          o1[c] = (uint8_t)min(max((u1 + 2) >> 2, 0), 255);
        }
      }
    }
  }
};

// The same bilinear for one-channel images on warp tiles of 128 output
// pixels (4 per lane) x `rows` rows. For each output row the two source rows'
// byte spans the tile needs are copied to shared memory with 16-byte cp.async
// (coalesced, kRing - 1 rows ahead), and the lanes read their taps from
// there. Tiles whose span exceeds kSpan bytes (shrinking by more than ~3.9x),
// or sources whose rows are not 16-byte aligned, read their taps directly.
struct OpLinearStrip {
  static constexpr int kThreads = 128, kMinBlocks = 6;
  static constexpr bool kWarpTiles = true;
  static constexpr int kPX = 4, kTW = 32 * kPX, kSpan = 512, kRing = 4;
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }

  static __device__ __forceinline__ uint32_t px(uint32_t a, uint32_t b, uint32_t c, uint32_t e, const int4 &t,
                                                int w0, int w1) {
    const int h0 = ((int)a * t.z + (int)b * t.w) >> 4;
    const int h1 = ((int)c * t.z + (int)e * t.w) >> 4;
    const int v = ((h0 * w0) >> 16) + ((h1 * w1) >> 16);
    return (uint32_t)min(max((v + 2) >> 2, 0), 255);
  }

  static __device__ __forceinline__ void put(const DImg &d, int y, int x, int dw, uint32_t out) {
    uint8_t *o = row_ptr<uint8_t>(d, y) + x;
    if (x + kPX <= dw && ((uintptr_t)o & 3) == 0) {
      *reinterpret_cast<uint32_t *>(o) = out;
    } else {
      for (int k = 0; k < kPX && x + k < dw; k++) o[k] = (uint8_t)(out >> (8 * k));
    }
  }

  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, int lane) {
    __shared__ __align__(16) uint8_t s_buf[4][kRing][2][kSpan];
    const DImg s = im.s, d = im.d;
    const int dw = d.w;
    const int x = tx * kTW + lane * kPX;
    const int ybeg = ty * a.rows, yend = min(d.h, ybeg + a.rows);
    const int4 *xt = static_cast<const int4 *>(im.t0);
    const LinTap *yt = static_cast<const LinTap *>(im.t1);
    int4 t[kPX];
#pragma unroll
    for (int k = 0; k < kPX; k++) t[k] = xt[min(x + k, dw - 1)];
    // The tile's source span [lo, hi] (x taps are monotonic; pixels past dw
    // repeat the last one).
    const int lo = (int)__reduce_min_sync(strip::kFull, (unsigned)t[0].x);
    const int hi = (int)__reduce_max_sync(strip::kFull, (unsigned)t[kPX - 1].y);
    const int a0 = lo & ~15;
    const int nb = hi + 1 - a0;
    const bool staged = nb <= kSpan && (((uintptr_t)s.p | (uintptr_t)s.stride) & 15) == 0;
    if (!staged) {
      for (int y = ybeg; y < yend; y++) {
        const LinTap r = yt[y];
        const uint8_t *q0 = row_ptr<const uint8_t>(s, r.o0), *q1 = row_ptr<const uint8_t>(s, r.o1);
        uint32_t out = 0;
#pragma unroll
        for (int k = 0; k < kPX; k++)
          out |= px(__ldg(q0 + t[k].x), __ldg(q0 + t[k].y), __ldg(q1 + t[k].x), __ldg(q1 + t[k].y), t[k], r.w0, r.w1)
                 << (8 * k);
        if (x < dw) put(d, y, x, dw, out);
      }
      return;
    }
    const int nch = (nb + 15) >> 4;  // 16-byte chunks per source row (<= 32)
    uint8_t(*buf)[2][kSpan] = s_buf[(threadIdx.x >> 5) & 3];
    // Copies of output row y's two source spans into ring slot y % kRing
    // (an empty group past the tile, so every row waits the same way).
    auto issue = [&](int y) {
      if (y < yend && lane < nch) {
        const LinTap r = yt[y];
        const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(&buf[y % kRing][0][lane * 16]);
        const uint32_t d1 = (uint32_t)__cvta_generic_to_shared(&buf[y % kRing][1][lane * 16]);
        const uint8_t *g0 = row_ptr<const uint8_t>(s, r.o0) + a0 + lane * 16;
        const uint8_t *g1 = row_ptr<const uint8_t>(s, r.o1) + a0 + lane * 16;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d0), "l"(g0));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d1), "l"(g1));
      }
      asm volatile("cp.async.commit_group;\n");
    };
    int o0[kPX], o1[kPX];
#pragma unroll
    for (int k = 0; k < kPX; k++) {
      o0[k] = t[k].x - a0;
      o1[k] = t[k].y - a0;
    }
#pragma unroll 1
    for (int k = 0; k < kRing - 1; k++) issue(ybeg + k);
#pragma unroll 1
    for (int y = ybeg; y < yend; y++) {
      issue(y + kRing - 1);
      asm volatile("cp.async.wait_group %0;\n" ::"n"(kRing - 1));  // row y's copies (this lane's) landed
      __syncwarp();                                                 // ... and every lane's
      const LinTap r = yt[y];
      const uint8_t *b0 = buf[y % kRing][0], *b1 = buf[y % kRing][1];
      uint32_t out = 0;
#pragma unroll
      for (int k = 0; k < kPX; k++) out |= px(b0[o0[k]], b0[o1[k]], b1[o0[k]], b1[o1[k]], t[k], r.w0, r.w1) << (8 * k);
      if (x < dw) put(d, y, x, dw, out);
      __syncwarp();  // every lane has read slot y % kRing before it is refilled
    }
  }
};

struct LutArgs {
  int rows;
  const uint8_t *lut;
};

// u8 threshold through a 256-entry table (threshold.zig:39-60), P = 8 or 16
// samples per thread.
template <int P>
struct OpLut {
  static constexpr int kThreads = 256, kMinBlocks = 5;  // <= 48 registers
  using Args = LutArgs;
  static size_t smem(const Args &) { return 256; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *smem) {
    uint8_t *t = smem;
    t[threadIdx.x] = a.lut[threadIdx.x];
    __syncthreads();
    const RowSpan r = row_span<kThreads, P>(im, a.rows, tx, ty, im.s.h);
    const long long n = (long long)im.s.w * im.s.cn;
    if (r.x0 >= n) return;
    const bool full = r.x0 + P <= n;
    for (int y = r.y; y < r.yend; y += 2 * r.step) {
      const int y2 = y + r.step;
      const bool two = y2 < r.yend;
      const uint8_t *s0 = row_ptr<const uint8_t>(im.s, y) + r.x0;
      const uint8_t *s1 = row_ptr<const uint8_t>(im.s, two ? y2 : y) + r.x0;
      uint8_t *d0 = row_ptr<uint8_t>(im.d, y) + r.x0;
      uint8_t *d1 = row_ptr<uint8_t>(im.d, two ? y2 : y) + r.x0;
      if (full && (((uintptr_t)s0 | (uintptr_t)s1 | (uintptr_t)d0 | (uintptr_t)d1) % P) == 0) {
        Vb<P, 1> v0, v1;
        v0.load(s0);
        v1.load(s1);
#pragma unroll
        for (int q = 0; q < P / 4; q++) {
          uint32_t w0 = 0, w1 = 0;
#pragma unroll
          for (int i = 0; i < 4; i++) {
            w0 |= (uint32_t)t[v0.byte(q * 4 + i)] << (8 * i);
            w1 |= (uint32_t)t[v1.byte(q * 4 + i)] << (8 * i);
          }
          v0.word(q) = w0;
          v1.word(q) = w1;
        }
        v0.store(d0);
        if (two) v1.store(d1);
      } else {
        for (long long k = 0; k < P && r.x0 + k < n; k++) {
          d0[k] = t[s0[k]];
          if (two) d1[k] = t[s1[k]];
        }
      }
    }
  }
};

// A byte copy of an image into a pitched pool image (any source alignment):
// the batched form repacks inputs whose rows are not 8-byte aligned before
// the stencils that need aligned rows. 16 bytes per thread.
struct CopyArgs {
  int rows;
  int esize;  // bytes per sample
};

struct OpCopy {
  static constexpr int kThreads = 256, kMinBlocks = 5, P = 16;
  using Args = CopyArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const RowSpan r = row_span<kThreads, P>(im, a.rows, tx, ty, im.s.h);
    const long long n = (long long)im.s.w * im.s.cn * a.esize;
    if (r.x0 >= n) return;
    const bool full = r.x0 + P <= n;
    for (int y = r.y; y < r.yend; y += r.step) {
      const uint8_t *sp = row_ptr<const uint8_t>(im.s, y) + r.x0;
      uint8_t *dp = row_ptr<uint8_t>(im.d, y) + r.x0;
      if (full && ((uintptr_t)dp & 15) == 0) {
        uint4 v;
        if (((uintptr_t)sp & 15) == 0) {
          v = __ldg(reinterpret_cast<const uint4 *>(sp));
        } else if (((uintptr_t)sp & 3) == 0) {
          const uint32_t *w = reinterpret_cast<const uint32_t *>(sp);
          v = make_uint4(__ldg(w), __ldg(w + 1), __ldg(w + 2), __ldg(w + 3));
        } else {
          uint32_t w[4];
#pragma unroll
          for (int q = 0; q < 4; q++)
            w[q] = (uint32_t)__ldg(sp + 4 * q) | ((uint32_t)__ldg(sp + 4 * q + 1) << 8) |
                   ((uint32_t)__ldg(sp + 4 * q + 2) << 16) | ((uint32_t)__ldg(sp + 4 * q + 3) << 24);
          v = make_uint4(w[0], w[1], w[2], w[3]);
        }
        *reinterpret_cast<uint4 *>(dp) = v;
      } else {
        for (long long k = 0; k < P && r.x0 + k < n; k++) dp[k] = sp[k];
      }
    }
  }
};

// f32 BGR / BGRA -> gray: b*0.114 + g*0.587 + r*0.299, unfused, in that
// order (color.zig:400); 4 pixels per thread.
template <int SCN>
struct OpGrayF {
  static constexpr int kThreads = 256, kMinBlocks = 4, P = 4;
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const RowSpan r = row_span<kThreads, P>(im, a.rows, tx, ty, im.s.h);
    const int w = im.s.w;
    if (r.x0 >= w) return;
    for (int y = r.y; y < r.yend; y += r.step) {
      const float *sp = row_ptr<const float>(im.s, y) + (long long)r.x0 * SCN;
      float *dp = row_ptr<float>(im.d, y) + r.x0;
#pragma unroll
      for (int i = 0; i < P; i++) {
        if (r.x0 + i >= w) break;
        const float *p = sp + i * SCN;
        dp[i] = __fadd_rn(__fadd_rn(__fmul_rn(__ldg(p), 0.114f), __fmul_rn(__ldg(p + 1), 0.587f)),
                          __fmul_rn(__ldg(p + 2), 0.299f));
      }
    }
  }
};

// Generic bilinear for f32 (resize.zig:284-423): f32 weights, h = s0*a0 +
// s1*a1, out = h0*b0 + h1*b1, unfused; one output pixel per thread.
template <int CN>
struct OpLinearF {
  static constexpr int kThreads = 256, kMinBlocks = 4;
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const RowSpan r = row_span<kThreads, 1>(im, a.rows, tx, ty, im.d.h);
    const int x = r.x0;
    if (x >= im.d.w) return;
    const FLinTap tq = static_cast<const FLinTap *>(im.t0)[x];
    const FLinTap *yt = static_cast<const FLinTap *>(im.t1);
    const long long a0 = (long long)tq.o0 * CN, a1 = (long long)tq.o1 * CN;
    for (int y = r.y; y < r.yend; y += r.step) {
      const FLinTap t = yt[y];
      const float *r0 = row_ptr<const float>(im.s, t.o0), *r1 = row_ptr<const float>(im.s, t.o1);
      float *o = row_ptr<float>(im.d, y) + (long long)x * CN;
#pragma unroll
      for (int c = 0; c < CN; c++) {
        const float h0 = __fadd_rn(__fmul_rn(__ldg(r0 + a0 + c), tq.a0), __fmul_rn(__ldg(r0 + a1 + c), tq.a1));
        const float h1 = __fadd_rn(__fmul_rn(__ldg(r1 + a0 + c), tq.a0), __fmul_rn(__ldg(r1 + a1 + c), tq.a1));
        o[c] = __fadd_rn(__fmul_rn(h0, t.a0), __fmul_rn(h1, t.a1));
      }
    }
  }
};

struct MorphFArgs {
  int rows;
  int kw, kh;  // rectangle, anchored at its centre
  bool is_max;
};

// f32 erode / dilate with a kw x kh rectangle, one pixel (all channels) per
// thread reading its window directly; pixels outside the image are ignored
// (morph.zig:473-474: the identity), min / max as fminf / fmaxf.
template <int CN>
struct OpMorphF {
  static constexpr int kThreads = 256, kMinBlocks = 4;
  using Args = MorphFArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const RowSpan r = row_span<kThreads, 1>(im, a.rows, tx, ty, im.s.h);
    const int x = r.x0, w = im.s.w, h = im.s.h;
    if (x >= w) return;
    const int xs0 = max(0, x - a.kw / 2), xs1 = min(w - 1, x - a.kw / 2 + a.kw - 1);
    const float id = a.is_max ? -__int_as_float(0x7f800000) : __int_as_float(0x7f800000);
    for (int y = r.y; y < r.yend; y += r.step) {
      const int ys0 = max(0, y - a.kh / 2), ys1 = min(h - 1, y - a.kh / 2 + a.kh - 1);
      float v[CN];
#pragma unroll
      for (int c = 0; c < CN; c++) v[c] = id;
      for (int sy = ys0; sy <= ys1; sy++) {
        const float *row = row_ptr<const float>(im.s, sy);
        for (int sx = xs0; sx <= xs1; sx++) {
#pragma unroll
          for (int c = 0; c < CN; c++) {
            const float u = __ldg(row + (long long)sx * CN + c);
            v[c] = a.is_max ? fmaxf(v[c], u) : fminf(v[c], u);
          }
        }
      }
      float *o = row_ptr<float>(im.d, y) + (long long)x * CN;
#pragma unroll
      for (int c = 0; c < CN; c++) o[c] = v[c];
    }
  }
};

// u8 Gaussian with binomial taps on warp strips (strip.cuh).
template <int K, int CN, int RH>
struct OpGaussStrip {
  static constexpr int kThreads = 128, kMinBlocks = 6;  // <= 85 registers (no spills)
  static constexpr bool kWarpTiles = true;
  using Args = strip::GaussArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, int lane) {
    strip::gauss_strip<K, CN, RH>(im.s, im.d, a.border, tx, ty, lane);
  }
};

struct NoArgs {
  int unused;
};

// Erode / dilate (one pass, or two fused) with a compiled element profile
// on warp strips (strip.cuh).
template <class P1, class P2, int CN, int RH, bool MAX1, bool FUSED>
struct OpMorphStrip {
  static constexpr int kThreads = 128, kMinBlocks = FUSED && P1::KH >= 7 ? 4 : FUSED ? 5 : 6;  // <= 128 / 102 / 85 registers
  static constexpr bool kWarpTiles = true;
  using Args = NoArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &, int tx, int ty, int lane) {
    strip::MorphStrip<P1, P2, CN, RH, MAX1, FUSED>::run(im.s, im.d, tx, ty, lane);
  }
};

struct WarpArgs {
  int interp, border;
  int rows;  // OpWarp4: tile height (a multiple of 32)
};

// warpAffine / warpPerspective on 32 x 32 output tiles; a warp covers 8 x 4
// pixels (the per-call kernels' footprint).
template <class T, int CN, bool PERSP>
struct OpWarp {
  static constexpr int kThreads = 256, TS = 32, kMinBlocks = 4;  // <= 64 registers
  using Args = WarpArgs;
  static size_t smem(const Args &) { return 0; }
  static int tiles_x(int w) { return (int)ceil_div(w, TS); }
  static int tiles_y(int h) { return (int)ceil_div(h, TS); }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const int y = ty * TS + (int)(threadIdx.x >> 3);
    if (y >= im.d.h) return;
    if constexpr (PERSP) {
      wp::PerArgs pa;
#pragma unroll
      for (int i = 0; i < 9; i++) pa.m[i] = im.md[i];
      pa.interp = a.interp;
      pa.border = a.border;
      pa.cv = im.cv;
#pragma unroll 1
      for (int k = 0; k < TS / 8; k++) {
        const int x = tx * TS + k * 8 + (int)(threadIdx.x & 7);
        if (x < im.d.w) wp::persp_px<T, CN>(im.s, im.d, pa, im.wide, x, y);
      }
    } else {
      wp::AffArgs aa;
#pragma unroll
      for (int i = 0; i < 6; i++) aa.m[i] = im.mf[i];
      aa.interp = a.interp;
      aa.border = a.border;
      aa.cv = im.cv;
#pragma unroll 1
      for (int k = 0; k < TS / 8; k++) {
        const int x = tx * TS + k * 8 + (int)(threadIdx.x & 7);
        if (x < im.d.w) wp::affine_px<T, CN>(im.s, im.d, aa, im.wide, x, y);
      }
    }
  }
};

// One-channel u8 warpAffine / warpPerspective, INTER_LINEAR, on 32 x 32
// output tiles of four consecutive pixels per thread (wp::warp4_u8: the
// taps of four pixels in flight together, 4-byte stores); a warp covers
// 32 x 4 pixels.
template <bool PERSP>
struct OpWarp4 {
  // Tiles of 32 x a.rows output pixels; a thread takes 4 consecutive pixels
  // in every 32nd row of its tile, so the tile's setup (queue ticket, image
  // record, matrix) is paid once per 4 x rows / 32 pixels.
  static constexpr int kThreads = 256, TS = 32, kDefaultRows = 128, kMinBlocks = 3;  // <= 85 registers (no spills)
  using Args = WarpArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const int x0 = tx * TS + (int)(threadIdx.x & 7) * 4;
    const int y0 = ty * a.rows, y1 = min(y0 + a.rows, im.d.h);
    if (x0 >= im.d.w) return;
    wp::PerArgs pa{};
    wp::AffArgs aa{};
    if constexpr (PERSP) {
#pragma unroll
      for (int i = 0; i < 9; i++) pa.m[i] = im.md[i];
      pa.interp = a.interp;
      pa.border = a.border;
      pa.cv = im.cv;
    } else {
#pragma unroll
      for (int i = 0; i < 6; i++) aa.m[i] = im.mf[i];
      aa.interp = a.interp;
      aa.border = a.border;
      aa.cv = im.cv;
    }
#pragma unroll 1
    for (int y = y0 + (int)(threadIdx.x >> 3); y < y1; y += kThreads / 8)
      wp::warp4_u8<PERSP>(im.s, im.d, pa, aa, im.wide, x0, y);
  }
};

// ----------------------------------------------------------- launching

template <class Op>
auto kernel_of() {
  if constexpr (WarpTiles<Op>::value) return k_batch_warp<Op>;
  else return k_batch<Op>;
}

// What one persistent launch needs: the queue, CTAs per SM (0: as many as
// fit) and the SM count; the grid launched is reported in *grid.
struct LaunchRun {
  TileQ q;
  int per_sm;
  int num_sms;
  int *grid;
};

// Launches Op's persistent kernel: the grid is the SMs times the CTAs per SM
// that fit (or the tuned count), capped by the tiles (per warp for
// warp-tile operations).
template <class Op>
cudaError_t launch_op(const LaunchRun &r, const typename Op::Args &a, cudaStream_t st) {
  const size_t smem = Op::smem(a);
  constexpr bool kWarp = WarpTiles<Op>::value;
  auto kern = kernel_of<Op>();
  static int occ = -1;  // per instantiation; same device type everywhere
  if (occ < 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, Op::kThreads, smem);
    if (e != cudaSuccess) return e;
    occ = o;
  }
  const int per_sm = r.per_sm > 0 ? std::min(r.per_sm, std::max(occ, 1)) : std::max(occ, 1);
  const int units = kWarp ? (int)ceil_div(r.q.total, Op::kThreads / 32) : r.q.total;
  const int grid = std::max(1, std::min(units, r.num_sms * per_sm));
  if (r.grid) *r.grid = grid;
  kern<<<grid, Op::kThreads, smem, st>>>(r.q, a);
  note_launch();
  return cudaGetLastError();
}

// Strip launches (batch_strip*.cu). prof: strip::ProfileId of the element.
cudaError_t launch_gauss_strip(const LaunchRun &r, int k, int cn, int rows, int border, cudaStream_t st);
cudaError_t launch_morph_strip(const LaunchRun &r, int prof, int cn, int rows, bool max1, bool fused, cudaStream_t st);

// The morphology strip launches of one channel count (one translation unit
// each, to spread the compile).
template <int CN>
cudaError_t launch_morph_strip_cn(const LaunchRun &r, int prof, int rows, bool max1, bool fused, cudaStream_t st);

template <class PR, int CN, int RH>
cudaError_t launch_morph_strip_rh(const LaunchRun &r, bool max1, bool fused, cudaStream_t st) {
  const NoArgs a{0};
  if (fused)
    return max1 ? launch_op<OpMorphStrip<PR, PR, CN, RH, true, true>>(r, a, st)
                : launch_op<OpMorphStrip<PR, PR, CN, RH, false, true>>(r, a, st);
  return max1 ? launch_op<OpMorphStrip<PR, PR, CN, RH, true, false>>(r, a, st)
              : launch_op<OpMorphStrip<PR, PR, CN, RH, false, false>>(r, a, st);
}

template <class PR, int CN>
cudaError_t launch_morph_strip_prof(const LaunchRun &r, int rows, bool max1, bool fused, cudaStream_t st) {
  if (rows == 8) return launch_morph_strip_rh<PR, CN, 8>(r, max1, fused, st);
  if constexpr (CN == 1) {  // 64- and 128-row tiles: one-channel images only (compile time)
    if (rows == 64) return launch_morph_strip_rh<PR, CN, 64>(r, max1, fused, st);
    if (rows == 128) return launch_morph_strip_rh<PR, CN, 128>(r, max1, fused, st);
  }
  return launch_morph_strip_rh<PR, CN, 32>(r, max1, fused, st);
}

// The one-channel profiles are instantiated in units of their own
// (batch_strip1a/b/c.cu).
#define VB_MORPH_PROF1(P) \
  extern template cudaError_t launch_morph_strip_prof<strip::P, 1>(const LaunchRun &, int, bool, bool, cudaStream_t);
VB_MORPH_PROF1(ProfRect3)
VB_MORPH_PROF1(ProfRect5)
VB_MORPH_PROF1(ProfRect7)
VB_MORPH_PROF1(ProfCross3)
VB_MORPH_PROF1(ProfCross5)
VB_MORPH_PROF1(ProfEll5)
VB_MORPH_PROF1(ProfEll7)
#undef VB_MORPH_PROF1

template <int CN>
cudaError_t launch_morph_strip_cn(const LaunchRun &r, int prof, int rows, bool max1, bool fused, cudaStream_t st) {
  using namespace strip;
  switch (prof) {
    case kRect3: return launch_morph_strip_prof<ProfRect3, CN>(r, rows, max1, fused, st);
    case kRect5: return launch_morph_strip_prof<ProfRect5, CN>(r, rows, max1, fused, st);
    case kRect7: return launch_morph_strip_prof<ProfRect7, CN>(r, rows, max1, fused, st);
    case kCross3: return launch_morph_strip_prof<ProfCross3, CN>(r, rows, max1, fused, st);
    case kCross5: return launch_morph_strip_prof<ProfCross5, CN>(r, rows, max1, fused, st);
    case kEll5: return launch_morph_strip_prof<ProfEll5, CN>(r, rows, max1, fused, st);
    case kEll7: return launch_morph_strip_prof<ProfEll7, CN>(r, rows, max1, fused, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace bt
}  // namespace vb
