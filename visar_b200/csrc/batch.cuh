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

template <class Op>
__global__ void __launch_bounds__(Op::kThreads) k_batch(TileQ q, typename Op::Args a) {
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
    const BImg &im = q.imgs[img];
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
    const BImg &im = q.imgs[img];
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

// Row-tiled elementwise operations: a tile is `rows` rows x (kThreads * P) pixels.
struct RowArgs {
  int rows;
};

__device__ __forceinline__ uint32_t gray_px(uint32_t b, uint32_t g, uint32_t r) {
  return (b * kB2G + g * kG2G + r * kR2G + (1u << (kGrayShift - 1))) >> kGrayShift;
}

// BGR / BGRA -> gray, 16 pixels per thread (color.zig:324-403 arithmetic).
template <int SCN>
struct OpGray {
  static constexpr int kThreads = 256, P = 16;
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  static int tiles_x(int w) { return (int)ceil_div(w, kThreads * P); }
  static int tiles_y(int h, const Args &a) { return (int)ceil_div(h, a.rows); }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const int x0 = tx * (kThreads * P) + (int)threadIdx.x * P;
    if (x0 >= im.s.w) return;
    const bool full = x0 + P <= im.s.w;
    for (int r = 0; r < a.rows; r++) {
      const int y = ty * a.rows + r;
      if (y >= im.s.h) break;
      const uint8_t *sp = row_ptr<const uint8_t>(im.s, y) + (long long)x0 * SCN;
      uint8_t *dp = row_ptr<uint8_t>(im.d, y) + x0;
      if (full && (((uintptr_t)sp | (uintptr_t)dp) % 16) == 0) {
        uint4 v[SCN];
#pragma unroll
        for (int k = 0; k < SCN; k++) v[k] = reinterpret_cast<const uint4 *>(sp)[k];
        const uint8_t *b = reinterpret_cast<const uint8_t *>(v);
        uint32_t o[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          uint32_t w = 0;
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int p = q * 4 + i;
            w |= gray_px(b[p * SCN], b[p * SCN + 1], b[p * SCN + 2]) << (8 * i);
          }
          o[q] = w;
        }
        *reinterpret_cast<uint4 *>(dp) = make_uint4(o[0], o[1], o[2], o[3]);
      } else {
        for (int i = 0; i < P && x0 + i < im.s.w; i++) dp[i] = (uint8_t)gray_px(sp[i * SCN], sp[i * SCN + 1], sp[i * SCN + 2]);
      }
    }
  }
};

// Exact halving (resize_u8.zig:381-447), 4 output pixels per thread.
template <int CN>
struct OpHalf {
  static constexpr int kThreads = 256, P = 4;
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  static int tiles_x(int dw) { return (int)ceil_div(dw, kThreads * P); }
  static int tiles_y(int dh, const Args &a) { return (int)ceil_div(dh, a.rows); }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const int x0 = tx * (kThreads * P) + (int)threadIdx.x * P;
    if (x0 >= im.d.w) return;
    const bool full = x0 + P <= im.d.w;
    for (int r = 0; r < a.rows; r++) {
      const int y = ty * a.rows + r;
      if (y >= im.d.h) break;
      const uint8_t *ra = row_ptr<const uint8_t>(im.s, 2LL * y) + (size_t)x0 * 2 * CN;
      const uint8_t *rb = row_ptr<const uint8_t>(im.s, 2LL * y + 1) + (size_t)x0 * 2 * CN;
      uint8_t *o = row_ptr<uint8_t>(im.d, y) + (size_t)x0 * CN;
      if (full && (((uintptr_t)ra | (uintptr_t)rb) % 8) == 0 && ((uintptr_t)o % 4) == 0) {
        uint2 va[CN], vb2[CN];
#pragma unroll
        for (int k = 0; k < CN; k++) {
          va[k] = reinterpret_cast<const uint2 *>(ra)[k];
          vb2[k] = reinterpret_cast<const uint2 *>(rb)[k];
        }
        const uint8_t *ba = reinterpret_cast<const uint8_t *>(va);
        const uint8_t *bb = reinterpret_cast<const uint8_t *>(vb2);
        uint32_t out[CN];
#pragma unroll
        for (int k = 0; k < CN; k++) {
          uint32_t w = 0;
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const int oi = k * 4 + j;  // output sample index within the 4 pixels
            const int p = oi / CN, c = oi % CN;
            const int i = 2 * p * CN + c;
            w |= (((uint32_t)ba[i] + ba[i + CN] + bb[i] + bb[i + CN] + 2u) >> 2) << (8 * j);
          }
          out[k] = w;
        }
#pragma unroll
        for (int k = 0; k < CN; k++) reinterpret_cast<uint32_t *>(o)[k] = out[k];
      } else {
        for (int p = 0; p < P && x0 + p < im.d.w; p++)
          for (int c = 0; c < CN; c++) {
            const int i = 2 * p * CN + c;
            o[p * CN + c] = (uint8_t)(((uint32_t)ra[i] + ra[i + CN] + rb[i] + rb[i + CN] + 2u) >> 2);
          }
      }
    }
  }
};

// OpenCV's fixed-point bilinear for u8 (resize_u8.zig:651-711) from the
// image's tap tables (t0: x taps in pixels, t1: y taps in rows).
template <int CN>
struct OpLinear {
  static constexpr int kThreads = 256, P = 1;
  using Args = RowArgs;
  static size_t smem(const Args &) { return 0; }
  static int tiles_x(int dw) { return (int)ceil_div(dw, kThreads); }
  static int tiles_y(int dh, const Args &a) { return (int)ceil_div(dh, a.rows); }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *) {
    const int x = tx * kThreads + (int)threadIdx.x;
    if (x >= im.d.w) return;
    const int4 tq = reinterpret_cast<const int4 *>(im.t0)[x];
    const LinTap *yt = static_cast<const LinTap *>(im.t1);
    const int a0 = tq.x * CN, a1 = tq.y * CN;
    for (int r = 0; r < a.rows; r++) {
      const int y = ty * a.rows + r;
      if (y >= im.d.h) break;
      const LinTap ty2 = yt[y];
      const uint8_t *r0 = row_ptr<const uint8_t>(im.s, ty2.o0);
      const uint8_t *r1 = row_ptr<const uint8_t>(im.s, ty2.o1);
      uint8_t *o = row_ptr<uint8_t>(im.d, y) + (size_t)x * CN;
#pragma unroll
      for (int c = 0; c < CN; c++) {
        const int h0 = ((int)r0[a0 + c] * tq.z + (int)r0[a1 + c] * tq.w) >> 4;
        const int h1 = ((int)r1[a0 + c] * tq.z + (int)r1[a1 + c] * tq.w) >> 4;
        const int t = ((h0 * ty2.w0) >> 16) + ((h1 * ty2.w1) >> 16);
        o[c] = (uint8_t)min(max((t + 2) >> 2, 0), 255);
      }
    }
  }
};

struct LutArgs {
  int rows;
  const uint8_t *lut;
};

// u8 threshold through a 256-entry table (threshold.zig:39-60), 16 samples per thread.
struct OpLut {
  static constexpr int kThreads = 256, P = 16;
  using Args = LutArgs;
  static size_t smem(const Args &) { return 256; }
  static int tiles_x(long long n) { return (int)ceil_div(n, kThreads * P); }
  static int tiles_y(int h, const Args &a) { return (int)ceil_div(h, a.rows); }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &a, int tx, int ty, unsigned char *smem) {
    uint8_t *t = smem;
    t[threadIdx.x] = a.lut[threadIdx.x];
    __syncthreads();
    const long long n = (long long)im.s.w * im.s.cn;
    const long long i0 = (long long)tx * (kThreads * P) + threadIdx.x * P;
    if (i0 >= n) return;
    for (int r = 0; r < a.rows; r++) {
      const int y = ty * a.rows + r;
      if (y >= im.s.h) break;
      const uint8_t *sp = row_ptr<const uint8_t>(im.s, y) + i0;
      uint8_t *dp = row_ptr<uint8_t>(im.d, y) + i0;
      if (i0 + P <= n && (((uintptr_t)sp | (uintptr_t)dp) % 16) == 0) {
        uint4 v = *reinterpret_cast<const uint4 *>(sp);
        uint8_t *b = reinterpret_cast<uint8_t *>(&v);
#pragma unroll
        for (int k = 0; k < P; k++) b[k] = t[b[k]];
        *reinterpret_cast<uint4 *>(dp) = v;
      } else {
        for (long long k = 0; k < P && i0 + k < n; k++) dp[k] = t[sp[k]];
      }
    }
  }
};

// u8 Gaussian with binomial taps on warp strips (strip.cuh).
template <int K, int CN, int RH>
struct OpGaussStrip {
  static constexpr int kThreads = 128, kMinBlocks = 4;  // <= 128 registers (no spills)
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
  static constexpr int kThreads = 128, kMinBlocks = FUSED ? 5 : 6;  // 102 / 85 registers
  static constexpr bool kWarpTiles = true;
  using Args = NoArgs;
  static size_t smem(const Args &) { return 0; }
  static __device__ __forceinline__ void tile(const BImg &im, const Args &, int tx, int ty, int lane) {
    strip::MorphStrip<P1, P2, CN, RH, MAX1, FUSED>::run(im.s, im.d, tx, ty, lane);
  }
};

struct WarpArgs {
  int interp, border;
};

// warpAffine / warpPerspective on 32 x 32 output tiles; a warp covers 8 x 4
// pixels (the per-call kernels' footprint).
template <class T, int CN, bool PERSP>
struct OpWarp {
  static constexpr int kThreads = 256, TS = 32;
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
  return rows == 8 ? launch_morph_strip_rh<PR, CN, 8>(r, max1, fused, st)
                   : launch_morph_strip_rh<PR, CN, 32>(r, max1, fused, st);
}

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
