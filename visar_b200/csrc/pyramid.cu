// Gaussian pyramid steps (src/imgproc/pyramid.zig): pyrDown (:73-96) and
// pyrUp (:408-426) for u8 / u16 / i16 / f32 images of any channel count.
//
// pyrDown: out(x, y) = sum over i, j in 0..4 of k_i k_j src(map(2x+i-2),
// map(2y+j-2)), k = [1 4 6 4 1], coordinates mapped by the border rule;
// integers finish with (v + 128) >> 8 (exact accumulators, so the pass order
// does not matter), f32 sums vertically first, per column
// ((r0 + r4) + (r1 + r3) * 4) + r2 * 6, then the same form horizontally, then
// * (1/256) (pyramid.zig:298-320, 335-344): the same operations in the same
// order here, each rounded on its own.
//
// pyrUp: the same kernel over the source upsampled with zeros and reflected
// about its own edges: per source row y, even output row 2y takes
// (r[y-1] + r[y+1]) + r[y] * 6 and odd row 2y+1 takes (r[y] + r[y+1]) * 4
// (rows mapped: -1 -> 1, h -> h-1); horizontally even pixel 2p takes
// (q[p-1] + q[p+1]) + q[p] * 6 and odd 2p+1 takes (q[p] + q[p+1]) * 4;
// integers finish with (v + 32) >> 6, f32 with * (1/64) (pyramid.zig:466-518).
//
// Layout: a CTA owns a tile of output rows and pixels. Phase 1 computes the
// vertical sums of every source element column under the tile (all channels
// interleaved) into shared memory, coalesced along the row; phase 2 combines
// them horizontally (taps cn elements apart) and stores the tile. Images with
// more than 16 channels use a direct kernel (one output element per thread).
#include "vb.h"

namespace vb {
namespace {

template <class T> struct PyrAcc { using A = int; };
template <> struct PyrAcc<float> { using A = float; };

template <class T, int S>
__device__ __forceinline__ T pyr_finish(int v) {
  return (T)((v + (1 << (S - 1))) >> S);  // arithmetic shift: floor for negative sums
}
template <class T, int S>
__device__ __forceinline__ T pyr_finish(float v) {
  return __fmul_rn(v, 1.0f / (float)(1 << S));
}

// ((a + e) + (b + d) * 4) + c * 6, each step rounded (f32) or exact (int).
__device__ __forceinline__ int tap5(int a, int b, int c, int d, int e) { return ((a + e) + (b + d) * 4) + c * 6; }
__device__ __forceinline__ float tap5(float a, float b, float c, float d, float e) {
  return __fadd_rn(__fadd_rn(__fadd_rn(a, e), __fmul_rn(__fadd_rn(b, d), 4.0f)), __fmul_rn(c, 6.0f));
}
__device__ __forceinline__ int up_even(int a, int b, int c) { return (a + c) + b * 6; }
__device__ __forceinline__ float up_even(float a, float b, float c) { return __fadd_rn(__fadd_rn(a, c), __fmul_rn(b, 6.0f)); }
__device__ __forceinline__ int up_odd(int b, int c) { return (b + c) * 4; }
__device__ __forceinline__ float up_odd(float b, float c) { return __fmul_rn(__fadd_rn(b, c), 4.0f); }

template <class T>
__device__ __forceinline__ typename PyrAcc<T>::A ld(const uint8_t *base, long long stride, int y, int e) {
  return (typename PyrAcc<T>::A)reinterpret_cast<const T *>(base + (long long)y * stride)[e];
}

constexpr int kDownRows = 8;      // output rows per tile
constexpr int kDownElems = 256;   // output elements (pixels x channels) per tile, about
constexpr int kThreads = 256;

// pyrDown tile: output rows [oy0, oy0 + kDownRows), output pixels [ox0, ox0 + twp).
// CN_: the channel count when compiled in (1, 3, 4), else 0 (cn at run time).
// vec: u8 destination rows 4-byte aligned and tiles of a multiple of 4
// output pixels; svec: source rows 4-byte aligned.
template <class T, int CN_>
__global__ void __launch_bounds__(kThreads) k_pyr_down(const uint8_t *__restrict__ src, long long sstride, int sw, int sh,
                                                       uint8_t *__restrict__ dst, long long dstride, int dw, int dh,
                                                       int cn_rt, int twp, int border, int vec, int svec) {
  using A = typename PyrAcc<T>::A;
  const int cn = CN_ > 0 ? CN_ : cn_rt;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *V = reinterpret_cast<A *>(smem_raw);
  const int ox0 = blockIdx.x * twp;
  const int oy0 = blockIdx.y * kDownRows;
  const int npx = min(twp, dw - ox0);
  const int nrows = min(kDownRows, dh - oy0);
  const int spx = 2 * npx + 3;  // source pixels 2*ox0-2 .. 2*(ox0+npx-1)+2
  const int span = spx * cn;
  // The tile's 2 * nrows + 3 source rows, border-mapped once.
  constexpr int NS = 2 * kDownRows + 3;
  __shared__ const uint8_t *s_row[NS];
  if (threadIdx.x < NS) s_row[threadIdx.x] = src + (long long)border_map(2 * oy0 - 2 + (int)threadIdx.x, sh, border) * sstride;
  __syncthreads();
  // Columns need the border map only in a row's first and last tiles.
  const bool inner = 2 * ox0 - 2 >= 0 && 2 * (ox0 + npx - 1) + 2 < sw;
  const int e0 = (2 * ox0 - 2) * cn;
  // Phase 1: vertical sums, V[r * span + e]; every row of a column is loaded
  // before the sums, so the loads are in flight together. u8 inner tiles
  // whose words stay inside the row take 4 bytes per thread and row (32-bit
  // loads from 4-byte aligned rows), summed as two 16-bit pair lanes
  // (sums <= 255 * 16, no carry between lanes).
  bool done = false;
  if constexpr (sizeof(T) == 1) {
    const int w0 = e0 & ~3;
    const int nw = (e0 + span - w0 + 3) >> 2;
    if (svec && inner && w0 + 4 * nw <= sw * cn) {
      for (int wi = threadIdx.x; wi < nw; wi += kThreads) {
        const int wb = w0 + 4 * wi;
        uint32_t r[NS];
#pragma unroll
        for (int k = 0; k < NS; k++) r[k] = k < 2 * nrows + 3 ? *reinterpret_cast<const uint32_t *>(s_row[k] + wb) : 0u;
        const int e = wb - e0;  // span element of the word's byte 0
#pragma unroll
        for (int rr = 0; rr < kDownRows; rr++) {
          if (rr >= nrows) break;
          uint32_t lo[5], hi[5];
#pragma unroll
          for (int t = 0; t < 5; t++) {
            lo[t] = r[2 * rr + t] & 0x00FF00FFu;         // bytes 0, 2
            hi[t] = (r[2 * rr + t] >> 8) & 0x00FF00FFu;  // bytes 1, 3
          }
          const uint32_t sl = ((lo[0] + lo[4]) + (lo[1] + lo[3]) * 4u) + lo[2] * 6u;
          const uint32_t sh8 = ((hi[0] + hi[4]) + (hi[1] + hi[3]) * 4u) + hi[2] * 6u;
          const int v4[4] = {(int)(sl & 0xFFFFu), (int)(sh8 & 0xFFFFu), (int)(sl >> 16), (int)(sh8 >> 16)};
#pragma unroll
          for (int b = 0; b < 4; b++)
            if (e + b >= 0 && e + b < span) V[rr * span + e + b] = v4[b];
        }
      }
      done = true;
    }
  }
  for (int e = threadIdx.x; e < span && !done; e += kThreads) {
    int se = e0 + e;
    if (!inner) {
      const int px = 2 * ox0 - 2 + e / cn;
      se = border_map(px, sw, border) * cn + (e - (e / cn) * cn);
    }
    A r[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) r[k] = k < 2 * nrows + 3 ? (A) reinterpret_cast<const T *>(s_row[k])[se] : (A)0;
#pragma unroll
    for (int rr = 0; rr < kDownRows; rr++)
      if (rr < nrows) V[rr * span + e] = tap5(r[2 * rr], r[2 * rr + 1], r[2 * rr + 2], r[2 * rr + 3], r[2 * rr + 4]);
  }
  __syncthreads();
  // Phase 2: output element j of the tile row sits over padded element 2j - j % cn + 2cn.
  if constexpr (sizeof(T) == 1 && CN_ > 0) {
    if (vec) {
      // u8: per thread and output row, four output pixels 4g .. 4g + 3 of
      // the tile (4 * CN bytes, CN aligned 32-bit stores); output element j
      // sits over padded element 2j - j % CN + 2CN.
      constexpr int CN = CN_;
      const int ng = (npx + 3) >> 2;
      for (int t = threadIdx.x; t < nrows * ng; t += kThreads) {
        const int r = t / ng, g = t - r * ng;
        const A *v = V + r * span + (8 * g + 2) * CN;  // output pixel 4g's channel 0
        const int npo = min(4, npx - 4 * g);
        uint32_t w[CN];
#pragma unroll
        for (int k = 0; k < CN; k++) w[k] = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          if (k >= npo) break;
#pragma unroll
          for (int c = 0; c < CN; c++) {
            const A *x = v + 2 * k * CN + c;
            const int byte = k * CN + c;
            w[byte >> 2] |= (uint32_t)pyr_finish<T, 8>(tap5(x[-2 * CN], x[-CN], x[0], x[CN], x[2 * CN])) << (8 * (byte & 3));
          }
        }
        uint8_t *o = dst + (long long)(oy0 + r) * dstride + (long long)(ox0 + 4 * g) * CN;
        if (npo == 4) {
#pragma unroll
          for (int k = 0; k < CN; k++) reinterpret_cast<uint32_t *>(o)[k] = w[k];
        } else {
          for (int b = 0; b < npo * CN; b++) o[b] = (uint8_t)(w[b >> 2] >> (8 * (b & 3)));
        }
      }
      return;
    }
  }
  const int ne = npx * cn;
  for (int r = 0; r < nrows; r++) {
    T *orow = reinterpret_cast<T *>(dst + (long long)(oy0 + r) * dstride) + (long long)ox0 * cn;
    for (int j = threadIdx.x; j < ne; j += kThreads) {
      const int c = 2 * j - j % cn + 2 * cn;
      const A *v = V + r * span + c;
      orow[j] = pyr_finish<T, 8>(tap5(v[-2 * cn], v[-cn], v[0], v[cn], v[2 * cn]));
    }
  }
}

// pyrDown for any channel count: one output element per thread, 25 loads.
template <class T>
__global__ void k_pyr_down_direct(const uint8_t *__restrict__ src, long long sstride, int sw, int sh,
                                  uint8_t *__restrict__ dst, long long dstride, int dw, int dh, int cn, int border) {
  using A = typename PyrAcc<T>::A;
  const long long ne = (long long)dw * cn;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ne * dh; i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / ne);
    const int j = (int)(i - (long long)y * ne);
    const int x = j / cn, ch = j - x * cn;
    A p[5];
    for (int t = 0; t < 5; t++) {
      const int se = border_map(2 * x + t - 2, sw, border) * cn + ch;
      A r[5];
      for (int k = 0; k < 5; k++) r[k] = ld<T>(src, sstride, border_map(2 * y + k - 2, sh, border), se);
      p[t] = tap5(r[0], r[1], r[2], r[3], r[4]);
    }
    reinterpret_cast<T *>(dst + (long long)y * dstride)[j] = pyr_finish<T, 8>(tap5(p[0], p[1], p[2], p[3], p[4]));
  }
}

constexpr int kUpRows = 8;  // source rows per tile (16 output rows)

__device__ __forceinline__ int up_row(int y, int h) { return y < 0 ? (h > 1 ? 1 : 0) : y >= h ? h - 1 : y; }

// pyrUp tile: source rows [sy0, sy0 + kUpRows), source pixels [sx0, sx0 + twp).
// vec: u8 destination rows 4-byte aligned (tiles start on 4-byte boundaries:
// 2 * twp * cn is a multiple of 4).
template <class T, int CN_>
__global__ void __launch_bounds__(kThreads) k_pyr_up(const uint8_t *__restrict__ src, long long sstride, int sw, int sh,
                                                     uint8_t *__restrict__ dst, long long dstride, int cn_rt, int twp, int vec) {
  using A = typename PyrAcc<T>::A;
  const int cn = CN_ > 0 ? CN_ : cn_rt;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int sx0 = blockIdx.x * twp;
  const int sy0 = blockIdx.y * kUpRows;
  const int npx = min(twp, sw - sx0);
  const int nrows = min(kUpRows, sh - sy0);
  const int span = (npx + 2) * cn;  // source pixels sx0-1 .. sx0+npx
  A *E = reinterpret_cast<A *>(smem_raw);
  A *O = E + kUpRows * span;
  // The tile's nrows + 2 source rows, mapped once.
  constexpr int NS = kUpRows + 2;
  __shared__ const uint8_t *s_row[NS];
  if (threadIdx.x < NS) s_row[threadIdx.x] = src + (long long)up_row(sy0 - 1 + (int)threadIdx.x, sh) * sstride;
  __syncthreads();
  const bool inner = sx0 - 1 >= 0 && sx0 + npx < sw;
  // Every row of a column is loaded before the sums (loads in flight together).
  for (int e = threadIdx.x; e < span; e += kThreads) {
    int se = (sx0 - 1) * cn + e;
    if (!inner) {
      const int px = sx0 - 1 + e / cn;
      const int mx = px < 0 ? (sw > 1 ? 1 : 0) : px >= sw ? sw - 1 : px;
      se = mx * cn + (e - (e / cn) * cn);
    }
    A r[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) r[k] = k < nrows + 2 ? (A) reinterpret_cast<const T *>(s_row[k])[se] : (A)0;
#pragma unroll
    for (int rr = 0; rr < kUpRows; rr++) {
      if (rr < nrows) {
        E[rr * span + e] = up_even(r[rr], r[rr + 1], r[rr + 2]);
        O[rr * span + e] = up_odd(r[rr + 1], r[rr + 2]);
      }
    }
  }
  __syncthreads();
  if constexpr (sizeof(T) == 1 && CN_ > 0) {
    if (vec) {
      constexpr int CN = CN_;
      // u8: per thread and output row, the four output pixels over source
      // pixels p0 = 2g and p0 + 1 of the tile (4 * CN bytes, CN aligned
      // 32-bit stores); q[k * CN + c] is source pixel p0 + k, k = -1 .. 2.
      const int ng = (npx + 1) >> 1;
      for (int t = threadIdx.x; t < 2 * nrows * ng; t += kThreads) {
        const int rr = t / ng, g = t - rr * ng;
        const A *q = ((rr & 1) ? O : E) + (rr >> 1) * span + (2 * g + 1) * CN;
        const int npo = min(4, 2 * npx - 4 * g);  // output pixels of the group inside the tile (4 or 2)
        uint32_t w[CN];
#pragma unroll
        for (int k = 0; k < CN; k++) w[k] = 0;
#pragma unroll
        for (int op = 0; op < 4; op++) {
          if (op >= npo) break;
          const int pp = op >> 1;
#pragma unroll
          for (int c = 0; c < CN; c++) {
            const A s = (op & 1) ? up_odd(q[pp * CN + c], q[(pp + 1) * CN + c])
                                 : up_even(q[(pp - 1) * CN + c], q[pp * CN + c], q[(pp + 1) * CN + c]);
            const int byte = op * CN + c;
            w[byte >> 2] |= (uint32_t)pyr_finish<T, 6>(s) << (8 * (byte & 3));
          }
        }
        uint8_t *o = dst + (long long)(2 * sy0 + rr) * dstride + (long long)(2 * sx0 + 4 * g) * CN;
        if (npo == 4) {
#pragma unroll
          for (int k = 0; k < CN; k++) reinterpret_cast<uint32_t *>(o)[k] = w[k];
        } else {
#pragma unroll
          for (int b = 0; b < 2 * CN; b++) o[b] = (uint8_t)(w[b >> 2] >> (8 * (b & 3)));
        }
      }
      return;
    }
  }
  // Output pixel 2p (+1) of tile row r; q[p] is smem element (p - sx0 + 1) * cn.
  const int ne = 2 * npx * cn;
  for (int rr = 0; rr < 2 * nrows; rr++) {  // output row within the tile
    T *orow = reinterpret_cast<T *>(dst + (long long)(2 * sy0 + rr) * dstride) + (long long)2 * sx0 * cn;
    const A *qrow = ((rr & 1) ? O : E) + (rr >> 1) * span;
    for (int j = threadIdx.x; j < ne; j += kThreads) {
      const int opx = j / cn, ch = j - opx * cn;
      const A *q = qrow + ((opx >> 1) + 1) * cn + ch;
      const A s = (opx & 1) ? up_odd(q[0], q[cn]) : up_even(q[-cn], q[0], q[cn]);
      orow[j] = pyr_finish<T, 6>(s);
    }
  }
}

template <class T>
__global__ void k_pyr_up_direct(const uint8_t *__restrict__ src, long long sstride, int sw, int sh,
                                uint8_t *__restrict__ dst, long long dstride, int cn) {
  using A = typename PyrAcc<T>::A;
  const long long ne = 2LL * sw * cn;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ne * 2 * sh; i += (long long)gridDim.x * blockDim.x) {
    const int oy = (int)(i / ne);
    const int j = (int)(i - (long long)oy * ne);
    const int opx = j / cn, ch = j - opx * cn;
    const int y = oy >> 1, p = opx >> 1;
    auto col = [&](int px) -> A {
      const int mx = px < 0 ? (sw > 1 ? 1 : 0) : px >= sw ? sw - 1 : px;
      const int se = mx * cn + ch;
      const A a = ld<T>(src, sstride, up_row(y - 1, sh), se);
      const A b = ld<T>(src, sstride, y, se);
      const A c = ld<T>(src, sstride, up_row(y + 1, sh), se);
      return (oy & 1) ? up_odd(b, c) : up_even(a, b, c);
    };
    const A s = (opx & 1) ? up_odd(col(p), col(p + 1)) : up_even(col(p - 1), col(p), col(p + 1));
    reinterpret_cast<T *>(dst + (long long)oy * dstride)[j] = pyr_finish<T, 6>(s);
  }
}

template <class T>
cudaError_t pyr_down_t(const DImg &s, const DImg &d, int border, cudaStream_t st) {
  using A = typename PyrAcc<T>::A;
  note_launch();
  if (s.cn > 16) {
    const long long n = (long long)d.w * d.cn * d.h;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 64);
    k_pyr_down_direct<T><<<blocks, 256, 0, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, s.cn, border);
    return cudaGetLastError();
  }
  // Tiles of a multiple of 4 output pixels (4-byte aligned u8 tile rows).
  const int twp = std::max(4, (kDownElems / s.cn) & ~3);
  const size_t smem = (size_t)kDownRows * (2 * twp + 3) * s.cn * sizeof(A);
  dim3 grid((d.w + twp - 1) / twp, (d.h + kDownRows - 1) / kDownRows);
  const int vec = (uintptr_t)d.p % 4 == 0 && d.stride % 4 == 0;
  const int svec = (uintptr_t)s.p % 4 == 0 && s.stride % 4 == 0;
  switch (s.cn) {
    case 1: k_pyr_down<T, 1><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, 1, twp, border, vec, svec); break;
    case 3: k_pyr_down<T, 3><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, 3, twp, border, vec, svec); break;
    case 4: k_pyr_down<T, 4><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, 4, twp, border, vec, svec); break;
    default: k_pyr_down<T, 0><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, s.cn, twp, border, vec, svec);
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t pyr_up_t(const DImg &s, const DImg &d, cudaStream_t st) {
  using A = typename PyrAcc<T>::A;
  note_launch();
  if (s.cn > 16) {
    const long long n = (long long)d.w * d.cn * d.h;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 64);
    k_pyr_up_direct<T><<<blocks, 256, 0, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, s.cn);
    return cudaGetLastError();
  }
  const int twp = std::max(1, 128 / s.cn);
  const size_t smem = (size_t)2 * kUpRows * (twp + 2) * s.cn * sizeof(A);
  dim3 grid((s.w + twp - 1) / twp, (s.h + kUpRows - 1) / kUpRows);
  const int vec = (uintptr_t)d.p % 4 == 0 && d.stride % 4 == 0 && (2 * twp * s.cn) % 4 == 0;
  switch (s.cn) {
    case 1: k_pyr_up<T, 1><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, 1, twp, vec); break;
    case 3: k_pyr_up<T, 3><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, 3, twp, vec); break;
    case 4: k_pyr_up<T, 4><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, 4, twp, vec); break;
    default: k_pyr_up<T, 0><<<grid, kThreads, smem, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, s.cn, twp, vec);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pyr_down(const DImg &s, const DImg &d, int depth, int border, cudaStream_t st) {
  switch (depth) {
    case k8U: return pyr_down_t<uint8_t>(s, d, border, st);
    case k16U: return pyr_down_t<uint16_t>(s, d, border, st);
    case k16S: return pyr_down_t<int16_t>(s, d, border, st);
    case k32F: return pyr_down_t<float>(s, d, border, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_pyr_up(const DImg &s, const DImg &d, int depth, cudaStream_t st) {
  switch (depth) {
    case k8U: return pyr_up_t<uint8_t>(s, d, st);
    case k16U: return pyr_up_t<uint16_t>(s, d, st);
    case k16S: return pyr_up_t<int16_t>(s, d, st);
    case k32F: return pyr_up_t<float>(s, d, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace vb
