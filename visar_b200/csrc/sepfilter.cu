// Separable filtering: GaussianBlur, boxFilter, Sobel and sepFilter2D
// (src/imgproc/filter.zig:118-341).
//
// VISAR filters vertically first into one row of accumulators, replicates
// the filtered columns across the horizontal border, then filters
// horizontally and finishes (filter.zig:168-205). Integer accumulators are
// exact, so any order gives the same result and the GPU sums freely. f32
// accumulators are order-sensitive: VISAR's 16-lane vector body folds
// mirrored taps (centre first, then pairs from the edge inwards,
// filter.zig:232-252) while the scalar tail of each row (the last
// rowLen % 16 samples) sums taps left to right (filter.zig:254-258). Both
// orders are reproduced per sample position, so f32 results are bit-exact.
//
// GPU layout: one CTA computes a tile of TW samples x TH rows. The source
// tile with its halo (TH + 2ry rows, TW + 2rx*cn samples, borders resolved
// by border_map) is staged in shared memory, the vertical pass writes its
// accumulators to shared memory, and the horizontal pass reads them.
#include <algorithm>
#include <cstring>

#include "vb.h"

namespace vb {

namespace {

constexpr int kMaxTaps = 255;
constexpr int kTileW = 128;  // samples per tile row

template <class K>
struct SepArgs {
  int nkx, nky, rx, ry, border;
  int n16;         // samples [n16, rowLen) of a row use the scalar-tail order
  int symx, symy;  // 0 none, 1 even, 2 odd (filter.zig:213-229)
  int shift;
  float scalef;
  K kx[kMaxTaps];
  K ky[kMaxTaps];
};

template <class A>
__device__ __forceinline__ float as_float(A v) {
  return (float)v;
}

// Weighted sum of nk taps; ld(j) returns tap j's input. For f32 the order
// follows tapsV (vector body, by symmetry) or tapsS (scalar tail).
template <class A, class K, class F>
__device__ __forceinline__ A taps_sum(F ld, const K *k, int nk, int sym, bool tail) {
  if constexpr (IsFloat<A>::v) {
    if (tail) {
      float a = __fmul_rn(k[0], ld(0));
      for (int j = 1; j < nk; j++) a = __fadd_rn(a, __fmul_rn(k[j], ld(j)));
      return a;
    }
    const int r = nk / 2;
    if (sym == 1) {
      float a = __fmul_rn(ld(r), k[r]);
      for (int i = 0; i < r; i++) a = __fadd_rn(a, __fmul_rn(__fadd_rn(ld(i), ld(nk - 1 - i)), k[i]));
      return a;
    }
    if (sym == 2) {
      float a = 0.0f;
      for (int i = 0; i < r; i++) a = __fadd_rn(a, __fmul_rn(__fsub_rn(ld(nk - 1 - i), ld(i)), k[nk - 1 - i]));
      return a;
    }
    float a = 0.0f;
    for (int j = 0; j < nk; j++) a = __fadd_rn(a, __fmul_rn(ld(j), k[j]));
    return a;
  } else {
    A a = 0;
    for (int j = 0; j < nk; j++) a += (A)k[j] * ld(j);
    return a;
  }
}

template <class D, class A, int FIN>
__device__ __forceinline__ D finish(A v, int shift, float scalef) {
  if constexpr (FIN == kFinShift) {
    unsigned long long u = (unsigned long long)v;
    u = (u + (1ULL << (shift - 1))) >> shift;
    const unsigned long long hi = (unsigned long long)Lim<D>::hi;
    return (D)(u < hi ? u : hi);
  } else if constexpr (FIN == kFinCast) {
    if constexpr (IsFloat<A>::v) return satv_f<D>(v);
    else return satv_i<D>((long long)v);
  } else {
    return satv_f<D>(__fmul_rn(as_float(v), scalef));
  }
}

__device__ __forceinline__ long long floor_div(long long a, int b) {
  long long q = a / b;
  if ((a % b) != 0 && ((a < 0) != (b < 0))) q--;
  return q;
}

template <class S, class D, class A, class K, int FIN>
__global__ void __launch_bounds__(256) k_sep_tiled(DImg s, DImg d, SepArgs<K> a, int th) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int cn = s.cn, W = s.w, H = s.h;
  const long long n = (long long)W * cn;
  const int halo = a.rx * cn;
  const int twh = kTileW + 2 * halo;
  const int ih = th + 2 * a.ry;
  const long long x0s = (long long)blockIdx.x * kTileW;
  const int y0 = blockIdx.y * th;
  S *in = reinterpret_cast<S *>(smem);
  size_t in_bytes = ((size_t)ih * twh * sizeof(S) + 15) & ~(size_t)15;
  A *V = reinterpret_cast<A *>(smem + in_bytes);

  for (int idx = threadIdx.x; idx < ih * twh; idx += blockDim.x) {
    const int r = idx / twh, c = idx - r * twh;
    const long long gs = x0s - halo + c;
    const long long px = floor_div(gs, cn);
    const int ch = (int)(gs - px * cn);
    const int mx = border_map(px, W, a.border);
    const int my = border_map((long long)y0 - a.ry + r, H, a.border);
    S v = S(0);
    if (mx >= 0 && my >= 0) v = row_ptr<const S>(s, my)[(long long)mx * cn + ch];
    in[idx] = v;
  }
  __syncthreads();

  for (int idx = threadIdx.x; idx < th * twh; idx += blockDim.x) {
    const int r = idx / twh, c = idx - r * twh;
    const long long gs = x0s - halo + c;
    const long long px = floor_div(gs, cn);
    const int ch = (int)(gs - px * cn);
    const int mx = border_map(px, W, a.border);
    A v = A(0);
    if (mx >= 0) {
      const long long msi = (long long)mx * cn + ch;  // the column's own sample index
      const S *col = in + r * twh + c;
      v = taps_sum<A, K>([&](int j) { return (A)col[j * twh]; }, a.ky, a.nky, a.symy, msi >= a.n16);
    }
    V[idx] = v;
  }
  __syncthreads();

  for (int idx = threadIdx.x; idx < th * kTileW; idx += blockDim.x) {
    const int r = idx / kTileW, c = idx - r * kTileW;
    const int y = y0 + r;
    const long long xo = x0s + c;
    if (y >= H || xo >= n) continue;
    const A *vr = V + r * twh + c;
    const A v = taps_sum<A, K>([&](int i) { return vr[i * cn]; }, a.kx, a.nkx, a.symx, xo >= a.n16);
    row_ptr<D>(d, y)[xo] = finish<D, A, FIN>(v, a.shift, a.scalef);
  }
}

// Fallback for halos too wide for a shared-memory tile: one thread per
// output sample, vertical sums computed on demand from global memory.
template <class S, class D, class A, class K, int FIN>
__global__ void __launch_bounds__(256) k_sep_direct(DImg s, DImg d, SepArgs<K> a) {
  const long long n = (long long)s.w * s.cn;
  const long long xo = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (xo >= n) return;
  const int cn = s.cn;
  const long long px0 = xo / cn;
  const int ch = (int)(xo - px0 * cn);
  auto vcol = [&](int i) -> A {
    const int mx = border_map(px0 - a.rx + i, s.w, a.border);
    if (mx < 0) return A(0);
    const long long msi = (long long)mx * cn + ch;
    return taps_sum<A, K>(
        [&](int j) -> A {
          const int my = border_map((long long)y - a.ry + j, s.h, a.border);
          return my < 0 ? A(0) : (A)row_ptr<const S>(s, my)[msi];
        },
        a.ky, a.nky, a.symy, msi >= a.n16);
  };
  const A v = taps_sum<A, K>(vcol, a.kx, a.nkx, a.symx, xo >= a.n16);
  row_ptr<D>(d, y)[xo] = finish<D, A, FIN>(v, a.shift, a.scalef);
}

template <class K>
int symmetry(const std::vector<K> &k, bool is_unsigned) {
  const int n = (int)k.size();
  bool even = true, odd = true;
  for (int i = 0; i < n / 2; i++) {
    const K x = k[i], y = k[n - 1 - i];
    if (x != y) even = false;
    if (is_unsigned) odd = false;
    else if (x != -y) odd = false;
  }
  if (n % 2 == 1 && k[n / 2] != 0) odd = false;
  return even ? 1 : odd ? 2 : 0;
}

template <class S, class D, class A, class K, int FIN>
cudaError_t run(const DImg &s, const DImg &d, const SepArgs<K> &a, cudaStream_t st) {
  const long long n = (long long)s.w * s.cn;
  const int halo = a.rx * s.cn;
  const int twh = kTileW + 2 * halo;
  size_t smem = 0;
  int th = 0;
  for (int cand : {32, 16, 8, 4, 2, 1}) {
    const int ih = cand + 2 * a.ry;
    const size_t in_b = (((size_t)ih * twh * sizeof(S)) + 15) & ~(size_t)15;
    const size_t need = in_b + (size_t)cand * twh * sizeof(A);
    if (need <= 160 * 1024 && (size_t)ih * twh < (1u << 30)) {
      th = cand;
      smem = need;
      break;
    }
  }
  if (th > 0 && halo < (1 << 20)) {
    auto kfn = k_sep_tiled<S, D, A, K, FIN>;
    cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(ceil_div(n, kTileW), ceil_div(s.h, th));
    kfn<<<grid, 256, smem, st>>>(s, d, a, th);
    note_launch();
    return cudaGetLastError();
  }
  dim3 grid(ceil_div(n, 256), s.h);
  k_sep_direct<S, D, A, K, FIN><<<grid, 256, 0, st>>>(s, d, a);
  note_launch();
  return cudaGetLastError();
}

template <class K>
SepArgs<K> make_args(const DImg &s, const std::vector<K> &kx, const std::vector<K> &ky, const SepSpec &sp, bool uns) {
  SepArgs<K> a;
  std::memset(&a, 0, sizeof(a));
  a.nkx = (int)kx.size();
  a.nky = (int)ky.size();
  a.rx = a.nkx / 2;
  a.ry = a.nky / 2;
  a.border = sp.border;
  const long long n = (long long)s.w * s.cn;
  a.n16 = (int)(n - n % 16);
  a.symx = symmetry(kx, uns);
  a.symy = symmetry(ky, uns);
  a.shift = sp.shift;
  a.scalef = (float)sp.scale;
  for (int i = 0; i < a.nkx; i++) a.kx[i] = kx[i];
  for (int i = 0; i < a.nky; i++) a.ky[i] = ky[i];
  return a;
}

template <class S, class D>
cudaError_t run_float_cast(const DImg &s, const DImg &d, const SepArgs<float> &a, cudaStream_t st) {
  return run<S, D, float, float, kFinCast>(s, d, a, st);
}

template <class S>
cudaError_t run_float_cast_d(const DImg &s, const DImg &d, int ddepth, const SepArgs<float> &a, cudaStream_t st) {
  switch (ddepth) {
    case k8U: return run_float_cast<S, uint8_t>(s, d, a, st);
    case k16U: return run_float_cast<S, uint16_t>(s, d, a, st);
    case k16S: return run_float_cast<S, int16_t>(s, d, a, st);
    case k32F: return run_float_cast<S, float>(s, d, a, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_sep_filter(const DImg &s, const DImg &d, const SepSpec &sp, cudaStream_t st) {
  if (s.w == 0 || s.h == 0) return cudaSuccess;
  {
    const cudaError_t e = launch_sep_fast(s, d, sp, 0, st);
    if (e != cudaErrorNotSupported) return e;
  }
  if (sp.acc == kAccF32) {
    if ((int)sp.kxf.size() > kMaxTaps || (int)sp.kyf.size() > kMaxTaps) return cudaErrorInvalidValue;
    const SepArgs<float> a = make_args<float>(s, sp.kxf, sp.kyf, sp, false);
    if (sp.fin == kFinCast) {
      switch (sp.sdepth) {
        case k8U: return run_float_cast_d<uint8_t>(s, d, sp.ddepth, a, st);
        case k16U: return run_float_cast_d<uint16_t>(s, d, sp.ddepth, a, st);
        case k16S: return run_float_cast_d<int16_t>(s, d, sp.ddepth, a, st);
        case k32F: return run_float_cast_d<float>(s, d, sp.ddepth, a, st);
      }
      return cudaErrorInvalidValue;
    }
    if (sp.fin == kFinScaled) {
      if (sp.ddepth == k32F) {
        switch (sp.sdepth) {
          case k8U: return run<uint8_t, float, float, float, kFinScaled>(s, d, a, st);
          case k16U: return run<uint16_t, float, float, float, kFinScaled>(s, d, a, st);
          case k16S: return run<int16_t, float, float, float, kFinScaled>(s, d, a, st);
          case k32F: return run<float, float, float, float, kFinScaled>(s, d, a, st);
        }
      }
      if (sp.sdepth == k8U && sp.ddepth == k16S) return run<uint8_t, int16_t, float, float, kFinScaled>(s, d, a, st);
    }
    return cudaErrorInvalidValue;
  }
  if ((int)sp.kxi.size() > kMaxTaps || (int)sp.kyi.size() > kMaxTaps) return cudaErrorInvalidValue;
  const SepArgs<int> a = make_args<int>(s, sp.kxi, sp.kyi, sp, false);
  if (sp.acc == kAccI32) {
    if (sp.sdepth == k8U && sp.ddepth == k8U) {
      if (sp.fin == kFinShift) return run<uint8_t, uint8_t, int, int, kFinShift>(s, d, a, st);
      if (sp.fin == kFinScaled) return run<uint8_t, uint8_t, int, int, kFinScaled>(s, d, a, st);
    }
    if (sp.sdepth == k8U && sp.ddepth == k16S) {
      if (sp.fin == kFinCast) return run<uint8_t, int16_t, int, int, kFinCast>(s, d, a, st);
      if (sp.fin == kFinScaled) return run<uint8_t, int16_t, int, int, kFinScaled>(s, d, a, st);
    }
    return cudaErrorInvalidValue;
  }
  // kAccI64
  if (sp.sdepth == k16U && sp.ddepth == k16U) {
    if (sp.fin == kFinShift) return run<uint16_t, uint16_t, long long, int, kFinShift>(s, d, a, st);
    if (sp.fin == kFinScaled) return run<uint16_t, uint16_t, long long, int, kFinScaled>(s, d, a, st);
  }
  if (sp.sdepth == k16S && sp.ddepth == k16S && sp.fin == kFinScaled)
    return run<int16_t, int16_t, long long, int, kFinScaled>(s, d, a, st);
  if (sp.sdepth == k8U && sp.ddepth == k16S) {
    if (sp.fin == kFinCast) return run<uint8_t, int16_t, long long, int, kFinCast>(s, d, a, st);
    if (sp.fin == kFinScaled) return run<uint8_t, int16_t, long long, int, kFinScaled>(s, d, a, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace vb
