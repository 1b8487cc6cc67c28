// erode / dilate passes and the saturating subtract of morphologyEx
// (src/imgproc/morph.zig). Output (x, y) is the min (erode) or max (dilate)
// over the element's "on" cells of src(x + kx - ax, y + ky - ay); pixels
// outside the image are ignored (morph.zig:1-3), i.e. they hold the
// operation's identity. min/max are exact, so any evaluation order gives
// VISAR's result (morph.zig:489-519 is the per-tap definition).
//
// The element arrives as horizontal runs of on-cells (ky, x0, len). A CTA
// stages a tile plus halo in shared memory (identity outside the image) and
// reduces over the runs; a full rectangle is reduced separably (row pass,
// then column pass).
#include "vb.h"

namespace vb {

namespace {

constexpr int kTW = 128;  // samples per tile row
constexpr int kMaxRuns = 1024;

template <class T>
__device__ __forceinline__ T ident(bool is_max) {
  if constexpr (IsFloat<T>::v) return is_max ? -__int_as_float(0x7f800000) : __int_as_float(0x7f800000);
  else return is_max ? T(Lim<T>::lo) : T(Lim<T>::hi);
}

template <class T>
__device__ __forceinline__ T op2(T a, T b, bool is_max) {
  if constexpr (IsFloat<T>::v) return is_max ? fmaxf(a, b) : fminf(a, b);
  else return is_max ? (a > b ? a : b) : (a < b ? a : b);
}

struct MorphArgs {
  int kw, kh, ax, ay, nruns;
  bool is_max, rect;
};

template <class T>
__global__ void __launch_bounds__(256) k_morph_tiled(DImg s, DImg d, MorphArgs a, const MorphRun *runs, int th) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int cn = s.cn;
  const long long n = (long long)s.w * cn;
  const int hl = a.ax * cn;                  // left halo (samples)
  const int iw = kTW + (a.kw - 1) * cn;      // staged width (samples)
  const int ih = th + a.kh - 1;              // staged rows
  const long long x0s = (long long)blockIdx.x * kTW;
  const int y0 = blockIdx.y * th;
  const bool mx = a.is_max;
  const T id = ident<T>(mx);
  T *in = reinterpret_cast<T *>(smem);
  for (int idx = threadIdx.x; idx < ih * iw; idx += blockDim.x) {
    const int r = idx / iw, c = idx - r * iw;
    const long long gs = x0s - hl + c;
    const long long gy = (long long)y0 - a.ay + r;
    T v = id;
    if (gs >= 0 && gs < n && gy >= 0 && gy < s.h) v = row_ptr<const T>(s, gy)[gs];
    in[idx] = v;
  }
  __syncthreads();
  if (a.rect) {
    // Row pass into the second buffer, then the column pass.
    T *hrow = in + ((size_t)ih * iw);
    for (int idx = threadIdx.x; idx < ih * kTW; idx += blockDim.x) {
      const int r = idx / kTW, c = idx - r * kTW;
      const T *p = in + r * iw + c;
      T v = p[0];
      for (int k = 1; k < a.kw; k++) v = op2(v, p[k * cn], mx);
      hrow[idx] = v;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < th * kTW; idx += blockDim.x) {
      const int r = idx / kTW, c = idx - r * kTW;
      const int y = y0 + r;
      const long long xo = x0s + c;
      if (y >= s.h || xo >= n) continue;
      T v = hrow[r * kTW + c];
      for (int k = 1; k < a.kh; k++) v = op2(v, hrow[(r + k) * kTW + c], mx);
      row_ptr<T>(d, y)[xo] = v;
    }
    return;
  }
  for (int idx = threadIdx.x; idx < th * kTW; idx += blockDim.x) {
    const int r = idx / kTW, c = idx - r * kTW;
    const int y = y0 + r;
    const long long xo = x0s + c;
    if (y >= s.h || xo >= n) continue;
    T v = id;
    for (int q = 0; q < a.nruns; q++) {
      const MorphRun ru = runs[q];
      const T *p = in + (r + ru.ky) * iw + c + ru.x0 * cn;
      for (int k = 0; k < ru.len; k++) v = op2(v, p[k * cn], mx);
    }
    row_ptr<T>(d, y)[xo] = v;
  }
}

// Fallback for elements whose halo does not fit a shared-memory tile.
template <class T>
__global__ void __launch_bounds__(256) k_morph_direct(DImg s, DImg d, MorphArgs a, const MorphRun *runs) {
  const long long n = (long long)s.w * s.cn;
  const long long xo = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (xo >= n) return;
  const int cn = s.cn;
  const long long px = xo / cn;
  const int ch = (int)(xo - px * cn);
  const bool mx = a.is_max;
  T v = ident<T>(mx);
  for (int q = 0; q < a.nruns; q++) {
    const MorphRun ru = runs[q];
    const long long sy = (long long)y + ru.ky - a.ay;
    if (sy < 0 || sy >= s.h) continue;
    const T *r = row_ptr<const T>(s, sy);
    for (int k = 0; k < ru.len; k++) {
      const long long sx = px + ru.x0 + k - a.ax;
      if (sx < 0 || sx >= s.w) continue;
      v = op2(v, r[sx * cn + ch], mx);
    }
  }
  row_ptr<T>(d, y)[xo] = v;
}

// d = saturate(a - b) (morph.zig:573-593): floats subtract; integers give
// a -| b where a > b, else 0.
template <class T>
__global__ void __launch_bounds__(256) k_sub_sat(DImg a, DImg b, DImg d) {
  const long long n = (long long)d.w * d.cn;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (i >= n) return;
  const T x = row_ptr<const T>(a, y)[i], z = row_ptr<const T>(b, y)[i];
  T o;
  if constexpr (IsFloat<T>::v) o = __fsub_rn(x, z);
  else o = x > z ? satv_i<T>((long long)x - (long long)z) : T(0);
  row_ptr<T>(d, y)[i] = o;
}

template <class T>
cudaError_t run_pass(const DImg &s, const DImg &d, const MorphArgs &a, const MorphRun *runs, cudaStream_t st) {
  const long long n = (long long)s.w * s.cn;
  const long long iw = kTW + (long long)(a.kw - 1) * s.cn;
  for (int th : {32, 16, 8, 4, 2, 1}) {
    const long long ih = th + a.kh - 1;
    size_t need = (size_t)(ih * iw) * sizeof(T);
    if (a.rect) need += (size_t)ih * kTW * sizeof(T);
    if (need <= 160 * 1024) {
      auto kfn = k_morph_tiled<T>;
      cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
      if (e != cudaSuccess) return e;
      kfn<<<dim3(ceil_div(n, kTW), ceil_div(s.h, th)), 256, need, st>>>(s, d, a, runs, th);
      note_launch();
      return cudaGetLastError();
    }
  }
  k_morph_direct<T><<<dim3(ceil_div(n, 256), s.h), 256, 0, st>>>(s, d, a, runs);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_morph_pass(const DImg &s, const DImg &d, int depth, bool is_max, int kw, int kh, int ax, int ay,
                              const MorphRun *runs, int nruns, bool rect, cudaStream_t st) {
  if (s.w == 0 || s.h == 0) return cudaSuccess;
  MorphArgs a{kw, kh, ax, ay, nruns, is_max, rect};
  switch (depth) {
    case k8U: return run_pass<uint8_t>(s, d, a, runs, st);
    case k16U: return run_pass<uint16_t>(s, d, a, runs, st);
    case k16S: return run_pass<int16_t>(s, d, a, runs, st);
    case k32F: return run_pass<float>(s, d, a, runs, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_sub_sat(const DImg &a, const DImg &b, const DImg &d, int depth, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  dim3 g(ceil_div((long long)d.w * d.cn, 256), d.h);
  switch (depth) {
    case k8U: k_sub_sat<uint8_t><<<g, 256, 0, st>>>(a, b, d); break;
    case k16U: k_sub_sat<uint16_t><<<g, 256, 0, st>>>(a, b, d); break;
    case k16S: k_sub_sat<int16_t><<<g, 256, 0, st>>>(a, b, d); break;
    case k32F: k_sub_sat<float><<<g, 256, 0, st>>>(a, b, d); break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return cudaGetLastError();
}

}  // namespace vb
