// The tracker's per-frame tail (demos/track_lib.zig:533-553 in VISAR):
// equalizeHist (src/imgproc/hist.zig:20-45), the compare of
// adaptiveThreshold (src/imgproc/threshold.zig:307-360), the running-average
// background model (src/video/track.zig:17-82) and
// connectedComponentsWithStats (src/imgproc/components.zig).
#include <climits>

#include "vb.h"

namespace vb {
namespace {

constexpr int kHistThreads = 256;

// 256-bin histogram: per-block shared bins, then one atomic per bin.
__global__ void k_hist256(const uint8_t *__restrict__ s, long long stride, int w, int h, uint32_t *hist) {
  __shared__ uint32_t bins[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) bins[i] = 0;
  __syncthreads();
  for (int y = blockIdx.y; y < h; y += gridDim.y) {
    const uint8_t *r = s + (long long)y * stride;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < w; x += gridDim.x * blockDim.x) atomicAdd(&bins[r[x]], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (bins[i]) atomicAdd(&hist[i], bins[i]);
}

// equalizeHist's LUT (hist.zig:24-44), one block of 256 threads: the first
// occupied bin i maps to 0, bin k > i to sat.cast(f32(cumulative) * scale);
// an image of one value keeps it.
__global__ void k_equalize_lut(const uint32_t *__restrict__ hist, unsigned long long total, uint8_t *lut) {
  __shared__ uint32_t h[256];
  __shared__ int first;
  const int t = threadIdx.x;
  h[t] = hist[t];
  if (t == 0) first = 256;
  __syncthreads();
  if (h[t] != 0) atomicMin(&first, t);
  __syncthreads();
  const int i = first;
  if (t != 0 || i >= 256) return;
  if (h[i] == total) {
    for (int k = 0; k < 256; k++) lut[k] = (uint8_t)i;
    return;
  }
  const float scale = __fdiv_rn(255.0f, (float)(total - h[i]));
  for (int k = 0; k < 256; k++) lut[k] = 0;
  unsigned long long acc = 0;
  for (int k = i + 1; k < 256; k++) {
    acc += h[k];
    lut[k] = (uint8_t)fminf(fmaxf(rintf(__fmul_rn((float)acc, scale)), 0.0f), 255.0f);
  }
}

// adaptiveThreshold's compare (threshold.zig:346-359): imax where
// s + idelta > mean (binary) or s + idelta <= mean (binary_inv), else 0.
__global__ void k_adaptive_cmp(const uint8_t *__restrict__ s, long long ss, const uint8_t *__restrict__ m, long long ms,
                               uint8_t *__restrict__ d, long long ds, int w, int h, int idelta, int inv, uint8_t imax) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  for (int y = blockIdx.y; y < h; y += gridDim.y) {
    const int sv = s[(long long)y * ss + x], mv = m[(long long)y * ms + x];
    const bool gt = sv + idelta > mv;
    d[(long long)y * ds + x] = (gt != (inv != 0)) ? imax : 0;
  }
}

// f32 -> u8 with sat.cast (rint, clamp; NaN -> 0) and u8 -> f32.
__global__ void k_f32_to_u8(const uint8_t *__restrict__ s, long long ss, uint8_t *__restrict__ d, long long ds, int w, int h) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  for (int y = blockIdx.y; y < h; y += gridDim.y) {
    const float v = reinterpret_cast<const float *>(s + (long long)y * ss)[x];
    d[(long long)y * ds + x] = (uint8_t)(v != v ? 0.0f : fminf(fmaxf(rintf(v), 0.0f), 255.0f));
  }
}
__global__ void k_u8_to_f32(const uint8_t *__restrict__ s, long long ss, uint8_t *__restrict__ d, long long ds, int w, int h) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  for (int y = blockIdx.y; y < h; y += gridDim.y)
    reinterpret_cast<float *>(d + (long long)y * ds)[x] = (float)s[(long long)y * ss + x];
}

// Background.apply (track.zig:33-81). First frame: the model takes f << 8
// and the mask is cleared. Then per pixel: fg = |f - (b >> 8)| > t; the mask
// is 255 on fg; b += ((f << 8) - b) >> (shift + (fg ? 2 : 0)) (arithmetic
// shift of the signed difference).
__global__ void k_background(const uint8_t *__restrict__ f, long long fs, uint8_t *__restrict__ m, long long ms,
                             uint16_t *__restrict__ model, int w, int h, int t, int shift, int primed) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  for (int y = blockIdx.y; y < h; y += gridDim.y) {
    const int fv = f[(long long)y * fs + x];
    uint16_t &b = model[(long long)y * w + x];
    if (!primed) {
      b = (uint16_t)(fv << 8);
      m[(long long)y * ms + x] = 0;
      continue;
    }
    const int bv = b;
    const bool fg = abs(fv - (bv >> 8)) > t;
    m[(long long)y * ms + x] = fg ? 255 : 0;
    b = (uint16_t)(bv + (((fv << 8) - bv) >> (shift + (fg ? 2 : 0))));
  }
}

}  // namespace

cudaError_t launch_equalize_hist(const DImg &s, const DImg &d, uint32_t *hist_dev, uint8_t *lut_dev, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(hist_dev, 0, 256 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  dim3 grid((s.w + kHistThreads * 4 - 1) / (kHistThreads * 4), std::min(s.h, 148 * 4));
  note_launch(2);
  k_hist256<<<grid, kHistThreads, 0, st>>>(s.p, s.stride, s.w, s.h, hist_dev);
  k_equalize_lut<<<1, 256, 0, st>>>(hist_dev, (unsigned long long)s.w * s.h, lut_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return launch_threshold_lut_u8(s, d, lut_dev, st);
}

cudaError_t launch_adaptive_cmp(const DImg &s, const DImg &m, const DImg &d, int idelta, bool inv, uint8_t imax,
                                cudaStream_t st) {
  dim3 grid((s.w + 255) / 256, std::min(s.h, 65535));
  note_launch();
  k_adaptive_cmp<<<grid, 256, 0, st>>>(s.p, s.stride, m.p, m.stride, d.p, d.stride, s.w, s.h, idelta, inv ? 1 : 0, imax);
  return cudaGetLastError();
}

cudaError_t launch_convert_u8_f32(const DImg &s, const DImg &d, bool to_f32, cudaStream_t st) {
  dim3 grid((s.w + 255) / 256, std::min(s.h, 65535));
  note_launch();
  if (to_f32) k_u8_to_f32<<<grid, 256, 0, st>>>(s.p, s.stride, d.p, d.stride, s.w, s.h);
  else k_f32_to_u8<<<grid, 256, 0, st>>>(s.p, s.stride, d.p, d.stride, s.w, s.h);
  return cudaGetLastError();
}

cudaError_t launch_background(const DImg &f, const DImg &m, uint16_t *model, int t, int shift, bool primed, cudaStream_t st) {
  dim3 grid((f.w + 255) / 256, std::min(f.h, 65535));
  note_launch();
  k_background<<<grid, 256, 0, st>>>(f.p, f.stride, m.p, m.stride, model, f.w, f.h, t, shift, primed ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace vb

// ----------------------------------------------------- connected components
//
// Labels follow OpenCV (components.zig:1-10): 4-connected components are
// numbered in raster order of their first pixel, 8-connected ones in
// block-raster order of their first 2x2 block. Union-find over pixel indices
// links the larger root under the smaller with atomicMin, so every root ends
// as its component's first pixel in raster order (Playne and Hawick's
// union-find); an 8-connected component's key is the smallest block index
// (y/2) * ceil(w/2) + x/2 of its pixels (only its first block row can hold
// it). A component's label is 1 + the number of keys below its own: an
// exclusive prefix sum over a flag per key. Statistics are exact integer
// sums (twice the x sum, as VISAR keeps them) gathered run by run.

namespace vb {
namespace {

constexpr int kUfLimit = 1 << 24;  // unions retry at most this often (never reached: each retry lowers a root)

__device__ __forceinline__ int uf_find(const int *P, int p) {
  int q = __ldcg(P + p);
  while (q != p) {
    p = q;
    q = __ldcg(P + p);
  }
  return p;
}

__device__ __forceinline__ void uf_unite(int *P, int a, int b, int *err) {
  for (int it = 0; it < kUfLimit; it++) {
    a = uf_find(P, a);
    b = uf_find(P, b);
    if (a == b) return;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(P + a, b);  // a > b: link a under b
    if (old == a) return;
    a = old;  // a had been linked meanwhile: join its new parent instead
  }
  atomicExch(err, 1);
}

__global__ void k_cc_init(const uint8_t *__restrict__ s, long long ss, int *P, int w, int h) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  for (int y = blockIdx.y; y < h; y += gridDim.y) {
    const int p = y * w + x;
    P[p] = s[(long long)y * ss + x] ? p : -1;
  }
}

__global__ void k_cc_union(const uint8_t *__restrict__ s, long long ss, int *P, int w, int h, int eight, int *err) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  for (int y = blockIdx.y; y < h; y += gridDim.y) {
    const uint8_t *r = s + (long long)y * ss;
    if (!r[x]) continue;
    const int p = y * w + x;
    if (x > 0 && r[x - 1]) uf_unite(P, p, p - 1, err);
    if (y > 0) {
      const uint8_t *u = r - ss;
      if (u[x]) uf_unite(P, p, p - w, err);
      if (eight) {
        if (x > 0 && u[x - 1]) uf_unite(P, p, p - w - 1, err);
        if (x + 1 < w && u[x + 1]) uf_unite(P, p, p - w + 1, err);
      }
    }
  }
}

// Every pixel to its root; roots start their key at INT_MAX (8-connected).
__global__ void k_cc_flatten(int *P, int *K, int n, int eight) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    if (P[p] < 0) continue;
    const int r = uf_find(P, p);
    P[p] = r;
    if (eight && r == p) K[p] = INT_MAX;
  }
}

__global__ void k_cc_keys(const int *__restrict__ P, int *K, int w, int h) {
  const int wb = (w + 1) / 2;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < w * h; p += gridDim.x * blockDim.x) {
    const int r = P[p];
    if (r < 0) continue;
    const int y = p / w, ry = r / w;
    if ((y >> 1) != (ry >> 1)) continue;
    atomicMin(K + r, (y >> 1) * wb + ((p - y * w) >> 1));
  }
}

__global__ void k_cc_flags(const int *__restrict__ P, const int *__restrict__ K, uint32_t *F, int n, int eight) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    if (P[p] == p) F[eight ? K[p] : p] = 1;
}

// Exclusive scan of n u32 in blocks of kScanItems: per-block scans with the
// block totals in part[], which the next level scans.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanItems = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads) k_scan_block(const uint32_t *__restrict__ in, uint32_t *out, long long n,
                                                              uint32_t *part) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  const long long base = (long long)blockIdx.x * kScanItems + (long long)threadIdx.x * kScanPer;
  uint32_t v[kScanPer], sum = 0;
#pragma unroll
  for (int i = 0; i < kScanPer; i++) {
    v[i] = base + i < n ? in[base + i] : 0u;
    sum += v[i];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, t, o);
      if (lane >= o) t += u;
    }
    warp_tot[lane] = t;  // inclusive warp totals
  }
  __syncthreads();
  uint32_t run = inc - sum + (wid > 0 ? warp_tot[wid - 1] : 0u);
#pragma unroll
  for (int i = 0; i < kScanPer; i++) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
  if (threadIdx.x == kScanThreads - 1) part[blockIdx.x] = run;
}

__global__ void k_scan_add(uint32_t *out, long long n, const uint32_t *__restrict__ part) {
  const long long i = (long long)blockIdx.x * kScanItems + threadIdx.x;
  const uint32_t a = part[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanPer; k++)
    if (i + (long long)k * kScanThreads < n) out[i + (long long)k * kScanThreads] += a;
}

__global__ void k_cc_total(const uint32_t *F, const uint32_t *R, long long n, uint32_t *total) { *total = R[n - 1] + F[n - 1]; }

__global__ void k_cc_labels(const int *__restrict__ P, const int *__restrict__ K, const uint32_t *__restrict__ R,
                            uint8_t *lab, long long ls, int w, int h, int eight) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  for (int y = blockIdx.y; y < h; y += gridDim.y) {
    const int r = P[y * w + x];
    reinterpret_cast<int *>(lab + (long long)y * ls)[x] = r < 0 ? 0 : 1 + (int)R[eight ? K[r] : r];
  }
}

struct CcAcc {
  long long x0, y0, x1, y1;
  unsigned long long area, sx2, sy, pad;
};

__global__ void k_cc_stats_init(CcAcc *a, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    a[i] = CcAcc{LLONG_MAX, LLONG_MAX, 0, 0, 0, 0, 0, 0};
}

__device__ __forceinline__ void cc_flush(CcAcc *a, int l, long long xs, long long xe, long long ys, long long ye,
                                         unsigned long long area, unsigned long long sx2, unsigned long long sy) {
  atomicMin(&a[l].x0, xs);
  atomicMax(&a[l].x1, xe);
  atomicMin(&a[l].y0, ys);
  atomicMax(&a[l].y1, ye);
  atomicAdd(&a[l].area, area);
  atomicAdd(&a[l].sx2, sx2);
  atomicAdd(&a[l].sy, sy);
}

constexpr int kCcSeg = 64;  // pixels of a row per thread in the statistics pass

// Foreground runs flush per run; the background is summed over the thread's
// segments and then over the block before one flush.
__global__ void __launch_bounds__(256) k_cc_stats(const uint8_t *__restrict__ lab, long long ls, int w, int h, CcAcc *a) {
  const int nseg = (w + kCcSeg - 1) / kCcSeg;
  const long long total = (long long)nseg * h;
  long long bx0 = LLONG_MAX, by0 = LLONG_MAX, bx1 = -1, by1 = -1;
  unsigned long long barea = 0, bsx2 = 0, bsy = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(t / nseg);
    const int x0 = (int)(t - (long long)y * nseg) * kCcSeg;
    const int x1 = min(w, x0 + kCcSeg);
    const int *row = reinterpret_cast<const int *>(lab + (long long)y * ls);
    int x = x0;
    while (x < x1) {
      const int l = row[x];
      int e = x + 1;
      while (e < x1 && row[e] == l) e++;
      const unsigned long long len = (unsigned long long)(e - x);
      const unsigned long long s2 = len * (unsigned long long)(x + e - 1);
      if (l == 0) {
        bx0 = min(bx0, (long long)x);
        bx1 = max(bx1, (long long)(e - 1));
        by0 = min(by0, (long long)y);
        by1 = max(by1, (long long)y);
        barea += len;
        bsx2 += s2;
        bsy += len * (unsigned long long)y;
      } else {
        cc_flush(a, l, x, e - 1, y, y, len, s2, len * (unsigned long long)y);
      }
      x = e;
    }
  }
  // Background over the block (256 threads, 8 warps).
  __shared__ long long s_min[2][8], s_max[2][8];
  __shared__ unsigned long long s_sum[3][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    bx0 = min(bx0, __shfl_xor_sync(0xFFFFFFFFu, bx0, o));
    by0 = min(by0, __shfl_xor_sync(0xFFFFFFFFu, by0, o));
    bx1 = max(bx1, __shfl_xor_sync(0xFFFFFFFFu, bx1, o));
    by1 = max(by1, __shfl_xor_sync(0xFFFFFFFFu, by1, o));
    barea += __shfl_xor_sync(0xFFFFFFFFu, barea, o);
    bsx2 += __shfl_xor_sync(0xFFFFFFFFu, bsx2, o);
    bsy += __shfl_xor_sync(0xFFFFFFFFu, bsy, o);
  }
  if (lane == 0) {
    s_min[0][wid] = bx0;
    s_min[1][wid] = by0;
    s_max[0][wid] = bx1;
    s_max[1][wid] = by1;
    s_sum[0][wid] = barea;
    s_sum[1][wid] = bsx2;
    s_sum[2][wid] = bsy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) {
      bx0 = min(bx0, s_min[0][i]);
      by0 = min(by0, s_min[1][i]);
      bx1 = max(bx1, s_max[0][i]);
      by1 = max(by1, s_max[1][i]);
      barea += s_sum[0][i];
      bsx2 += s_sum[1][i];
      bsy += s_sum[2][i];
    }
    if (barea) cc_flush(a, 0, bx0, bx1, by0, by1, barea, bsx2, bsy);
  }
}

cudaError_t scan_u32(const uint32_t *in, uint32_t *out, long long n, uint32_t *tmp, cudaStream_t st) {
  const long long nb = (n + kScanItems - 1) / kScanItems;
  note_launch();
  k_scan_block<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, tmp);
  if (nb > 1) {
    const cudaError_t e = scan_u32(tmp, tmp + nb, nb, tmp + 2 * nb, st);
    if (e != cudaSuccess) return e;
    note_launch();
    k_scan_add<<<(unsigned)nb, kScanThreads, 0, st>>>(out, n, tmp + nb);
  }
  return cudaGetLastError();
}

}  // namespace

size_t cc_scan_tmp_words(long long n) {
  long long nb = (n + kScanItems - 1) / kScanItems, words = 64;
  while (true) {
    words += 2 * nb;
    if (nb <= 1) break;
    nb = (nb + kScanItems - 1) / kScanItems;
  }
  return (size_t)words;
}

size_t cc_acc_bytes() { return sizeof(CcAcc); }

cudaError_t launch_cc_phase1(const DImg &s, bool eight, const CcBuffers &b, cudaStream_t st) {
  const int w = s.w, h = s.h, n = w * h;
  const long long nkeys = eight ? (long long)((w + 1) / 2) * ((h + 1) / 2) : (long long)n;
  dim3 g2((w + 255) / 256, std::min(h, 65535));
  const int g1 = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  cudaError_t e;
  if ((e = cudaMemsetAsync(b.err, 0, sizeof(int), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(b.F, 0, (size_t)nkeys * sizeof(uint32_t), st)) != cudaSuccess) return e;
  note_launch(eight ? 5 : 4);
  k_cc_init<<<g2, 256, 0, st>>>(s.p, s.stride, b.P, w, h);
  k_cc_union<<<g2, 256, 0, st>>>(s.p, s.stride, b.P, w, h, eight ? 1 : 0, b.err);
  k_cc_flatten<<<g1, 256, 0, st>>>(b.P, b.K, n, eight ? 1 : 0);
  if (eight) k_cc_keys<<<g1, 256, 0, st>>>(b.P, b.K, w, h);
  k_cc_flags<<<g1, 256, 0, st>>>(b.P, b.K, b.F, n, eight ? 1 : 0);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan_u32(b.F, b.R, nkeys, b.tmp, st)) != cudaSuccess) return e;
  note_launch();
  k_cc_total<<<1, 1, 0, st>>>(b.F, b.R, nkeys, b.total);
  return cudaGetLastError();
}

cudaError_t launch_cc_phase2(const DImg &labels, bool eight, const CcBuffers &b, void *acc, int nlabels, cudaStream_t st) {
  const int w = labels.w, h = labels.h;
  dim3 g2((w + 255) / 256, std::min(h, 65535));
  CcAcc *a = static_cast<CcAcc *>(acc);
  note_launch(3);
  k_cc_labels<<<g2, 256, 0, st>>>(b.P, b.K, b.R, labels.p, labels.stride, w, h, eight ? 1 : 0);
  k_cc_stats_init<<<std::max(1, std::min((nlabels + 255) / 256, 148 * 8)), 256, 0, st>>>(a, nlabels);
  const long long segs = (long long)((w + kCcSeg - 1) / kCcSeg) * h;
  k_cc_stats<<<(int)std::max<long long>(1, std::min<long long>((segs + 255) / 256, 148LL * 16)), 256, 0, st>>>(
      labels.p, labels.stride, w, h, a);
  return cudaGetLastError();
}

void cc_read_acc(const void *host_acc, int i, long long out[7]) {
  const CcAcc &a = static_cast<const CcAcc *>(host_acc)[i];
  out[0] = a.x0;
  out[1] = a.y0;
  out[2] = a.x1;
  out[3] = a.y1;
  out[4] = (long long)a.area;
  out[5] = (long long)a.sx2;
  out[6] = (long long)a.sy;
}

}  // namespace vb
