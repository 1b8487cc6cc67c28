// threshold (src/imgproc/threshold.zig:25-261). u8 images always go through
// a 256-entry table built from the integer threshold, which is what VISAR's
// compare path and its out-of-range LUT (threshold.zig:39-60) both compute.
// Otsu and triangle run their f64 scans in one device thread, in VISAR's
// operation order, so the whole call stays on the stream.
#include "vb.h"

namespace vb {

namespace {

__global__ void __launch_bounds__(256) k_lut_u8(DImg s, DImg d, const uint8_t *lut) {
  __shared__ uint8_t t[256];
  t[threadIdx.x] = lut[threadIdx.x];
  __syncthreads();
  const long long n = (long long)s.w * s.cn;
  const int y = blockIdx.y;
  const uint8_t *sp = row_ptr<const uint8_t>(s, y);
  uint8_t *dp = row_ptr<uint8_t>(d, y);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dp[i] = t[sp[i]];
}

// 16 samples per thread with 16-byte accesses (rows 16-byte aligned).
__global__ void __launch_bounds__(256) k_lut_u8_v16(DImg s, DImg d, const uint8_t *lut, long long groups) {
  __shared__ uint8_t t[256];
  t[threadIdx.x] = lut[threadIdx.x];
  __syncthreads();
  const long long n = (long long)s.w * s.cn;
  const int y = blockIdx.y;
  const uint8_t *sp = row_ptr<const uint8_t>(s, y);
  uint8_t *dp = row_ptr<uint8_t>(d, y);
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups) return;
  const long long i0 = g * 16;
  if (i0 + 16 <= n) {
    uint4 v = *reinterpret_cast<const uint4 *>(sp + i0);
    uint8_t *b = reinterpret_cast<uint8_t *>(&v);
#pragma unroll
    for (int k = 0; k < 16; k++) b[k] = t[b[k]];
    *reinterpret_cast<uint4 *>(dp + i0) = v;
  } else {
    for (long long i = i0; i < n; i++) dp[i] = t[sp[i]];
  }
}

// threshOne (threshold.zig:84-100) on u16 / i16 / f32.
template <class T>
__global__ void __launch_bounds__(256) k_thresh_cmp(DImg s, DImg d, int type, T t, T m) {
  const long long n = (long long)s.w * s.cn;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (i >= n) return;
  const T v = row_ptr<const T>(s, y)[i];
  const bool gt = v > t;
  T o;
  switch (type) {
    case 0: o = gt ? m : T(0); break;
    case 1: o = gt ? T(0) : m; break;
    case 2: o = gt ? t : v; break;
    case 3: o = gt ? v : T(0); break;
    default: o = gt ? T(0) : v; break;
  }
  row_ptr<T>(d, y)[i] = o;
}

template <class T>
__global__ void __launch_bounds__(256) k_fill(DImg d, T v) {
  const long long n = (long long)d.w * d.cn;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) row_ptr<T>(d, blockIdx.y)[i] = v;
}

__global__ void __launch_bounds__(256) k_hist_u8(DImg s, uint32_t *hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long n = (long long)s.w;  // one channel
  for (int y = blockIdx.y; y < s.h; y += gridDim.y) {
    const uint8_t *sp = row_ptr<const uint8_t>(s, y);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      atomicAdd(&h[sp[i]], 1u);
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// getThreshVal_Otsu_8u (threshold.zig:190-215).
__device__ double otsu(const uint32_t *hist, double total) {
  const double scale = __ddiv_rn(1.0, total);
  double mu = 0;
  for (int i = 0; i < 256; i++) mu = __dadd_rn(mu, __dmul_rn((double)i, (double)hist[i]));
  mu = __dmul_rn(mu, scale);
  double mu1 = 0, q1 = 0, max_sigma = 0, max_val = 0;
  const double eps = 2.220446049250313e-16;
  for (int i = 0; i < 256; i++) {
    const double p_i = __dmul_rn((double)hist[i], scale);
    mu1 = __dmul_rn(mu1, q1);
    q1 = __dadd_rn(q1, p_i);
    const double q2 = __dsub_rn(1.0, q1);
    if (fmin(q1, q2) < eps || fmax(q1, q2) > __dsub_rn(1.0, eps)) continue;
    mu1 = __ddiv_rn(__dadd_rn(mu1, __dmul_rn((double)i, p_i)), q1);
    const double mu2 = __ddiv_rn(__dsub_rn(mu, __dmul_rn(q1, mu1)), q2);
    const double dm = __dsub_rn(mu1, mu2);
    const double sigma = __dmul_rn(__dmul_rn(__dmul_rn(q1, q2), dm), dm);
    if (sigma > max_sigma) {
      max_sigma = sigma;
      max_val = (double)i;
    }
  }
  return max_val;
}

// getThreshVal_Triangle_8u (threshold.zig:217-261).
__device__ double triangle(const uint32_t *hist) {
  int left = 0, right = 0, max_ind = 0;
  uint32_t mx = 0;
  for (int i = 0; i < 256; i++)
    if (hist[i] > 0) {
      left = i;
      break;
    }
  if (left > 0) left -= 1;
  for (int i = 255; i > 0; i--)
    if (hist[i] > 0) {
      right = i;
      break;
    }
  if (right < 255) right += 1;
  for (int j = 0; j < 256; j++)
    if (hist[j] > mx) {
      mx = hist[j];
      max_ind = j;
    }
  bool flip = false;
  if (max_ind - left < right - max_ind) {
    flip = true;
    left = 255 - right;
    max_ind = 255 - max_ind;
  }
  int thresh = left;
  const double a = (double)mx;
  const double b = (double)(left - max_ind);
  double dist = 0;
  for (int j = left + 1; j <= max_ind; j++) {
    const uint32_t hj = flip ? hist[255 - j] : hist[j];
    const double td = __dadd_rn(__dmul_rn(a, (double)j), __dmul_rn(b, (double)hj));
    if (td > dist) {
      dist = td;
      thresh = j;
    }
  }
  thresh -= 1;
  if (flip) thresh = 255 - thresh;
  return (double)thresh;
}

__device__ void build_lut(uint8_t *lut, int ti, int type, uint8_t m) {
  const uint8_t tsat = (uint8_t)min(max(ti, 0), 255);
  for (int i = 0; i < 256; i++) {
    const bool gt = i > ti;
    uint8_t v = (uint8_t)i, o;
    switch (type) {
      case 0: o = gt ? m : 0; break;
      case 1: o = gt ? 0 : m; break;
      case 2: o = gt ? tsat : v; break;
      case 3: o = gt ? v : 0; break;
      default: o = gt ? 0 : v; break;
    }
    lut[i] = o;
  }
}

__global__ void k_auto_thresh(const uint32_t *hist, double total, int method, int type, uint8_t m, double *thresh_out,
                              uint8_t *lut) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double t = method == 0 ? otsu(hist, total) : triangle(hist);
  *thresh_out = t;
  build_lut(lut, (int)floor(t), type, m);
}

template <class T>
cudaError_t run_cmp(const DImg &s, const DImg &d, int type, double t, double m, cudaStream_t st) {
  k_thresh_cmp<T><<<dim3(ceil_div((long long)s.w * s.cn, 256), s.h), 256, 0, st>>>(s, d, type, (T)t, (T)m);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_threshold_lut_u8(const DImg &s, const DImg &d, const uint8_t *lut, cudaStream_t st) {
  if (s.w == 0 || s.h == 0) return cudaSuccess;
  const long long n = (long long)s.w * s.cn;
  const bool aligned = ((uintptr_t)s.p % 16 == 0) && ((uintptr_t)d.p % 16 == 0) && (s.stride % 16 == 0) && (d.stride % 16 == 0);
  if (aligned) {
    const long long groups = (n + 15) / 16;
    k_lut_u8_v16<<<dim3(ceil_div(groups, 256), s.h), 256, 0, st>>>(s, d, lut, groups);
  } else {
    k_lut_u8<<<dim3(ceil_div(n, 256), s.h), 256, 0, st>>>(s, d, lut);
  }
  note_launch();
  return cudaGetLastError();
}

// t and m are already converted to the sample type by the caller.
cudaError_t launch_threshold_cmp(const DImg &s, const DImg &d, int depth, int type, double t, double m, cudaStream_t st) {
  if (s.w == 0 || s.h == 0) return cudaSuccess;
  switch (depth) {
    case k16U: return run_cmp<uint16_t>(s, d, type, t, m, st);
    case k16S: return run_cmp<int16_t>(s, d, type, t, m, st);
    case k32F: return run_cmp<float>(s, d, type, t, m, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_fill(const DImg &d, int depth, double v, cudaStream_t st) {
  if (d.w == 0 || d.h == 0) return cudaSuccess;
  dim3 g(ceil_div((long long)d.w * d.cn, 256), d.h);
  switch (depth) {
    case k8U: k_fill<uint8_t><<<g, 256, 0, st>>>(d, (uint8_t)v); break;
    case k16U: k_fill<uint16_t><<<g, 256, 0, st>>>(d, (uint16_t)v); break;
    case k16S: k_fill<int16_t><<<g, 256, 0, st>>>(d, (int16_t)v); break;
    case k32F: k_fill<float><<<g, 256, 0, st>>>(d, (float)v); break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_threshold_auto_u8(const DImg &s, int method, int type, double maxval, uint32_t *hist, double *thresh_dev,
                                     uint8_t *lut_dev, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(hist, 0, 256 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  const int gx = (int)ceil_div(s.w, 256);
  const int gy = s.h < 512 ? s.h : 512;
  k_hist_u8<<<dim3(gx < 4 ? gx : 4, gy), 256, 0, st>>>(s, hist);
  note_launch();
  // maxval -> u8 with sat.cast (round half to even, clamp, NaN -> 0).
  uint8_t m;
  if (maxval != maxval) m = 0;
  else {
    const double r = std::nearbyint(maxval);
    m = r <= 0 ? 0 : r >= 255 ? 255 : (uint8_t)(int)r;
  }
  k_auto_thresh<<<1, 32, 0, st>>>(hist, (double)s.w * (double)s.h, method, type, m, thresh_dev, lut_dev);
  note_launch();
  return cudaGetLastError();
}

}  // namespace vb
