// Lens undistortion and remapping (src/calib3d/undistort.zig): undistort
// (:204-281), initUndistortRectifyMap (:84-110) and remap (:288-327) of u8
// images with 1-4 channels.
//
// Map (MapParams.row, :44-81), per destination pixel (j, i), in f64, every
// operation rounded on its own:
//   x = (i*ir1 + ir2) + j*ir0,  y = (i*ir4 + ir5) + j*ir3
//   unless (ir6, ir7, ir8) = (0, 0, 1): w = 1 / ((i*ir7 + ir8) + j*ir6), x *= w, y *= w
//   r2 = x*x + y*y, 2xy = (2*x)*y
//   kr = 1 + ((k4*r2 + k1)*r2 + k0)*r2   [/ (1 + ((k7*r2 + k6)*r2 + k5)*r2) if k5..k7 != 0]
//   xd = (x*kr + k2*2xy) + k3*(r2 + 2*x*x),  yd = (y*kr + k2*(r2 + 2*y*y)) + k3*2xy
//   u = fx*xd + u0,  v = fy*yd + v0
// undistort (OpenCV's stripes of 4096 / width rows: the new camera's
// principal point moves up by the stripe's first row, and i counts rows from
// there) rounds u, v to 1/32 pixel half to even and blends with 15-bit
// integer weights ((s + 512) >> 10, constant 0 border, :136-172);
// initUndistortRectifyMap stores f32(u), f32(v); remap takes f32 map
// coordinates and blends with the fma chain of warpAffine (constant border
// `value`, :366-392).
#include <cmath>

#include "vb.h"

namespace vb {
namespace {

struct UndistParams {
  double ir[9];
  double fx, fy, u0, v0;
  double k[8];
  bool persp;   // the projective row of ir is not (0, 0, 1)
  bool ratio;   // k5..k7 used
  bool skip;    // singular camera matrix: VISAR leaves these rows as they are
};

__device__ __forceinline__ void map_px(const UndistParams &p, double i, double j, double &u, double &v) {
  const double *ir = p.ir;
  double x = __dadd_rn(__dadd_rn(__dmul_rn(i, ir[1]), ir[2]), __dmul_rn(j, ir[0]));
  double y = __dadd_rn(__dadd_rn(__dmul_rn(i, ir[4]), ir[5]), __dmul_rn(j, ir[3]));
  if (p.persp) {
    const double w0 = __dadd_rn(__dadd_rn(__dmul_rn(i, ir[7]), ir[8]), __dmul_rn(j, ir[6]));
    const double w = __ddiv_rn(1.0, w0);
    x = __dmul_rn(x, w);
    y = __dmul_rn(y, w);
  }
  const double *k = p.k;
  const double x2 = __dmul_rn(x, x), y2 = __dmul_rn(y, y);
  const double r2 = __dadd_rn(x2, y2);
  const double xy2 = __dmul_rn(__dmul_rn(2.0, x), y);
  double kr = __dadd_rn(1.0, __dmul_rn(__dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(k[4], r2), k[1]), r2), k[0]), r2));
  if (p.ratio)
    kr = __ddiv_rn(kr, __dadd_rn(1.0, __dmul_rn(__dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(k[7], r2), k[6]), r2), k[5]), r2)));
  const double xd = __dadd_rn(__dadd_rn(__dmul_rn(x, kr), __dmul_rn(k[2], xy2)),
                              __dmul_rn(k[3], __dadd_rn(r2, __dmul_rn(2.0, x2))));
  const double yd = __dadd_rn(__dadd_rn(__dmul_rn(y, kr), __dmul_rn(k[2], __dadd_rn(r2, __dmul_rn(2.0, y2)))),
                              __dmul_rn(k[3], xy2));
  u = __dadd_rn(__dmul_rn(p.fx, xd), p.u0);
  v = __dadd_rn(__dmul_rn(p.fy, yd), p.v0);
}

// OpenCV's saturate_cast<int>(v * 32): clamped, rounded half to even. The
// rounding is an add of 1.5 * 2^52 (exact for |s| < 2^51, the sum's low word
// then holds the integer): the same value as __double2int_rn without the
// conversion unit.
__device__ __forceinline__ int fix32(double v) {
  const double s = fmin(fmax(__dmul_rn(v, 32.0), -2147483647.0), 2147483647.0);
  return (int)__double2loint(__dadd_rn(s, 6755399441055744.0));
}

// The camera of an undistort stripe: the inverse of the new camera matrix
// with its principal point moved up by the stripe's first row, as
// linalg.inv3 computes it (src/calib3d/linalg.zig:417-426; the host restatement
// inv3 below evaluates the same expressions in the same order, each product
// and sum rounded on its own, 1 / det correctly rounded).
struct UndistBase {
  double ar[9];  // the new camera matrix (new_k, else K)
  double fx, fy, u0, v0;
  double k[8];
  bool ratio;
};

__device__ __forceinline__ double dif2(double a, double b, double c, double d) {
  return __dsub_rn(__dmul_rn(a, b), __dmul_rn(c, d));  // a*b - c*d
}

__device__ void stripe_params(const UndistBase &b, int first_row, UndistParams &p) {
  double a[9];
#pragma unroll
  for (int i = 0; i < 9; i++) a[i] = b.ar[i];
  a[5] = __dsub_rn(b.ar[5], (double)first_row);
  const double det = __dadd_rn(__dsub_rn(__dmul_rn(a[0], dif2(a[4], a[8], a[7], a[5])), __dmul_rn(a[1], dif2(a[3], a[8], a[6], a[5]))),
                               __dmul_rn(a[2], dif2(a[3], a[7], a[6], a[4])));
  p.fx = b.fx;
  p.fy = b.fy;
  p.u0 = b.u0;
  p.v0 = b.v0;
#pragma unroll
  for (int i = 0; i < 8; i++) p.k[i] = b.k[i];
  p.ratio = b.ratio;
  p.skip = det == 0;
  if (p.skip) {
    p.persp = false;
    return;
  }
  const double d = __drcp_rn(det);
  p.ir[0] = __dmul_rn(dif2(a[4], a[8], a[5], a[7]), d);
  p.ir[1] = __dmul_rn(dif2(a[2], a[7], a[1], a[8]), d);
  p.ir[2] = __dmul_rn(dif2(a[1], a[5], a[2], a[4]), d);
  p.ir[3] = __dmul_rn(dif2(a[5], a[6], a[3], a[8]), d);
  p.ir[4] = __dmul_rn(dif2(a[0], a[8], a[2], a[6]), d);
  p.ir[5] = __dmul_rn(dif2(a[2], a[3], a[0], a[5]), d);
  p.ir[6] = __dmul_rn(dif2(a[3], a[7], a[4], a[6]), d);
  p.ir[7] = __dmul_rn(dif2(a[1], a[6], a[0], a[7]), d);
  p.ir[8] = __dmul_rn(dif2(a[0], a[4], a[1], a[3]), d);
  p.persp = !(p.ir[6] == 0 && p.ir[7] == 0 && p.ir[8] == 1);
}

// The CN bytes of pixel x and of pixel x + 1 of row r. 3- and 4-channel
// rows with 8-byte aligned starts (`wide`) take two aligned 8-byte loads
// when the 16-byte window stays inside the row, and pick the bytes by
// permutes; otherwise bytewise.
template <int CN>
__device__ __forceinline__ void tap_pair(const uint8_t *r, int x, int row_bytes, bool wide, int (&p)[CN], int (&q)[CN]) {
  if constexpr (CN == 3 || CN == 4) {
    const int b = x * CN, a8 = b & ~7;
    if (wide && a8 + 16 <= row_bytes) {
      const uint2 lo = __ldg(reinterpret_cast<const uint2 *>(r + a8));
      const uint2 hi = __ldg(reinterpret_cast<const uint2 *>(r + a8 + 8));
      const int off = b - a8;  // 0..7
      const uint32_t wa = off >= 4 ? lo.y : lo.x, wb = off >= 4 ? hi.x : lo.y, wc = off >= 4 ? hi.y : hi.x;
      const unsigned sel = 0x3210u + 0x1111u * (unsigned)(off & 3);
      const uint32_t b0 = __byte_perm(wa, wb, sel), b1 = __byte_perm(wb, wc, sel);  // bytes off .. off + 7
#pragma unroll
      for (int c = 0; c < CN; c++) {
        p[c] = (int)((b0 >> (8 * c)) & 0xFFu);
        const int k = c + CN;
        q[c] = (int)(((k < 4 ? b0 : b1) >> (8 * (k & 3))) & 0xFFu);
      }
      return;
    }
  }
#pragma unroll
  for (int c = 0; c < CN; c++) {
    p[c] = r[x * CN + c];
    q[c] = r[x * CN + CN + c];
  }
}

template <int CN>
__device__ __forceinline__ void sample_fixed(const uint8_t *__restrict__ src, long long stride, int W, int H, int iu, int iv,
                                             uint8_t *o, bool wide = false) {
  const int sx = iu >> 5, sy = iv >> 5;
  const int a = iu & 31, b = iv & 31;
  const int w0 = (32 - a) * (32 - b), w1 = a * (32 - b), w2 = (32 - a) * b, w3 = a * b;
  if (sx >= 0 && sx < W - 1 && sy >= 0 && sy < H - 1) {
    const uint8_t *r0 = src + (long long)sy * stride;
    int p0[CN], q0[CN], p1[CN], q1[CN];
    tap_pair<CN>(r0, sx, W * CN, wide, p0, q0);
    tap_pair<CN>(r0 + stride, sx, W * CN, wide, p1, q1);
#pragma unroll
    for (int c = 0; c < CN; c++) o[c] = (uint8_t)((p0[c] * w0 + q0[c] * w1 + p1[c] * w2 + q1[c] * w3 + 512) >> 10);
    return;
  }
  if (sx >= W || sx + 1 < 0 || sy >= H || sy + 1 < 0) {
#pragma unroll
    for (int c = 0; c < CN; c++) o[c] = 0;
    return;
  }
  const int wq[4] = {w0, w1, w2, w3};
#pragma unroll
  for (int c = 0; c < CN; c++) {
    int s = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int px = sx + (q & 1), py = sy + (q >> 1);
      const int v = (px >= 0 && px < W && py >= 0 && py < H) ? src[(long long)py * stride + (long long)px * CN + c] : 0;
      s += v * wq[q];
    }
    o[c] = (uint8_t)((s + 512) >> 10);
  }
}

// undistort: four consecutive destination pixels per thread (their map
// arithmetic and taps interleave); a block of 32 x 8 threads covers 8 rows,
// whose stripes' cameras (at most 8) its first threads compute into shared
// memory.
constexpr int kUndRows = 8;

template <int CN>
__global__ void __launch_bounds__(256) k_undistort(const uint8_t *__restrict__ src, long long sstride, uint8_t *__restrict__ dst,
                                                   long long dstride, int W, int H, int stripe, UndistBase base, int wide) {
  __shared__ UndistParams sp[kUndRows];
  const int y0 = blockIdx.y * kUndRows;
  const int s0 = y0 / stripe, s1 = min(y0 + kUndRows - 1, H - 1) / stripe;
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  if (t <= s1 - s0) stripe_params(base, (s0 + t) * stripe, sp[t]);
  __syncthreads();
  const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  const int y = y0 + threadIdx.y;
  if (x0 >= W || y >= H) return;
  const int s = y / stripe;
  const UndistParams &p = sp[s - s0];
  if (p.skip) return;
  const double i = (double)(y - s * stripe);
  uint8_t *o = dst + (long long)y * dstride + (long long)x0 * CN;
  int iu[4], iv[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    double u, v;
    map_px(p, i, (double)(x0 + q), u, v);
    iu[q] = fix32(u);
    iv[q] = fix32(v);
  }
  uint8_t px[4][CN];
#pragma unroll
  for (int q = 0; q < 4; q++) sample_fixed<CN>(src, sstride, W, H, iu[q], iv[q], px[q], wide != 0);
#pragma unroll
  for (int q = 0; q < 4; q++)
    if (x0 + q < W) {
#pragma unroll
      for (int c = 0; c < CN; c++) o[q * CN + c] = px[q][c];
    }
}

__global__ void k_init_map(float *__restrict__ mx, long long mxs, float *__restrict__ my, long long mys, int W, int H,
                           UndistParams p) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  double u, v;
  map_px(p, (double)y, (double)x, u, v);
  reinterpret_cast<float *>(reinterpret_cast<uint8_t *>(mx) + (long long)y * mxs)[x] = __double2float_rn(u);
  reinterpret_cast<float *>(reinterpret_cast<uint8_t *>(my) + (long long)y * mys)[x] = __double2float_rn(v);
}

// remap: linearF32 (:366-392).
template <int CN>
__global__ void k_remap(const uint8_t *__restrict__ src, long long sstride, int sw, int sh, uint8_t *__restrict__ dst,
                        long long dstride, int dw, int dh, const uint8_t *__restrict__ mxp, long long mxs,
                        const uint8_t *__restrict__ myp, long long mys, uint8_t bv) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  const float sx = reinterpret_cast<const float *>(mxp + (long long)y * mxs)[x];
  const float sy = reinterpret_cast<const float *>(myp + (long long)y * mys)[x];
  uint8_t *o = dst + (long long)y * dstride + (long long)x * CN;
  const float fx = floorf(sx), fy = floorf(sy);
  if (!(fx >= -1.0f && fy >= -1.0f && fx < (float)sw && fy < (float)sh)) {
#pragma unroll
    for (int c = 0; c < CN; c++) o[c] = bv;
    return;
  }
  const float ax = __fsub_rn(sx, fx), ay = __fsub_rn(sy, fy);
  const int ix = (int)fx, iy = (int)fy;
#pragma unroll
  for (int c = 0; c < CN; c++) {
    float p[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int px = ix + (q & 1), py = iy + (q >> 1);
      p[q] = (px >= 0 && px < sw && py >= 0 && py < sh) ? (float)src[(long long)py * sstride + (long long)px * CN + c]
                                                         : (float)bv;
    }
    const float v0 = __fmaf_rn(ax, __fsub_rn(p[1], p[0]), p[0]);
    const float v1 = __fmaf_rn(ax, __fsub_rn(p[3], p[2]), p[2]);
    const float v = __fmaf_rn(ay, __fsub_rn(v1, v0), v0);
    o[c] = (uint8_t)fminf(fmaxf(rintf(v), 0.0f), 255.0f);
  }
}

}  // namespace

// ------------------------------------------------------------------ host side

namespace {

bool inv3(const double a[9], double out[9]) {
  // linalg.inv3 (src/calib3d/linalg.zig:417-426).
  const double det = a[0] * (a[4] * a[8] - a[7] * a[5]) - a[1] * (a[3] * a[8] - a[6] * a[5]) + a[2] * (a[3] * a[7] - a[6] * a[4]);
  if (det == 0) return false;
  const double d = 1 / det;
  const double r[9] = {(a[4] * a[8] - a[5] * a[7]) * d, (a[2] * a[7] - a[1] * a[8]) * d, (a[1] * a[5] - a[2] * a[4]) * d,
                       (a[5] * a[6] - a[3] * a[8]) * d, (a[0] * a[8] - a[2] * a[6]) * d, (a[2] * a[3] - a[0] * a[5]) * d,
                       (a[3] * a[7] - a[4] * a[6]) * d, (a[1] * a[6] - a[0] * a[7]) * d, (a[0] * a[4] - a[1] * a[3]) * d};
  for (int i = 0; i < 9; i++) out[i] = r[i];
  return true;
}

void mul3(const double a[9], const double b[9], double r[9]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
}

void fill_params(UndistParams &p, const double ir[9], const double K[9], const double k[8]) {
  for (int i = 0; i < 9; i++) p.ir[i] = ir[i];
  p.fx = K[0];
  p.fy = K[4];
  p.u0 = K[2];
  p.v0 = K[5];
  for (int i = 0; i < 8; i++) p.k[i] = k[i];
  p.persp = !(ir[6] == 0 && ir[7] == 0 && ir[8] == 1);
  p.ratio = k[5] != 0 || k[6] != 0 || k[7] != 0;
  p.skip = false;
}

}  // namespace

int undistort_stripe_rows(int width, int height) {
  const int s = std::max(1, 4096 / std::max(width, 1));
  return std::min(s, height);
}

bool undistort_any_singular(const double *new_k, const double K[9], int width, int height) {
  // The stripes' cameras (inverted on the device): singular when det = 0,
  // which, as det is linear in the principal point, is at most one stripe
  // (or every stripe).
  const int stripe = undistort_stripe_rows(width, height);
  const int n = (height + stripe - 1) / stripe;
  const double *ar0 = new_k ? new_k : K;
  for (int s = 0; s < n; s++) {
    double a[9];
    for (int i = 0; i < 9; i++) a[i] = ar0[i];
    a[5] = ar0[5] - (double)(s * stripe);
    const double det =
        a[0] * (a[4] * a[8] - a[7] * a[5]) - a[1] * (a[3] * a[8] - a[6] * a[5]) + a[2] * (a[3] * a[7] - a[6] * a[4]);
    if (det == 0) return true;
  }
  return false;
}

bool undistort_map_params(const double K[9], const double k8[8], const double *R, const double *new_k, std::vector<uint8_t> &out) {
  const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double m[9], ir[9];
  mul3(new_k ? new_k : K, R ? R : eye, m);
  if (!inv3(m, ir)) return false;
  out.assign(sizeof(UndistParams), 0);
  fill_params(*reinterpret_cast<UndistParams *>(out.data()), ir, K, k8);
  return true;
}

cudaError_t launch_undistort(const DImg &s, const DImg &d, const double K[9], const double k8[8], const double *new_k,
                             cudaStream_t st) {
  const int stripe = undistort_stripe_rows(s.w, s.h);
  UndistBase b{};
  const double *ar0 = new_k ? new_k : K;
  for (int i = 0; i < 9; i++) b.ar[i] = ar0[i];
  b.fx = K[0];
  b.fy = K[4];
  b.u0 = K[2];
  b.v0 = K[5];
  for (int i = 0; i < 8; i++) b.k[i] = k8[i];
  b.ratio = k8[5] != 0 || k8[6] != 0 || k8[7] != 0;
  const int wide = ((uintptr_t)s.p % 8 == 0) && (s.stride % 8 == 0);
  dim3 block(32, kUndRows), grid((d.w + 127) / 128, (d.h + kUndRows - 1) / kUndRows);
  note_launch();
  switch (s.cn) {
    case 1: k_undistort<1><<<grid, block, 0, st>>>(s.p, s.stride, d.p, d.stride, s.w, s.h, stripe, b, wide); break;
    case 2: k_undistort<2><<<grid, block, 0, st>>>(s.p, s.stride, d.p, d.stride, s.w, s.h, stripe, b, wide); break;
    case 3: k_undistort<3><<<grid, block, 0, st>>>(s.p, s.stride, d.p, d.stride, s.w, s.h, stripe, b, wide); break;
    default: k_undistort<4><<<grid, block, 0, st>>>(s.p, s.stride, d.p, d.stride, s.w, s.h, stripe, b, wide); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_init_undistort_map(const std::vector<uint8_t> &params, const DImg &mx, const DImg &my, cudaStream_t st) {
  const UndistParams p = *reinterpret_cast<const UndistParams *>(params.data());
  dim3 block(32, 8), grid((mx.w + 31) / 32, (mx.h + 7) / 8);
  note_launch();
  k_init_map<<<grid, block, 0, st>>>(reinterpret_cast<float *>(mx.p), mx.stride, reinterpret_cast<float *>(my.p), my.stride,
                                     mx.w, mx.h, p);
  return cudaGetLastError();
}

cudaError_t launch_remap(const DImg &s, const DImg &d, const DImg &mx, const DImg &my, uint8_t value, cudaStream_t st) {
  dim3 block(32, 8), grid((d.w + 31) / 32, (d.h + 7) / 8);
  note_launch();
  switch (s.cn) {
    case 1: k_remap<1><<<grid, block, 0, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, mx.p, mx.stride, my.p, my.stride, value); break;
    case 2: k_remap<2><<<grid, block, 0, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, mx.p, mx.stride, my.p, my.stride, value); break;
    case 3: k_remap<3><<<grid, block, 0, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, mx.p, mx.stride, my.p, my.stride, value); break;
    default: k_remap<4><<<grid, block, 0, st>>>(s.p, s.stride, s.w, s.h, d.p, d.stride, d.w, d.h, mx.p, mx.stride, my.p, my.stride, value); break;
  }
  return cudaGetLastError();
}

}  // namespace vb
