// INTER_LINEAR resize of u8 device images with its tap tables in a fixed,
// statically reserved device buffer, for callers that must not allocate
// device memory during a call: a cudaMalloc/cudaFree synchronises the whole
// device (stalling every other stream of a latency-bound pipeline), can fail
// once a pre-reserved memory budget has taken the rest of HBM, and changes
// the footprint a memory-admission scheme has accounted for. The per-call
// visar_resize instead grows per-device scratch buffers on demand.
//
// The output is the one visar_resize gives (resize.zig:181-214 taps,
// resize_u8.zig:651-711 arithmetic): exact halving and same-size copies take
// the same table-free kernels, every other size computes its taps on the
// device into the static buffer and runs the same linear kernel.
//
// The buffer is one per device and per process: two calls in flight at once
// on one device (different streams, or different host threads) overwrite
// each other's tables and race. Callers serialise them (one stream, or one
// call at a time).
#include <mutex>

#include "vb.h"

namespace vb {

namespace {

// Destination widths and heights up to this many pixels: 2 x 16384 taps of 16
// bytes = 512 KiB of device memory reserved when the module loads.
constexpr int kMaxSide = kNoAllocMaxSide;

// x taps at [0, kMaxSide), y taps at [kMaxSide, 2 kMaxSide). Nothing in it
// needs to start at zero: each call writes every entry it reads, before the
// resize kernel reads it, in stream order.
static __device__ __align__(256) LinTap g_taps[2 * kMaxSide];

std::mutex g_sym_mu;
LinTap *g_sym[64] = {nullptr};

// sat.cast(i16, f32) (src/core/saturate.zig:20-49).
__device__ __forceinline__ int sat_i16_dev(float x) {
  if (x != x) return 0;
  const float r = rintf(x);
  if (r <= -32768.0f) return -32768;
  if (r >= 32767.0f) return 32767;
  return (int)r;
}

// linearTapU8 without the area branch (src/imgproc/resize.zig:181-214): the
// source coordinate in f32 from the f64 scale, floor, the x axis pinned to the
// image, each weight rounded to 11 bits on its own.
__device__ __forceinline__ LinTap tap_u8(long long d, unsigned ssize, unsigned dsize, bool pin) {
  const double inv = (double)dsize / (double)ssize;
  const double scale = 1.0 / inv;
  float fx = (float)(((double)d + 0.5) * scale - 0.5);
  const float fl = floorf(fx);
  long long sx = (long long)fl;
  fx = fx - fl;
  const long long last = (long long)ssize - 1;
  if (pin && sx < 0) {
    sx = 0;
    fx = 0.0f;
  }
  if (pin && sx >= last) {
    sx = last;
    fx = 0.0f;
  }
  LinTap t;
  t.w0 = sat_i16_dev((1.0f - fx) * 2048.0f);
  t.w1 = sat_i16_dev(fx * 2048.0f);
  t.o0 = (int)min(max(sx, 0LL), last);
  t.o1 = (int)min(max(sx + 1, 0LL), last);
  return t;
}

__global__ void k_static_taps(LinTap *taps, unsigned sw, unsigned dw, unsigned sh, unsigned dh) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < dw) taps[i] = tap_u8(i, sw, dw, true);
  else if (i < dw + dh) taps[kMaxSide + (i - dw)] = tap_u8(i - dw, sh, dh, false);
}

}  // namespace

// The scratch address on the current device. The first call on a device
// resolves it with cudaGetSymbolAddress, which may load this module onto the
// device; that first call belongs before any stream capture on the device.
cudaError_t static_taps_on_device(int dev, LinTap **out) {
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_sym_mu);
  if (!g_sym[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_taps);
    if (e != cudaSuccess) return e;
    g_sym[dev] = static_cast<LinTap *>(p);
  }
  *out = g_sym[dev];
  return cudaSuccess;
}

// s, d: u8 device images with equal channel counts (1-4), d no larger than
// kNoAllocMaxSide on either axis (checked by the caller).
cudaError_t launch_resize_linear_u8_static(const DImg &s, const DImg &d, LinTap *taps, cudaStream_t st) {
  if (s.w == d.w && s.h == d.h) return launch_copy_image(s, d, k8U, st);
  if (s.w == 2 * d.w && s.h == 2 * d.h) return launch_resize_u8_half(s, d, st);
  const unsigned n = (unsigned)d.w + (unsigned)d.h;
  k_static_taps<<<ceil_div(n, 256), 256, 0, st>>>(taps, s.w, d.w, s.h, d.h);
  note_launch();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_resize_u8_linear(s, d, taps, taps + kMaxSide, st);
}

}  // namespace vb
