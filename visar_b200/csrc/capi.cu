// The C ABI (include/visar.h): descriptor validation with VISAR's status codes
// and error names (src/capi.zig:38-144), host/device pointer handling, the
// host-side tables (resize taps, Gaussian taps, structuring elements) built
// exactly as VISAR builds them, and dispatch to the CUDA kernels.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/visar.h"
#include "vb.h"

namespace vb {

namespace {

std::atomic<unsigned long long> g_launches{0};

// ------------------------------------------------------------------ errors

thread_local char t_last_error[256] = {0};

// A failed call: status code and VISAR's error name.
struct Fail {
  int status;
  const char *name;
};

[[noreturn]] void fail(int status, const char *name) { throw Fail{status, name}; }
[[noreturn]] void unsupported() { fail(VISAR_UNSUPPORTED, "Unsupported"); }
[[noreturn]] void invalid_arg() { fail(VISAR_INVALID_ARGUMENT, "InvalidArgument"); }
[[noreturn]] void invalid_size() { fail(VISAR_INVALID_ARGUMENT, "InvalidSize"); }
[[noreturn]] void invalid_kernel() { fail(VISAR_INVALID_ARGUMENT, "InvalidKernel"); }
[[noreturn]] void size_mismatch() { fail(VISAR_SIZE_MISMATCH, "SizeMismatch"); }
[[noreturn]] void unsupported_channels() { fail(VISAR_UNSUPPORTED, "UnsupportedChannels"); }

void set_error(const char *msg) {
  std::snprintf(t_last_error, sizeof(t_last_error), "%s", msg);
}

void ck(cudaError_t e) {
  if (e == cudaSuccess) return;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    fail(VISAR_OUT_OF_MEMORY, "OutOfMemory");
  }
  static thread_local char buf[200];
  std::snprintf(buf, sizeof(buf), "CudaError: %s", cudaGetErrorName(e));
  fail(VISAR_INTERNAL, buf);
}

// The device of the current call: the one owning its device-resident
// images (set while validating them), else the thread's current device.
thread_local int t_hint_dev = -1;

struct DevCtx;
void record_call_done();

template <class F>
int guarded(F &&f) {
  t_hint_dev = -1;
  int rc = VISAR_OK;
  try {
    f();
  } catch (const Fail &e) {
    set_error(e.name);
    rc = e.status;
  } catch (const std::bad_alloc &) {
    set_error("OutOfMemory");
    rc = VISAR_OUT_OF_MEMORY;
  } catch (...) {
    set_error("Internal");
    rc = VISAR_INTERNAL;
  }
  record_call_done();
  return rc;
}

// -------------------------------------------------------- device context

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};


enum Slot { kSrc, kDst, kTmp1, kTmp2, kTmp3, kTmp4, kTab1, kTab2, kTab3, kTab4, kSmall, kNumSlots };

struct DevCtx {
  bool init = false;
  cudaStream_t own = nullptr;
  // Recorded after every call's work: the next call, on whatever stream,
  // waits for it on the device, so the shared scratch buffers are never used
  // by two streams at once. An event (not the last stream's handle) keeps
  // this safe when the caller destroys a stream it passed in.
  cudaEvent_t done = nullptr;
  bool has_done = false;
  DevBuf slot[kNumSlots];
};

std::mutex g_mu;
DevCtx g_ctx[64];
thread_local cudaStream_t t_stream = nullptr;
thread_local int t_async = 0;
// The call in progress on this thread (its context and stream), for the
// completion event guarded() records.
thread_local DevCtx *t_call_ctx = nullptr;
thread_local cudaStream_t t_call_st = nullptr;
int g_threads = 0;

struct Call {
  DevCtx *ctx;
  cudaStream_t st;
  int dev;
};

Call begin_call() {
  int dev = 0;
  if (t_hint_dev >= 0) {
    ck(cudaSetDevice(t_hint_dev));
    dev = t_hint_dev;
  } else {
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) ck(e);
  }
  if (dev < 0 || dev >= 64) fail(VISAR_INTERNAL, "CudaError: device index");
  DevCtx &c = g_ctx[dev];
  if (!c.init) {
    ck(cudaStreamCreateWithFlags(&c.own, cudaStreamNonBlocking));
    ck(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
    c.init = true;
  }
  cudaStream_t st = t_stream ? t_stream : c.own;
  // Scratch buffers are shared by all calls on this device: this call's work
  // starts after the previous call's, whichever stream that used.
  if (c.has_done) ck(cudaStreamWaitEvent(st, c.done, 0));
  t_call_ctx = &c;
  t_call_st = st;
  return Call{&c, st, dev};
}

// Marks the end of the thread's call in progress on its stream.
void record_call_done() {
  if (!t_call_ctx) return;
  if (cudaEventRecord(t_call_ctx->done, t_call_st) == cudaSuccess) t_call_ctx->has_done = true;
  else cudaGetLastError();
  t_call_ctx = nullptr;
  t_call_st = nullptr;
}

void *scratch(Call &call, Slot s, size_t bytes) {
  DevBuf &b = call.ctx->slot[s];
  if (bytes == 0) bytes = 16;
  if (b.cap < bytes) {
    ck(cudaStreamSynchronize(call.st));
    if (b.p) ck(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
    const size_t want = (bytes + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
    ck(cudaMalloc(&b.p, want));
    b.cap = want;
  }
  return b.p;
}

template <class T>
T *upload(Call &call, Slot s, const std::vector<T> &v) {
  T *p = static_cast<T *>(scratch(call, s, v.size() * sizeof(T)));
  // Tables are small: a copy from pageable memory costs the device less than
  // a DMA from a pinned buffer would.
  if (!v.empty()) ck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, call.st));
  return p;
}

// ------------------------------------------------------------ descriptors

// A validated image: its typed view (capi.zig:123-132) and where it lives.
struct View {
  const visar_image *c;
  int depth;
  int esize;
  bool host;
  DImg dev;  // device view (after staging for host images)
};

bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const bool dev = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
  if (dev && a.device >= 0) {
    if (t_hint_dev >= 0 && t_hint_dev != a.device) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument");
    t_hint_dev = a.device;
  }
  return dev;
}

// typed(T, c): the checks of src/capi.zig:123-132 and Image.fromSliceStrided
// (src/core/image.zig:70-77, 172-176), in that order.
View typed(const visar_image *c, int depth) {
  if (!c || !c->data) invalid_arg();
  if ((int)c->depth != depth) unsupported();
  if (c->channels == 0 || c->channels > 512) invalid_arg();
  const int es = depth_size(depth);
  if (c->stride % es != 0) invalid_arg();
  if (c->width == 0 || c->height == 0) invalid_size();
  const unsigned long long row = (unsigned long long)c->width * c->channels * es;
  if (c->stride < row) invalid_size();
  View v;
  v.c = c;
  v.depth = depth;
  v.esize = es;
  v.host = !is_device_ptr(c->data);
  v.dev = DImg{static_cast<uint8_t *>(c->data), (long long)c->stride, (int)c->width, (int)c->height, (int)c->channels};
  return v;
}

// The depths VISAR's C ABI dispatches on (capi.zig:136-144).
int src_depth(const visar_image *c) {
  if (!c) invalid_arg();
  switch (c->depth) {
    case 0: case 2: case 3: case 5: return (int)c->depth;
  }
  unsupported();
}

long long row_bytes(const View &v) { return (long long)v.c->width * v.c->channels * v.esize; }

size_t pitch_for(long long rb) { return (size_t)((rb + 255) & ~255LL); }

// Host input -> device copy; device input used in place.
void stage_in(Call &call, View &v, Slot s) {
  if (!v.host) return;
  const long long rb = row_bytes(v);
  const size_t pitch = pitch_for(rb);
  uint8_t *p = static_cast<uint8_t *>(scratch(call, s, pitch * v.c->height));
  ck(cudaMemcpy2DAsync(p, pitch, v.c->data, v.c->stride, rb, v.c->height, cudaMemcpyHostToDevice, call.st));
  v.dev.p = p;
  v.dev.stride = (long long)pitch;
}

void stage_out(Call &call, View &v, Slot s) {
  if (!v.host) return;
  const size_t pitch = pitch_for(row_bytes(v));
  v.dev.p = static_cast<uint8_t *>(scratch(call, s, pitch * v.c->height));
  v.dev.stride = (long long)pitch;
}

void finish_out(Call &call, View &v) {
  if (v.host)
    ck(cudaMemcpy2DAsync(v.c->data, v.c->stride, v.dev.p, v.dev.stride, row_bytes(v), v.c->height, cudaMemcpyDeviceToHost,
                         call.st));
}

void end_call(Call &call, bool any_host) {
  ck(cudaGetLastError());
  if (any_host || !t_async) ck(cudaStreamSynchronize(call.st));
}

bool overlaps(const View &a, const View &b) {
  if (a.host || b.host) return false;  // host images are staged separately
  const uintptr_t a0 = (uintptr_t)a.dev.p, b0 = (uintptr_t)b.dev.p;
  const uintptr_t a1 = a0 + (uintptr_t)((a.dev.h - 1) * a.dev.stride + row_bytes(a));
  const uintptr_t b1 = b0 + (uintptr_t)((b.dev.h - 1) * b.dev.stride + row_bytes(b));
  return a0 < b1 && b0 < a1;
}

// A private device copy of a device-resident source that overlaps dst.
void detach_src(Call &call, View &src, Slot s) {
  const long long rb = row_bytes(src);
  const size_t pitch = pitch_for(rb);
  uint8_t *p = static_cast<uint8_t *>(scratch(call, s, pitch * src.c->height));
  ck(cudaMemcpy2DAsync(p, pitch, src.dev.p, src.dev.stride, rb, src.c->height, cudaMemcpyDeviceToDevice, call.st));
  src.dev.p = p;
  src.dev.stride = (long long)pitch;
}

DImg temp_like(Call &call, const View &v, Slot s) {
  const size_t pitch = pitch_for(row_bytes(v));
  DImg d = v.dev;
  d.p = static_cast<uint8_t *>(scratch(call, s, pitch * v.c->height));
  d.stride = (long long)pitch;
  return d;
}

int border_arg(int b) {
  if (b < 0 || b > 4) unsupported();
  return b;
}

// ------------------------------------------------------------- cvtColor

// capi.zig:148-161: OpenCV COLOR_* code -> conversion.
bool color_info(int code, ColorInfo &ci) {
  switch (code) {
    case 0: ci = {3, 4, 0, 0, kReorder}; return true;   // BGR2BGRA
    case 1: ci = {4, 3, 0, 0, kReorder}; return true;   // BGRA2BGR
    case 2: ci = {3, 4, 0, 2, kReorder}; return true;   // BGR2RGBA
    case 3: ci = {4, 3, 0, 2, kReorder}; return true;   // RGBA2BGR
    case 4: ci = {3, 3, 0, 2, kReorder}; return true;   // BGR2RGB
    case 5: ci = {4, 4, 0, 2, kReorder}; return true;   // BGRA2RGBA
    case 6: ci = {3, 1, 0, 0, kGray}; return true;      // BGR2GRAY
    case 7: ci = {3, 1, 2, 0, kGray}; return true;      // RGB2GRAY
    case 8: ci = {1, 3, 0, 0, kFromGray}; return true;  // GRAY2BGR
    case 9: ci = {1, 4, 0, 0, kFromGray}; return true;  // GRAY2BGRA
    case 10: ci = {4, 1, 0, 0, kGray}; return true;     // BGRA2GRAY
    case 11: ci = {4, 1, 2, 0, kGray}; return true;     // RGBA2GRAY
    case 36: ci = {3, 3, 0, 0, kYcrcb}; return true;    // BGR2YCrCb
    case 37: ci = {3, 3, 2, 0, kYcrcb}; return true;    // RGB2YCrCb
    case 38: ci = {3, 3, 0, 0, kFromYcrcb}; return true;
    case 39: ci = {3, 3, 0, 2, kFromYcrcb}; return true;
    case 40: ci = {3, 3, 0, 0, kHsv}; return true;
    case 41: ci = {3, 3, 2, 0, kHsv}; return true;
    case 54: ci = {3, 3, 0, 0, kFromHsv}; return true;
    case 55: ci = {3, 3, 0, 2, kFromHsv}; return true;
  }
  return false;
}

// Depths each family implements (color.zig:107-114).
bool color_supported(int depth, ColorKind k) {
  switch (k) {
    case kReorder: case kFromGray: return true;
    case kGray: return depth == k8U || depth == k16U || depth == k32F;
    default: return depth == k8U || depth == k32F;
  }
}

// --------------------------------------------------------------- resize

void cubic_coeffs(float x, float c[4]) {
  const float A = -0.75f;
  c[0] = ((A * (x + 1) - 5 * A) * (x + 1) + 8 * A) * (x + 1) - 4 * A;
  c[1] = ((A + 2) * x - (A + 3)) * x * x + 1;
  c[2] = ((A + 2) * (1 - x) - (A + 3)) * (1 - x) * (1 - x) + 1;
  c[3] = 1 - c[0] - c[1] - c[2];
}

std::vector<CubTap> cubic_tab_u8(uint32_t ssize, uint32_t dsize) {
  std::vector<CubTap> t(dsize);
  const double scale = 1.0 / ((double)dsize / (double)ssize);
  for (uint32_t i = 0; i < dsize; i++) {
    float fx = (float)(((double)i + 0.5) * scale - 0.5);
    const float sx = std::floor(fx);
    fx -= sx;
    const long long isx = (long long)sx;
    float cf[4];
    cubic_coeffs(fx, cf);
    for (int k = 0; k < 4; k++) {
      t[i].w[k] = sat_i16(cf[k] * 2048.0f);
      t[i].o[k] = (int)std::min(std::max(isx - 1 + k, 0LL), (long long)ssize - 1);
    }
  }
  return t;
}

std::vector<FCubTap> cubic_tab_f(uint32_t ssize, uint32_t dsize) {
  std::vector<FCubTap> t(dsize);
  const double scale = (double)ssize / (double)dsize;
  for (uint32_t i = 0; i < dsize; i++) {
    const double fx = ((double)i + 0.5) * scale - 0.5;
    const long long sx = (long long)std::floor(fx);
    cubic_coeffs((float)(fx - (double)sx), t[i].w);
    for (int k = 0; k < 4; k++) t[i].o[k] = (int)std::min(std::max(sx - 1 + k, 0LL), (long long)ssize - 1);
  }
  return t;
}

// computeResizeAreaTab (resize.zig:470-493).
std::vector<AreaEnt> area_tab(uint32_t ssize, uint32_t dsize, double scale) {
  std::vector<AreaEnt> v;
  for (uint32_t dx = 0; dx < dsize; dx++) {
    const double fsx1 = (double)dx * scale;
    const double fsx2 = fsx1 + scale;
    const double cellw = std::min(scale, (double)ssize - fsx1);
    long long sx1 = (long long)std::ceil(fsx1);
    const long long sx2 = (long long)std::floor(fsx2);
    const long long sx2c = std::min(sx2, (long long)ssize - 1);
    sx1 = std::min(sx1, (long long)ssize - 1);
    if ((double)sx1 - fsx1 > 1e-3) v.push_back({(int)dx, (int)(sx1 - 1), (float)(((double)sx1 - fsx1) / cellw)});
    for (long long sx = sx1; sx < sx2; sx++) v.push_back({(int)dx, (int)sx, (float)(1.0 / cellw)});
    if (fsx2 - (double)sx2 > 1e-3)
      v.push_back({(int)dx, (int)sx2c, (float)(std::min(std::min(fsx2 - (double)sx2, 1.0), cellw) / cellw)});
  }
  return v;
}

std::vector<int> starts_of(const std::vector<AreaEnt> &t, uint32_t dsize) {
  std::vector<int> st(dsize + 1);
  size_t k = 0;
  for (uint32_t d = 0; d < dsize; d++) {
    st[d] = (int)k;
    while (k < t.size() && t[k].di == (int)d) k++;
  }
  st[dsize] = (int)k;
  return st;
}

void resize_impl(Call &call, const DImg &s, const DImg &d, int depth, int interp) {
  const uint32_t sw = s.w, sh = s.h, dw = d.w, dh = d.h;
  const int cn = s.cn;
  if (sw == dw && sh == dh) {
    ck(launch_copy_image(s, d, depth, call.st));
    return;
  }
  const bool u8fast = depth == k8U && cn <= 4;
  const bool exact_half = sw == 2 * dw && sh == 2 * dh;
  auto u8_linear = [&](bool area) {
    std::vector<LinTap> xt(dw), yt(dh);
    for (uint32_t x = 0; x < dw; x++) xt[x] = lin_tap_u8(x, sw, dw, area, true);
    for (uint32_t y = 0; y < dh; y++) yt[y] = lin_tap_u8(y, sh, dh, area, false);
    ck(launch_resize_u8_linear(s, d, upload(call, kTab1, xt), upload(call, kTab2, yt), call.st));
  };
  auto generic_linear = [&](bool area) {
    if (depth == k8U) return u8_linear(area);
    std::vector<FLinTap> xt(dw), yt(dh);
    for (uint32_t x = 0; x < dw; x++) xt[x] = lin_tap_f(x, sw, dw, area, true);
    for (uint32_t y = 0; y < dh; y++) yt[y] = lin_tap_f(y, sh, dh, area, false);
    ck(launch_resize_linear_generic(s, d, depth, upload(call, kTab1, xt), upload(call, kTab2, yt), call.st));
  };
  auto area_frac = [&]() {
    const std::vector<AreaEnt> xt = area_tab(sw, dw, (double)sw / (double)dw);
    const std::vector<AreaEnt> yt = area_tab(sh, dh, (double)sh / (double)dh);
    const std::vector<int> xs = starts_of(xt, dw), ys = starts_of(yt, dh);
    ck(launch_resize_area_frac(s, d, depth, upload(call, kTab1, xt), (int)xt.size(), upload(call, kTab2, xs),
                               upload(call, kTab3, yt), upload(call, kTab4, ys), call.st));
  };
  if (u8fast) {
    switch (interp) {
      case 1:
        if (exact_half) ck(launch_resize_u8_half(s, d, call.st));
        else u8_linear(false);
        return;
      case 3: {
        if (dw > sw || dh > sh) return u8_linear(true);
        if (exact_half) {
          ck(launch_resize_u8_half(s, d, call.st));
          return;
        }
        const uint32_t ix = sw / dw, iy = sh / dh;
        if (ix * dw == sw && iy * dh == sh) {
          ck(launch_resize_area_int(s, d, depth, (int)ix, (int)iy, true, call.st));
          return;
        }
        return area_frac();
      }
      case 2: {
        const std::vector<CubTap> xt = cubic_tab_u8(sw, dw), yt = cubic_tab_u8(sh, dh);
        ck(launch_resize_u8_cubic(s, d, upload(call, kTab1, xt), upload(call, kTab2, yt), call.st));
        return;
      }
      default: break;
    }
  }
  switch (interp) {
    case 0: {
      // nearest (resize.zig:64-105)
      std::vector<int> xo(dw), yo(dh);
      const double ifx = (double)sw / (double)dw, ify = (double)sh / (double)dh;
      for (uint32_t x = 0; x < dw; x++) xo[x] = (int)std::min((uint32_t)std::floor((double)x * ifx), sw - 1);
      for (uint32_t y = 0; y < dh; y++) yo[y] = (int)std::min((uint32_t)std::floor((double)y * ify), sh - 1);
      ck(launch_resize_nearest(s, d, depth, upload(call, kTab1, xo), upload(call, kTab2, yo), call.st));
      return;
    }
    case 1: return generic_linear(false);
    case 3: {
      if (dw > sw || dh > sh) return generic_linear(true);
      const uint32_t ix = sw / dw, iy = sh / dh;
      if (ix * dw == sw && iy * dh == sh) {
        ck(launch_resize_area_int(s, d, depth, (int)ix, (int)iy, false, call.st));
        return;
      }
      return area_frac();
    }
    case 2: {
      const std::vector<FCubTap> xt = cubic_tab_f(sw, dw), yt = cubic_tab_f(sh, dh);
      ck(launch_resize_cubic_generic(s, d, depth, upload(call, kTab1, xt), upload(call, kTab2, yt), call.st));
      return;
    }
  }
  unsupported();  // lanczos4
}

// -------------------------------------------------------- morphology

std::vector<MorphRun> element_runs(const std::vector<uint8_t> &m, int w, int h) {
  std::vector<MorphRun> runs;
  for (int ky = 0; ky < h; ky++) {
    int x = 0;
    while (x < w) {
      if (!m[(size_t)ky * w + x]) {
        x++;
        continue;
      }
      const int x0 = x;
      while (x < w && m[(size_t)ky * w + x]) x++;
      runs.push_back({ky, x0, x - x0});
    }
  }
  return runs;
}

}  // namespace

void note_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

cudaStream_t thread_stream() { return t_stream; }
int thread_async() { return t_async; }
void set_thread_stream(cudaStream_t st, int async) {
  t_stream = st;
  t_async = async;
}

int report_error(int status, const char *msg) {
  set_error(msg);
  return status;
}

}  // namespace vb

using namespace vb;

// ====================================================================== ABI

extern "C" {

const char *visar_version(void) { return "0.1.0-b200"; }

const char *visar_build_info(void) { return "visar-b200 CUDA sm_100a (B200), bit-exact VISAR imgproc"; }

const char *visar_last_error(void) { return t_last_error; }

void visar_set_num_threads(int n) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_threads = n <= 0 ? 0 : n;
}

int visar_get_num_threads(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_threads > 0) return g_threads;
  const unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)hc : 1;
}

int visar_cuda_set_stream(void *stream) {
  t_stream = static_cast<cudaStream_t>(stream);
  return VISAR_OK;
}

int visar_cuda_set_async(int async) {
  t_async = async ? 1 : 0;
  return VISAR_OK;
}

uint64_t visar_cuda_launch_count(void) { return g_launches.load(); }

int visar_cvt_color(const visar_image *src, const visar_image *dst, int code) {
  return guarded([&] {
    ColorInfo ci;
    if (code < 0 || code >= 56 || !color_info(code, ci)) unsupported();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    if (s.c->width != d.c->width || s.c->height != d.c->height) size_mismatch();
    if ((int)s.c->channels != ci.scn || (int)d.c->channels != ci.dcn) unsupported_channels();
    if (!color_supported(depth, ci.kind)) unsupported();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d) && !(s.dev.p == d.dev.p && s.dev.stride == d.dev.stride && ci.scn == ci.dcn)) detach_src(call, s, kTmp1);
    ck(launch_cvt_color(s.dev, d.dev, depth, ci, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_resize(const visar_image *src, const visar_image *dst, int interp) {
  return guarded([&] {
    if (interp < 0 || interp > 4) unsupported();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    if (s.c->channels != d.c->channels) size_mismatch();
    if (interp == 4 && !(s.c->width == d.c->width && s.c->height == d.c->height)) unsupported();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    resize_impl(call, s.dev, d.dev, depth, interp);
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_gaussian_blur(const visar_image *src, const visar_image *dst, int kw_in, int kh_in, double sx, double sy_arg,
                        int border) {
  return guarded([&] {
    const int bd = border_arg(border);
    if (kw_in < 0 || kh_in < 0) invalid_arg();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    // gaussianBlur (filter.zig:498-607)
    const double sy = sy_arg > 0 ? sy_arg : sx;
    int kw = kw_in > 0 ? kw_in : gaussian_ksize(sx, depth == k8U);
    int kh = kh_in > 0 ? kh_in : gaussian_ksize(sy, depth == k8U);
    if (kw <= 0 || kh <= 0 || kw % 2 == 0 || kh % 2 == 0 || kw > 127 || kh > 127) invalid_kernel();
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    if (bd != kConstant) {
      if (s.c->width == 1) kw = 1;
      if (s.c->height == 1) kh = 1;
    }
    SepSpec sp;
    sp.sdepth = depth;
    sp.ddepth = depth;
    sp.border = bd;
    sp.scale = 1.0;
    sp.shift = 0;
    if (depth == k8U || depth == k16U) {
      // Fixed-point taps (8 fractional bits for u8, 16 for u16); the exact
      // 2-D sum is rounded once: (v + 2^(2b-1)) >> 2b. This equals every
      // reduced-tap variant VISAR dispatches to (filter.zig:511-581).
      const int bits = depth == k8U ? 8 : 16;
      std::vector<int64_t> kx(kw), ky(kh);
      gaussian_kernel_fixed(kx.data(), kw, sx, bits);
      gaussian_kernel_fixed(ky.data(), kh, sy, bits);
      sp.kxi.assign(kx.begin(), kx.end());
      sp.kyi.assign(ky.begin(), ky.end());
      sp.acc = depth == k8U ? kAccI32 : kAccI64;
      sp.fin = kFinShift;
      sp.shift = 2 * bits;
    } else {
      std::vector<double> kx(kw), ky(kh);
      gaussian_kernel(kx.data(), kw, sx);
      gaussian_kernel(ky.data(), kh, sy);
      for (double v : kx) sp.kxf.push_back((float)v);
      for (double v : ky) sp.kyf.push_back((float)v);
      sp.acc = kAccF32;
      sp.fin = kFinCast;
    }
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_sep_filter(s.dev, d.dev, sp, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_box_filter(const visar_image *src, const visar_image *dst, int kw, int kh, int normalize, int border) {
  return guarded([&] {
    const int bd = border_arg(border);
    if (kw <= 0 || kh <= 0) invalid_arg();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    // boxFilter (filter.zig:619-633)
    if (kw > 255 || kh > 255 || kw % 2 == 0 || kh % 2 == 0) invalid_kernel();
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    SepSpec sp;
    sp.sdepth = depth;
    sp.ddepth = depth;
    sp.border = bd;
    sp.scale = normalize ? 1.0 / (double)(kw * kh) : 1.0;
    sp.shift = 0;
    sp.fin = kFinScaled;
    if (depth == k32F) {
      sp.acc = kAccF32;
      sp.kxf.assign(kw, 1.0f);
      sp.kyf.assign(kh, 1.0f);
    } else {
      sp.acc = depth == k8U ? kAccI32 : kAccI64;
      sp.kxi.assign(kw, 1);
      sp.kyi.assign(kh, 1);
    }
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_sep_filter(s.dev, d.dev, sp, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_sobel(const visar_image *src, const visar_image *dst, int dx, int dy, int ksize, double scale, int border) {
  return guarded([&] {
    const int bd = border_arg(border);
    if (dx < 0 || dy < 0) invalid_arg();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    if (!dst) invalid_arg();
    int ddepth;
    if (dst->depth == 3) {
      if (depth != k8U) unsupported();
      ddepth = k16S;
    } else if (dst->depth == 5) {
      ddepth = k32F;
    } else {
      unsupported();
    }
    View d = typed(dst, ddepth);
    // sobel (filter.zig:867-906)
    if (ksize > 31 || ksize < -1) invalid_kernel();
    const int n = ksize <= 1 ? 3 : ksize;
    const int nx = (ksize == 1 && dx > 0) ? 3 : n;
    const int ny = (ksize == 1 && dy > 0) ? 3 : n;
    std::vector<int> kx(nx), ky(ny);
    const int ksx = (ksize == 1 && dx == 0) ? 1 : (ksize == 1) ? 3 : ksize;
    const int ksy = (ksize == 1 && dy == 0) ? 1 : (ksize == 1) ? 3 : ksize;
    if (!deriv_kernel(kx.data(), nx, dx, ksx)) invalid_kernel();
    if (!deriv_kernel(ky.data(), ny, dy, ksy)) invalid_kernel();
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    if (nx % 2 == 0 || ny % 2 == 0) invalid_kernel();
    SepSpec sp;
    sp.sdepth = depth;
    sp.ddepth = ddepth;
    sp.border = bd;
    sp.scale = scale;
    sp.shift = 0;
    if (ddepth == k32F || depth == k32F) {
      sp.acc = kAccF32;
      sp.fin = kFinScaled;
      for (int v : kx) sp.kxf.push_back((float)v);
      for (int v : ky) sp.kyf.push_back((float)v);
    } else {
      // VISAR sums in i16 or i32 (filter.zig:886-905); where 255 * sum|kx| *
      // sum|ky| exceeds i32 (large apertures) its sums overflow, which Zig
      // leaves undefined. The exact sum is kept in 64 bits there.
      long long bx = 0, by = 0;
      for (int v : kx) bx += v < 0 ? -v : v;
      for (int v : ky) by += v < 0 ? -v : v;
      sp.acc = (255.0 * (double)bx * (double)by > 2147483647.0) ? kAccI64 : kAccI32;
      sp.kxi = kx;
      sp.kyi = ky;
      sp.fin = scale == 1.0 ? kFinCast : kFinScaled;
    }
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_sep_filter(s.dev, d.dev, sp, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_sep_filter_2d(const visar_image *src, const visar_image *dst, const float *kx, int nkx, const float *ky, int nky,
                        int border) {
  return guarded([&] {
    const int bd = border_arg(border);
    if (!kx || !ky || nkx < 0 || nky < 0) invalid_arg();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    const int ddepth = src_depth(dst);
    View d = typed(dst, ddepth);
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    if (nkx == 0 || nky == 0 || nkx % 2 == 0 || nky % 2 == 0 || nkx > 255 || nky > 255) invalid_kernel();
    SepSpec sp;
    sp.sdepth = depth;
    sp.ddepth = ddepth;
    sp.border = bd;
    sp.scale = 1.0;
    sp.shift = 0;
    sp.acc = kAccF32;
    sp.fin = kFinCast;
    sp.kxf.assign(kx, kx + nkx);
    sp.kyf.assign(ky, ky + nky);
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_sep_filter(s.dev, d.dev, sp, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_threshold(const visar_image *src, const visar_image *dst, double thresh, double maxval, int type, double *used) {
  double t_used = thresh;
  const int rc = guarded([&] {
    const int kind = type & 7;
    if (kind > 4) unsupported();
    const int method = (type & 8) ? 0 : (type & 16) ? 1 : -1;  // 0 otsu, 1 triangle
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    // threshold (threshold.zig:25-82)
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    if (method >= 0 && (depth != k8U || s.c->channels != 1)) unsupported();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (depth == k8U) {
      uint8_t *lut = static_cast<uint8_t *>(scratch(call, kTab1, 256));
      if (method >= 0) {
        uint8_t *small = static_cast<uint8_t *>(scratch(call, kSmall, 4096));
        uint32_t *hist = reinterpret_cast<uint32_t *>(small);
        double *tdev = reinterpret_cast<double *>(small + 1024);
        ck(launch_threshold_auto_u8(s.dev, method, kind, maxval, hist, tdev, lut, call.st));
        ck(launch_threshold_lut_u8(s.dev, d.dev, lut, call.st));
        double th = 0;
        ck(cudaMemcpyAsync(&th, tdev, sizeof(double), cudaMemcpyDeviceToHost, call.st));
        finish_out(call, d);
        ck(cudaStreamSynchronize(call.st));
        t_used = th;
        return;
      }
      const double fl = std::floor(thresh);
      const int ti = fl != fl ? 0 : fl < -1e9 ? -1000000000 : fl > 1e9 ? 1000000000 : (int)fl;
      uint8_t m;
      {
        const double r = std::nearbyint(maxval);
        m = maxval != maxval ? 0 : r <= 0 ? 0 : r >= 255 ? 255 : (uint8_t)(int)r;
      }
      std::vector<uint8_t> host_lut(256);
      const uint8_t tsat = (uint8_t)std::min(std::max(ti, 0), 255);
      for (int i = 0; i < 256; i++) {
        const bool gt = i > ti;
        const uint8_t v = (uint8_t)i;
        uint8_t o;
        switch (kind) {
          case 0: o = gt ? m : 0; break;
          case 1: o = gt ? 0 : m; break;
          case 2: o = gt ? tsat : v; break;
          case 3: o = gt ? v : 0; break;
          default: o = gt ? 0 : v; break;
        }
        host_lut[i] = o;
      }
      lut = upload(call, kTab1, host_lut);
      ck(launch_threshold_lut_u8(s.dev, d.dev, lut, call.st));
    } else if (depth == k32F) {
      ck(launch_threshold_cmp(s.dev, d.dev, depth, kind, (double)(float)thresh, (double)(float)maxval, call.st));
    } else {
      const int lo = depth == k16U ? 0 : -32768, hi = depth == k16U ? 65535 : 32767;
      auto satd = [&](double v) -> double {
        if (v != v) return 0;
        const double r = std::nearbyint(v);
        return r <= lo ? lo : r >= hi ? hi : r;
      };
      const double fl = std::floor(thresh);
      const double m = satd(maxval);
      if (fl < lo) {
        // Every value is above the threshold (threshold.zig:62-72).
        if (kind == 3) ck(launch_copy_image(s.dev, d.dev, depth, call.st));
        else ck(launch_fill(d.dev, depth, kind == 0 ? m : 0.0, call.st));
      } else {
        ck(launch_threshold_cmp(s.dev, d.dev, depth, kind, satd(fl), m, call.st));
      }
    }
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
  if (used) *used = t_used;
  return rc;
}

int visar_morphology(const visar_image *src, const visar_image *dst, int op, int shape, int kw, int kh, int iterations) {
  return guarded([&] {
    if (op < 0 || op > 6) unsupported();
    if (shape < 0 || shape > 2) unsupported();
    if (kw <= 0 || kh <= 0 || kw > 255 || kh > 255 || iterations < 0) invalid_arg();
    const std::vector<uint8_t> mask = structuring_element(shape, kw, kh);
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    const std::vector<MorphRun> runs = element_runs(mask, kw, kh);
    bool rect = true;
    for (uint8_t m : mask) rect = rect && m;
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    const MorphRun *runs_dev = upload(call, kTab1, runs);
    const int ax = kw / 2, ay = kh / 2;
    // One erode or dilate of `iterations` passes from a to b, ping-ponging
    // through tmp so the last pass lands in b (morph.zig:71-96).
    auto morph = [&](const DImg &a, const DImg &b, bool is_max, Slot tmp_slot) {
      if (iterations == 0) {
        ck(launch_copy_image(a, b, depth, call.st));
        return;
      }
      DImg tmp{};
      if (iterations > 1) tmp = temp_like(call, s, tmp_slot);
      DImg cur = a;
      for (int it = 0; it < iterations; it++) {
        const DImg out = ((iterations - 1 - it) % 2 == 0) ? b : tmp;
        if (runs.empty()) {
          // No on-cells: every output is the identity.
          double idv = 0;
          if (depth == k32F) idv = is_max ? -INFINITY : INFINITY;
          else idv = is_max ? (depth == k16S ? -32768 : 0) : (depth == k8U ? 255 : depth == k16U ? 65535 : 32767);
          ck(launch_fill(out, depth, idv, call.st));
        } else {
          cudaError_t e = cudaErrorNotSupported;
          if (depth == k8U) e = launch_morph_fast(cur, out, is_max, mask, kw, kh, call.st);
          if (e == cudaErrorNotSupported)
            e = launch_morph_pass(cur, out, depth, is_max, kw, kh, ax, ay, runs_dev, (int)runs.size(), rect, call.st);
          ck(e);
        }
        cur = out;
      }
    };
    switch (op) {
      case 0: morph(s.dev, d.dev, false, kTmp2); break;
      case 1: morph(s.dev, d.dev, true, kTmp2); break;
      case 2: {
        const DImg t = temp_like(call, s, kTmp3);
        morph(s.dev, t, false, kTmp2);
        morph(t, d.dev, true, kTmp2);
        break;
      }
      case 3: {
        const DImg t = temp_like(call, s, kTmp3);
        morph(s.dev, t, true, kTmp2);
        morph(t, d.dev, false, kTmp2);
        break;
      }
      case 4: {
        const DImg t = temp_like(call, s, kTmp3);
        morph(s.dev, t, false, kTmp2);
        morph(s.dev, d.dev, true, kTmp2);
        ck(launch_sub_sat(d.dev, t, d.dev, depth, call.st));
        break;
      }
      case 5: {
        const DImg t = temp_like(call, s, kTmp3);
        morph(s.dev, t, false, kTmp2);
        const DImg t2 = temp_like(call, s, kTmp4);
        morph(t, t2, true, kTmp2);
        ck(launch_sub_sat(s.dev, t2, d.dev, depth, call.st));
        break;
      }
      case 6: {
        const DImg t = temp_like(call, s, kTmp3);
        morph(s.dev, t, true, kTmp2);
        const DImg t2 = temp_like(call, s, kTmp4);
        morph(t, t2, false, kTmp2);
        ck(launch_sub_sat(t2, s.dev, d.dev, depth, call.st));
        break;
      }
    }
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_warp_affine(const visar_image *src, const visar_image *dst, const double m[6], int interp, int border, double value) {
  return guarded([&] {
    const int bd = border_arg(border);
    if (!m) invalid_arg();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    float mf[6];
    if (!affine_inverse_f32(m, mf)) unsupported();
    if (s.c->channels != d.c->channels) size_mismatch();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_warp_affine(s.dev, d.dev, depth, mf, interp == 0 ? 0 : 1, bd, value, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_warp_perspective(const visar_image *src, const visar_image *dst, const double m[9], int interp, int border,
                           double value) {
  return guarded([&] {
    const int bd = border_arg(border);
    if (!m) invalid_arg();
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    double inv[9];
    if (!perspective_inverse(m, inv)) unsupported();
    if (s.c->channels != d.c->channels) size_mismatch();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_warp_perspective(s.dev, d.dev, depth, inv, interp == 0 ? 0 : 1, bd, value, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

// capi.zig:176-182 -> frame.zig:169-174: k <= 0 is InvalidArgument; a factor
// above 16, a destination that is not one channel of (w / k) x (h / k), or a
// source that is not BGR / BGRA is SizeMismatch.
int visar_gray_downsample(const visar_image *src, const visar_image *dst, int k) {
  return guarded([&] {
    if (k <= 0) invalid_arg();
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, k8U);
    View d = typed(dst, k8U);
    if (k > 16 || d.c->channels != 1 || (s.c->channels != 3 && s.c->channels != 4)) size_mismatch();
    if (d.c->width != s.c->width / (uint32_t)k || d.c->height != s.c->height / (uint32_t)k) size_mismatch();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_gray_downsample(s.dev, d.dev, k, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

// capi.zig:234-249 -> pyramid.zig:73-80, 408-413: the border must be 0-4
// (Unsupported otherwise), pyrDown refuses BORDER_CONSTANT and pyrUp anything
// but BORDER_REFLECT_101 (Unsupported); dst must have the source's channels
// and ((w+1)/2, (h+1)/2) resp. (2w, 2h) pixels (SizeMismatch).
int visar_pyr_down(const visar_image *src, const visar_image *dst, int border) {
  return guarded([&] {
    const int bd = border_arg(border);
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    if (bd == 0) unsupported();
    if (d.c->channels != s.c->channels || d.c->width != (s.c->width + 1) / 2 || d.c->height != (s.c->height + 1) / 2)
      size_mismatch();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_pyr_down(s.dev, d.dev, depth, bd, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

int visar_pyr_up(const visar_image *src, const visar_image *dst, int border) {
  return guarded([&] {
    const int bd = border_arg(border);
    const int depth = src_depth(src);
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, depth);
    View d = typed(dst, depth);
    if (bd != 4) unsupported();
    if (d.c->channels != s.c->channels || (uint64_t)d.c->width != 2ull * s.c->width ||
        (uint64_t)d.c->height != 2ull * s.c->height)
      size_mismatch();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_pyr_up(s.dev, d.dev, depth, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

// camera.expandDist (src/calib3d/camera.zig:17-22) of distSlice
// (capi_calib3d.zig:93-95): a null `dist` is no coefficients; 0, 4, 5 or 8.
void expand_dist(const double *dist, size_t nd, double k8[8]) {
  for (int i = 0; i < 8; i++) k8[i] = 0;
  if (!dist) return;
  if (nd != 0 && nd != 4 && nd != 5 && nd != 8) invalid_arg();
  for (size_t i = 0; i < nd; i++) k8[i] = dist[i];
}

// capi_calib3d.zig:186-191 -> undistort.zig:204-209.
int visar_undistort(const visar_image *src, const visar_image *dst, const double k[9], const double *dist, size_t nd,
                    const double *new_k) {
  return guarded([&] {
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, k8U);
    View d = typed(dst, k8U);
    if (!k) invalid_arg();
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    if (s.c->channels < 1 || s.c->channels > 4) unsupported();
    double k8[8];
    expand_dist(dist, nd, k8);
    const bool keeps_rows = undistort_any_singular(new_k, k, (int)s.c->width, (int)s.c->height);
    Call call = begin_call();
    stage_in(call, s, kSrc);
    if (d.host && keeps_rows) {
      // Rows under a singular stripe camera are left as they are: start from dst.
      View dd = d;
      stage_in(call, dd, kDst);
      d.dev = dd.dev;
    } else {
      stage_out(call, d, kDst);
    }
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_undistort(s.dev, d.dev, k, k8, new_k, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

// capi_calib3d.zig:195-201: maps VISAR_32F, one channel, of equal shape.
int visar_init_undistort_rectify_map(const double k[9], const double *dist, size_t nd, const double *r, const double *new_k,
                                     const visar_image *mapx, const visar_image *mapy) {
  return guarded([&] {
    std::lock_guard<std::mutex> lk(g_mu);
    View mx = typed(mapx, k32F);
    View my = typed(mapy, k32F);
    if (!k) invalid_arg();
    double k8[8];
    expand_dist(dist, nd, k8);
    std::vector<uint8_t> params;
    if (!undistort_map_params(k, k8, r, new_k, params)) invalid_arg();
    if (mx.c->width != my.c->width || mx.c->height != my.c->height || mx.c->channels != my.c->channels ||
        mx.c->channels != 1)
      size_mismatch();
    Call call = begin_call();
    stage_out(call, mx, kDst);
    stage_out(call, my, kTmp2);
    ck(launch_init_undistort_map(params, mx.dev, my.dev, call.st));
    finish_out(call, mx);
    finish_out(call, my);
    end_call(call, mx.host || my.host);
  });
}

// capi_calib3d.zig:205-213 -> undistort.zig:288-291: value rounded half away
// from zero and clamped to 0..255 for every channel.
int visar_remap(const visar_image *src, const visar_image *dst, const visar_image *mapx, const visar_image *mapy,
                double value) {
  return guarded([&] {
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, k8U);
    View d = typed(dst, k8U);
    View mx = typed(mapx, k32F);
    View my = typed(mapy, k32F);
    const double rv = std::round(value);
    const uint8_t bv = (uint8_t)(rv != rv ? 0 : rv < 0 ? 0 : rv > 255 ? 255 : rv);
    if (d.c->width != mx.c->width || d.c->height != mx.c->height || mx.c->width != my.c->width ||
        mx.c->height != my.c->height || mx.c->channels != my.c->channels || mx.c->channels != 1)
      size_mismatch();
    if (s.c->channels != d.c->channels || s.c->channels < 1 || s.c->channels > 4) unsupported();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_in(call, mx, kTmp2);
    stage_in(call, my, kTmp3);
    stage_out(call, d, kDst);
    if (overlaps(s, d)) detach_src(call, s, kTmp1);
    ck(launch_remap(s.dev, d.dev, mx.dev, my.dev, bv, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host || mx.host || my.host);
  });
}

}  // extern "C"

// The background model's state: a u16 image on the device it was created on.
struct visar_background {
  int dev = 0;
  uint32_t w = 0, h = 0;
  int shift = 0;
  bool primed = false;
  uint16_t *model = nullptr;
};

extern "C" {

// capi.zig:446-469 -> track.zig:17-82.
int visar_background_create(uint32_t width, uint32_t height, int shift, visar_background **out) {
  return guarded([&] {
    if (!out) invalid_arg();
    *out = nullptr;
    if (shift < 0 || shift > 15) invalid_arg();
    std::unique_ptr<visar_background> b(new visar_background);
    ck(cudaGetDevice(&b->dev));
    b->w = width;
    b->h = height;
    b->shift = shift;
    if ((size_t)width * height > 0) ck(cudaMalloc(&b->model, (size_t)width * height * 2));
    *out = b.release();
  });
}

int visar_background_apply(visar_background *b, const visar_image *frame, const visar_image *mask, int threshold) {
  return guarded([&] {
    if (!b) invalid_arg();
    std::lock_guard<std::mutex> lk(g_mu);
    View f = typed(frame, k8U);
    View m = typed(mask, k8U);
    if (f.c->channels != 1 || f.c->width != m.c->width || f.c->height != m.c->height || f.c->channels != m.c->channels ||
        f.c->width != b->w || f.c->height != b->h)
      size_mismatch();
    if (t_hint_dev >= 0 && t_hint_dev != b->dev) invalid_arg();
    t_hint_dev = b->dev;
    Call call = begin_call();
    stage_in(call, f, kSrc);
    stage_out(call, m, kDst);
    ck(launch_background(f.dev, m.dev, b->model, std::min(std::max(threshold, 0), 255), b->shift, b->primed, call.st));
    b->primed = true;
    finish_out(call, m);
    end_call(call, f.host || m.host);
  });
}

void visar_background_free(visar_background *b) {
  if (!b) return;
  if (b->model) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(b->dev);
    cudaFree(b->model);
    cudaSetDevice(cur);
  }
  delete b;
}

// capi.zig:382-386 -> hist.zig:22-45.
int visar_equalize_hist(const visar_image *src, const visar_image *dst) {
  return guarded([&] {
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, k8U);
    View d = typed(dst, k8U);
    if (s.c->channels != 1 || s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels)
      size_mismatch();
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    uint8_t *tab = static_cast<uint8_t *>(scratch(call, kSmall, 2048));
    ck(launch_equalize_hist(s.dev, d.dev, reinterpret_cast<uint32_t *>(tab + 1024), tab, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

// capi.zig:326-337 -> threshold.zig:307-360: the mean (box, or the Gaussian of
// an f32 copy rounded back to 8 bits; replicated border), then the compare.
int visar_adaptive_threshold(const visar_image *src, const visar_image *dst, double maxval, int method, int type,
                             int block, double delta) {
  return guarded([&] {
    if (method != 0 && method != 1) invalid_arg();
    if (type != 0 && type != 1) invalid_arg();
    if (block < 3) invalid_arg();
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, k8U);
    View d = typed(dst, k8U);
    if (s.c->width != d.c->width || s.c->height != d.c->height || s.c->channels != d.c->channels) size_mismatch();
    if (s.c->channels != 1) unsupported_channels();
    if (block % 2 != 1) invalid_kernel();
    // The filters' own kernel limits (boxFilter: 255, f32 gaussianBlur: 127).
    if ((method == 0 && block > 255) || (method == 1 && block > 127)) invalid_kernel();
    const int W = (int)s.c->width, H = (int)s.c->height;
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, d, kDst);
    const size_t pitch = pitch_for(W);
    DImg mean{static_cast<uint8_t *>(scratch(call, kTmp2, pitch * H)), (long long)pitch, W, H, 1};
    SepSpec sp;
    sp.border = kReplicate;
    sp.shift = 0;
    if (method == 0) {
      sp.sdepth = sp.ddepth = k8U;
      sp.scale = 1.0 / (double)(block * block);
      sp.fin = kFinScaled;
      sp.acc = kAccI32;
      sp.kxi.assign(block, 1);
      sp.kyi.assign(block, 1);
      ck(launch_sep_filter(s.dev, mean, sp, call.st));
    } else {
      const size_t fp = pitch_for((long long)W * 4);
      DImg f{static_cast<uint8_t *>(scratch(call, kTmp3, fp * H)), (long long)fp, W, H, 1};
      DImg fb{static_cast<uint8_t *>(scratch(call, kTmp4, fp * H)), (long long)fp, W, H, 1};
      ck(launch_convert_u8_f32(s.dev, f, true, call.st));
      // gaussianBlur f32, sigma 0, kw = kh = block; a 1-pixel axis is not
      // filtered (filter.zig:507-510).
      const int kw = W == 1 ? 1 : block, kh = H == 1 ? 1 : block;
      std::vector<double> kx(kw), ky(kh);
      gaussian_kernel(kx.data(), kw, 0.0);
      gaussian_kernel(ky.data(), kh, 0.0);
      sp.sdepth = sp.ddepth = k32F;
      sp.scale = 1.0;
      sp.fin = kFinCast;
      sp.acc = kAccF32;
      for (double v : kx) sp.kxf.push_back((float)v);
      for (double v : ky) sp.kyf.push_back((float)v);
      ck(launch_sep_filter(f, fb, sp, call.st));
      ck(launch_convert_u8_f32(fb, mean, false, call.st));
    }
    const double rv = std::nearbyint(maxval);
    const uint8_t imax = (uint8_t)(rv != rv ? 0 : rv < 0 ? 0 : rv > 255 ? 255 : rv);
    double dl = type == 0 ? std::ceil(delta) : std::floor(delta);
    dl = dl != dl ? 0 : std::min(std::max(dl, -1024.0), 1024.0);
    ck(launch_adaptive_cmp(s.dev, mean, d.dev, (int)dl, type == 1, imax, call.st));
    finish_out(call, d);
    end_call(call, s.host || d.host);
  });
}

// capi.zig:529-551 -> components.zig:408-543.
int visar_connected_components(const visar_image *src, const visar_image *labels, int connectivity, int32_t *stats,
                               double *centroids, size_t max, size_t *count) {
  return guarded([&] {
    if (!count) invalid_arg();
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, k8U);
    View l = typed(labels, k32S);
    if (s.c->channels != 1 || l.c->channels != 1 || s.c->width != l.c->width || s.c->height != l.c->height)
      size_mismatch();
    const long long W = s.c->width, H = s.c->height, n = W * H;
    if (n >= (1LL << 31) - 1) fail(VISAR_INVALID_ARGUMENT, "InvalidSize");
    const bool eight = connectivity != 4;
    const long long nkeys = eight ? ((W + 1) / 2) * ((H + 1) / 2) : n;
    Call call = begin_call();
    stage_in(call, s, kSrc);
    stage_out(call, l, kDst);
    CcBuffers b;
    b.P = static_cast<int *>(scratch(call, kTmp1, (size_t)n * 4));
    b.K = static_cast<int *>(scratch(call, kTmp2, (size_t)n * 4));
    b.F = static_cast<uint32_t *>(scratch(call, kTmp3, (size_t)nkeys * 4));
    b.R = static_cast<uint32_t *>(scratch(call, kTmp4, (size_t)nkeys * 4));
    b.tmp = static_cast<uint32_t *>(scratch(call, kTab1, cc_scan_tmp_words(nkeys) * 4));
    uint32_t *small = static_cast<uint32_t *>(scratch(call, kSmall, 64));
    b.err = reinterpret_cast<int *>(small);
    b.total = small + 1;
    ck(launch_cc_phase1(s.dev, eight, b, call.st));
    uint32_t hs[2] = {0, 0};
    ck(cudaMemcpyAsync(hs, small, 8, cudaMemcpyDeviceToHost, call.st));
    ck(cudaStreamSynchronize(call.st));
    if (hs[0]) fail(VISAR_INTERNAL, "Internal: union-find did not settle");
    const int nl = (int)hs[1] + 1;
    void *acc = scratch(call, kTab2, (size_t)nl * cc_acc_bytes());
    ck(launch_cc_phase2(l.dev, eight, b, acc, nl, call.st));
    const size_t want = std::min<size_t>(max, (size_t)nl);
    std::vector<uint8_t> hacc(want * cc_acc_bytes());
    if (want && (stats || centroids))
      ck(cudaMemcpyAsync(hacc.data(), acc, hacc.size(), cudaMemcpyDeviceToHost, call.st));
    finish_out(call, l);
    ck(cudaGetLastError());
    ck(cudaStreamSynchronize(call.st));
    *count = (size_t)nl;
    if (!stats && !centroids) return;
    for (size_t i = 0; i < want; i++) {
      long long a[7];
      cc_read_acc(hacc.data(), (int)i, a);
      const long long area = a[4];
      if (stats) {
        int32_t *o = stats + i * 5;
        if (area == 0) {
          o[0] = -1; o[1] = INT32_MAX; o[2] = 0; o[3] = 0; o[4] = 0;
        } else {
          o[0] = (int32_t)a[0]; o[1] = (int32_t)a[1]; o[2] = (int32_t)(a[2] - a[0] + 1); o[3] = (int32_t)(a[3] - a[1] + 1);
          o[4] = (int32_t)area;
        }
      }
      if (centroids) {
        const double ar = (double)std::max<long long>(area, 1);
        centroids[2 * i] = area == 0 ? NAN : (double)a[5] / 2.0 / ar;
        centroids[2 * i + 1] = area == 0 ? NAN : (double)a[6] / ar;
      }
    }
  });
}

// visar_resize(src, dst, INTER_LINEAR) for u8 device images without any
// device allocation: the tap tables go to a static device buffer
// (noalloc.cu). Host images would need staging buffers and overlapping images
// a private source copy, so both are refused rather than allocated.
int visar_resize_linear_u8_noalloc(const visar_image *src, const visar_image *dst) {
  return guarded([&] {
    if (!src || !dst) invalid_arg();
    if (src->depth != VISAR_8U || dst->depth != VISAR_8U) unsupported();
    std::lock_guard<std::mutex> lk(g_mu);
    View s = typed(src, k8U);
    View d = typed(dst, k8U);
    if (s.c->channels != d.c->channels) size_mismatch();
    if (s.c->channels > 4) unsupported_channels();
    if (s.host || d.host) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument: noalloc resize needs device-resident images");
    if (d.c->width > (uint32_t)kNoAllocMaxSide || d.c->height > (uint32_t)kNoAllocMaxSide)
      fail(VISAR_INVALID_ARGUMENT, "InvalidSize: noalloc resize destination is limited to 16384 x 16384");
    if (overlaps(s, d)) fail(VISAR_INVALID_ARGUMENT, "InvalidArgument: noalloc resize needs src and dst apart");
    const int dev = t_hint_dev;
    ck(cudaSetDevice(dev));
    LinTap *taps = nullptr;
    ck(static_taps_on_device(dev, &taps));
    // The thread's stream, else the library's stream if it exists (no stream
    // is created here), else the legacy default stream; ordered after the
    // previous call's stream as begin_call orders calls.
    DevCtx &c = g_ctx[dev];
    const cudaStream_t st = t_stream ? t_stream : c.init ? c.own : cudaStreamLegacy;
    if (c.has_done) ck(cudaStreamWaitEvent(st, c.done, 0));
    if (c.init) {
      t_call_ctx = &c;
      t_call_st = st;
    }
    ck(launch_resize_linear_u8_static(s.dev, d.dev, taps, st));
    ck(cudaGetLastError());
    if (!t_async) ck(cudaStreamSynchronize(st));
  });
}

}  // extern "C"
