// Host-side structures of the batched form, shared by the batch plans
// (batch.cu) and the server (serve.cu): image buffers, shape-class launches,
// per-image fallbacks, stages, the device pool of a plan and the builder
// that turns stages into launches.
#pragma once
#include <cstring>
#include <string>
#include <vector>

#include "../../include/visar_batch.h"
#include "batch.cuh"

namespace vb {
namespace bt {

struct Buf {
  DImg v;
  int depth;
  int input = -1;  // index of the plan input this buffer is, else -1
  // Engine-owned pitched image: every row can be read and written up to its
  // pitch (at least its length rounded up to 8 samples).
  bool padded = false;
};

enum OpKind {
  kOpGauss, kOpMorph, kOpGray, kOpHalf, kOpLinear, kOpLut, kOpWarpAff, kOpWarpPer, kOpGaussStrip, kOpMorphStrip,
  kOpCopy, kOpMorphF
};

inline const char *op_name(int op) {
  switch (op) {
    case kOpGauss: return "gauss";
    case kOpMorph: return "morph";
    case kOpGray: return "gray";
    case kOpHalf: return "half";
    case kOpLinear: return "linear";
    case kOpLut: return "lut";
    case kOpWarpAff: return "warp_affine";
    case kOpWarpPer: return "warp_perspective";
    case kOpGaussStrip: return "gauss_strip";
    case kOpMorphStrip: return "morph_strip";
    case kOpCopy: return "copy";
    case kOpMorphF: return "morph_f";
  }
  return "?";
}

// One persistent launch: one shape class of one stage pass.
struct Launch {
  int op = 0;
  int depth = k8U;
  int cn = 1;
  int k = 0;        // kernel size (Gaussian) / element height (morphology)
  bool is_max = false;
  int rows = 8;     // tile rows (Gaussian band height, elementwise rows)
  int per_sm = 0;   // CTAs per SM (0: as many as fit)
  int vec = 16;     // row-tiled operations: samples (pixels) per thread
  fast::FastArgs fa{};
  fast::MFArgs ma{};
  bool fused = false;
  int sub = 0;      // strip::ProfileId of a morphology strip launch
  int border = 0;
  WarpArgs wa{};
  const uint8_t *lut = nullptr;
  std::vector<BImg> imgs;
  std::vector<int> src_input;  // per image: the plan input it reads, else -1
  size_t bytes = 0;  // algorithmic bytes
  int stage = 0;
  mutable int grid = 0;
  std::string tkey;  // tuning key with the size class (launch_key + ".S|M|L")
  BImg *d_imgs = nullptr;
  int *d_start = nullptr;
  int total = 0;
  int counter = 0;
};

// A per-image call through the per-call entry point.
struct Fallback {
  visar_stage st;
  Buf s, d;
  double m[9];
};

struct Step {
  std::vector<Launch> launches;  // in order (morphology passes are ordered)
  std::vector<Fallback> fallbacks;
};

// Device allocations of a plan: one block, sub-allocated.
struct Pool {
  uint8_t *base = nullptr;
  size_t cap = 0, used = 0;
  void *take(size_t bytes) {
    const size_t off = (used + 255) & ~(size_t)255;
    if (off + bytes > cap) return nullptr;
    used = off + bytes;
    return base + off;
  }
};

// One image of a restriding copy (contiguous host-copy staging <-> pitched
// plan images): rb bytes per row, h rows.
struct StageCopy {
  const uint8_t *src;
  uint8_t *dst;
  long long sstride, dstride;
  int rb, h;
};

// Device staging for host transfers: the images laid out contiguously, so
// each image crosses PCIe as one 1D copy (2D copies of short pitched rows
// run at about half the link rate), then a kernel restrides them.
struct XferStaging {
  uint8_t *buf = nullptr;
  StageCopy *table = nullptr;          // device copy of `rows`
  std::vector<StageCopy> rows;         // as built (pitched side per image)
  std::vector<size_t> off;             // image offsets in buf
  int maxh = 0;
  ~XferStaging() {
    if (buf) cudaFree(buf);
    if (table) cudaFree(table);
  }
};

struct Plan {
  int dev = 0;
  int num_sms = 148;
  std::vector<Buf> inputs;
  std::vector<std::vector<Buf>> outs;  // [stage][image]
  std::vector<Step> steps;
  Pool pool;
  int *counters = nullptr;
  int ncounters = 0;
  size_t pixels_in = 0, bytes = 0, nlaunch = 0, nfallback = 0;
  cudaStream_t own = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool prof = false;
  bool prof_valid = false;
  std::vector<cudaEvent_t> evs;  // 2 per launch when profiling
  XferStaging up, down;          // visar_batch_upload / _download
  ~Plan() {
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
    if (graph) cudaGraphExecDestroy(graph);
    if (pool.base) cudaFree(pool.base);
    if (own) cudaStreamDestroy(own);
  }
};

inline size_t pitch_of(long long rb) { return (size_t)((rb + 255) & ~255LL); }

// Sizes the pool: first pass counts bytes, second pass takes them.
struct Sizer {
  size_t bytes = 0;
  void add(size_t b) { bytes = ((bytes + 255) & ~(size_t)255) + b; }
};

struct Builder {
  Plan &P;
  bool sizing;
  Sizer sz;
  // Host copies of the per-launch device data, uploaded after the pool exists.
  struct Upload {
    void *dst;
    std::vector<uint8_t> data;
  };
  std::vector<Upload> uploads;

  // An external allocator (the server's pool) replaces the plan pool.
  void *(*ext_alloc)(void *ctx, size_t bytes) = nullptr;
  void *ext_ctx = nullptr;

  void *take(size_t bytes) {
    if (sizing) {
      sz.add(bytes);
      return nullptr;
    }
    if (ext_alloc) return ext_alloc(ext_ctx, bytes);
    return P.pool.take(bytes);
  }
  bool image(int w, int h, int cn, int depth, Buf &out) {
    const size_t pitch = pitch_of((long long)w * cn * depth_size(depth));
    void *p = take(pitch * (size_t)h);
    if (!sizing && !p) return false;
    out = Buf{DImg{static_cast<uint8_t *>(p), (long long)pitch, w, h, cn}, depth};
    out.padded = true;
    return true;
  }
  template <class T>
  T *table(const std::vector<T> &v) {
    const size_t bytes = sizeof(T) * std::max<size_t>(1, v.size());
    void *p = take(bytes);
    if (sizing || !p) return static_cast<T *>(p);
    Upload u;
    u.dst = p;
    u.data.resize(bytes);
    if (!v.empty()) std::memcpy(u.data.data(), v.data(), sizeof(T) * v.size());
    uploads.push_back(std::move(u));
    return static_cast<T *>(p);
  }
};


// Stage building and running (batch.cu).
int build_stage(Builder &B, const visar_stage &st, const std::vector<Buf> &cur, std::vector<Buf> &next, Step &step);
cudaError_t run_launch(const Plan &P, const Launch &L, cudaStream_t st);
int run_fallback(const Fallback &f);
int cuda_status(cudaError_t e);
std::string launch_key(const Launch &L);
const char *launch_suffix(const Launch &L);
visar_image cimg(const Buf &b);

}  // namespace bt
}  // namespace vb
