// Host side of the batched form (include/visar_batch.h): plan building,
// shape classes, the device pool, launches, CUDA graph replay and the tuning
// table. Device side: batch.cuh.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/visar_batch.h"
#include "batch.cuh"
#include "batch_plan.h"

namespace vb {
namespace bt {
namespace {

// --------------------------------------------------------------- tuning

std::mutex g_tune_mu;
std::map<std::string, int> g_tune;

int tune_get(const std::string &key, int fallback) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const auto it = g_tune.find(key);
  return it == g_tune.end() ? fallback : it->second;
}

// Reads the flat JSON object the autotuner writes: "key": integer pairs
// (other values are skipped).
bool parse_tune_json(const std::string &txt, std::map<std::string, int> &out) {
  size_t i = 0;
  const size_t n = txt.size();
  while (i < n) {
    const size_t q0 = txt.find('"', i);
    if (q0 == std::string::npos) break;
    const size_t q1 = txt.find('"', q0 + 1);
    if (q1 == std::string::npos) return false;
    const std::string key = txt.substr(q0 + 1, q1 - q0 - 1);
    size_t j = q1 + 1;
    while (j < n && (txt[j] == ' ' || txt[j] == '\t' || txt[j] == '\n' || txt[j] == '\r')) j++;
    if (j < n && txt[j] == ':') {
      j++;
      while (j < n && (txt[j] == ' ' || txt[j] == '\t' || txt[j] == '\n' || txt[j] == '\r')) j++;
      if (j < n && (txt[j] == '-' || (txt[j] >= '0' && txt[j] <= '9'))) {
        char *end = nullptr;
        const long v = std::strtol(txt.c_str() + j, &end, 10);
        out[key] = (int)v;
        j = (size_t)(end - txt.c_str());
      } else if (j < n && txt[j] == '"') {
        const size_t e = txt.find('"', j + 1);  // string value: skipped
        if (e == std::string::npos) return false;
        j = e + 1;
      }
    }
    i = j;
  }
  return true;
}

}  // namespace

// ----------------------------------------------------------------- plan

// Size class of a launch: mean destination pixels per image, S < 0.25 MP <=
// M < 2 MP <= L, with "1" appended for a single image (a lone frame needs
// short tiles to fill the GPU where a batch of the same images does not).
std::string size_class(const std::vector<BImg> &imgs) {
  double px = 0;
  for (const BImg &b : imgs) px += (double)b.d.w * b.d.h;
  px /= std::max<size_t>(1, imgs.size());
  std::string sc = px < 250e3 ? "S" : px < 2e6 ? "M" : "L";
  if (imgs.size() == 1) sc += "1";
  return sc;
}

const char *launch_suffix(const Launch &L) {
  if (L.op != kOpMorph && L.op != kOpMorphStrip && L.op != kOpMorphF) return "";
  if (L.fused) return L.is_max ? ".close" : ".open";
  return L.is_max ? ".max" : ".min";
}

// Tuning key of a launch class: op.depth.c<channels>.k<size>, the compiled
// element profile of a morphology strip, the pass (.min/.max/.open/.close).
std::string launch_key(const Launch &L) {
  static const char *const prof[strip::kProfileCount] = {"rect3", "rect5", "rect7", "cross3",
                                                         "cross5", "ell5", "ell7"};
  char buf[96];
  std::snprintf(buf, sizeof(buf), "%s.%s.c%d.k%d%s%s%s", op_name(L.op), L.depth == k32F ? "f32" : "u8", L.cn, L.k,
                L.op == kOpMorphStrip ? "." : "",
                L.op == kOpMorphStrip && L.sub >= 0 && L.sub < strip::kProfileCount ? prof[L.sub] : "",
                launch_suffix(L));
  return buf;
}

Launch *class_of(std::vector<Launch> &ls, int op, int depth, int cn, int k, bool is_max, bool fused = false,
                 int sub = 0) {
  for (Launch &l : ls)
    if (l.op == op && l.depth == depth && l.cn == cn && l.k == k && l.is_max == is_max && l.fused == fused &&
        l.sub == sub)
      return &l;
  ls.emplace_back();
  Launch &l = ls.back();
  l.sub = sub;
  l.op = op;
  l.depth = depth;
  l.cn = cn;
  l.k = k;
  l.is_max = is_max;
  l.fused = fused;
  return &l;
}

// The packed strip Gaussian applies when the fixed taps are g * binomial(k)
// with g = 256 / 2^(k-1) (the sigma <= 0 tables of 3x3 and 5x5).
bool binomial_taps(const std::vector<int64_t> &t) {
  const int k = (int)t.size();
  if (k != 3 && k != 5) return false;
  static const int b3[3] = {1, 2, 1}, b5[5] = {1, 4, 6, 4, 1};
  const int *b = k == 3 ? b3 : b5;
  const int64_t g = k == 3 ? 64 : 16;
  for (int j = 0; j < k; j++)
    if (t[j] != g * b[j]) return false;
  return true;
}

// Per-row half-widths of an element made of runs centred on the anchor
// column (-1: empty row); false for any other element.
bool row_profile(const std::vector<uint8_t> &mask, int kw, int kh, int *d) {
  if (kw % 2 == 0 || kh % 2 == 0 || kh > 16) return false;
  const int ax = kw / 2;
  for (int y = 0; y < kh; y++) {
    int j1 = -1, j2 = -1;
    for (int x = 0; x < kw; x++)
      if (mask[(size_t)y * kw + x]) {
        if (j1 < 0) j1 = x;
        j2 = x;
      }
    if (j1 < 0) {
      d[y] = -1;
      continue;
    }
    for (int x = j1; x <= j2; x++)
      if (!mask[(size_t)y * kw + x]) return false;
    if (ax - j1 != j2 - ax) return false;
    d[y] = ax - j1;
  }
  return true;
}

// Strip halo words of a morphology launch (strip.cuh MorphStrip::HALO).
int strip_halo(int prof, int cn, bool fused) {
  const int m = strip::profile_maxd(prof) * (fused ? 2 : 1) * cn;
  return std::max(1, (m + strip::kSPL - 1) / strip::kSPL);
}

int gauss_tiles_x(int w, int cn, int k) {
  const int hw = ((k / 2) * cn + 3) / 4;
  return (int)ceil_div(((long long)w * cn + 3) / 4, 128 - 2 * hw);
}

// Row-tiled operations (256 threads, P samples per thread): threads per row
// = the smallest power of two covering the row's units, at most 256.
void row_tiles(BImg &b, long long units, int P, int rows, int h) {
  const long long per = ceil_div(units, P);
  int lg = 0;
  while (lg < 8 && (1LL << lg) < per) lg++;
  b.lanes = lg;
  b.tiles_x = (int)ceil_div(per, 1LL << lg);
  b.tiles_y = (int)ceil_div(h, (long long)rows * (256 >> lg));
}

// One-channel u8 warps with linear interpolation run OpWarp4 (4 pixels per
// thread, tiles of 32 x L.wa.rows).
bool warp4_class(const Launch &L) {
  return (L.op == kOpWarpAff || L.op == kOpWarpPer) && L.depth == k8U && L.cn == 1 && L.wa.interp != 0;
}

// Tiles per image of an operation, for the launch's tuned parameters.
void set_tiles(const Launch &L, BImg &b) {
  switch (L.op) {
    case kOpGauss:
      b.tiles_x = gauss_tiles_x(b.s.w, L.cn, L.k);
      b.tiles_y = (int)ceil_div(b.s.h, L.rows);
      break;
    case kOpMorph:
      b.tiles_x = (int)ceil_div(((long long)b.s.w * L.cn + 3) / 4, 126);
      b.tiles_y = (int)ceil_div(b.s.h, 8);
      break;
    case kOpGray: row_tiles(b, b.s.w, L.vec, L.rows, b.s.h); break;
    case kOpCopy: row_tiles(b, (long long)b.s.w * b.s.cn * depth_size(L.depth), OpCopy::P, L.rows, b.s.h); break;
    case kOpMorphF: row_tiles(b, b.s.w, 1, L.rows, b.s.h); break;
    case kOpHalf: row_tiles(b, b.d.w, L.vec, L.rows, b.d.h); break;
    case kOpLinear:
      if (L.cn == 1 && L.depth == k8U) {  // OpLinearStrip warp tiles
        b.tiles_x = (int)ceil_div(b.d.w, OpLinearStrip::kTW);
        b.tiles_y = (int)ceil_div(b.d.h, L.rows);
      } else {
        row_tiles(b, b.d.w, 1, L.rows, b.d.h);
      }
      break;
    case kOpLut: row_tiles(b, (long long)b.s.w * b.s.cn, L.vec, L.rows, b.s.h); break;
    case kOpGaussStrip: {
      const int halo = ((L.k / 2) * L.cn + strip::kSPL - 1) / strip::kSPL;
      b.tiles_x = (int)ceil_div((long long)b.s.w * L.cn, strip::kSPL * (32 - 2 * halo));
      b.tiles_y = (int)ceil_div(b.s.h, L.rows);
      break;
    }
    case kOpMorphStrip:
      b.tiles_x = (int)ceil_div((long long)b.s.w * L.cn, strip::kSPL * (32 - 2 * strip_halo(L.sub, L.cn, L.fused)));
      b.tiles_y = (int)ceil_div(b.s.h, L.rows);
      break;
    case kOpWarpAff: case kOpWarpPer:
      b.tiles_x = (int)ceil_div(b.d.w, 32);
      b.tiles_y = (int)ceil_div(b.d.h, warp4_class(L) ? L.wa.rows : 32);
      break;
    default:
      b.tiles_x = (int)ceil_div(b.d.w, 32);
      b.tiles_y = (int)ceil_div(b.d.h, 32);
  }
}

// Applies the tuning table to a finished class, then tiles its images.
long long total_tiles(const Launch &L) {
  long long t = 0;
  for (const BImg &b : L.imgs) t += (long long)b.tiles_x * b.tiles_y;
  return t;
}

// Applies the tuning table to a finished class, then tiles its images. A
// tuned value wins; otherwise tile heights shrink until the class has
// enough tiles to occupy the GPU (single large frames need short tiles,
// large batches take tall ones, which cut halo re-reads and queue traffic).
void tune_and_tile(Launch &L, int num_sms) {
  const std::string key = launch_key(L);
  const std::string sc = size_class(L.imgs);
  L.tkey = key + "." + sc;
  auto get = [&](const char *field, int def) {
    return tune_get(L.tkey + "." + field, tune_get(key + "." + field, def));
  };
  auto retile = [&]() {
    for (BImg &b : L.imgs) set_tiles(L, b);
  };
  const int tuned = get("rows", -1);
  switch (L.op) {
    case kOpGauss:
      L.rows = tuned == 8 || tuned == 16 || tuned == 32 ? tuned : 16;
      retile();
      break;
    case kOpLinear:
      if (L.cn == 1 && L.depth == k8U) {
        // Warp tiles: the tallest of 32..4 rows leaving ~8 tiles per warp slot.
        L.vec = 1;
        if (tuned > 0) {
          L.rows = std::min(tuned, 64);
          retile();
          break;
        }
        for (const int rh : {32, 16, 8, 4}) {
          L.rows = rh;
          retile();
          if (total_tiles(L) >= 8LL * num_sms * 24) break;
        }
        break;
      }
      [[fallthrough]];
    case kOpGray: case kOpHalf: case kOpLut: case kOpCopy: case kOpMorphF: {
      // Samples per thread (vector width): 8 or 16 bytes for u8 gray and the
      // LUT, 4 or 8 output pixels for the halving (fixed for the others).
      const int vec = get("vec", -1);
      if (L.op == kOpHalf) L.vec = vec == 8 ? 8 : 4;
      else if (L.op == kOpLinear) L.vec = 1;
      else if (L.op == kOpCopy) L.vec = OpCopy::P;
      else if (L.op == kOpMorphF) L.vec = 1;
      else if (L.op == kOpGray && L.depth == k32F) L.vec = OpGrayF<3>::P;
      else L.vec = vec == 8 ? 8 : 16;
      // Enough CTA tiles for ~8 per SM.
      L.rows = tuned > 0 ? std::min(tuned, 64) : 8;
      retile();
      while (tuned <= 0 && L.rows > 1 && total_tiles(L) < 8LL * num_sms) {
        L.rows /= 2;
        retile();
      }
      break;
    }
    case kOpGaussStrip: case kOpMorphStrip: {
      // Warp tiles of 128 (one-channel images), 64 (Gaussian, one-channel
      // morphology), 32 or 8 rows: by default the tallest that leaves ~4
      // (128 rows) or ~8 (shorter tiles) tiles per resident warp slot --
      // taller tiles re-read fewer halo rows, and 128-row tiles save enough
      // of them to outweigh a longer tail.
      const bool has64 = L.op == kOpGaussStrip || L.cn == 1;
      if (tuned == 8 || tuned == 32 || (tuned == 64 && has64) || (tuned == 128 && L.cn == 1)) {
        L.rows = tuned;
        retile();
        break;
      }
      for (const int rh : {128, 64, 32, 8}) {
        if ((rh == 64 && !has64) || (rh == 128 && L.cn != 1)) continue;
        L.rows = rh;
        retile();
        if (total_tiles(L) >= (rh == 128 ? 4LL : 8LL) * num_sms * 24) break;
      }
      break;
    }
    case kOpWarpAff: case kOpWarpPer:
      // One-channel u8 linear warps (OpWarp4): tiles of 32 x 32..256 rows.
      L.rows = 8;
      L.wa.rows = tuned == 32 || tuned == 64 || tuned == 128 || tuned == 256 ? tuned : OpWarp4<true>::kDefaultRows;
      retile();
      break;
    default:
      L.rows = 8;
      retile();
  }
  L.per_sm = std::max(0, get("per_sm", 0));
}

bool u8_aligned4(const DImg &v) { return ((uintptr_t)v.p % 4 == 0) && (v.stride % 4 == 0); }
bool u8_aligned8(const DImg &v) { return ((uintptr_t)v.p % 8 == 0) && (v.stride % 8 == 0); }
bool aligned16(const DImg &v) { return ((uintptr_t)v.p % 16 == 0) && (v.stride % 16 == 0); }

BImg bimg(const DImg &s, const DImg &d) {
  BImg b{};
  b.s = s;
  b.d = d;
  return b;
}

void add_img(Launch *l, const BImg &b, int input) {
  l->imgs.push_back(b);
  l->src_input.push_back(input);
}

void u8_bytes(Launch &L, const DImg &s, const DImg &d, int esize) {
  L.bytes += ((size_t)s.w * s.h * s.cn + (size_t)d.w * d.h * d.cn) * (size_t)esize;
}

// ------------------------------------------------------------- stages

// Builds one stage over `cur`, writing its outputs to `next`. Returns a
// VISAR status.
int build_stage(Builder &B, const visar_stage &st, const std::vector<Buf> &cur, std::vector<Buf> &next, Step &step) {
  const size_t n = cur.size();
  next.resize(n);
  std::vector<Launch> ls;
  auto fallback = [&](size_t i, const Buf &out, const double *m) {
    Fallback f;
    f.st = st;
    f.s = cur[i];
    f.d = out;
    std::memset(f.m, 0, sizeof(f.m));
    if (m) std::memcpy(f.m, m, sizeof(double) * (st.kind == VISAR_STAGE_WARP_AFFINE ? 6 : 9));
    step.fallbacks.push_back(f);
  };
  // u8 inputs whose rows are not 8-byte aligned and f32 inputs whose rows are
  // not 16-byte aligned (caller-owned images) are first copied, in one
  // batched launch, into pitched pool images, so the stencil classes that
  // need aligned rows take them instead of the per-call fallback.
  std::vector<Buf> src(cur.begin(), cur.end());
  // ragged: also u8 images of the caller whose rows are not a multiple of 8
  // bytes (the strips read rows up to that rounding; plan images are padded
  // to it).
  auto repack_unaligned = [&](bool ragged = false) -> int {
    for (size_t i = 0; i < n; i++) {
      const Buf &im = cur[i];
      // u8 rows that are not 8-byte aligned (strips), f32 rows that are not
      // 16-byte aligned (band kernels).
      const bool unaligned =
          im.depth == k8U ? !u8_aligned8(im.v) || (ragged && !im.padded && ((long long)im.v.w * im.v.cn) % 8 != 0)
                          : im.depth == k32F && !aligned16(im.v);
      if (!unaligned || im.v.w < 2 || im.v.h < 2) continue;
      if (im.v.cn != 1 && im.v.cn != 3 && im.v.cn != 4) continue;
      Buf t;
      if (!B.image(im.v.w, im.v.h, im.v.cn, im.depth, t)) return VISAR_OUT_OF_MEMORY;
      Launch *l = class_of(ls, kOpCopy, im.depth, im.v.cn, 0, false);
      add_img(l, bimg(im.v, t.v), im.input);
      u8_bytes(*l, im.v, t.v, depth_size(im.depth));
      src[i] = t;
    }
    for (Launch &l : ls) {
      tune_and_tile(l, B.P.num_sms);
      step.launches.push_back(std::move(l));
    }
    ls.clear();
    return VISAR_OK;
  };
  switch (st.kind) {
    case VISAR_STAGE_GRAY: {
      for (size_t i = 0; i < n; i++) {
        const Buf &im = cur[i];
        if (im.v.cn == 1) {
          next[i] = im;
          continue;
        }
        if (im.v.cn != 3 && im.v.cn != 4) return VISAR_UNSUPPORTED;
        if (!B.image(im.v.w, im.v.h, 1, im.depth, next[i])) return VISAR_OUT_OF_MEMORY;
        if (im.depth != k8U && im.depth != k32F) {
          fallback(i, next[i], nullptr);
          continue;
        }
        Launch *l = class_of(ls, kOpGray, im.depth, im.v.cn, 0, false);
        add_img(l, bimg(im.v, next[i].v), im.input);
        u8_bytes(*l, im.v, next[i].v, depth_size(im.depth));
      }
      break;
    }
    case VISAR_STAGE_GAUSSIAN: {
      const int kw_in = st.i[0], kh_in = st.i[1], border = st.i[2];
      const double sx = st.d[0], sy = st.d[1] > 0 ? st.d[1] : st.d[0];
      if (border < 0 || border > 4) return VISAR_UNSUPPORTED;
      if (kw_in < 0 || kh_in < 0) return VISAR_INVALID_ARGUMENT;
      if (const int rc = repack_unaligned(true); rc != VISAR_OK) return rc;
      // The taps depend only on the size and the depth class: computed once
      // per stage (a served round holds hundreds of images of one stage).
      std::map<int, std::vector<int64_t>> fixed_taps;
      std::map<int, std::vector<double>> f_taps;
      auto fixed_of = [&](int kw) -> const std::vector<int64_t> & {
        auto it = fixed_taps.find(kw);
        if (it == fixed_taps.end()) {
          std::vector<int64_t> t(kw);
          gaussian_kernel_fixed(t.data(), kw, sx, 8);
          it = fixed_taps.emplace(kw, std::move(t)).first;
        }
        return it->second;
      };
      auto float_of = [&](int kw) -> const std::vector<double> & {
        auto it = f_taps.find(kw);
        if (it == f_taps.end()) {
          std::vector<double> t(kw);
          gaussian_kernel(t.data(), kw, sx);
          it = f_taps.emplace(kw, std::move(t)).first;
        }
        return it->second;
      };
      for (size_t i = 0; i < n; i++) {
        const Buf &im = src[i];
        if (!B.image(im.v.w, im.v.h, im.v.cn, im.depth, next[i])) return VISAR_OUT_OF_MEMORY;
        const bool u8 = im.depth == k8U;
        const int kw = kw_in > 0 ? kw_in : gaussian_ksize(sx, u8);
        const int kh = kh_in > 0 ? kh_in : gaussian_ksize(sy, u8);
        if (kw <= 0 || kh <= 0 || kw % 2 == 0 || kh % 2 == 0 || kw > 127 || kh > 127) return VISAR_INVALID_ARGUMENT;
        bool ok = (im.depth == k8U || im.depth == k32F) && kw == kh && sx == sy && (kw == 3 || kw == 5 || kw == 7) &&
                  (im.v.cn == 1 || im.v.cn == 3 || im.v.cn == 4) && im.v.w > 1 && im.v.h > 1;
        ok = ok && (u8 ? u8_aligned4(im.v) : aligned16(im.v));
        fast::FastArgs a{};
        if (ok) {
          a.border = border;
          a.symx = a.symy = 1;
          if (u8) {
            const std::vector<int64_t> &t = fixed_of(kw);
            long long sum = 0;
            for (int j = 0; j < kw; j++) {
              ok = ok && t[j] >= 0 && t[j] == t[kw - 1 - j];
              sum += t[j];
              a.kx[j] = a.ky[j] = (float)t[j];
            }
            ok = ok && sum <= 256;
            a.shift = 16;
          } else {
            const std::vector<double> &t = float_of(kw);
            for (int j = 0; j < kw; j++) {
              const float f = (float)t[j];
              ok = ok && f >= 0.0f && f == (float)t[kw - 1 - j];
              a.kx[j] = a.ky[j] = f;
            }
          }
        }
        if (!ok) {
          fallback(i, next[i], nullptr);
          continue;
        }
        if (u8) {
          const std::vector<int64_t> &t = fixed_of(kw);
          // Strips map rows past the bottom edge in closed form (images taller
          // than the radius), take border columns from their own row window
          // (not the far end of the row: no wrap), and read and write whole
          // 8-byte words (padded rows or rows of 8-byte multiples).
          const bool words = im.padded || ((long long)im.v.w * im.v.cn) % 8 == 0;
          if (binomial_taps(t) && u8_aligned8(im.v) && im.v.h > kw / 2 && border != kWrap && next[i].padded && words) {
            Launch *l = class_of(ls, kOpGaussStrip, k8U, im.v.cn, kw, false);
            l->border = border;
            add_img(l, bimg(im.v, next[i].v), im.input);
            u8_bytes(*l, im.v, next[i].v, 1);
            continue;
          }
        }
        Launch *l = class_of(ls, kOpGauss, im.depth, im.v.cn, kw, false);
        l->fa = a;
        add_img(l, bimg(im.v, next[i].v), im.input);
        u8_bytes(*l, im.v, next[i].v, depth_size(im.depth));
      }
      break;
    }
    case VISAR_STAGE_MORPHOLOGY: {
      const int op = st.i[0], shape = st.i[1], kw = st.i[2], kh = st.i[3], it = st.i[4];
      if (op < 0 || op > 6 || shape < 0 || shape > 2) return VISAR_UNSUPPORTED;
      if (kw <= 0 || kh <= 0 || kw > 255 || kh > 255 || it < 0) return VISAR_INVALID_ARGUMENT;
      const std::vector<uint8_t> mask = structuring_element(shape, kw, kh);
      // The passes of ops 0-3 (morph.zig:71-96, 560-593): erode/dilate `it` times each.
      std::vector<bool> passes;
      auto add = [&](bool mx) {
        for (int j = 0; j < it; j++) passes.push_back(mx);
      };
      if (op == 0) add(false);
      else if (op == 1) add(true);
      else if (op == 2) { add(false); add(true); }
      else if (op == 3) { add(true); add(false); }
      const bool kernel_ok = op <= 3 && !passes.empty();
      // OPEN / CLOSE of one iteration whose two horizontal reaches fit one
      // halo word run as one fused strip launch; other covered shapes run
      // pass by pass (ping-ponging through temporaries).
      // Elements with a compiled profile run on warp strips: OPEN / CLOSE of
      // one iteration as one fused launch, other cases pass by pass
      // (ping-ponging through temporaries); other centred-run elements with
      // a short reach use the band kernel pass by pass.
      int dprof[16];
      const int prof = row_profile(mask, kw, kh, dprof) ? strip::profile_of(dprof, kh) : strip::kProfileCount;
      std::vector<std::vector<Buf>> tmp(n);
      std::vector<int> mode(n, 0);  // 0 fallback, 1 strip passes, 2 fused strip, 3 band passes, 4 f32 rectangle passes
      const bool rect = std::all_of(mask.begin(), mask.end(), [](uint8_t m) { return m != 0; });
      if (kernel_ok) {
        if (const int rc = repack_unaligned(true); rc != VISAR_OK) return rc;
      }
      for (size_t i = 0; i < n; i++) {
        const Buf &im = src[i];
        if (!B.image(im.v.w, im.v.h, im.v.cn, im.depth, next[i])) return VISAR_OUT_OF_MEMORY;
        const bool u8ok = kernel_ok && im.depth == k8U && (im.v.cn == 1 || im.v.cn == 3 || im.v.cn == 4) &&
                          u8_aligned4(im.v);
        fast::MFArgs ma;
        // Strips read and write whole 8-byte words (padded rows or rows of
        // 8-byte multiples).
        const bool strip_ok = u8ok && prof < strip::kProfileCount && u8_aligned8(im.v) && next[i].padded &&
                              (im.padded || ((long long)im.v.w * im.v.cn) % 8 == 0);
        if (strip_ok && strip_halo(prof, im.v.cn, true) <= 8 && (op == 2 || op == 3) && it == 1) {
          mode[i] = 2;
          Launch *l = class_of(ls, kOpMorphStrip, k8U, im.v.cn, kh, op == 3, true, prof);
          add_img(l, bimg(im.v, next[i].v), im.input);
          u8_bytes(*l, im.v, next[i].v, 1);
          continue;
        }
        if (strip_ok) mode[i] = 1;
        else if (u8ok && fast::morph_fast_args(mask, kw, kh, im.v.cn, im.v.w, ma)) mode[i] = 3;
        else if (kernel_ok && im.depth == k32F && rect && kw <= 15 && kh <= 15 && im.v.cn <= 4) mode[i] = 4;
        if (mode[i] == 0) {
          fallback(i, next[i], nullptr);
          continue;
        }
        const size_t ntmp = std::min<size_t>(passes.size() - 1, 2);
        tmp[i].resize(ntmp);
        for (size_t k = 0; k < ntmp; k++)
          if (!B.image(im.v.w, im.v.h, im.v.cn, im.depth, tmp[i][k])) return VISAR_OUT_OF_MEMORY;
      }
      for (Launch &l : ls) {
        tune_and_tile(l, B.P.num_sms);
        step.launches.push_back(std::move(l));
      }
      ls.clear();
      const size_t np = passes.size();
      for (size_t p = 0; p < np && kernel_ok; p++) {
        std::vector<Launch> pl;
        for (size_t i = 0; i < n; i++) {
          if (mode[i] != 1 && mode[i] != 3 && mode[i] != 4) continue;
          const Buf &im = src[i];
          const DImg from = p == 0 ? im.v : tmp[i][(p - 1) % 2].v;
          const DImg dst = p + 1 == np ? next[i].v : tmp[i][p % 2].v;
          Launch *l;
          if (mode[i] == 1) {
            l = class_of(pl, kOpMorphStrip, k8U, im.v.cn, kh, passes[p], false, prof);
          } else if (mode[i] == 4) {
            l = class_of(pl, kOpMorphF, k32F, im.v.cn, kh, passes[p], false, kw);
          } else {
            l = class_of(pl, kOpMorph, k8U, im.v.cn, kh, passes[p]);
            fast::morph_fast_args(mask, kw, kh, im.v.cn, im.v.w, l->ma);
          }
          add_img(l, bimg(from, dst), p == 0 ? im.input : -1);
          u8_bytes(*l, from, dst, depth_size(im.depth));
        }
        for (Launch &l : pl) {
          tune_and_tile(l, B.P.num_sms);
          step.launches.push_back(std::move(l));
        }
      }
      return VISAR_OK;
    }
    case VISAR_STAGE_RESIZE: {
      const int interp = st.i[0];
      const double fx = st.d[0], fy = st.d[1];
      if (interp < 0 || interp > 4) return VISAR_UNSUPPORTED;
      if (!(fx > 0) || !(fy > 0) || !std::isfinite(fx) || !std::isfinite(fy)) return VISAR_INVALID_ARGUMENT;
      // Tap tables depend only on (source, destination) lengths per axis:
      // images of equal sizes share one device table (read only).
      std::map<std::tuple<int, int, int, int>, const void *> tabs;  // (f32, axis, src, dst)
      auto table_of = [&](bool f32, int axis, int sn, int dn) -> const void * {
        const auto key = std::make_tuple(f32 ? 1 : 0, axis, sn, dn);
        auto it = tabs.find(key);
        if (it != tabs.end()) return it->second;
        const void *t;
        if (f32) {
          std::vector<FLinTap> v(dn);
          for (int k = 0; k < dn; k++) v[k] = lin_tap_f(k, sn, dn, false, axis == 0);
          t = B.table(v);
        } else {
          std::vector<LinTap> v(dn);
          for (int k = 0; k < dn; k++) v[k] = lin_tap_u8(k, sn, dn, false, axis == 0);
          t = B.table(v);
        }
        tabs.emplace(key, t);
        return t;
      };
      for (size_t i = 0; i < n; i++) {
        const Buf &im = cur[i];
        const double wd = std::floor((double)im.v.w * fx), hd = std::floor((double)im.v.h * fy);
        if (wd > 1e9 || hd > 1e9) return VISAR_INVALID_ARGUMENT;
        const int dw = std::max(1, (int)wd), dh = std::max(1, (int)hd);
        if (dw == im.v.w && dh == im.v.h && interp != 4) {
          next[i] = im;  // VISAR copies; the pixels are the input's
          continue;
        }
        if (interp == 4) return VISAR_UNSUPPORTED;
        if (!B.image(dw, dh, im.v.cn, im.depth, next[i])) return VISAR_OUT_OF_MEMORY;
        const bool f32lin = im.depth == k32F && im.v.cn <= 4 && interp == 1;
        if (f32lin) {  // the generic f32 path (resize.zig:284-423), exact halves included
          BImg b = bimg(im.v, next[i].v);
          b.t0 = table_of(true, 0, im.v.w, dw);
          b.t1 = table_of(true, 1, im.v.h, dh);
          if (!B.sizing && (!b.t0 || !b.t1)) return VISAR_OUT_OF_MEMORY;
          Launch *l = class_of(ls, kOpLinear, k32F, im.v.cn, 0, false);
          add_img(l, b, im.input);
          u8_bytes(*l, im.v, next[i].v, 4);
          continue;
        }
        const bool u8lin = im.depth == k8U && im.v.cn <= 4 && interp == 1;
        if (!u8lin) {
          fallback(i, next[i], nullptr);
          continue;
        }
        if (im.v.w == 2 * dw && im.v.h == 2 * dh) {
          Launch *l = class_of(ls, kOpHalf, k8U, im.v.cn, 0, false);
          add_img(l, bimg(im.v, next[i].v), im.input);
          u8_bytes(*l, im.v, next[i].v, 1);
        } else {
          BImg b = bimg(im.v, next[i].v);
          b.t0 = table_of(false, 0, im.v.w, dw);
          b.t1 = table_of(false, 1, im.v.h, dh);
          if (!B.sizing && (!b.t0 || !b.t1)) return VISAR_OUT_OF_MEMORY;
          Launch *l = class_of(ls, kOpLinear, k8U, im.v.cn, 0, false);
          add_img(l, b, im.input);
          u8_bytes(*l, im.v, next[i].v, 1);
        }
      }
      break;
    }
    case VISAR_STAGE_THRESHOLD: {
      const int type = st.i[0];
      const int kind = type & 7;
      if (kind > 4) return VISAR_UNSUPPORTED;
      const bool autoth = (type & 24) != 0;
      const double fl = std::floor(st.d[0]);
      const int ti = fl != fl ? 0 : fl < -1e9 ? -1000000000 : fl > 1e9 ? 1000000000 : (int)fl;
      const double r = std::nearbyint(st.d[1]);
      const uint8_t m = st.d[1] != st.d[1] ? 0 : r <= 0 ? 0 : r >= 255 ? 255 : (uint8_t)(int)r;
      // threshold.zig:39-60: the u8 table of every type.
      std::vector<uint8_t> lut(256);
      const uint8_t tsat = (uint8_t)std::min(std::max(ti, 0), 255);
      for (int v = 0; v < 256; v++) {
        const bool gt = v > ti;
        switch (kind) {
          case 0: lut[v] = gt ? m : 0; break;
          case 1: lut[v] = gt ? 0 : m; break;
          case 2: lut[v] = gt ? tsat : (uint8_t)v; break;
          case 3: lut[v] = gt ? (uint8_t)v : 0; break;
          default: lut[v] = gt ? 0 : (uint8_t)v; break;
        }
      }
      const uint8_t *dlut = nullptr;
      for (size_t i = 0; i < n; i++) {
        const Buf &im = cur[i];
        if (!B.image(im.v.w, im.v.h, im.v.cn, im.depth, next[i])) return VISAR_OUT_OF_MEMORY;
        if (im.depth != k8U || autoth) {
          fallback(i, next[i], nullptr);
          continue;
        }
        if (!dlut) {
          dlut = B.table(lut);
          if (!B.sizing && !dlut) return VISAR_OUT_OF_MEMORY;
        }
        Launch *l = class_of(ls, kOpLut, k8U, 0, 0, false);
        l->lut = dlut;
        add_img(l, bimg(im.v, next[i].v), im.input);
        u8_bytes(*l, im.v, next[i].v, 1);
      }
      break;
    }
    case VISAR_STAGE_WARP_AFFINE:
    case VISAR_STAGE_WARP_PERSPECTIVE: {
      const bool persp = st.kind == VISAR_STAGE_WARP_PERSPECTIVE;
      const int interp = st.i[0] == 0 ? 0 : 1, border = st.i[1];
      if (border < 0 || border > 4) return VISAR_UNSUPPORTED;
      const double value = persp ? st.d[9] : st.d[6];
      const int nm = persp ? 9 : 6;
      for (size_t i = 0; i < n; i++) {
        const Buf &im = cur[i];
        const double *m = st.per_image ? st.per_image + i * nm : st.d;
        BImg b = bimg(im.v, DImg{});
        if (persp) {
          if (!perspective_inverse(m, b.md)) return VISAR_UNSUPPORTED;
        } else {
          if (!affine_inverse_f32(m, b.mf)) return VISAR_UNSUPPORTED;
        }
        if (!B.image(im.v.w, im.v.h, im.v.cn, im.depth, next[i])) return VISAR_OUT_OF_MEMORY;
        b.d = next[i].v;
        const bool ok = (im.depth == k8U || im.depth == k32F) && (im.v.cn == 1 || im.v.cn == 3 || im.v.cn == 4) &&
                        (im.depth != k8U || im.v.cn != 4 || u8_aligned4(im.v)) &&
                        (im.depth != k32F || ((uintptr_t)im.v.p % 4 == 0 && im.v.stride % 4 == 0));
        if (!ok) {
          fallback(i, next[i], m);
          continue;
        }
        b.cv = im.depth == k8U ? wp::sat_value_host<uint8_t>(value) : wp::sat_value_host<float>(value);
        b.wide = ((uintptr_t)im.v.p % 8 == 0) && (im.v.stride % 8 == 0);
        Launch *l = class_of(ls, persp ? kOpWarpPer : kOpWarpAff, im.depth, im.v.cn, 0, false);
        l->wa = WarpArgs{interp, border, 32};
        add_img(l, b, im.input);
        u8_bytes(*l, im.v, next[i].v, depth_size(im.depth));
      }
      break;
    }
    default:
      return VISAR_UNSUPPORTED;
  }
  for (Launch &l : ls) {
    tune_and_tile(l, B.P.num_sms);
    step.launches.push_back(std::move(l));
  }
  return VISAR_OK;
}

int build_all(Builder &B, const std::vector<visar_stage> &stages) {
  Plan &P = B.P;
  P.steps.clear();
  P.outs.clear();
  std::vector<Buf> cur = P.inputs;
  for (const visar_stage &st : stages) {
    Step step;
    std::vector<Buf> next;
    const int rc = build_stage(B, st, cur, next, step);
    if (rc != VISAR_OK) return rc;
    for (Launch &l : step.launches) l.stage = (int)P.steps.size();
    P.steps.push_back(std::move(step));
    P.outs.push_back(next);
    cur = next;
  }
  return VISAR_OK;
}

// ------------------------------------------------------------------ run

LaunchRun run_of(const Plan &P, const Launch &L) {
  return LaunchRun{TileQ{L.d_imgs, L.d_start, (int)L.imgs.size(), L.total, P.counters + L.counter}, L.per_sm, P.num_sms,
                   &L.grid};
}

template <class Op>
cudaError_t run_op(const Plan &P, const Launch &L, const typename Op::Args &a, cudaStream_t st) {
  return launch_op<Op>(run_of(P, L), a, st);
}

template <class S, int K, int CN>
cudaError_t run_gauss_rows(const Plan &P, const Launch &L, cudaStream_t st) {
  switch (L.rows) {
    case 8: return run_op<OpGauss<S, K, CN, 8>>(P, L, L.fa, st);
    case 32: return run_op<OpGauss<S, K, CN, 32>>(P, L, L.fa, st);
    default: return run_op<OpGauss<S, K, CN, 16>>(P, L, L.fa, st);
  }
}

template <class S, int CN>
cudaError_t run_gauss_k(const Plan &P, const Launch &L, cudaStream_t st) {
  switch (L.k) {
    case 3: return run_gauss_rows<S, 3, CN>(P, L, st);
    case 5: return run_gauss_rows<S, 5, CN>(P, L, st);
    case 7: return run_gauss_rows<S, 7, CN>(P, L, st);
  }
  return cudaErrorNotSupported;
}

template <class S>
cudaError_t run_gauss(const Plan &P, const Launch &L, cudaStream_t st) {
  switch (L.cn) {
    case 1: return run_gauss_k<S, 1>(P, L, st);
    case 3: return run_gauss_k<S, 3>(P, L, st);
    case 4: return run_gauss_k<S, 4>(P, L, st);
  }
  return cudaErrorNotSupported;
}

template <int CN, bool MAX>
cudaError_t run_morph_kh(const Plan &P, const Launch &L, cudaStream_t st) {
  switch (L.k) {
    case 1: return run_op<OpMorph<CN, 1, MAX>>(P, L, L.ma, st);
    case 3: return run_op<OpMorph<CN, 3, MAX>>(P, L, L.ma, st);
    case 5: return run_op<OpMorph<CN, 5, MAX>>(P, L, L.ma, st);
    case 7: return run_op<OpMorph<CN, 7, MAX>>(P, L, L.ma, st);
    case 9: return run_op<OpMorph<CN, 9, MAX>>(P, L, L.ma, st);
  }
  return cudaErrorNotSupported;
}

template <int CN>
cudaError_t run_morph(const Plan &P, const Launch &L, cudaStream_t st) {
  return L.is_max ? run_morph_kh<CN, true>(P, L, st) : run_morph_kh<CN, false>(P, L, st);
}

template <class T, bool PERSP>
cudaError_t run_warp(const Plan &P, const Launch &L, cudaStream_t st) {
  // Pool destinations are pitched (4-byte aligned rows).
  if (warp4_class(L)) return run_op<OpWarp4<PERSP>>(P, L, L.wa, st);
  switch (L.cn) {
    case 1: return run_op<OpWarp<T, 1, PERSP>>(P, L, L.wa, st);
    case 3: return run_op<OpWarp<T, 3, PERSP>>(P, L, L.wa, st);
    case 4: return run_op<OpWarp<T, 4, PERSP>>(P, L, L.wa, st);
  }
  return cudaErrorNotSupported;
}

template <int PX>
cudaError_t run_half(const Plan &P, const Launch &L, const RowArgs &ra, cudaStream_t st) {
  switch (L.cn) {
    case 1: return run_op<OpHalf<1, PX>>(P, L, ra, st);
    case 2: return run_op<OpHalf<2, PX>>(P, L, ra, st);
    case 3: return run_op<OpHalf<3, PX>>(P, L, ra, st);
    default: return run_op<OpHalf<4, PX>>(P, L, ra, st);
  }
}

cudaError_t run_launch(const Plan &P, const Launch &L, cudaStream_t st) {
  if (L.total == 0) return cudaSuccess;
  const RowArgs ra{L.rows};
  switch (L.op) {
    case kOpGaussStrip: return launch_gauss_strip(run_of(P, L), L.k, L.cn, L.rows, L.border, st);
    case kOpMorphStrip: return launch_morph_strip(run_of(P, L), L.sub, L.cn, L.rows, L.is_max, L.fused, st);
    case kOpGauss: return L.depth == k8U ? run_gauss<uint8_t>(P, L, st) : run_gauss<float>(P, L, st);
    case kOpMorph:
      if (L.cn == 1) return run_morph<1>(P, L, st);
      if (L.cn == 3) return run_morph<3>(P, L, st);
      return run_morph<4>(P, L, st);
    case kOpCopy: return run_op<OpCopy>(P, L, CopyArgs{L.rows, depth_size(L.depth)}, st);
    case kOpMorphF: {
      const MorphFArgs a{L.rows, L.sub, L.k, L.is_max};
      switch (L.cn) {
        case 1: return run_op<OpMorphF<1>>(P, L, a, st);
        case 2: return run_op<OpMorphF<2>>(P, L, a, st);
        case 3: return run_op<OpMorphF<3>>(P, L, a, st);
        default: return run_op<OpMorphF<4>>(P, L, a, st);
      }
    }
    case kOpGray:
      if (L.depth == k32F) return L.cn == 3 ? run_op<OpGrayF<3>>(P, L, ra, st) : run_op<OpGrayF<4>>(P, L, ra, st);
      if (L.vec == 8) return L.cn == 3 ? run_op<OpGray<3, 8>>(P, L, ra, st) : run_op<OpGray<4, 8>>(P, L, ra, st);
      return L.cn == 3 ? run_op<OpGray<3, 16>>(P, L, ra, st) : run_op<OpGray<4, 16>>(P, L, ra, st);
    case kOpHalf:
      if (L.vec == 8) return run_half<8>(P, L, ra, st);
      return run_half<4>(P, L, ra, st);
    case kOpLinear:
      if (L.depth == k32F) {
        switch (L.cn) {
          case 1: return run_op<OpLinearF<1>>(P, L, ra, st);
          case 2: return run_op<OpLinearF<2>>(P, L, ra, st);
          case 3: return run_op<OpLinearF<3>>(P, L, ra, st);
          default: return run_op<OpLinearF<4>>(P, L, ra, st);
        }
      }
      switch (L.cn) {
        case 1: return run_op<OpLinearStrip>(P, L, ra, st);
        case 2: return run_op<OpLinear<2>>(P, L, ra, st);
        case 3: return run_op<OpLinear<3>>(P, L, ra, st);
        default: return run_op<OpLinear<4>>(P, L, ra, st);
      }
    case kOpLut:
      if (L.vec == 8) return run_op<OpLut<8>>(P, L, LutArgs{L.rows, L.lut}, st);
      return run_op<OpLut<16>>(P, L, LutArgs{L.rows, L.lut}, st);
    case kOpWarpAff: return L.depth == k8U ? run_warp<uint8_t, false>(P, L, st) : run_warp<float, false>(P, L, st);
    case kOpWarpPer: return L.depth == k8U ? run_warp<uint8_t, true>(P, L, st) : run_warp<float, true>(P, L, st);
  }
  return cudaErrorNotSupported;
}

visar_image cimg(const Buf &b) {
  visar_image c;
  c.width = (uint32_t)b.v.w;
  c.height = (uint32_t)b.v.h;
  c.channels = (uint32_t)b.v.cn;
  c.depth = (uint32_t)b.depth;
  c.stride = (size_t)b.v.stride;
  c.data = b.v.p;
  return c;
}

int run_fallback(const Fallback &f) {
  const visar_image s = cimg(f.s), d = cimg(f.d);
  const visar_stage &st = f.st;
  switch (st.kind) {
    case VISAR_STAGE_GRAY: return visar_cvt_color(&s, &d, f.s.v.cn == 4 ? 10 : 6);
    case VISAR_STAGE_GAUSSIAN: return visar_gaussian_blur(&s, &d, st.i[0], st.i[1], st.d[0], st.d[1], st.i[2]);
    case VISAR_STAGE_MORPHOLOGY: return visar_morphology(&s, &d, st.i[0], st.i[1], st.i[2], st.i[3], st.i[4]);
    case VISAR_STAGE_RESIZE: return visar_resize(&s, &d, st.i[0]);
    case VISAR_STAGE_THRESHOLD: return visar_threshold(&s, &d, st.d[0], st.d[1], st.i[0], nullptr);
    case VISAR_STAGE_WARP_AFFINE: return visar_warp_affine(&s, &d, f.m, st.i[0], st.i[1], st.d[6]);
    case VISAR_STAGE_WARP_PERSPECTIVE: return visar_warp_perspective(&s, &d, f.m, st.i[0], st.i[1], st.d[9]);
  }
  return VISAR_UNSUPPORTED;
}

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return VISAR_OK;
  static thread_local char buf[160];
  std::snprintf(buf, sizeof(buf), "CudaError: %s", cudaGetErrorName(e));
  if (e == cudaErrorMemoryAllocation) return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory");
  return report_error(VISAR_INTERNAL, buf);
}

// Enqueues the whole plan on st. Fallback calls run on st in async mode.
int enqueue(Plan &P, cudaStream_t st, bool timed) {
  if (P.ncounters > 0) {
    const cudaError_t e = cudaMemsetAsync(P.counters, 0, sizeof(int) * (size_t)P.ncounters, st);
    if (e != cudaSuccess) return cuda_status(e);
  }
  size_t j = 0;
  for (const Step &s : P.steps) {
    for (const Launch &L : s.launches) {
      if (timed) cudaEventRecord(P.evs[2 * j], st);
      const cudaError_t e = run_launch(P, L, st);
      if (e != cudaSuccess) return cuda_status(e);
      if (timed) cudaEventRecord(P.evs[2 * j + 1], st);
      j++;
    }
    if (!s.fallbacks.empty()) {
      const cudaStream_t old = thread_stream();
      const int old_async = thread_async();
      set_thread_stream(st, 1);
      int rc = VISAR_OK;
      for (const Fallback &f : s.fallbacks) {
        rc = run_fallback(f);
        if (rc != VISAR_OK) break;
      }
      set_thread_stream(old, old_async);
      if (rc != VISAR_OK) return rc;
    }
  }
  return VISAR_OK;
}

// Points the source of descriptor j at p (input rebinding).
__global__ void k_patch_src(BImg *imgs, int j, uint8_t *p) { imgs[j].s.p = p; }

bool same_shape(const visar_image &c, const Buf &b) {
  return c.width == (uint32_t)b.v.w && c.height == (uint32_t)b.v.h && c.channels == (uint32_t)b.v.cn &&
         c.depth == (uint32_t)b.depth;
}

cudaStream_t run_stream(Plan &P) {
  const cudaStream_t t = thread_stream();
  return t ? t : P.own;
}

int finish(cudaStream_t st) {
  if (thread_async()) return VISAR_OK;
  return cuda_status(cudaStreamSynchronize(st));
}

}  // namespace bt
}  // namespace vb

using namespace vb;
using namespace vb::bt;

namespace vb {
namespace bt {

// Rows of one image per warp, 16 bytes per lane: source words are read
// aligned and funnel-shifted (never past the row), destination written as
// one 16-byte store when aligned, else by words or bytes.
__global__ void __launch_bounds__(256) k_restride(const StageCopy *t, int n) {
  const int i = blockIdx.y;
  if (i >= n) return;
  const StageCopy c = t[i];
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < c.h; r += warps) {
    const uint8_t *s = c.src + (long long)r * c.sstride;
    uint8_t *d = c.dst + (long long)r * c.dstride;
    for (int x = lane * 16; x < c.rb; x += 32 * 16) {
      if (x + 20 <= c.rb) {
        const uintptr_t a = (uintptr_t)(s + x);
        const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
        const uint32_t sh = (uint32_t)(a & 3) * 8;
        uint32_t q[5];
#pragma unroll
        for (int k = 0; k < 5; k++) q[k] = __ldg(w + k);
        uint32_t o[4];
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = __funnelshift_r(q[k], q[k + 1], sh);
        uint8_t *p = d + x;
        if (((uintptr_t)p & 15) == 0) {
          *reinterpret_cast<uint4 *>(p) = make_uint4(o[0], o[1], o[2], o[3]);
        } else if (((uintptr_t)p & 3) == 0) {
#pragma unroll
          for (int k = 0; k < 4; k++) reinterpret_cast<uint32_t *>(p)[k] = o[k];
        } else {
#pragma unroll
          for (int k = 0; k < 16; k++) p[k] = (uint8_t)(o[k >> 2] >> (8 * (k & 3)));
        }
      } else {
        for (int k = x; k < c.rb && k < x + 16; k++) d[k] = s[k];
      }
    }
  }
}

namespace {

// Staged transfers apply when every host image's rows are contiguous and
// the plan has at most 65535 images (one grid row each).
bool staged_ok(const visar_image *host, size_t n, const std::vector<StageCopy> &imgs) {
  if (n == 0 || n > 65535) return false;
  for (size_t i = 0; i < n; i++)
    if ((long long)host[i].stride != (long long)imgs[i].rb) return false;
  return true;
}

// Builds (or reuses) the staging buffer and the restride table for these
// images; `in`: staging -> plan images, else plan images -> staging. The
// table is rebuilt (a synchronous upload) only when the images changed.
int staging_prepare(XferStaging &S, std::vector<StageCopy> &imgs, bool in) {
  size_t total = 0;
  std::vector<size_t> off(imgs.size());
  for (size_t i = 0; i < imgs.size(); i++) {
    off[i] = total;
    total += ((size_t)imgs[i].rb * imgs[i].h + 255) & ~(size_t)255;
  }
  bool same = S.buf != nullptr && S.rows.size() == imgs.size();
  for (size_t i = 0; same && i < imgs.size(); i++) {
    const StageCopy &a = S.rows[i], &b = imgs[i];
    same = (in ? a.dst == b.dst && a.dstride == b.dstride : a.src == b.src && a.sstride == b.sstride) && a.rb == b.rb &&
           a.h == b.h;
  }
  if (same) return VISAR_OK;
  if (S.buf) cudaFree(S.buf);
  if (S.table) cudaFree(S.table);
  S.buf = nullptr;
  S.table = nullptr;
  S.rows.clear();
  cudaError_t e = cudaMalloc(&S.buf, std::max<size_t>(total, 256));
  if (e == cudaSuccess) e = cudaMalloc(&S.table, sizeof(StageCopy) * imgs.size());
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (S.buf) cudaFree(S.buf);
    S.buf = nullptr;
    return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory: transfer staging");
  }
  S.maxh = 0;
  for (size_t i = 0; i < imgs.size(); i++) {
    if (in) imgs[i].src = S.buf + off[i];
    else imgs[i].dst = S.buf + off[i];
    S.maxh = std::max(S.maxh, imgs[i].h);
  }
  if ((e = cudaMemcpy(S.table, imgs.data(), sizeof(StageCopy) * imgs.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_status(e);
  S.rows = imgs;
  S.off = off;
  return VISAR_OK;
}

cudaError_t launch_restride(const XferStaging &S, cudaStream_t st) {
  const int n = (int)S.rows.size();
  const int gx = std::max(1, std::min(64, (S.maxh + 7) / 8));
  k_restride<<<dim3(gx, n), 256, 0, st>>>(S.table, n);
  note_launch();
  return cudaGetLastError();
}

}  // namespace
}  // namespace bt
}  // namespace vb

struct visar_batch {
  Plan plan;
};

extern "C" {

int visar_batch_create(const visar_image *inputs, size_t n, const visar_stage *stages, size_t nstages,
                       visar_batch **out) {
  if (!out || (n > 0 && !inputs) || (nstages > 0 && !stages) || n > (size_t)INT32_MAX)
    return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  *out = nullptr;
  std::unique_ptr<visar_batch> b(new (std::nothrow) visar_batch);
  if (!b) return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory");
  Plan &P = b->plan;
  // Inputs: device images of one device, or plan-owned (data == NULL).
  int dev = -1;
  for (size_t i = 0; i < n; i++) {
    const visar_image &c = inputs[i];
    if (!(c.depth == 0 || c.depth == 2 || c.depth == 3 || c.depth == 5)) return report_error(VISAR_UNSUPPORTED, "Unsupported");
    if (c.channels == 0 || c.channels > 4) return report_error(VISAR_UNSUPPORTED, "UnsupportedChannels");
    if (c.width == 0 || c.height == 0 || c.width > (1u << 30) || c.height > (1u << 30))
      return report_error(VISAR_INVALID_ARGUMENT, "InvalidSize");
    if (!c.data) continue;
    const int es = depth_size((int)c.depth);
    if (c.stride % es != 0 || c.stride < (size_t)c.width * c.channels * es) return report_error(VISAR_INVALID_ARGUMENT, "InvalidSize");
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, c.data) != cudaSuccess || !(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged)) {
      cudaGetLastError();
      return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: batch inputs must be device memory");
    }
    if (dev >= 0 && a.device != dev) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: batch inputs on several devices");
    dev = a.device;
  }
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return cuda_status(cudaGetLastError());
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) return cuda_status(e);
  P.dev = dev;
  cudaDeviceGetAttribute(&P.num_sms, cudaDevAttrMultiProcessorCount, dev);
  std::vector<visar_stage> st(stages, stages + nstages);

  // Pass 1 sizes the pool (inputs owned by the plan, outputs, tables,
  // descriptors); pass 2 builds the plan inside it.
  P.inputs.resize(n);
  Builder sizing{P, true, {}, {}};
  for (size_t i = 0; i < n; i++) {
    const visar_image &c = inputs[i];
    if (c.data) P.inputs[i] = Buf{DImg{static_cast<uint8_t *>(c.data), (long long)c.stride, (int)c.width, (int)c.height, (int)c.channels}, (int)c.depth};
    else sizing.image((int)c.width, (int)c.height, (int)c.channels, (int)c.depth, P.inputs[i]);
    P.inputs[i].input = (int)i;
  }
  int rc = build_all(sizing, st);
  if (rc != VISAR_OK) return report_error(rc, rc == VISAR_UNSUPPORTED ? "Unsupported" : "InvalidArgument");
  size_t desc_bytes = 0;
  int nl = 0;
  for (const Step &s : P.steps)
    for (const Launch &L : s.launches) {
      desc_bytes += ((sizeof(BImg) * L.imgs.size() + 255) & ~(size_t)255) + ((sizeof(int) * (L.imgs.size() + 1) + 255) & ~(size_t)255);
      nl++;
    }
  const size_t total = sizing.sz.bytes + desc_bytes + sizeof(int) * (size_t)(nl + 1) + 4096;
  e = cudaMalloc(&P.pool.base, total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory");
  }
  P.pool.cap = total;
  Builder B{P, false, {}, {}};
  for (size_t i = 0; i < n; i++) {
    if (!inputs[i].data && !B.image((int)inputs[i].width, (int)inputs[i].height, (int)inputs[i].channels, (int)inputs[i].depth, P.inputs[i]))
      return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory");
    P.inputs[i].input = (int)i;
  }
  rc = build_all(B, st);
  if (rc != VISAR_OK) return report_error(rc, rc == VISAR_OUT_OF_MEMORY ? "OutOfMemory" : "InvalidArgument");
  // Descriptors and prefix sums of every launch.
  P.ncounters = 0;
  for (Step &s : P.steps) {
    for (Launch &L : s.launches) {
      std::vector<int> start(L.imgs.size() + 1, 0);
      for (size_t i = 0; i < L.imgs.size(); i++) start[i + 1] = start[i] + L.imgs[i].tiles_x * L.imgs[i].tiles_y;
      L.total = start.back();
      L.d_imgs = B.table(L.imgs);
      L.d_start = B.table(start);
      if (!L.d_imgs || !L.d_start) return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory");
      L.counter = P.ncounters++;
      P.bytes += L.bytes;
      P.nlaunch++;
    }
    P.nfallback += s.fallbacks.size();
    for (const Fallback &f : s.fallbacks)
      P.bytes += ((size_t)f.s.v.w * f.s.v.h * f.s.v.cn + (size_t)f.d.v.w * f.d.v.h * f.d.v.cn) * (size_t)depth_size(f.s.depth);
  }
  P.counters = static_cast<int *>(P.pool.take(sizeof(int) * (size_t)std::max(1, P.ncounters)));
  if (!P.counters) return report_error(VISAR_OUT_OF_MEMORY, "OutOfMemory");
  for (const Builder::Upload &u : B.uploads) {
    e = cudaMemcpy(u.dst, u.data.data(), u.data.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e);
  }
  for (size_t i = 0; i < n; i++) P.pixels_in += (size_t)inputs[i].width * inputs[i].height;
  e = cudaStreamCreateWithFlags(&P.own, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_status(e);
  *out = b.release();
  return VISAR_OK;
}

int visar_batch_input(const visar_batch *b, size_t i, visar_image *out) {
  if (!b || !out || i >= b->plan.inputs.size()) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  *out = cimg(b->plan.inputs[i]);
  return VISAR_OK;
}

int visar_batch_stage_output(const visar_batch *b, size_t stage, size_t i, visar_image *out) {
  if (!b || !out || stage >= b->plan.outs.size() || i >= b->plan.inputs.size())
    return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  *out = cimg(b->plan.outs[stage][i]);
  return VISAR_OK;
}

int visar_batch_output(const visar_batch *b, size_t i, visar_image *out) {
  if (!b || !out || i >= b->plan.inputs.size()) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  *out = cimg(b->plan.outs.empty() ? b->plan.inputs[i] : b->plan.outs.back()[i]);
  return VISAR_OK;
}

int visar_batch_run(visar_batch *b) {
  if (!b) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  Plan &P = b->plan;
  cudaError_t e = cudaSetDevice(P.dev);
  if (e != cudaSuccess) return cuda_status(e);
  const cudaStream_t st = run_stream(P);
  const bool timed = P.prof && P.evs.size() == 2 * P.nlaunch;
  const int rc = enqueue(P, st, timed);
  if (rc != VISAR_OK) return rc;
  P.prof_valid = timed;
  return finish(st);
}

int visar_batch_run_graph(visar_batch *b) {
  if (!b) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  Plan &P = b->plan;
  if (P.nfallback > 0) return visar_batch_run(b);
  cudaError_t e = cudaSetDevice(P.dev);
  if (e != cudaSuccess) return cuda_status(e);
  const cudaStream_t st = run_stream(P);
  if (!P.graph) {
    // Capture on the plan's own stream (never the legacy default stream).
    e = cudaStreamBeginCapture(P.own, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e);
    const int rc = enqueue(P, P.own, false);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(P.own, &g);
    if (rc != VISAR_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaGraphInstantiate(&P.graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      P.graph = nullptr;
      return cuda_status(e);
    }
  }
  e = cudaGraphLaunch(P.graph, st);
  if (e != cudaSuccess) return cuda_status(e);
  return finish(st);
}

int visar_batch_get_info(const visar_batch *b, visar_batch_info *info) {
  if (!b || !info) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  const Plan &P = b->plan;
  info->images = P.inputs.size();
  info->stages = P.steps.size();
  info->launches = P.nlaunch;
  info->fallback_calls = P.nfallback;
  info->pool_bytes = P.pool.cap;
  info->bytes_moved = P.bytes;
  info->pixels_in = P.pixels_in;
  return VISAR_OK;
}

void visar_batch_destroy(visar_batch *b) {
  if (!b) return;
  cudaSetDevice(b->plan.dev);
  cudaStreamSynchronize(b->plan.own);
  delete b;
}

int visar_batch_set_input(visar_batch *b, size_t i, const visar_image *img) {
  if (!b || !img || !img->data || i >= b->plan.inputs.size()) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  Plan &P = b->plan;
  if (!same_shape(*img, P.inputs[i])) return report_error(VISAR_SIZE_MISMATCH, "SizeMismatch");
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, img->data) != cudaSuccess ||
      !(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) || a.device != P.dev) {
    cudaGetLastError();
    return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: batch inputs must be device memory of the plan's device");
  }
  uint8_t *np = static_cast<uint8_t *>(img->data);
  const long long nstride = (long long)img->stride;
  // Kernel choices depend on the source layout; a new pointer must keep it.
  const uint8_t *op = P.inputs[i].v.p;
  const long long ostride = P.inputs[i].v.stride;
  if (nstride != ostride) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: rebound input has another stride");
  for (int al : {16, 8, 4})
    if ((uintptr_t)op % al == 0 && (uintptr_t)np % al != 0)
      return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: rebound input is less aligned than the original");
  cudaError_t e = cudaSetDevice(P.dev);
  if (e != cudaSuccess) return cuda_status(e);
  const cudaStream_t st = run_stream(P);
  for (Step &s : P.steps) {
    for (Launch &L : s.launches)
      for (size_t j = 0; j < L.imgs.size(); j++)
        if (L.src_input[j] == (int)i) {
          L.imgs[j].s.p = np;
          k_patch_src<<<1, 1, 0, st>>>(L.d_imgs, (int)j, np);
          note_launch();
          e = cudaGetLastError();
          if (e != cudaSuccess) return cuda_status(e);
        }
    for (Fallback &f : s.fallbacks)
      if (f.s.input == (int)i) f.s.v.p = np;
  }
  for (auto &stage : P.outs)
    if (stage[i].input == (int)i) stage[i].v.p = np;  // pass-through stages
  P.inputs[i].v.p = np;
  return finish(st);
}

int visar_batch_upload(visar_batch *b, const visar_image *host, size_t n) {
  if (!b || (n > 0 && !host) || n != b->plan.inputs.size()) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  Plan &P = b->plan;
  cudaError_t e = cudaSetDevice(P.dev);
  if (e != cudaSuccess) return cuda_status(e);
  const cudaStream_t st = run_stream(P);
  for (size_t i = 0; i < n; i++)
    if (!host[i].data || !same_shape(host[i], P.inputs[i])) return report_error(VISAR_SIZE_MISMATCH, "SizeMismatch");
  std::vector<StageCopy> imgs(n);
  for (size_t i = 0; i < n; i++) {
    const Buf &d = P.inputs[i];
    const int rb = d.v.w * d.v.cn * depth_size(d.depth);
    imgs[i] = StageCopy{nullptr, d.v.p, rb, (long long)d.v.stride, rb, d.v.h};
  }
  if (staged_ok(host, n, imgs)) {
    const int rc = staging_prepare(P.up, imgs, true);
    if (rc != VISAR_OK) return rc;
    for (size_t i = 0; i < n; i++) {
      e = cudaMemcpyAsync(P.up.buf + P.up.off[i], host[i].data, (size_t)imgs[i].rb * imgs[i].h, cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return cuda_status(e);
    }
    if ((e = launch_restride(P.up, st)) != cudaSuccess) return cuda_status(e);
    return finish(st);
  }
  for (size_t i = 0; i < n; i++) {
    const Buf &d = P.inputs[i];
    e = cudaMemcpy2DAsync(d.v.p, (size_t)d.v.stride, host[i].data, host[i].stride, (size_t)imgs[i].rb, (size_t)d.v.h,
                          cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return finish(st);
}

int visar_batch_download(visar_batch *b, const visar_image *host, size_t n) {
  if (!b || (n > 0 && !host) || n != b->plan.inputs.size()) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  Plan &P = b->plan;
  cudaError_t e = cudaSetDevice(P.dev);
  if (e != cudaSuccess) return cuda_status(e);
  const cudaStream_t st = run_stream(P);
  std::vector<StageCopy> imgs(n);
  for (size_t i = 0; i < n; i++) {
    const Buf &s = P.outs.empty() ? P.inputs[i] : P.outs.back()[i];
    if (!host[i].data || !same_shape(host[i], s)) return report_error(VISAR_SIZE_MISMATCH, "SizeMismatch");
    const int rb = s.v.w * s.v.cn * depth_size(s.depth);
    imgs[i] = StageCopy{s.v.p, nullptr, (long long)s.v.stride, rb, rb, s.v.h};
  }
  if (staged_ok(host, n, imgs)) {
    const int rc = staging_prepare(P.down, imgs, false);
    if (rc != VISAR_OK) return rc;
    if ((e = launch_restride(P.down, st)) != cudaSuccess) return cuda_status(e);
    for (size_t i = 0; i < n; i++) {
      e = cudaMemcpyAsync(host[i].data, P.down.buf + P.down.off[i], (size_t)imgs[i].rb * imgs[i].h, cudaMemcpyDeviceToHost, st);
      if (e != cudaSuccess) return cuda_status(e);
    }
    return finish(st);
  }
  for (size_t i = 0; i < n; i++) {
    const Buf &s = P.outs.empty() ? P.inputs[i] : P.outs.back()[i];
    e = cudaMemcpy2DAsync(host[i].data, host[i].stride, s.v.p, (size_t)s.v.stride, (size_t)imgs[i].rb, (size_t)s.v.h,
                          cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return finish(st);
}

int visar_batch_profile(visar_batch *b, int enable) {
  if (!b) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  Plan &P = b->plan;
  cudaError_t e = cudaSetDevice(P.dev);
  if (e != cudaSuccess) return cuda_status(e);
  P.prof = enable != 0;
  P.prof_valid = false;
  while (P.prof && P.evs.size() < 2 * P.nlaunch) {
    cudaEvent_t ev;
    e = cudaEventCreate(&ev);
    if (e != cudaSuccess) return cuda_status(e);
    P.evs.push_back(ev);
  }
  return VISAR_OK;
}

int visar_batch_launch_stat_get(const visar_batch *b, size_t i, visar_batch_launch_stat *out) {
  if (!b || !out || i >= b->plan.nlaunch) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  const Plan &P = b->plan;
  size_t j = 0;
  for (const Step &s : P.steps)
    for (const Launch &L : s.launches) {
      if (j++ != i) continue;
      std::memset(out, 0, sizeof(*out));
      std::snprintf(out->name, sizeof(out->name), "%s", L.tkey.c_str());
      out->stage = L.stage;
      out->images = L.imgs.size();
      out->tiles = (size_t)L.total;
      out->bytes = L.bytes;
      out->grid = L.grid;
      if (P.prof_valid) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, P.evs[2 * i], P.evs[2 * i + 1]) == cudaSuccess) out->ms = ms;
        else cudaGetLastError();
      }
      return VISAR_OK;
    }
  return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
}

int visar_tune_load(const char *path) {
  std::map<std::string, int> m;
  if (path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument: tuning file not readable");
    std::string txt;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) txt.append(buf, k);
    std::fclose(f);
    if (!parse_tune_json(txt, m)) return report_error(VISAR_INVALID_DATA, "InvalidData: tuning file");
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune = std::move(m);
  return VISAR_OK;
}

int visar_tune_set(const char *key, int value) {
  if (!key) return report_error(VISAR_INVALID_ARGUMENT, "InvalidArgument");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = value;
  return VISAR_OK;
}

int visar_tune_get(const char *key, int fallback) {
  if (!key) return fallback;
  return tune_get(key, fallback);
}

}  // extern "C"
