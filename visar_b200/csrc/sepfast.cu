// Host launchers of the fast separable filter (device code: sepfast.cuh).
#include "sepfast.cuh"

namespace vb {

namespace {

using namespace fast;

template <class S, int K, int CN, int NT, int RH, bool EXACT, int SYM>
cudaError_t launch_band(const DImg &s, const DImg &d, const FastArgs &a, unsigned bx, cudaStream_t st) {
  using WT = typename Word<S>::T;
  constexpr int NR = RH + K - 1;
  const size_t smem = sizeof(WT) == sizeof(float4) ? sizeof(WT) * NR * NT : sizeof(WT) * NR * NT + sizeof(float4) * RH * NT;
  auto kfn = k_sep_fast<S, K, K, CN, NT, RH, EXACT, SYM, SYM>;
  const cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kfn<<<dim3(bx, ceil_div(s.h, RH)), NT, smem, st>>>(s, d, a);
  note_launch();
  return cudaGetLastError();
}

template <class S, int K, int CN, bool EXACT, int SYM>
cudaError_t go(const DImg &s, const DImg &d, FastArgs a, cudaStream_t st) {
  constexpr int NT = 128;
  constexpr int HW = ((K / 2) * CN + 3) / 4;
  constexpr int OW = NT - 2 * HW;
  const long long nwords = (a.n + 3) / 4;
  const unsigned bx = ceil_div(nwords, OW);
  // Taller bands cut the re-read halo rows; keep at least ~2 CTAs per SM.
  if ((long long)bx * ceil_div(s.h, 32) >= 2 * 148) return launch_band<S, K, CN, NT, 32, EXACT, SYM>(s, d, a, bx, st);
  if ((long long)bx * ceil_div(s.h, 16) >= 2 * 148) return launch_band<S, K, CN, NT, 16, EXACT, SYM>(s, d, a, bx, st);
  return launch_band<S, K, CN, NT, 8, EXACT, SYM>(s, d, a, bx, st);
}

template <class S, bool EXACT, int SYM>
cudaError_t dispatch_k(const DImg &s, const DImg &d, const FastArgs &a, int k, cudaStream_t st) {
  switch (s.cn * 16 + k) {
    case 16 + 3: return go<S, 3, 1, EXACT, SYM>(s, d, a, st);
    case 16 + 5: return go<S, 5, 1, EXACT, SYM>(s, d, a, st);
    case 16 + 7: return go<S, 7, 1, EXACT, SYM>(s, d, a, st);
    case 48 + 3: return go<S, 3, 3, EXACT, SYM>(s, d, a, st);
    case 48 + 5: return go<S, 5, 3, EXACT, SYM>(s, d, a, st);
    case 48 + 7: return go<S, 7, 3, EXACT, SYM>(s, d, a, st);
    case 64 + 3: return go<S, 3, 4, EXACT, SYM>(s, d, a, st);
    case 64 + 5: return go<S, 5, 4, EXACT, SYM>(s, d, a, st);
    case 64 + 7: return go<S, 7, 4, EXACT, SYM>(s, d, a, st);
  }
  return cudaErrorNotSupported;
}

bool aligned(const DImg &im, int bytes) {
  return ((uintptr_t)im.p % bytes == 0) && (im.stride % bytes == 0);
}

}  // namespace

// Returns cudaErrorNotSupported when the shape is not one the fast kernel
// handles; the caller then uses the general kernel.
cudaError_t launch_sep_fast(const DImg &s, const DImg &d, const SepSpec &sp, int rows_hint, cudaStream_t st) {
  const int cn = s.cn;
  if (!(cn == 1 || cn == 3 || cn == 4)) return cudaErrorNotSupported;
  FastArgs a{};
  a.border = sp.border;
  a.n = (long long)s.w * cn;
  a.n16 = (int)(a.n - a.n % 16);
  a.shift = sp.shift;
  if (sp.acc == kAccI32 && sp.sdepth == k8U && sp.ddepth == k8U && sp.fin == kFinShift && sp.shift == 16) {
    const int k = (int)sp.kxi.size();
    if (k != (int)sp.kyi.size() || !(k == 3 || k == 5 || k == 7)) return cudaErrorNotSupported;
    long long sx = 0, sy = 0;
    for (int i = 0; i < k; i++) {
      if (sp.kxi[i] < 0 || sp.kyi[i] < 0 || sp.kxi[i] != sp.kxi[k - 1 - i] || sp.kyi[i] != sp.kyi[k - 1 - i])
        return cudaErrorNotSupported;
      sx += sp.kxi[i];
      sy += sp.kyi[i];
      a.kx[i] = (float)sp.kxi[i];
      a.ky[i] = (float)sp.kyi[i];
    }
    if (sx > 256 || sy > 256) return cudaErrorNotSupported;  // exactness bound of the f32 sums
    if (!aligned(s, 4) || !aligned(d, 4)) return cudaErrorNotSupported;
    (void)rows_hint;
    return dispatch_k<uint8_t, true, 1>(s, d, a, k, st);
  }
  if (sp.acc == kAccF32 && sp.sdepth == k32F && sp.ddepth == k32F && sp.fin == kFinCast) {
    const int k = (int)sp.kxf.size();
    if (k != (int)sp.kyf.size() || !(k == 3 || k == 5 || k == 7)) return cudaErrorNotSupported;
    if (!aligned(s, 16) || !aligned(d, 16)) return cudaErrorNotSupported;
    auto sym = [](const std::vector<float> &v) {
      const int m = (int)v.size();
      bool even = true, odd = true;
      for (int i = 0; i < m / 2; i++) {
        if (v[i] != v[m - 1 - i]) even = false;
        if (v[i] != -v[m - 1 - i]) odd = false;
      }
      if (m % 2 == 1 && v[m / 2] != 0) odd = false;
      return even ? 1 : odd ? 2 : 0;
    };
    for (int i = 0; i < k; i++) {
      // Non-negative taps: an out-of-image column under BORDER_CONSTANT then
      // filters to +0 exactly as VISAR's constant column value does.
      if (!(sp.kxf[i] >= 0.0f) || !(sp.kyf[i] >= 0.0f)) return cudaErrorNotSupported;
      a.kx[i] = sp.kxf[i];
      a.ky[i] = sp.kyf[i];
    }
    a.symx = sym(sp.kxf);
    a.symy = sym(sp.kyf);
    if (a.symx != 1 || a.symy != 1) return cudaErrorNotSupported;
    (void)rows_hint;
    return dispatch_k<float, false, 1>(s, d, a, k, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace vb
