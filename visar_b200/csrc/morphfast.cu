// Host launcher of the fast u8 morphology pass (device code: morphfast.cuh).
#include "morphfast.cuh"

namespace vb {

namespace {

using namespace fast;

template <int CN, int KH, bool MAX>
cudaError_t go(const DImg &s, const DImg &d, const MFArgs &a, cudaStream_t st) {
  constexpr int NT = 128, RH = 8;
  const long long nwords = (a.n + 3) / 4;
  dim3 grid(ceil_div(nwords, NT - 2), ceil_div(s.h, RH));
  k_morph_fast<CN, KH, NT, RH, MAX><<<grid, NT, 0, st>>>(s, d, a);
  note_launch();
  return cudaGetLastError();
}

template <int CN, bool MAX>
cudaError_t by_kh(const DImg &s, const DImg &d, const MFArgs &a, int kh, cudaStream_t st) {
  switch (kh) {
    case 1: return go<CN, 1, MAX>(s, d, a, st);
    case 3: return go<CN, 3, MAX>(s, d, a, st);
    case 5: return go<CN, 5, MAX>(s, d, a, st);
    case 7: return go<CN, 7, MAX>(s, d, a, st);
    case 9: return go<CN, 9, MAX>(s, d, a, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace

// mask: kh x kw structuring element (row-major, nonzero = on), anchor at
// (kw/2, kh/2). Returns cudaErrorNotSupported for shapes this kernel does not
// cover; the caller then runs the general pass.
cudaError_t launch_morph_fast(const DImg &s, const DImg &d, bool is_max, const std::vector<uint8_t> &mask, int kw, int kh,
                              cudaStream_t st) {
  const int cn = s.cn;
  if (((uintptr_t)s.p | (uintptr_t)d.p | (uintptr_t)s.stride | (uintptr_t)d.stride) % 4 != 0) return cudaErrorNotSupported;
  MFArgs a{};
  if (!fast::morph_fast_args(mask, kw, kh, cn, s.w, a)) return cudaErrorNotSupported;
  switch (cn * 2 + (is_max ? 1 : 0)) {
    case 2: return by_kh<1, false>(s, d, a, kh, st);
    case 3: return by_kh<1, true>(s, d, a, kh, st);
    case 6: return by_kh<3, false>(s, d, a, kh, st);
    case 7: return by_kh<3, true>(s, d, a, kh, st);
    case 8: return by_kh<4, false>(s, d, a, kh, st);
    case 9: return by_kh<4, true>(s, d, a, kh, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace vb
