// Strip launches of the batched form: the Gaussian strips and the
// one-channel morphology strips, and the dispatch over channel counts.
#include "batch.cuh"

namespace vb {
namespace bt {

template <int K, int CN>
static cudaError_t gauss_rows(const LaunchRun &r, int rows, int border, cudaStream_t st) {
  const strip::GaussArgs a{border};
  if (rows == 8) return launch_op<OpGaussStrip<K, CN, 8>>(r, a, st);
  if (rows == 64) return launch_op<OpGaussStrip<K, CN, 64>>(r, a, st);
  return launch_op<OpGaussStrip<K, CN, 32>>(r, a, st);
}

template <int CN>
static cudaError_t gauss_k(const LaunchRun &r, int k, int rows, int border, cudaStream_t st) {
  return k == 3 ? gauss_rows<3, CN>(r, rows, border, st) : gauss_rows<5, CN>(r, rows, border, st);
}

cudaError_t launch_gauss_strip(const LaunchRun &r, int k, int cn, int rows, int border, cudaStream_t st) {
  switch (cn) {
    case 1: return gauss_k<1>(r, k, rows, border, st);
    case 3: return gauss_k<3>(r, k, rows, border, st);
    case 4: return gauss_k<4>(r, k, rows, border, st);
  }
  return cudaErrorNotSupported;
}

template cudaError_t launch_morph_strip_cn<1>(const LaunchRun &, int, int, bool, bool, cudaStream_t);

cudaError_t launch_morph_strip(const LaunchRun &r, int prof, int cn, int rows, bool max1, bool fused, cudaStream_t st) {
  switch (cn) {
    case 1: return launch_morph_strip_cn<1>(r, prof, rows, max1, fused, st);
    case 3: return launch_morph_strip_cn<3>(r, prof, rows, max1, fused, st);
    case 4: return launch_morph_strip_cn<4>(r, prof, rows, max1, fused, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace bt
}  // namespace vb
