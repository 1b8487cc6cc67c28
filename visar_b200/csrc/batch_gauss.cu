// Gaussian strip launches of the batched form (3x3 / 5x5 binomial, 1 / 3 / 4
// channels, 8 / 32 / 64-row warp tiles).
#include "batch.cuh"

namespace vb {
namespace bt {

template <int K, int CN>
static cudaError_t gauss_rows(const LaunchRun &r, int rows, int border, cudaStream_t st) {
  const strip::GaussArgs a{border};
  if (rows == 8) return launch_op<OpGaussStrip<K, CN, 8>>(r, a, st);
  if constexpr (CN == 1) {  // 128-row tiles: one-channel images only (compile time)
    if (rows == 128) return launch_op<OpGaussStrip<K, CN, 128>>(r, a, st);
  }
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

}  // namespace bt
}  // namespace vb
