// Morphology strip launches of the batched form: the dispatch over channel
// counts and profiles (the kernels are instantiated in batch_strip1a/b/c.cu,
// batch_strip3.cu and batch_strip4.cu).
#include "batch.cuh"

namespace vb {
namespace bt {

template cudaError_t launch_morph_strip_cn<1>(const LaunchRun &, int, int, bool, bool, cudaStream_t);
// Instantiated in batch_strip3.cu and batch_strip4.cu.
extern template cudaError_t launch_morph_strip_cn<3>(const LaunchRun &, int, int, bool, bool, cudaStream_t);
extern template cudaError_t launch_morph_strip_cn<4>(const LaunchRun &, int, int, bool, bool, cudaStream_t);

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
