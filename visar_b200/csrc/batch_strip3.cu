// Morphology strip launches of the batched form for 3-channel images.
#include "batch.cuh"

namespace vb {
namespace bt {

template cudaError_t launch_morph_strip_cn<3>(const LaunchRun &, int, int, bool, bool, cudaStream_t);

}  // namespace bt
}  // namespace vb
