// Morphology strip launches of the batched form for one-channel images:
// elements Rect3, Rect5.
#include "batch.cuh"

namespace vb {
namespace bt {

template cudaError_t launch_morph_strip_prof<strip::ProfRect3, 1>(const LaunchRun &, int, bool, bool, cudaStream_t);
template cudaError_t launch_morph_strip_prof<strip::ProfRect5, 1>(const LaunchRun &, int, bool, bool, cudaStream_t);

}  // namespace bt
}  // namespace vb
