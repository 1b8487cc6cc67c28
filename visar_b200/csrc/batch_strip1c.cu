// Morphology strip launches of the batched form for one-channel images:
// elements Ell5, Ell7.
#include "batch.cuh"

namespace vb {
namespace bt {

template cudaError_t launch_morph_strip_prof<strip::ProfEll5, 1>(const LaunchRun &, int, bool, bool, cudaStream_t);
template cudaError_t launch_morph_strip_prof<strip::ProfEll7, 1>(const LaunchRun &, int, bool, bool, cudaStream_t);

}  // namespace bt
}  // namespace vb
