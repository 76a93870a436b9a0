// Stage kernel at CBD_PRECISION_FAST.
#include "stage_launch.cuh"

namespace cbd {

cudaError_t launch_stage_fast(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                              cudaStream_t stream)
{
    return launch_stage<CBD_PRECISION_FAST>(s, k, st, a, stream);
}

}  // namespace cbd
