// Stage kernel at CBD_PRECISION_FAST.
#include "stage_launch.cuh"

namespace cbd {

cudaError_t launch_stage_fast(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                              int role, cudaStream_t stream)
{
    return launch_stage<CBD_PRECISION_FAST>(s, k, st, a, role, stream);
}

}  // namespace cbd
