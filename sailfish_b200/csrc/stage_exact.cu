// Stage kernel at CBD_PRECISION_EXACT.
// Built with -fmad=false so that no a*b+c is contracted into an FMA.
#include "stage_launch.cuh"

namespace cbd {

cudaError_t launch_stage_exact(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                              int role, cudaStream_t stream)
{
    return launch_stage<CBD_PRECISION_EXACT>(s, k, st, a, role, stream);
}

}  // namespace cbd
