// Batched stage kernel at CBD_PRECISION_EXACT (built with -fmad=false).
#include "batched.cuh"

namespace cbd {

cudaError_t launch_batched_exact(const BatchArgs &a, int ctas, int role, cudaStream_t s)
{
    return launch_batched<CBD_PRECISION_EXACT>(a, ctas, role, s);
}

}  // namespace cbd
