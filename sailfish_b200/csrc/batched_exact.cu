// Batched stage kernel at CBD_PRECISION_EXACT (built with -fmad=false).
#include "batched.cuh"

namespace cbd {

cudaError_t launch_batched_exact(const BatchArgs &a, int ctas, cudaStream_t s)
{
    batched_stage_kernel<128, 6, CBD_PRECISION_EXACT><<<ctas, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace cbd
