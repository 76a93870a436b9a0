// Instantiates the stage kernel for the supported strip widths at precision PREC.
#pragma once

#include "cbd_internal.h"

namespace cbd {

template <int PREC>
cudaError_t launch_stage(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                         cudaStream_t stream)
{
    switch (s.bj) {
    case 64:
        stage_kernel<64, PREC><<<s.grid, 64, 0, stream>>>(k, st, a);
        break;
    case 128:
        stage_kernel<128, PREC><<<s.grid, 128, 0, stream>>>(k, st, a);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace cbd
