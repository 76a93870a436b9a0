// Instantiates the stage kernel for the supported strip widths and occupancy
// targets at precision PREC.
#pragma once

#include "cbd_internal.h"

namespace cbd {

template <int BJ, int MINB, int PREC>
cudaError_t launch_one(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                       cudaStream_t stream)
{
    stage_kernel<BJ, MINB, PREC><<<s.grid, BJ, 0, stream>>>(k, st, a);
    return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_stage(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                         cudaStream_t stream)
{
    // minb = target resident CTAs per SM, which caps registers per thread
    if (s.bj == 128) {
        switch (s.minb) {
        case 5:
            return launch_one<128, 5, PREC>(s, k, st, a, stream);
        case 6:
            return launch_one<128, 6, PREC>(s, k, st, a, stream);
        default:
            return launch_one<128, 1, PREC>(s, k, st, a, stream);
        }
    }
    if (s.bj == 64) {
        switch (s.minb) {
        case 10:
            return launch_one<64, 10, PREC>(s, k, st, a, stream);
        case 12:
            return launch_one<64, 12, PREC>(s, k, st, a, stream);
        default:
            return launch_one<64, 1, PREC>(s, k, st, a, stream);
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace cbd
