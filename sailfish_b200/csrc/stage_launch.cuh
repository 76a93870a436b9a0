// Instantiates the stage kernel for the supported strip widths, occupancy
// targets and face-cache roles at precision PREC.
#pragma once

#include "cbd_internal.h"

namespace cbd {

template <int BJ, int MINB, int PREC>
cudaError_t launch_one(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a, int role,
                       cudaStream_t stream)
{
    // a stage with an epilogue runs as the stage without it, then the
    // epilogue kernel over the same tiles (the same bits as fusing them)
    const bool epi = k.want_ws || k.num_diag > 0;
    switch (role) {
    case ROLE_WRITER:
        stage_kernel<BJ, MINB, PREC, ROLE_WRITER, false><<<s.grid, BJ, 0, stream>>>(k, st, a);
        break;
    case ROLE_READER: {
        // the fill over the stage's own tiles, then the stage
        const int tiles = s.grid.x * s.grid.y;
        const int per_sm = FILL_WARPS_PER_SM * 32 / BJ;
        const int fill_ctas = tiles < 148 * per_sm ? tiles : 148 * per_sm;
        face_cache_fill_kernel<BJ, PREC><<<fill_ctas, BJ, 0, stream>>>(k, st, a.stage_dev, a.fcache, s.grid.x, tiles);
        stage_kernel<BJ, MINB, PREC, ROLE_READER, false><<<s.grid, BJ, 0, stream>>>(k, st, a);
        break;
    }
    default:
        stage_kernel<BJ, MINB, PREC, ROLE_NONE, false><<<s.grid, BJ, 0, stream>>>(k, st, a);
        break;
    }
    if (epi)
        stage_epilogue_kernel<BJ, PREC><<<s.grid, BJ, 0, stream>>>(k, st, a);
    return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_stage(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a, int role,
                         cudaStream_t stream)
{
    // minb = target resident CTAs per SM, which caps registers per thread
    if (s.bj == 128) {
        switch (s.minb) {
        case 5:
            return launch_one<128, 5, PREC>(s, k, st, a, role, stream);
        case 6:
            return launch_one<128, 6, PREC>(s, k, st, a, role, stream);
        default:
            return launch_one<128, 1, PREC>(s, k, st, a, role, stream);
        }
    }
    if (s.bj == 64) {
        switch (s.minb) {
        case 10:
            return launch_one<64, 10, PREC>(s, k, st, a, role, stream);
        case 12:
            return launch_one<64, 12, PREC>(s, k, st, a, role, stream);
        default:
            return launch_one<64, 1, PREC>(s, k, st, a, role, stream);
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace cbd
