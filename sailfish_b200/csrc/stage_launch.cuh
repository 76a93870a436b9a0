// Instantiates the stage kernel for the supported strip widths, occupancy
// targets and face-cache roles at precision PREC.
#pragma once

#include "cbd_internal.h"

namespace cbd {

// Raises the kernel's dynamic shared memory limit to what its march takes,
// once per device (a no-op for strips whose march fits the static 48 KB).
template <int BJ, int MINB, int PREC, int ROLE, bool P2>
cudaError_t prepare_stage_kernel()
{
    constexpr size_t bytes = march_dynamic_smem<BJ>();
    if (bytes == 0)
        return cudaSuccess;
    static bool ready[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= 64)
        return cudaErrorInvalidDevice;
    if (!ready[dev]) {
        e = cudaFuncSetAttribute(stage_kernel<BJ, MINB, PREC, ROLE, false, P2>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess)
            return e;
        ready[dev] = true;
    }
    return cudaSuccess;
}

template <int BJ, int MINB, int PREC, bool P2>
cudaError_t launch_one_p2(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a, int role,
                          cudaStream_t stream)
{
    constexpr size_t smem = march_dynamic_smem<BJ>();
    cudaError_t e = role == ROLE_WRITER   ? prepare_stage_kernel<BJ, MINB, PREC, ROLE_WRITER, P2>()
                    : role == ROLE_READER ? prepare_stage_kernel<BJ, MINB, PREC, ROLE_READER, P2>()
                                          : prepare_stage_kernel<BJ, MINB, PREC, ROLE_NONE, P2>();
    if (e != cudaSuccess)
        return e;
    // a stage with an epilogue runs as the stage without it, then the
    // epilogue kernel over the same tiles (the same bits as fusing them)
    switch (role) {
    case ROLE_WRITER:
        stage_kernel<BJ, MINB, PREC, ROLE_WRITER, false, P2><<<s.grid, BJ, smem, stream>>>(k, st, a);
        break;
    case ROLE_READER: {
        // the fill over the stage's own tiles, then the stage
        const int tiles = s.grid.x * s.grid.y;
        const int per_sm = FILL_WARPS_PER_SM * 32 / BJ;
        const int fill_ctas = tiles < 148 * per_sm ? tiles : 148 * per_sm;
        face_cache_fill_kernel<BJ, PREC><<<fill_ctas, BJ, 0, stream>>>(k, st, a.stage_dev, a.fcache, s.grid.x, tiles);
        stage_kernel<BJ, MINB, PREC, ROLE_READER, false, P2><<<s.grid, BJ, smem, stream>>>(k, st, a);
        break;
    }
    default:
        stage_kernel<BJ, MINB, PREC, ROLE_NONE, false, P2><<<s.grid, BJ, smem, stream>>>(k, st, a);
        break;
    }
    if (k.want_ws || k.num_diag > 0) {
        if (k.rates_only)
            stage_epilogue_kernel<BJ, PREC, true><<<s.grid, BJ, 0, stream>>>(k, st, a);
        else
            stage_epilogue_kernel<BJ, PREC, false><<<s.grid, BJ, 0, stream>>>(k, st, a);
    }
    return cudaGetLastError();
}

// Grids whose spacings are powers of two take the kernels without the
// correction steps of the divisions by dx and dy (FAST has none anyway).
template <int BJ, int MINB, int PREC>
cudaError_t launch_one(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a, int role,
                       cudaStream_t stream)
{
    if (PREC != CBD_PRECISION_FAST && k.spacing_pow2)
        return launch_one_p2<BJ, MINB, PREC, true>(s, k, st, a, role, stream);
    return launch_one_p2<BJ, MINB, PREC, false>(s, k, st, a, role, stream);
}

template <int PREC>
cudaError_t launch_stage(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a, int role,
                         cudaStream_t stream)
{
    // minb = target resident CTAs per SM, which caps registers per thread
    if (s.bj == 256)
        return launch_one<256, 3, PREC>(s, k, st, a, role, stream);
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
