// Internal launch interface shared by the host shim (capi.cu) and the three
// precision-specific translation units of the stage kernel.
#pragma once

#include "cbd_stencil.cuh"

namespace cbd {

struct LaunchShape {
    int bj;        // threads per CTA = columns per strip (64, 128)
    int rows;      // rows per CTA
    int minb;      // occupancy target (resident CTAs per SM) the kernel is compiled for; 1 = none
    dim3 grid;
};

cudaError_t launch_stage_exact(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                               int role, cudaStream_t stream);
cudaError_t launch_stage_fma(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                             int role, cudaStream_t stream);
cudaError_t launch_stage_fast(const LaunchShape &s, const Consts &k, const StageDev &st, const StageArgs &a,
                              int role, cudaStream_t stream);

// Kernel constants of a grid (mesh, EOS, options, buffer), with host-side
// reciprocals of the constant divisors; and the diagnostics of an epilogue
// (entries first .. first + count - 1) copied into them.
Consts consts_from_grid(const cbd_grid_t *g);
int set_diagnostics(Consts &k, const cbd_epilogue_t *ep, int first, int count);

// The stream the drop-in kernels launch on (cbdiso_b200_set_stream).
cudaStream_t drop_in_stream();

}  // namespace cbd
