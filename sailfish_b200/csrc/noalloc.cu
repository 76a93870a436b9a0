// cbdiso_b200_advance_stage_noalloc: the fused RK stage for callers that
// cannot allocate device memory. The only device memory the stage needs
// beyond the caller's inputs and outputs is the reductions scratch of its
// epilogue (a counter and one partial per CTA); here it is a fixed-size array
// in the library's own device memory instead of a caller buffer.
#include <mutex>

#include "cbd_internal.h"

namespace {

// 5 MiB: enough for every grid whose cbdiso_b200_scratch_bytes() is at most
// this, which includes 4096 x 4096. Each GPU that loads the library holds it
// until the process exits.
constexpr size_t kStaticScratchBytes = size_t(5) << 20;
static __device__ __align__(256) double g_stage_scratch[kStaticScratchBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_address[kMaxDevices] = {};

// The array's name is a host-side stand-in in host code, not a device
// address; its device address is looked up once per device, with that device
// current, and handed to the kernel. The address is kept for the life of the
// process: after cudaDeviceReset (which unloads the library's device code)
// it would be stale, so calls after a reset are not supported.
int static_scratch(double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return CBD_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices)
        return CBD_ERR_CAPACITY;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_address[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_stage_scratch) != cudaSuccess || !p)
            return CBD_ERR_CUDA;
        g_scratch_address[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_address[dev];
    return CBD_OK;
}

}  // namespace

extern "C" int cbdiso_b200_advance_stage_noalloc(
    const cbd_grid_t *grid, const cbd_stage_t *stage, const void *stage_dev,
    const double *primitive_rd, const double *primitive_n, double *primitive_wr,
    const cbd_epilogue_t *epilogue, double *result, void *stream)
{
    const size_t need = cbdiso_b200_scratch_bytes(grid);
    if (need == 0)
        return CBD_ERR_ARGUMENT;
    double *scratch = nullptr;
    if (epilogue) {
        // only the epilogue uses scratch: a stage without one has no size limit here
        if (need > kStaticScratchBytes)
            return CBD_ERR_CAPACITY;
        const int rc = static_scratch(&scratch);
        if (rc != CBD_OK)
            return rc;
        // The array keeps the previous call's contents; the last-CTA counter
        // in its first word must start at zero.
        if (cudaMemsetAsync(scratch, 0, 64, static_cast<cudaStream_t>(stream)) != cudaSuccess)
            return CBD_ERR_CUDA;
    }
    return cbdiso_b200_advance_stage(grid, stage, stage_dev, primitive_rd, primitive_n, primitive_wr, epilogue,
                                     scratch, result, stream);
}
