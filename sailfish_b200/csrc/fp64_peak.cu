// FP64 issue-rate probe: the denominator of the stencil kernels' FP64
// roofline. Every thread runs eight independent FMA chains (enough to cover
// the pipe's dependency latency at full occupancy), so the kernel's run time
// is set by the FP64 pipe alone; x <- x m + c with 0 < m < 1 stays finite.
#include <cuda_runtime.h>

#include "cbdiso_b200.h"

namespace {

constexpr int PROBE_THREADS = 256;
constexpr int PROBE_CHAINS = 8;

__global__ void __launch_bounds__(PROBE_THREADS) fma_chains(long iterations, double m, double c, double *out)
{
    double x[PROBE_CHAINS];
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; ++k)
        x[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    for (long n = 0; n < iterations; ++n) {
#pragma unroll
        for (int k = 0; k < PROBE_CHAINS; ++k)
            x[k] = fma(x[k], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; ++k)
        s += x[k];
    if (s == 12345.678)  // never true for these inputs; keeps the chains live
        out[blockIdx.x] = s;
}

}  // namespace

extern "C" {

int cbdiso_b200_fp64_probe(long iterations, int blocks, double *out, void *stream)
{
    if (iterations <= 0 || blocks <= 0 || !out)
        return CBD_ERR_ARGUMENT;
    fma_chains<<<blocks, PROBE_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(iterations, 0.999999, 1e-6, out);
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

long cbdiso_b200_fp64_probe_fmas(long iterations, int blocks)
{
    return iterations * (long)blocks * PROBE_THREADS * PROBE_CHAINS;
}

}  // extern "C"
