// Launchers of the zone-wise kernels (elementwise.cu).
#pragma once

#include "cbd_stencil.cuh"

namespace cbd {

cudaError_t launch_p2c(int ni, int nj, const double *p, double *u, cudaStream_t s);
cudaError_t launch_source(int ni, int nj, double xl, double yl, double dx, double dy, const MassDev &m,
                          const double *p, double *rate, cudaStream_t s);
cudaError_t launch_wavespeed(const Consts &k, const MassDev &m0, const MassDev &m1, const double *p, double *ws,
                             cudaStream_t s);
cudaError_t launch_fill_guards(int ni, int nj, double *p, cudaStream_t s);
int reduce_ctas(int ni, int nj);
cudaError_t launch_primitives(long n, const double *a, const double *b, double *out, cudaStream_t s);
cudaError_t launch_reduce(const Consts &k, const StageDev &st, const double *p, double *scratch, double *out0,
                          double *out_rest, cudaStream_t s);

}  // namespace cbd
