// Zone-wise kernels: the three smaller drop-in kernels of the reference
// (cbdiso_2d.c:606-722), the guard-zone fill, and the standalone reduction of
// the CFL wavespeed and diagnostics. Built with -fmad=false so their
// arithmetic matches the reference's CPU build operation for operation.
#include "cbd_internal.h"
#include "elementwise.h"

namespace cbd {

namespace {

__device__ __forceinline__ size_t zoff(int i, int j, int nj)
{
    return ((size_t)(i + NG) * (size_t)(nj + 2 * NG) + (size_t)(j + NG)) * NQ;
}

// Threads map to zones with j (the contiguous axis) fastest.
__global__ void p2c_kernel(int ni, int nj, const double *p, double *u)
{
    const long n = (long)ni * nj;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < n; z += (long)gridDim.x * blockDim.x) {
        const int i = (int)(z / nj), j = (int)(z - (long)i * nj);
        const size_t o = zoff(i, j, nj);
        const double rho = p[o];
        u[o] = rho;
        u[o + 1] = p[o + 1] * rho;
        u[o + 2] = p[o + 2] * rho;
    }
}

__global__ void source_kernel(int ni, int nj, double xl, double yl, double dx, double dy, MassDev m,
                              const double *p, double *rate)
{
    const long n = (long)ni * nj;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < n; z += (long)gridDim.x * blockDim.x) {
        const int i = (int)(z / nj), j = (int)(z - (long)i * nj);
        const size_t o = zoff(i, j, nj);
        const double xc = xl + (i + 0.5) * dx;
        const double yc = yl + (j + 0.5) * dy;
        double du[3] = {rate[o], rate[o + 1], rate[o + 2]};
        mass_source<false>(m, xc, yc, 1.0, p + o, du);
        rate[o] = du[0];
        rate[o + 1] = du[1];
        rate[o + 2] = du[2];
    }
}

__global__ void wavespeed_kernel(int ni, int nj, Consts k, MassDev m0, MassDev m1, const double *p, double *ws)
{
    const long n = (long)ni * nj;
    MassDev m[2] = {m0, m1};
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < n; z += (long)gridDim.x * blockDim.x) {
        const int i = (int)(z / nj), j = (int)(z - (long)i * nj);
        const double xc = k.xl + (i + 0.5) * k.dx;
        const double yc = k.yl + (j + 0.5) * k.dy;
        const double c2 = sound_speed2<false>(k, m, xc, yc);
        ws[(size_t)(i + NG) * (nj + 2 * NG) + (j + NG)] = max_wavespeed(p + zoff(i, j, nj), c2);
    }
}

__global__ void fill_guards_kernel(int ni, int nj, double *p)
{
    const long wi = ni + 2 * NG, wj = nj + 2 * NG;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < wi * wj; z += (long)gridDim.x * blockDim.x) {
        const int ii = (int)(z / wj) - NG, jj = (int)(z % wj) - NG;
        if (ii >= 0 && ii < ni && jj >= 0 && jj < nj)
            continue;
        const int ci = ii < 0 ? 0 : (ii >= ni ? ni - 1 : ii);
        const int cj = jj < 0 ? 0 : (jj >= nj ? nj - 1 : jj);
        const size_t src = zoff(ci, cj, nj), dst = zoff(ii, jj, nj);
        p[dst] = p[src];
        p[dst + 1] = p[src + 1];
        p[dst + 2] = p[src + 2];
    }
}

template <int BJ>
__global__ void __launch_bounds__(BJ) reduce_kernel(const Consts k, const StageDev st, const double *p,
                                                    double *scratch, double *out0, double *out_rest)
{
    __shared__ double sred[PARTIAL_STRIDE * (BJ / 32)];
    double acc[PARTIAL_STRIDE];
#pragma unroll
    for (int v = 0; v < PARTIAL_STRIDE; ++v)
        acc[v] = 0.0;
    const long n = (long)k.ni * k.nj;
    for (long z = blockIdx.x * (long)BJ + threadIdx.x; z < n; z += (long)gridDim.x * BJ) {
        const int i = (int)(z / k.nj), j = (int)(z - (long)i * k.nj);
        const double *pc = p + zoff(i, j, k.nj);
        const double pz[3] = {pc[0], pc[1], pc[2]};
        const double xc = k.xl + (i + 0.5) * k.dx;
        const double yc = k.yl + (j + 0.5) * k.dy;
        accumulate_zone<false>(k, st.e, xc, yc, pz, acc);
    }
    double red[PARTIAL_STRIDE];
    block_reduce<BJ>(acc, sred, red);
    grid_finish<BJ>(red, 1 + 2 * k.num_diag, scratch, out0, out_rest, sred);
}

// Evaluates the stencil's correctly rounded arithmetic on arrays, so tests
// can compare it with IEEE division and high-precision powers:
// out[4i] = a / b, out[4i+1] = a^-1.5, out[4i+2] = a^4, out[4i+3] = the
// limited slope of (a, b, a + b) with theta = 1.5.
__global__ void primitives_kernel(long n, const double *a, const double *b, double *out)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        out[4 * i] = div_rn<false>(a[i], b[i]);
        out[4 * i + 1] = pow_m15_rn(a[i]);
        out[4 * i + 2] = pow4_rn(a[i]);
        out[4 * i + 3] = limited_slope(a[i], b[i], a[i] + b[i], 1.5);
    }
}

inline int blocks_for(long n, int bs, int cap)
{
    long b = (n + bs - 1) / bs;
    if (b < 1)
        b = 1;
    return (int)(b < cap ? b : cap);
}

}  // namespace

cudaError_t launch_p2c(int ni, int nj, const double *p, double *u, cudaStream_t s)
{
    p2c_kernel<<<blocks_for((long)ni * nj, 256, 148 * 16), 256, 0, s>>>(ni, nj, p, u);
    return cudaGetLastError();
}

cudaError_t launch_source(int ni, int nj, double xl, double yl, double dx, double dy, const MassDev &m,
                          const double *p, double *rate, cudaStream_t s)
{
    source_kernel<<<blocks_for((long)ni * nj, 256, 148 * 16), 256, 0, s>>>(ni, nj, xl, yl, dx, dy, m, p, rate);
    return cudaGetLastError();
}

cudaError_t launch_wavespeed(const Consts &k, const MassDev &m0, const MassDev &m1, const double *p, double *ws,
                             cudaStream_t s)
{
    wavespeed_kernel<<<blocks_for((long)k.ni * k.nj, 256, 148 * 16), 256, 0, s>>>(k.ni, k.nj, k, m0, m1, p, ws);
    return cudaGetLastError();
}

cudaError_t launch_fill_guards(int ni, int nj, double *p, cudaStream_t s)
{
    const long n = (long)(ni + 2 * NG) * (nj + 2 * NG);
    fill_guards_kernel<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(ni, nj, p);
    return cudaGetLastError();
}

cudaError_t launch_primitives(long n, const double *a, const double *b, double *out, cudaStream_t s)
{
    primitives_kernel<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, a, b, out);
    return cudaGetLastError();
}

int reduce_ctas(int ni, int nj)
{
    return blocks_for((long)ni * nj, 256, 148 * 8);
}

cudaError_t launch_reduce(const Consts &k, const StageDev &st, const double *p, double *scratch, double *out0,
                          double *out_rest, cudaStream_t s)
{
    reduce_kernel<256><<<reduce_ctas(k.ni, k.nj), 256, 0, s>>>(k, st, p, scratch, out0, out_rest);
    return cudaGetLastError();
}

}  // namespace cbd
