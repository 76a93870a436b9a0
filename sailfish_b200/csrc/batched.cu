// Batched (many-disk) entry points: disk records, the persistent stage launch
// at FMA / FAST precision, the per-disk reduction of tile partials, and the
// per-disk step prologue.
#include <cstring>

#include "batched.cuh"
#include "cbd_internal.h"
#include "stepper.h"

namespace cbd {

cudaError_t launch_batched_fma(const BatchArgs &a, int ctas, int role, cudaStream_t s)
{
    return launch_batched<CBD_PRECISION_FMA>(a, ctas, role, s);
}

cudaError_t launch_batched_fast(const BatchArgs &a, int ctas, int role, cudaStream_t s)
{
    return launch_batched<CBD_PRECISION_FAST>(a, ctas, role, s);
}

namespace {

// One CTA per disk: the disk's tile partials, in tile order, into its result
// row (slot 0 the wavespeed maximum, then the diagnostic sums).
__global__ void __launch_bounds__(128) batched_finalize_kernel(const DiskDev *disks, const double *partials,
                                                               double *results, int result_stride)
{
    __shared__ double sred[PARTIAL_STRIDE * 4];
    const DiskDev &D = disks[blockIdx.x];
    const int n = D.strips * D.segments;
    double acc[PARTIAL_STRIDE];
#pragma unroll
    for (int v = 0; v < PARTIAL_STRIDE; ++v)
        acc[v] = 0.0;
    for (int u = threadIdx.x; u < n; u += 128) {
        const double *p = partials + (size_t)(D.unit_begin + u) * PARTIAL_STRIDE;
#pragma unroll
        for (int v = 0; v < PARTIAL_STRIDE; ++v)
            acc[v] = v == 0 ? max_nan(acc[v], p[v]) : acc[v] + p[v];
    }
    double red[PARTIAL_STRIDE];
    block_reduce<128>(acc, sred, red);
    if (threadIdx.x == 0) {
        double *r = results + (size_t)blockIdx.x * result_stride;
        for (int v = 0; v < PARTIAL_STRIDE && v < result_stride; ++v)
            r[v] = red[v];
    }
}

}  // namespace

}  // namespace cbd

using namespace cbd;

extern "C" {

size_t cbdiso_b200_batch_disk_bytes(void) { return sizeof(DiskDev); }

int cbdiso_b200_batch_disk_record(const cbd_grid_t *grid, const cbd_epilogue_t *diagnostics, int strip_width,
                                  int rows, long long offset, int unit_begin, int *units, void *record)
{
    if (!grid || !record || !units || grid->ni <= 0 || grid->nj <= 0 || !(grid->xr > grid->xl) ||
        !(grid->yr > grid->yl) || (grid->eos_type != 1 && grid->eos_type != 2) || strip_width < 32 ||
        strip_width > 128 || rows < 1 || offset < 0 || unit_begin < 0)
        return CBD_ERR_ARGUMENT;
    DiskDev d;
    std::memset(&d, 0, sizeof(d));
    d.k = consts_from_grid(grid);
    d.k.rows_per_cta = rows;
    d.k.write_guards = 1;
    if (diagnostics) {
        if (diagnostics->num_diag < 0 || diagnostics->num_diag > MAX_FUSED)
            return CBD_ERR_CAPACITY;
        d.k.want_ws = diagnostics->want_wavespeed ? 1 : 0;
        const int rc = set_diagnostics(d.k, diagnostics, 0, diagnostics->num_diag);
        if (rc != CBD_OK)
            return rc;
    } else {
        d.k.want_ws = 1;
    }
    d.offset = offset;
    d.strip_width = strip_width;
    d.strips = (grid->nj + strip_width - 1) / strip_width;
    d.segments = (grid->ni + rows - 1) / rows;
    d.unit_begin = unit_begin;
    d.cache_offset = -1;
    *units = d.strips * d.segments;
    std::memcpy(record, &d, sizeof(d));
    return CBD_OK;
}

int cbdiso_b200_batch_disk_set_face_cache(void *record, long long cache_offset)
{
    // pairs are moved as 16-byte vectors: an even offset in an aligned arena
    if (!record || cache_offset < 0 || (cache_offset & 1))
        return CBD_ERR_ARGUMENT;
    DiskDev d;
    std::memcpy(&d, record, sizeof(d));
    d.cache_offset = cache_offset;
    std::memcpy(record, &d, sizeof(d));
    return CBD_OK;
}

}  // extern "C"

namespace {

int batched_stage(const void *disks, int num_disks, int total_units, const double *primitive_rd,
                  const double *primitive_n, double *primitive_wr, const void *records, int num_stages, int stage,
                  int epilogue, double *partials, unsigned int *counters, int precision, double *face_cache,
                  int role, void *stream)
{
    if (!disks || num_disks <= 0 || total_units <= 0 || !primitive_rd || !primitive_wr || !records ||
        num_stages < 1 || num_stages > 3 || stage < 0 || stage >= num_stages || !counters ||
        (epilogue && !partials) || precision < CBD_PRECISION_EXACT || precision > CBD_PRECISION_FAST)
        return CBD_ERR_ARGUMENT;
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.disks = static_cast<const DiskDev *>(disks);
    a.num_disks = num_disks;
    a.total_units = total_units;
    a.prd = primitive_rd;
    a.un = primitive_n;
    a.pwr = primitive_wr;
    a.records = static_cast<const StageDev *>(records);
    a.num_stages = num_stages;
    a.stage = stage;
    a.epilogue = epilogue == 2 ? 2 : (epilogue ? 1 : 0);
    a.partials = partials;
    a.counters = counters;
    a.fcache = face_cache;
    int ctas = 148 * 6;
    if (total_units < ctas)
        ctas = total_units;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    switch (precision) {
    case CBD_PRECISION_EXACT:
        e = launch_batched_exact(a, ctas, role, s);
        break;
    case CBD_PRECISION_FMA:
        e = launch_batched_fma(a, ctas, role, s);
        break;
    default:
        e = launch_batched_fast(a, ctas, role, s);
        break;
    }
    return e == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

}  // namespace

extern "C" {

int cbdiso_b200_batched_stage(const void *disks, int num_disks, int total_units, const double *primitive_rd,
                              const double *primitive_n, double *primitive_wr, const void *records, int num_stages,
                              int stage, int epilogue, double *partials, unsigned int *counters, int precision,
                              void *stream)
{
    return batched_stage(disks, num_disks, total_units, primitive_rd, primitive_n, primitive_wr, records,
                         num_stages, stage, epilogue, partials, counters, precision, nullptr, ROLE_NONE, stream);
}

int cbdiso_b200_batched_stage_cached(const void *disks, int num_disks, int total_units, const double *primitive_rd,
                                     const double *primitive_n, double *primitive_wr, const void *records,
                                     int num_stages, int stage, int epilogue, double *partials,
                                     unsigned int *counters, int precision, double *face_cache, int role,
                                     void *stream)
{
    if (!face_cache || (reinterpret_cast<uintptr_t>(face_cache) & 15) != 0 || role < ROLE_NONE ||
        role > ROLE_READER)
        return CBD_ERR_ARGUMENT;
    return batched_stage(disks, num_disks, total_units, primitive_rd, primitive_n, primitive_wr, records,
                         num_stages, stage, epilogue, partials, counters, precision, face_cache, role, stream);
}

int cbdiso_b200_batched_finalize(const void *disks, int num_disks, const double *partials, double *results,
                                 int result_stride, void *stream)
{
    if (!disks || num_disks <= 0 || !partials || !results || result_stride < 1)
        return CBD_ERR_ARGUMENT;
    batched_finalize_kernel<<<num_disks, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const DiskDev *>(disks), partials, results, result_stride);
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

int cbdiso_b200_batched_prologue(void *steppers, int num_disks, const double *results, int result_stride,
                                 void *records, double *series, int num_values, int finalize, void *stream)
{
    if (!steppers || num_disks <= 0 || !results || result_stride < 1 || !records || num_values < 0 ||
        num_values > 2 * MAX_FUSED)
        return CBD_ERR_ARGUMENT;
    return launch_step_prologue(static_cast<StepperDev *>(steppers), num_disks, results, result_stride,
                                static_cast<StageDev *>(records), series, num_values, finalize,
                                static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? CBD_OK
               : CBD_ERR_CUDA;
}

}  // extern "C"
