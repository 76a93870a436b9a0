// Many grids ("disks") of different sizes and physics advanced by one
// persistent launch per RK stage. The work is the list of all tiles
// (disk, strip, segment), largest disks first; each CTA takes the next tile
// from an atomic counter, loads that disk's constants and stage record into
// shared memory and marches the tile with the same code as the single-grid
// kernel. Per-tile epilogue partials are reduced per disk afterwards, in tile
// order, by one CTA per disk.
#pragma once

#include "cbd_stencil.cuh"

namespace cbd {

struct DiskDev {
    Consts k;            // the disk's kernel constants (k.rows_per_cta = tile rows)
    long long offset;    // offset of the disk's state, in doubles, in the batch buffers
    int strip_width;     // tile columns (<= the kernel's thread count)
    int strips;
    int segments;
    int unit_begin;      // index of the disk's first tile in the batch's tile list
    long long cache_offset;  // offset of the disk's face cache in BatchArgs::fcache, in doubles; -1: none
};

struct BatchArgs {
    const DiskDev *disks;
    int num_disks;
    int total_units;
    const double *prd;
    const double *un;    // u_n source (primitive_n), or null for a = 0 stages
    double *pwr;
    const StageDev *records;  // records[disk * num_stages + stage]
    int num_stages;
    int stage;
    int epilogue;        // the step's last stage: 1, or 2 when every disk's diagnostics are source
                         // rates without a radial cut (Consts::rates_only; the launch then takes the
                         // kernel compiled for those)
    int _pad;
    double *partials;    // [total_units][PARTIAL_STRIDE]
    unsigned int *counters;  // [0] next tile, [1] CTAs finished; both return to zero at the end
    double *fcache;      // face-cache arena (disk d's cache at disks[d].cache_offset), or null
};

// ROLE (ROLE_*) is what the launch does with each disk's face cache: a writer
// stores into the caches of the disks that have one; a reader requires one
// for every disk (the batch's fill kernel ran before it), skips the tiles of
// a disk without one, and the disk's first tile records the key.
template <int BJ, int MINB, int PREC, int ROLE = ROLE_NONE, bool EPI = true, bool RATES = false>
__global__ void __launch_bounds__(BJ, MINB) batched_stage_kernel(const BatchArgs a)
{
    constexpr bool FAST = PREC == CBD_PRECISION_FAST;
    __shared__ Consts k;
    __shared__ StageDev st;
    __shared__ double sred[PARTIAL_STRIDE * (BJ / 32)];
    __shared__ int s_unit, s_disk;
    const int t = threadIdx.x;

    for (;;) {
        if (t == 0) {
            const int u = (int)atomicAdd(&a.counters[0], 1u);
            s_unit = u;
            if (u < a.total_units) {
                int lo = 0, hi = a.num_disks - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) / 2;
                    if (a.disks[mid].unit_begin <= u)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                s_disk = lo;
            }
        }
        __syncthreads();
        const int u = s_unit;
        if (u >= a.total_units)
            break;
        const DiskDev &D = a.disks[s_disk];
        {
            const double *src = reinterpret_cast<const double *>(&D.k);
            double *dst = reinterpret_cast<double *>(&k);
            for (int w = t; w < (int)(sizeof(Consts) / sizeof(double)); w += BJ)
                dst[w] = src[w];
            const double *rs = reinterpret_cast<const double *>(&a.records[(size_t)s_disk * a.num_stages + a.stage]);
            double *rd = reinterpret_cast<double *>(&st);
            for (int w = t; w < (int)(sizeof(StageDev) / sizeof(double)); w += BJ)
                rd[w] = rs[w];
        }
        __syncthreads();
        if (t == 0) {
            k.un_kind = a.un ? 1 : 0;
            k.write_guards = 1;
            if (!a.epilogue) {
                k.want_ws = 0;
                k.num_diag = 0;
            }
        }
        __syncthreads();
        const int local = u - D.unit_begin;
        const int strip = local % D.strips;
        const int seg = local / D.strips;
        StageArgs sa;
        sa.prd = a.prd + D.offset;
        sa.un = a.un ? a.un + D.offset : nullptr;
        sa.pwr = a.pwr + D.offset;
        sa.stage_dev = nullptr;
        sa.scratch = nullptr;
        sa.result = nullptr;
        const bool cached = ROLE != ROLE_NONE && a.fcache && D.cache_offset >= 0;
        sa.fcache = cached ? a.fcache + D.cache_offset : nullptr;
        double acc[PARTIAL_STRIDE];
#pragma unroll
        for (int v = 0; v < PARTIAL_STRIDE; ++v)
            acc[v] = 0.0;
        const int c0 = strip * D.strip_width, r0 = seg * k.rows_per_cta;
        if (st.halt) {
            // the disk's stepper stopped: no march, zero partials
        } else if (ROLE == ROLE_WRITER) {
            // the same answer in every thread; the disk's first tile writes the key
            const bool store = cached && cache_write_check<PREC>(k, st, sa.fcache, t == 0 && u == D.unit_begin);
            march_tile<BJ, FAST, CACHE_WRITE, EPI, false, false, RATES>(k, st, sa, c0, D.strip_width, r0, acc, store);
        } else if (ROLE == ROLE_READER) {
            if (cached) {
                march_tile<BJ, FAST, CACHE_READ, EPI, false, false, RATES>(k, st, sa, c0, D.strip_width, r0, acc);
                // the fill kernel ran before this launch; no tile reads the key
                if (t == 0 && u == D.unit_begin)
                    cache_write_key<PREC>(k, st, sa.fcache);
            }
        } else {
            march_tile<BJ, FAST, CACHE_NONE, EPI, false, false, RATES>(k, st, sa, c0, D.strip_width, r0, acc);
        }
        if (EPI) {
            double red[PARTIAL_STRIDE];
            block_reduce<BJ>(acc, sred, red);
            // a disk whose diagnostics the rates-only kernel cannot evaluate
            // (a wrong epilogue form from the caller): NaN sums, not wrong ones
            if (RATES && !k.rates_only) {
#pragma unroll
                for (int v = 1; v < PARTIAL_STRIDE; ++v)
                    red[v] = __longlong_as_double(0x7ff8000000000000LL);
            }
            if (t == 0) {
#pragma unroll
                for (int v = 0; v < PARTIAL_STRIDE; ++v)
                    a.partials[(size_t)u * PARTIAL_STRIDE + v] = red[v];
            }
        }
        __syncthreads();
    }
    if (t == 0) {
        __threadfence();
        const unsigned int done = atomicAdd(&a.counters[1], 1u);
        if (done == gridDim.x - 1) {
            a.counters[0] = 0u;
            a.counters[1] = 0u;
            __threadfence();
        }
    }
}

// The face caches of every disk valid for a reader stage (see
// face_cache_fill_kernel): CTA b takes tiles u = b, b + gridDim.x, ... of the
// batch's tile list (the same tiles as the stage) and fills tile u when its
// disk has a cache whose key does not match the disk's stage masses.
template <int BJ, int PREC>
__global__ void __launch_bounds__(BJ, FILL_WARPS_PER_SM * 32 / BJ) batched_fill_kernel(const BatchArgs a)
{
    constexpr bool FAST = PREC == CBD_PRECISION_FAST;
    __shared__ StageDev st;
    __shared__ int s_disk, fill;
    for (int u = blockIdx.x; u < a.total_units; u += gridDim.x) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = a.num_disks - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (a.disks[mid].unit_begin <= u)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            s_disk = lo;
            const DiskDev &D = a.disks[lo];
            st = a.records[(size_t)lo * a.num_stages + a.stage];
            fill = D.cache_offset >= 0 && !st.halt &&
                   !cache_key_matches<PREC>(D.k, st, a.fcache + D.cache_offset);
        }
        __syncthreads();
        if (fill) {
            const DiskDev &D = a.disks[s_disk];
            const int local = u - D.unit_begin;
            const int strip = local % D.strips;
            const int seg = local / D.strips;
            face_cache_fill_tile<BJ, FAST>(D.k, st.m, a.fcache + D.cache_offset, strip * D.strip_width,
                                           D.strip_width, seg * D.k.rows_per_cta, D.k.rows_per_cta);
        }
        // the shared record is rewritten for the next tile
        __syncthreads();
    }
}

cudaError_t launch_batched_exact(const BatchArgs &a, int ctas, int role, cudaStream_t s);
cudaError_t launch_batched_fma(const BatchArgs &a, int ctas, int role, cudaStream_t s);
cudaError_t launch_batched_fast(const BatchArgs &a, int ctas, int role, cudaStream_t s);

// One batched stage launch at precision PREC with a face-cache role; the
// reader is preceded by the fill kernel.
template <int PREC>
cudaError_t launch_batched(const BatchArgs &a, int ctas, int role, cudaStream_t s)
{
    switch (role) {
    case ROLE_WRITER:
        if (a.epilogue == 2)
            batched_stage_kernel<128, 6, PREC, ROLE_WRITER, true, true><<<ctas, 128, 0, s>>>(a);
        else if (a.epilogue)
            batched_stage_kernel<128, 6, PREC, ROLE_WRITER, true><<<ctas, 128, 0, s>>>(a);
        else
            batched_stage_kernel<128, 6, PREC, ROLE_WRITER, false><<<ctas, 128, 0, s>>>(a);
        break;
    case ROLE_READER:
        batched_fill_kernel<128, PREC><<<a.total_units < 148 * 8 ? a.total_units : 148 * 8, 128, 0, s>>>(a);
        if (a.epilogue == 2)
            batched_stage_kernel<128, 6, PREC, ROLE_READER, true, true><<<ctas, 128, 0, s>>>(a);
        else if (a.epilogue)
            batched_stage_kernel<128, 6, PREC, ROLE_READER, true><<<ctas, 128, 0, s>>>(a);
        else
            batched_stage_kernel<128, 6, PREC, ROLE_READER, false><<<ctas, 128, 0, s>>>(a);
        break;
    default:
        if (a.epilogue == 2)
            batched_stage_kernel<128, 6, PREC, ROLE_NONE, true, true><<<ctas, 128, 0, s>>>(a);
        else if (a.epilogue)
            batched_stage_kernel<128, 6, PREC, ROLE_NONE, true><<<ctas, 128, 0, s>>>(a);
        else
            batched_stage_kernel<128, 6, PREC, ROLE_NONE, false><<<ctas, 128, 0, s>>>(a);
        break;
    }
    return cudaGetLastError();
}

}  // namespace cbd
