// C-ABI of libcbdiso_b200.so (include/cbdiso_b200.h): argument checks,
// per-launch constants computed on the host, launch shapes, and dispatch to
// the precision-specific stage kernels.
#include <cmath>
#include <cstring>

#include "cbd_internal.h"
#include "elementwise.h"

using namespace cbd;

namespace {

cudaStream_t g_stream = nullptr;
double g_theta = 1.8;  // cbdiso_2d.c:11
int g_precision = CBD_PRECISION_EXACT;

int status_of(cudaError_t e) { return e == cudaSuccess ? CBD_OK : CBD_ERR_CUDA; }

MassDev mass_dev(const cbd_mass_t &m)
{
    MassDev d;
    d.x = m.x;
    d.y = m.y;
    d.vx = m.vx;
    d.vy = m.vy;
    d.mass = m.mass;
    d.soft2 = m.softening_length * m.softening_length;
    d.sink_rate = m.sink_rate;
    d.sink_radius = m.sink_radius;
    d.inv_sink_radius = 1.0 / m.sink_radius;
    d.sink_r4 = 4.0 * m.sink_radius;
    d.sink_hi2 = d.sink_r4 * d.sink_r4 * (1.0 + 1e-10);
    d.sink_model = m.sink_model;
    d._pad = 0;
    return d;
}

MassDev mass_dev(double x, double y, double vx, double vy, double mass, double soft, double rate, double rsink,
                 int model)
{
    cbd_mass_t m = {x, y, vx, vy, mass, soft, rate, rsink, model, 0};
    return mass_dev(m);
}

bool valid_grid(const cbd_grid_t *g)
{
    return g && g->ni > 0 && g->nj > 0 && (long)g->ni * (long)g->nj < (1L << 40) && g->xr > g->xl &&
           g->yr > g->yl && g->precision >= CBD_PRECISION_EXACT && g->precision <= CBD_PRECISION_FAST &&
           (g->eos_type == 1 || g->eos_type == 2);
}

}  // namespace

Consts cbd::consts_from_grid(const cbd_grid_t *g)
{
    Consts k;
    std::memset(&k, 0, sizeof(k));
    k.ni = g->ni;
    k.nj = g->nj;
    k.xl = g->xl;
    k.yl = g->yl;
    k.dx = (g->xr - g->xl) / g->ni;  // cbdiso_2d.c:440-441
    k.dy = (g->yr - g->yl) / g->nj;
    k.inv_dx = 1.0 / k.dx;
    k.inv_dy = 1.0 / k.dy;
    // a power of two has an exact reciprocal, and x * RN(1 / d) then rounds
    // as x / d does (the same real number, rounded once)
    int ex, ey;
    k.spacing_pow2 = std::frexp(k.dx, &ex) == 0.5 && std::frexp(k.dy, &ey) == 0.5 && std::isfinite(k.inv_dx) &&
                     std::isfinite(k.inv_dy) && k.inv_dx * k.dx == 1.0 && k.inv_dy * k.dy == 1.0;
    k.theta = g->plm_theta;
    k.eos = g->eos_type;
    k.cs2 = g->cs2;
    k.mach2 = g->mach2;
    k.inv_mach2 = 1.0 / g->mach2;
    k.neg_inv_mach2 = -1.0 / g->mach2;
    k.nu = g->nu;
    k.half_nu = 0.5 * g->nu;
    k.vmax = g->velocity_ceiling;
    k.rho_min = g->density_floor;
    k.buffer_on = g->buffer_is_enabled ? 1 : 0;
    k.buf_sigma = g->buffer_surface_density;
    k.buf_onset = g->buffer_outer_radius - g->buffer_onset_width;  // cbdiso_2d.c:229
    // zones with r^2 <= buf_lo2 are inside the onset radius whatever the
    // rounding of sqrt(r^2); the square root is taken only beyond it
    k.buf_lo2 = k.buf_onset > 0.0 ? k.buf_onset * k.buf_onset * (1.0 - 1e-10) : -1.0;
    k.buf_span = g->buffer_outer_radius - k.buf_onset;
    k.inv_buf_span = 1.0 / k.buf_span;
    return k;
}

namespace {

// driving_rate * omega_outer with omega_outer = sqrt(M onset^-3), evaluated
// with the host libm as the reference's CPU build does (cbdiso_2d.c:237-238).
double buffer_k(double driving_rate, double central_mass, double onset)
{
    return driving_rate * std::sqrt(central_mass * std::pow(onset, -3.0));
}

// Launch shape of the stage kernel. Defaults: 256-column strips (3 resident
// CTAs per SM) on grids of at least 2048^2 zones, 128-column strips compiled
// for 6 resident CTAs per SM below that (64-column strips and 12 CTAs for
// narrow grids), and rows per CTA chosen for whole waves (below). (Measured
// per step at 32 and 16 rows: 4096^2 2.188 -> 2.157 ms and 2048^2 0.657 ->
// 0.637 ms with 256 columns; 1024^2 0.232 -> 0.234 ms.)
LaunchShape stage_shape(int ni, int nj, int bj, int rows, int occupancy = 0)
{
    LaunchShape s;
    if (bj != 64 && bj != 128 && bj != 256) {
        bj = nj >= 2048 && (long)ni * nj >= 2048L * 2048 ? 256 : (nj > 96 ? 128 : 64);
        if (occupancy == 0)
            occupancy = bj == 128 ? 6 : 12;
    }
    s.minb = 1;
    // 256-column strips: 3 CTAs per SM (80 registers, 68 KB of shared memory each)
    if (bj == 256)
        s.minb = 3;
    if (bj == 128 && (occupancy == 5 || occupancy == 6))
        s.minb = occupancy;
    if (bj == 64 && (occupancy == 10 || occupancy == 12))
        s.minb = occupancy;
    const int strips = (nj + bj - 1) / bj;
    if (rows <= 0) {
        // The CTAs should fill whole waves of the resident slots: a last,
        // partial wave leaves SMs idle at the end of the launch (4096^2 at
        // 256 columns: 37 rows, 4.0 waves, 2.127 ms per step; 36 rows, 4.11
        // waves, 2.239 ms; 32 rows, 4.61 waves, 2.150 ms). Each CTA also
        // recomputes about two rows' worth of slopes and faces at its
        // segment's top, and a single wave starts every CTA at once
        // (2048^2: 19 rows in 1.95 waves 0.607 ms, 38 rows in 0.97 waves
        // 0.628 ms; 1024^2 at 128 columns: 10 rows in 0.93 waves 0.212 ms,
        // 5 rows in 1.85 waves 0.219 ms). Score of r rows in W waves:
        // (W / ceil(W)) (r / (r + 2)), times 0.95 below 1.5 waves.
        const int slots = 148 * (s.minb > 1 ? s.minb : 4);
        rows = 4;
        double best = -1.0;
        for (int r = 48; r >= 4; --r) {
            const double waves = (double)strips * ((ni + r - 1) / r) / slots;
            const double score = waves / std::ceil(waves) * r / (r + 2.0) * (waves < 1.5 ? 0.95 : 1.0);
            if (score > best * (1.0 + 1e-3)) {
                best = score;
                rows = r;
            }
        }
    }
    if (rows < 4)
        rows = 4;
    s.bj = bj;
    s.rows = rows;
    s.grid = dim3(strips, (ni + rows - 1) / rows, 1);
    return s;
}

cudaError_t dispatch_stage(int precision, const LaunchShape &s, const Consts &k, const StageDev &st,
                           const StageArgs &a, cudaStream_t stream, int role = ROLE_NONE)
{
    switch (precision) {
    case CBD_PRECISION_EXACT:
        return launch_stage_exact(s, k, st, a, role, stream);
    case CBD_PRECISION_FMA:
        return launch_stage_fma(s, k, st, a, role, stream);
    default:
        return launch_stage_fast(s, k, st, a, role, stream);
    }
}

StageDev stage_dev_from(const cbd_grid_t *g, const cbd_stage_t *stage, const cbd_epilogue_t *ep)
{
    StageDev st;
    std::memset(&st, 0, sizeof(st));
    st.m[0] = mass_dev(stage->mass[0]);
    st.m[1] = mass_dev(stage->mass[1]);
    if (ep) {
        st.e[0] = mass_dev(ep->mass[0]);
        st.e[1] = mass_dev(ep->mass[1]);
    }
    st.a = stage->a;
    st.one_minus_a = 1.0 - stage->a;
    st.dt = stage->dt;
    st.buffer_mass = stage->buffer_central_mass;
    st.buffer_k = g->buffer_is_enabled
                      ? buffer_k(g->buffer_driving_rate, stage->buffer_central_mass,
                                 g->buffer_outer_radius - g->buffer_onset_width)
                      : 0.0;
    return st;
}

}  // namespace

int cbd::set_diagnostics(Consts &k, const cbd_epilogue_t *ep, int first, int count)
{
    k.num_diag = count;
    k.need_rates = 0;
    k.rates_only = 1;
    for (int d = 0; d < count; ++d) {
        const cbd_diag_t &src = ep->diag[first + d];
        if (src.quantity < CBD_Q_MDOT || src.quantity > CBD_Q_POWER || src.which_mass < 1 || src.which_mass > 3)
            return CBD_ERR_ARGUMENT;
        k.diag[d] = src;
        const bool rate = src.quantity == CBD_Q_MDOT || src.quantity == CBD_Q_FX || src.quantity == CBD_Q_FY ||
                          src.quantity == CBD_Q_TORQUE || src.quantity == CBD_Q_POWER;
        if (rate)
            k.need_rates |= (src.which_mass & 3) << (src.accretion ? 2 : 0);
        if (!rate || src.has_cut)
            k.rates_only = 0;
    }
    return CBD_OK;
}

namespace cbd {
cudaStream_t drop_in_stream() { return g_stream; }
}  // namespace cbd

extern "C" {

int cbdiso_b200_version(void) { return 1; }

int cbdiso_b200_epilogue_rates_only(const cbd_epilogue_t *ep)
{
    if (!ep || ep->num_diag < 0 || ep->num_diag > MAX_FUSED)
        return -1;
    Consts k;
    std::memset(&k, 0, sizeof(k));
    return set_diagnostics(k, ep, 0, ep->num_diag) == CBD_OK ? k.rates_only : -1;
}

int cbdiso_b200_set_stream(void *stream)
{
    g_stream = static_cast<cudaStream_t>(stream);
    return CBD_OK;
}

int cbdiso_b200_set_plm_theta(double theta)
{
    if (!(theta >= 1.0 && theta <= 2.0))
        return CBD_ERR_ARGUMENT;
    g_theta = theta;
    return CBD_OK;
}

int cbdiso_b200_set_precision(int precision)
{
    if (precision < CBD_PRECISION_EXACT || precision > CBD_PRECISION_FAST)
        return CBD_ERR_ARGUMENT;
    g_precision = precision;
    return CBD_OK;
}

const char *cbdiso_b200_status_string(int status)
{
    switch (status) {
    case CBD_OK:
        return "success";
    case CBD_ERR_ARGUMENT:
        return "invalid argument";
    case CBD_ERR_CUDA:
        return "CUDA runtime error";
    case CBD_ERR_NONFINITE:
        return "non-finite value";
    case CBD_ERR_TIMEOUT:
        return "device wait timed out";
    case CBD_ERR_KEPLER:
        return "Kepler solve did not converge";
    case CBD_ERR_CAPACITY:
        return "request exceeds library capacity";
    default:
        return "unknown status";
    }
}

// --------------------------------------------------------------------------
// drop-in kernels
// --------------------------------------------------------------------------

int cbdiso_2d_advance_rk(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    double *conserved_rk, double *primitive_rd, double *primitive_wr,
    double buffer_surface_density, double buffer_central_mass, double buffer_driving_rate,
    double buffer_outer_radius, double buffer_onset_width, int buffer_is_enabled,
    double x1, double y1, double vx1, double vy1, double mass1, double softening_length1,
    double sink_rate1, double sink_radius1, int sink_model1,
    double x2, double y2, double vx2, double vy2, double mass2, double softening_length2,
    double sink_rate2, double sink_radius2, int sink_model2,
    double cs2, double mach_squared, int eos_type, double nu, double a, double dt,
    double velocity_ceiling, double density_floor)
{
    if (ni <= 0 || nj <= 0 || !conserved_rk || !primitive_rd || !primitive_wr || primitive_rd == primitive_wr)
        return CBD_ERR_ARGUMENT;
    cbd_grid_t g;
    std::memset(&g, 0, sizeof(g));
    g.ni = ni;
    g.nj = nj;
    g.xl = patch_xl;
    g.xr = patch_xr;
    g.yl = patch_yl;
    g.yr = patch_yr;
    g.plm_theta = g_theta;
    g.eos_type = eos_type;
    g.precision = g_precision;
    g.cs2 = cs2;
    g.mach2 = mach_squared;
    g.nu = nu;
    g.velocity_ceiling = velocity_ceiling;
    g.density_floor = density_floor;
    g.buffer_is_enabled = buffer_is_enabled;
    g.buffer_surface_density = buffer_surface_density;
    g.buffer_driving_rate = buffer_driving_rate;
    g.buffer_outer_radius = buffer_outer_radius;
    g.buffer_onset_width = buffer_onset_width;
    Consts k = consts_from_grid(&g);
    // The reference kernel returns 1.0 for an unknown EOS (cbdiso_2d.c:208-209);
    // keep that behaviour rather than rejecting.
    k.eos = eos_type;
    k.un_kind = 2;
    k.write_guards = 0;

    StageDev st;
    std::memset(&st, 0, sizeof(st));
    st.m[0] = mass_dev(x1, y1, vx1, vy1, mass1, softening_length1, sink_rate1, sink_radius1, sink_model1);
    st.m[1] = mass_dev(x2, y2, vx2, vy2, mass2, softening_length2, sink_rate2, sink_radius2, sink_model2);
    st.a = a;
    st.one_minus_a = 1.0 - a;
    st.dt = dt;
    st.buffer_mass = buffer_central_mass;
    st.buffer_k = buffer_is_enabled ? buffer_k(buffer_driving_rate, buffer_central_mass, k.buf_onset) : 0.0;

    const LaunchShape s = stage_shape(ni, nj, 0, 0);
    k.rows_per_cta = s.rows;
    StageArgs args = {primitive_rd, conserved_rk, primitive_wr, nullptr, nullptr, nullptr, nullptr};
    return status_of(dispatch_stage(g_precision, s, k, st, args, g_stream));
}

int cbdiso_2d_primitive_to_conserved(int ni, int nj, double *primitive, double *conserved)
{
    if (ni <= 0 || nj <= 0 || !primitive || !conserved)
        return CBD_ERR_ARGUMENT;
    return status_of(launch_p2c(ni, nj, primitive, conserved, g_stream));
}

int cbdiso_2d_point_mass_source_term(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    double x1, double y1, double vx1, double vy1, double mass1, double softening_length1,
    double sink_rate1, double sink_radius1, int sink_model1,
    double *primitive, double *cons_rate)
{
    if (ni <= 0 || nj <= 0 || !primitive || !cons_rate)
        return CBD_ERR_ARGUMENT;
    const double dx = (patch_xr - patch_xl) / ni;
    const double dy = (patch_yr - patch_yl) / nj;
    const MassDev m = mass_dev(x1, y1, vx1, vy1, mass1, softening_length1, sink_rate1, sink_radius1, sink_model1);
    return status_of(launch_source(ni, nj, patch_xl, patch_yl, dx, dy, m, primitive, cons_rate, g_stream));
}

int cbdiso_2d_wavespeed(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    double soundspeed2, double mach_squared, int eos_type,
    double x1, double y1, double vx1, double vy1, double mass1, double softening_length1,
    double sink_rate1, double sink_radius1, int sink_model1,
    double x2, double y2, double vx2, double vy2, double mass2, double softening_length2,
    double sink_rate2, double sink_radius2, int sink_model2,
    double *primitive, double *wavespeed)
{
    if (ni <= 0 || nj <= 0 || !primitive || !wavespeed)
        return CBD_ERR_ARGUMENT;
    Consts k;
    std::memset(&k, 0, sizeof(k));
    k.ni = ni;
    k.nj = nj;
    k.xl = patch_xl;
    k.yl = patch_yl;
    k.dx = (patch_xr - patch_xl) / ni;
    k.dy = (patch_yr - patch_yl) / nj;
    k.eos = eos_type;
    k.cs2 = soundspeed2;
    k.mach2 = mach_squared;
    k.inv_mach2 = 1.0 / mach_squared;
    k.neg_inv_mach2 = -1.0 / mach_squared;
    const MassDev m0 = mass_dev(x1, y1, vx1, vy1, mass1, softening_length1, sink_rate1, sink_radius1, sink_model1);
    const MassDev m1 = mass_dev(x2, y2, vx2, vy2, mass2, softening_length2, sink_rate2, sink_radius2, sink_model2);
    return status_of(launch_wavespeed(k, m0, m1, primitive, wavespeed, g_stream));
}

// --------------------------------------------------------------------------
// fused product path
// --------------------------------------------------------------------------

void cbdiso_b200_abi_sizes(size_t out[4])
{
    out[0] = sizeof(cbd_mass_t);
    out[1] = sizeof(cbd_grid_t);
    out[2] = sizeof(cbd_stage_t);
    out[3] = sizeof(cbd_epilogue_t);
}

size_t cbdiso_b200_scratch_bytes(const cbd_grid_t *grid)
{
    if (!valid_grid(grid))
        return 0;
    const LaunchShape s = stage_shape(grid->ni, grid->nj, 64, 4);
    size_t ctas = (size_t)s.grid.x * s.grid.y;
    const size_t r = (size_t)reduce_ctas(grid->ni, grid->nj);
    if (r > ctas)
        ctas = r;
    return 64 + ctas * PARTIAL_STRIDE * sizeof(double);
}

int cbdiso_b200_fill_guards(const cbd_grid_t *grid, double *primitive, void *stream)
{
    if (!valid_grid(grid) || !primitive)
        return CBD_ERR_ARGUMENT;
    return status_of(launch_fill_guards(grid->ni, grid->nj, primitive, static_cast<cudaStream_t>(stream)));
}

size_t cbdiso_b200_stage_record_bytes(void) { return sizeof(StageDev); }

int cbdiso_b200_stage_record(const cbd_grid_t *grid, const cbd_stage_t *stage, const cbd_epilogue_t *epilogue,
                             void *record)
{
    if (!valid_grid(grid) || !stage || !record)
        return CBD_ERR_ARGUMENT;
    StageDev st = stage_dev_from(grid, stage, epilogue);
    std::memcpy(record, &st, sizeof(st));
    return CBD_OK;
}

}  // extern "C"

namespace {

int advance_stage(const cbd_grid_t *grid, const cbd_stage_t *stage, const void *stage_dev,
                  const double *primitive_rd, const double *primitive_n, double *primitive_wr,
                  const cbd_epilogue_t *epilogue, double *scratch, double *result, double *face_cache,
                  int role, void *stream)
{
    if (!valid_grid(grid) || !stage || !primitive_rd || !primitive_wr || primitive_rd == primitive_wr)
        return CBD_ERR_ARGUMENT;
    if (!primitive_n && stage->a != 0.0 && !stage_dev)
        return CBD_ERR_ARGUMENT;
    Consts k = consts_from_grid(grid);
    k.un_kind = primitive_n ? 1 : 0;
    k.write_guards = 1;

    const StageDev st = stage_dev_from(grid, stage, epilogue);
    if (epilogue) {
        if (!scratch || !result)
            return CBD_ERR_ARGUMENT;
        if (epilogue->num_diag < 0 || epilogue->num_diag > MAX_FUSED)
            return CBD_ERR_CAPACITY;
        k.want_ws = epilogue->want_wavespeed ? 1 : 0;
        const int rc = set_diagnostics(k, epilogue, 0, epilogue->num_diag);
        if (rc != CBD_OK)
            return rc;
    }
    const LaunchShape s = stage_shape(grid->ni, grid->nj, grid->tile_columns, grid->tile_rows, grid->tile_occupancy);
    k.rows_per_cta = s.rows;
    StageArgs args = {primitive_rd, primitive_n, primitive_wr, static_cast<const StageDev *>(stage_dev), scratch,
                      result, face_cache};
    return status_of(dispatch_stage(grid->precision, s, k, st, args, static_cast<cudaStream_t>(stream), role));
}

}  // namespace

extern "C" {

int cbdiso_b200_advance_stage(
    const cbd_grid_t *grid, const cbd_stage_t *stage, const void *stage_dev,
    const double *primitive_rd, const double *primitive_n, double *primitive_wr,
    const cbd_epilogue_t *epilogue, double *scratch, double *result, void *stream)
{
    return advance_stage(grid, stage, stage_dev, primitive_rd, primitive_n, primitive_wr, epilogue, scratch,
                         result, nullptr, ROLE_NONE, stream);
}

size_t cbdiso_b200_face_cache_bytes(const cbd_grid_t *grid)
{
    if (!valid_grid(grid))
        return 0;
    return face_cache_doubles(grid->ni, grid->nj) * sizeof(double);
}

int cbdiso_b200_advance_stage_cached(
    const cbd_grid_t *grid, const cbd_stage_t *stage, const void *stage_dev,
    const double *primitive_rd, const double *primitive_n, double *primitive_wr,
    const cbd_epilogue_t *epilogue, double *scratch, double *result, double *face_cache, int role, void *stream)
{
    // the cache's pairs are loaded and stored as 16-byte vectors
    if (!face_cache || (reinterpret_cast<uintptr_t>(face_cache) & 15) != 0 || role < ROLE_NONE ||
        role > ROLE_READER)
        return CBD_ERR_ARGUMENT;
    return advance_stage(grid, stage, stage_dev, primitive_rd, primitive_n, primitive_wr, epilogue, scratch,
                         result, face_cache, role, stream);
}

int cbdiso_b200_reduce(
    const cbd_grid_t *grid, const cbd_epilogue_t *epilogue, const double *primitive,
    double *scratch, double *result, void *stream)
{
    if (!valid_grid(grid) || !epilogue || !primitive || !scratch || !result)
        return CBD_ERR_ARGUMENT;
    if (epilogue->num_diag < 0 || epilogue->num_diag > CBD_MAX_DIAG)
        return CBD_ERR_CAPACITY;
    Consts k = consts_from_grid(grid);
    StageDev st;
    std::memset(&st, 0, sizeof(st));
    st.e[0] = mass_dev(epilogue->mass[0]);
    st.e[1] = mass_dev(epilogue->mass[1]);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int first = 0;
    bool ws = epilogue->want_wavespeed != 0;
    do {
        const int count = epilogue->num_diag - first < MAX_FUSED ? epilogue->num_diag - first : MAX_FUSED;
        const int rc = set_diagnostics(k, epilogue, first, count);
        if (rc != CBD_OK)
            return rc;
        k.want_ws = ws ? 1 : 0;
        const cudaError_t e = launch_reduce(k, st, primitive, scratch, ws ? result : nullptr,
                                            result + 1 + 2 * first, s);
        if (e != cudaSuccess)
            return CBD_ERR_CUDA;
        ws = false;
        first += count;
    } while (first < epilogue->num_diag);
    return CBD_OK;
}

int cbdiso_b200_eval_primitives(long n, const double *a, const double *b, double *out, void *stream)
{
    if (n < 0 || (n > 0 && (!a || !b || !out)))
        return CBD_ERR_ARGUMENT;
    if (n == 0)
        return CBD_OK;
    return status_of(launch_primitives(n, a, b, out, static_cast<cudaStream_t>(stream)));
}

}  // extern "C"
