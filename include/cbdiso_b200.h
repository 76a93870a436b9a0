/*
 * cbdiso_b200: a B200 (sm_100a) implementation of sailfish's 2D isothermal
 * circumbinary-disk solver, cbdiso_2d, as a C-ABI shared library
 * (libcbdiso_b200.so).
 *
 * Two groups of entry points:
 *
 *  1. Drop-in kernels. Same symbol names and the same positional arguments as
 *     the four public kernels of sailfish/solvers/cbdiso_2d.c, so a binding
 *     written for the reference's kernel library can call them unchanged. The
 *     differences: array pointers are DEVICE pointers, launches go to the
 *     library's current stream (cbdiso_b200_set_stream), the PLM parameter
 *     theta is a library setting (cbdiso_b200_set_plm_theta, default 1.8 as in
 *     cbdiso_2d.c:11), and each returns an int status (0 = success) where the
 *     reference returns void.
 *
 *  2. The fused product path used by the Python solver: one kernel per RK
 *     stage with boundary conditions, the RK average and, on the final stage,
 *     the next step's CFL wavespeed and the diagnostics reductions fused in;
 *     plus the batched many-disk form and the tangent / adjoint kernels.
 *
 *  3. The gamma-law sibling, cbdgam_2d: its four drop-in kernels
 *     (sailfish/solvers/cbdgam_2d.c) and a product stage with fused guards.
 *
 * Arrays use the reference layout: C-contiguous (ni + 4, nj + 4, 3) float64,
 * two guard zones per side, j fastest, then the field (Sigma, vx, vy) or
 * (Sigma, Sigma vx, Sigma vy).
 */
#ifndef CBDISO_B200_H
#define CBDISO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * status codes
 * ---------------------------------------------------------------------- */
enum {
    CBD_OK = 0,
    CBD_ERR_ARGUMENT = 1,   /* bad sizes, null pointers, unsupported option */
    CBD_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    CBD_ERR_NONFINITE = 3,  /* a non-finite value was found where it must not be */
    CBD_ERR_TIMEOUT = 4,    /* a bounded device-side wait ran out */
    CBD_ERR_KEPLER = 5,     /* device Kepler solve did not converge in 10 steps */
    CBD_ERR_CAPACITY = 6    /* request exceeds a fixed capacity of the library */
};

/* arithmetic of the fused stencil */
enum {
    CBD_PRECISION_EXACT = 0, /* IEEE divide / sqrt, the reference's operation order, no FMA contraction */
    CBD_PRECISION_FMA = 1,   /* as EXACT but the compiler may contract a*b+c into FMA */
    CBD_PRECISION_FAST = 2   /* FMA, reciprocal multiplies, rsqrt-based gravity */
};

/* ------------------------------------------------------------------------
 * 1. drop-in kernels (sailfish/solvers/cbdiso_2d.c:385-722)
 * ---------------------------------------------------------------------- */

/* replaces cbdiso_2d_advance_rk, sailfish/solvers/cbdiso_2d.c:385-426 */
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
    double velocity_ceiling, double density_floor);

/* replaces cbdiso_2d_primitive_to_conserved, sailfish/solvers/cbdiso_2d.c:606-610 */
int cbdiso_2d_primitive_to_conserved(int ni, int nj, double *primitive, double *conserved);

/* replaces cbdiso_2d_point_mass_source_term, sailfish/solvers/cbdiso_2d.c:626-643 */
int cbdiso_2d_point_mass_source_term(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    double x1, double y1, double vx1, double vy1, double mass1, double softening_length1,
    double sink_rate1, double sink_radius1, int sink_model1,
    double *primitive, double *cons_rate);

/* replaces cbdiso_2d_wavespeed, sailfish/solvers/cbdiso_2d.c:666-695 */
int cbdiso_2d_wavespeed(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    double soundspeed2, double mach_squared, int eos_type,
    double x1, double y1, double vx1, double vy1, double mass1, double softening_length1,
    double sink_rate1, double sink_radius1, int sink_model1,
    double x2, double y2, double vx2, double vy2, double mass2, double softening_length2,
    double sink_rate2, double sink_radius2, int sink_model2,
    double *primitive, double *wavespeed);

/* library settings used by the drop-in kernels (no counterpart in the
 * reference, whose kernels take no stream and fix theta at compile time) */
int cbdiso_b200_set_stream(void *cuda_stream);
int cbdiso_b200_set_plm_theta(double theta);
int cbdiso_b200_set_precision(int precision);
const char *cbdiso_b200_status_string(int status);
int cbdiso_b200_version(void);

/* ------------------------------------------------------------------------
 * 2. fused product path
 * ---------------------------------------------------------------------- */

/* One point mass (sailfish/physics/circumbinary.py:41-95). */
typedef struct cbd_mass {
    double x, y, vx, vy;
    double mass;
    double softening_length;
    double sink_rate;
    double sink_radius;
    int sink_model;  /* 0 inactive, 1 acceleration-free, 2 torque-free, 3 force-free */
    int _pad0;
} cbd_mass_t;

/* Mesh, equation of state and solver options: constant over a run. */
typedef struct cbd_grid {
    int ni, nj;
    double xl, xr, yl, yr;  /* patch extent (vertex coordinates); dx = (xr - xl) / ni */
    double plm_theta;
    int eos_type;           /* 1 globally isothermal, 2 locally isothermal */
    int precision;          /* CBD_PRECISION_* */
    double cs2;             /* sound_speed^2 (eos 1) */
    double mach2;           /* mach_number^2 (eos 2) */
    double nu;              /* constant kinematic viscosity, 0 = inviscid */
    double velocity_ceiling;
    double density_floor;
    int buffer_is_enabled;
    int tile_columns;       /* CTA strip width: 64 or 128; 0 = library default */
    int tile_rows;          /* rows per CTA segment; 0 = library default */
    int tile_occupancy;     /* resident CTAs per SM the kernel is built for: 0 default, 5 or 6 (128 wide), 10 or 12 (64 wide) */
    double buffer_surface_density;
    double buffer_driving_rate;
    double buffer_outer_radius;
    double buffer_onset_width;
} cbd_grid_t;

/* Everything that changes per RK stage. */
typedef struct cbd_stage {
    cbd_mass_t mass[2];     /* point masses at the stage's start time */
    double a;               /* RK weight of u_n: u <- (1 - a) (u + du) + a u_n */
    double dt;
    double buffer_central_mass;  /* m1 + m2 */
} cbd_stage_t;

/* Diagnostics (sailfish/physics/circumbinary.py:24-38, cbdiso_2d.py:383-471) */
enum {
    CBD_Q_MDOT = 1, CBD_Q_FX = 2, CBD_Q_FY = 3, CBD_Q_TORQUE = 4, CBD_Q_SIGMA_M1 = 5,
    CBD_Q_ECCENTRICITY_VECTOR = 6, CBD_Q_ANGULAR_MOMENTUM = 7, CBD_Q_MASS = 8, CBD_Q_POWER = 9
};
#define CBD_MAX_DIAG 16

typedef struct cbd_diag {
    int quantity;           /* CBD_Q_* */
    int which_mass;         /* 1, 2, or 3 for 'both' */
    int gravity;            /* include the gravity term */
    int accretion;          /* include the accretion term */
    int has_cut;            /* radial cut r0 < r < r1 */
    int _pad;
    double r0, r1;
} cbd_diag_t;

/* Quantities computed on the updated state at the end of a step: the CFL
 * wavespeed maximum and the diagnostic sums, with point masses at `mass`
 * (the end-of-step time). Results land in `result`:
 *   result[0] = max wavespeed, result[1 + 2k], result[2 + 2k] = real and
 *   imaginary part of sum_cells f_k (not yet multiplied by dx dy). */
typedef struct cbd_epilogue {
    cbd_mass_t mass[2];
    int want_wavespeed;
    int num_diag;
    cbd_diag_t diag[CBD_MAX_DIAG];
} cbd_epilogue_t;

/* sizeof of cbd_mass_t, cbd_grid_t, cbd_stage_t, cbd_epilogue_t, for
 * bindings to check their struct layouts against. */
void cbdiso_b200_abi_sizes(size_t out[4]);

/* Bytes of device scratch the fused reductions need for this grid. */
size_t cbdiso_b200_scratch_bytes(const cbd_grid_t *grid);

/* Fill the two guard zones per side by zero-gradient extrapolation
 * (equivalent to cbdiso_2d.py:553-586 on one patch). */
int cbdiso_b200_fill_guards(const cbd_grid_t *grid, double *primitive, void *stream);

/* One fused RK stage: reads primitive_rd (guards valid), writes the interior
 * and the guard zones of primitive_wr. For a > 0 the stage's u_n is formed
 * from primitive_n (the state at the start of the step). primitive_wr may
 * equal primitive_n (in-place final stage). If `epilogue` is non-null its
 * quantities are reduced into `result` using `scratch`
 * (cbdiso_b200_scratch_bytes). `stage_dev`, when non-null, is a device-side
 * stage record written by the library's own device stepping kernels and read
 * instead of `stage` (used under CUDA graph capture). */
int cbdiso_b200_advance_stage(
    const cbd_grid_t *grid, const cbd_stage_t *stage, const void *stage_dev,
    const double *primitive_rd, const double *primitive_n, double *primitive_wr,
    const cbd_epilogue_t *epilogue, double *scratch, double *result, void *stream);

/* Size of the device-side stage record, and a host routine that fills one
 * from a stage (and the end-of-step masses of an epilogue, may be null). A
 * caller copies records to device memory and passes them as `stage_dev`, so
 * a step's inputs travel as one explicit host-to-device copy. */
size_t cbdiso_b200_stage_record_bytes(void);
int cbdiso_b200_stage_record(const cbd_grid_t *grid, const cbd_stage_t *stage, const cbd_epilogue_t *epilogue,
                             void *record);

/* cbdiso_b200_advance_stage with a face cache (no counterpart in the
 * reference, which recomputes these values in every stage,
 * cbdiso_2d.c:555-558 and :97-175).
 *
 * The face sound speeds and the zones' gravity factors depend only on the mesh,
 * the EOS constants and the point masses' positions, masses and softenings, so
 * a step's first stage can reuse what the previous step's last stage computed
 * for the same masses. `role`:
 *   0  no cache use (as cbdiso_b200_advance_stage);
 *   1  writer (RK2's second stage, RK3's second): when the stage's masses equal
 *      its record's end-of-step masses, also stores the values in `face_cache`
 *      with a key of everything they depend on;
 *   2  reader (a step's first stage): a fill pass before the stage computes
 *      the values when the key does not match the stage's masses; the stage
 *      loads them and records the key.
 * In EXACT precision the results are bit-identical to
 * cbdiso_b200_advance_stage (in FMA and FAST the compiler may contract the code
 * paths differently: equal to rounding). `face_cache` is a caller-owned,
 * 16-byte aligned device buffer of cbdiso_b200_face_cache_bytes(grid) bytes for
 * this grid only; zero its first 256 bytes before its first use. Calls on one
 * cache must be ordered on one stream. */
size_t cbdiso_b200_face_cache_bytes(const cbd_grid_t *grid);
int cbdiso_b200_advance_stage_cached(
    const cbd_grid_t *grid, const cbd_stage_t *stage, const void *stage_dev,
    const double *primitive_rd, const double *primitive_n, double *primitive_wr,
    const cbd_epilogue_t *epilogue, double *scratch, double *result, double *face_cache, int role,
    void *stream);

/* cbdiso_b200_advance_stage without a scratch argument (no counterpart in the
 * reference, whose kernels take only the solver's own arrays).
 *
 * Some callers cannot allocate device memory: a binding written against the
 * reference's kernel interface passes only the arrays its solver already owns
 * and has no buffer to offer as scratch, and host applications that account
 * for all device memory through their own pool do not let a library call
 * cudaMalloc behind their back. This entry point allocates nothing. The
 * epilogue's reductions scratch is a fixed 5 MiB array inside the library's
 * device memory (each GPU that loads the library holds it until the process
 * exits); the caller still passes the state arrays and `result`.
 *
 * Limit: a call with an epilogue on a grid whose cbdiso_b200_scratch_bytes()
 * exceeds 5 MiB is rejected with CBD_ERR_CAPACITY before anything is
 * launched; 4096 x 4096 fits. A call without an epilogue uses no scratch and
 * has no such limit.
 * The first call with an epilogue on a device looks up the array's device
 * address for that device and keeps it for the life of the process, so make
 * that first call before any stream capture, and make no call after
 * cudaDeviceReset (the kept address would be stale). All calls on a device
 * share the array, which keeps the last call's contents (each call clears the
 * counter it needs zeroed): calls that overlap on the GPU, from different
 * streams or threads, race on it. */
int cbdiso_b200_advance_stage_noalloc(
    const cbd_grid_t *grid, const cbd_stage_t *stage, const void *stage_dev,
    const double *primitive_rd, const double *primitive_n, double *primitive_wr,
    const cbd_epilogue_t *epilogue, double *result, void *stream);

/* ------------------------------------------------------------------------
 * device-resident stepping (no counterpart in the reference, whose driver
 * computes dt and the point masses on the host every step)
 * ---------------------------------------------------------------------- */

/* A binary on a Kepler orbit with identical sink / softening settings for
 * both components, as the circumbinary setups build it
 * (sailfish/setups/circumbinary_disk.py:185-212, binary_bondi.py:79-102). */
typedef struct cbd_orbit {
    double semimajor_axis, total_mass, mass_ratio, eccentricity;
    double softening_length, sink_rate, sink_radius;
    int sink_model;
    int has_x_offset;       /* shift both x positions by x_offset */
    double x_offset;
} cbd_orbit_t;

/* Size of the stepper's device record, and its initial contents (written to
 * host memory; the caller copies it to device memory). The stepper keeps the
 * time, the last dt and a status word; min_spacing is the mesh's
 * min(dx, dy) as the driver uses it; fixed_dt > 0 freezes dt. */
size_t cbdiso_b200_stepper_bytes(void);
int cbdiso_b200_stepper_init(const cbd_grid_t *grid, const cbd_orbit_t *orbit, int rk_order, double time,
                             double cfl, double min_spacing, double fixed_dt, int series_capacity, void *stepper);

/* Attach to a host copy of a stepper record (before copying it to the
 * device): a device array of dt_count time steps to use instead of the CFL
 * rule (a frozen dt sequence), and/or a device array of history_capacity *
 * rk_order stage records that receives every step's stage records. */
int cbdiso_b200_stepper_attach(void *stepper, const double *dt_sequence, int dt_count, void *history,
                               int history_capacity);

/* One step's prologue (a single-thread kernel): records the previous step's
 * time-series row [time, dt, max wavespeed, num_values reduction values] from
 * `result` into `series` (if non-null), then, unless `finalize`, takes
 * dt = min_spacing / max wavespeed * cfl, solves the Kepler orbit at every
 * stage time and at the end of the step, and writes the stage records that
 * cbdiso_b200_advance_stage reads as `stage_dev`. A Kepler solve that does
 * not converge sets the stepper's status to CBD_ERR_KEPLER and stops it. A
 * dt that is not finite and positive (a NaN, infinite or zero wavespeed, or
 * such an entry of a frozen dt sequence) sets CBD_ERR_NONFINITE, stops the
 * stepper and marks the step's stage records halted: stage launches that
 * read them return without touching any array, so a captured sequence of
 * steps leaves the state as it was before the failing step. (The reference's
 * driver has no such check, sailfish/driver.py:508-510.) */
int cbdiso_b200_step_prologue(void *stepper_dev, const double *result, void *records_dev, double *series,
                              int num_values, int finalize, void *stream);

/* ------------------------------------------------------------------------
 * batched: many disks of different sizes and physics per launch (no
 * counterpart in the reference, which advances one grid at a time)
 * ---------------------------------------------------------------------- */

/* Size of a disk record, and a host routine filling one: the disk's kernel
 * constants from `grid`, its fused diagnostics (up to four; null: wavespeed
 * only), its tile shape (strip_width in 32..128 columns, rows per tile), the
 * offset in doubles of its (ni + 4, nj + 4, 3) state in the batch buffers and
 * the index of its first tile in the batch; *units receives its tile count.
 * Records are copied to a device array ordered by unit_begin. */
size_t cbdiso_b200_batch_disk_bytes(void);
/* 1 when every diagnostic of `ep` is a source rate of the masses (mdot,
 * fx, fy, torque, power) without a radial cut, else 0; -1 for a null or
 * malformed epilogue or one of more than four diagnostics. The stage epilogue takes a kernel compiled
 * for such diagnostics by itself; the batched stage takes it on request
 * (`epilogue` 2). No counterpart in the reference. */
int cbdiso_b200_epilogue_rates_only(const cbd_epilogue_t *ep);
int cbdiso_b200_batch_disk_record(const cbd_grid_t *grid, const cbd_epilogue_t *diagnostics, int strip_width,
                                  int rows, long long offset, int unit_begin, int *units, void *record);

/* One RK stage of every disk in one persistent launch: CTAs take tiles from
 * counters[0] until all total_units are done (both counters return to zero).
 * Stage records are read from records[disk * num_stages + stage]; with
 * `epilogue` (1), each tile's wavespeed / diagnostic partial goes to
 * partials[tile * 9 ...]. `epilogue` 2 does the same with the kernel
 * compiled for diagnostics that are all source rates of the masses without
 * a radial cut (cbdiso_b200_epilogue_rates_only true for every disk's
 * diagnostics; fewer registers, the same values); a disk whose diagnostics
 * are not gets NaN sums. primitive_n (null for the a = 0 stage) gives u_n. */
int cbdiso_b200_batched_stage(const void *disks, int num_disks, int total_units, const double *primitive_rd,
                              const double *primitive_n, double *primitive_wr, const void *records, int num_stages,
                              int stage, int epilogue, double *partials, unsigned int *counters, int precision,
                              void *stream);

/* cbdiso_b200_batched_stage with face caches and a role (as in
 * cbdiso_b200_advance_stage_cached: 0 none, 1 writer, 2 reader, the reader
 * preceded by a fill pass over every disk's tiles). Disk d's cache lies at face_cache + its
 * record's cache offset, set by cbdiso_b200_batch_disk_set_face_cache (an even
 * number of doubles); it holds cbdiso_b200_face_cache_bytes(its grid) bytes
 * with its first 256 bytes zeroed before the first use, and `face_cache` is
 * 16-byte aligned. A reader needs a cache for every disk: it leaves the tiles
 * of a disk without one unwritten. No counterpart in the reference. */
int cbdiso_b200_batch_disk_set_face_cache(void *record, long long cache_offset);
int cbdiso_b200_batched_stage_cached(const void *disks, int num_disks, int total_units, const double *primitive_rd,
                                     const double *primitive_n, double *primitive_wr, const void *records,
                                     int num_stages, int stage, int epilogue, double *partials,
                                     unsigned int *counters, int precision, double *face_cache, int role,
                                     void *stream);

/* Per-disk reduction of the tile partials, in tile order: results[d * stride]
 * = max wavespeed, then the diagnostic sums. */
int cbdiso_b200_batched_finalize(const void *disks, int num_disks, const double *partials, double *results,
                                 int result_stride, void *stream);

/* Per-disk step prologue (see cbdiso_b200_step_prologue), one stepper record
 * per disk in `steppers`; each disk's series block holds its
 * series_capacity rows. */
int cbdiso_b200_batched_prologue(void *steppers, int num_disks, const double *results, int result_stride,
                                 void *records, double *series, int num_values, int finalize, void *stream);

/* ------------------------------------------------------------------------
 * differentiation: tangent and discrete adjoint of a stage and of the
 * objective (no counterpart in the reference)
 *
 * Parameter vectors have 12 entries: mass 1 (x, y, vx, vy, mass), mass 2
 * (x, y, vx, vy, mass), nu, sink rate. Stage records are device records as
 * written by cbdiso_b200_step_prologue / cbdiso_b200_stage_record.
 * ---------------------------------------------------------------------- */

/* Device workspace bytes for cbdiso_b200_stage_adjoint / objective_adjoint. */
size_t cbdiso_b200_adjoint_workspace_bytes(const cbd_grid_t *grid);

/* Records the branches the stage took (limiter choices, HLLE wave choices,
 * floor and ceiling) as one 32-bit word per zone of the padded layout, from
 * the stage's input and output states, for the adjoint to replay. */
int cbdiso_b200_stage_record_branches(const cbd_grid_t *grid, const void *stage_dev, const double *primitive_rd,
                                      const double *primitive_out, unsigned int *words, void *stream);

/* Forward-mode tangent of a stage: primitive_out and its derivative along
 * (dprimitive_rd, dprimitive_n, dmass[10], dnu, drate); guards of both
 * outputs are filled. primitive_n null means the a = 0 stage. */
int cbdiso_b200_stage_tangent(const cbd_grid_t *grid, const void *stage_dev, const double *dmass, double dnu,
                              double drate, const double *primitive_rd, const double *dprimitive_rd,
                              const double *primitive_n, const double *dprimitive_n, double *primitive_out,
                              double *dprimitive_out, void *stream);

/* Adjoint of a stage: given lam_out (adjoint of primitive_out, zero guards),
 * ADDS the adjoint of primitive_rd into lam_rd and of primitive_n into lam_n
 * (interior zones; guard contributions folded), and ADDS the 12 parameter
 * derivatives into params_out. */
int cbdiso_b200_stage_adjoint(const cbd_grid_t *grid, const void *stage_dev, const double *primitive_rd,
                              const double *primitive_n, const double *primitive_out, const unsigned int *words,
                              const double *lam_out, double *lam_rd, double *lam_n, double *params_out,
                              void *workspace, void *stream);

/* Objective F = sum over zones of w_mdot * (-(mdot_1 + mdot_2)) + w_torque *
 * torque, with the stage record's end-of-step masses (cbdiso_2d.py:383-471
 * rates). Tangent: per-block partial sums of dF into `partials`. Adjoint:
 * ADDS dF/dprimitive into lam and the 12 parameter derivatives into
 * params_out. */
int cbdiso_b200_objective_tangent(const cbd_grid_t *grid, const void *stage_dev, const double *dmass,
                                  double drate, const double *primitive, const double *dprimitive, double w_mdot,
                                  double w_torque, double *partials, int num_partials, void *stream);
int cbdiso_b200_objective_adjoint(const cbd_grid_t *grid, const void *stage_dev, const double *primitive,
                                  double w_mdot, double w_torque, double *lam, double *params_out, void *workspace,
                                  void *stream);

/* Chained forms for a whole reverse sweep: the stage adjoint records the
 * stage's branches itself (into the workspace); instead of 12 parameter
 * derivatives per call, the mass-parameter part is contracted on the device
 * with `jacobian` (device memory, 10 x 2 row-major: d(x, y, vx, vy, mass of
 * mass 1, then of mass 2) / d(q, e) at this stage's time) and ADDED per
 * block into `chain_acc` (device, cbdiso_b200_adjoint_chain_blocks(grid) x 4
 * doubles: d/dq, d/de, d/dnu, d/d(sink rate)), which the caller zeroes once
 * before the sweep. cbdiso_b200_adjoint_chain_finish ADDS the block sums, in
 * a fixed order, into out4 (device, 4 doubles). The chained objective's
 * weights are per unit time: each is multiplied by the record's dt. */
int cbdiso_b200_stage_adjoint_chained(const cbd_grid_t *grid, const void *stage_dev, const double *primitive_rd,
                                      const double *primitive_n, const double *primitive_out, const double *lam_out,
                                      double *lam_rd, double *lam_n, const double *jacobian, double *chain_acc,
                                      void *workspace, void *stream);
int cbdiso_b200_objective_adjoint_chained(const cbd_grid_t *grid, const void *stage_dev, const double *primitive,
                                          double w_mdot, double w_torque, double *lam, const double *jacobian,
                                          double *chain_acc, void *workspace, void *stream);
size_t cbdiso_b200_adjoint_chain_blocks(const cbd_grid_t *grid);

/* Test hook (no counterpart in the reference): 1 (default) runs each stage
 * adjoint as one fused row-marching kernel, 0 as separate passes over the
 * zones and faces; lambda_rd and lambda_n agree bit for bit, the parameter
 * sums to rounding. Process-wide. */
int cbdiso_b200_set_adjoint_variant(int fused);

/* Rows per CTA segment of the fused stage adjoint (no counterpart in the
 * reference). 0 (default): chosen per grid to finish a lone sweep soonest
 * (whole waves of CTAs; short segments on small grids); 4 .. 32: fixed, for
 * sweeps that share the GPU with others (several disks over streams), where
 * the total work of the longer segments counts. Process-wide; read when a
 * stage adjoint is launched or captured into a CUDA graph. */
int cbdiso_b200_set_adjoint_segment_rows(int rows);
int cbdiso_b200_adjoint_chain_finish(const double *chain_acc, int num_blocks, double *out4, void *stream);

/* The epilogue quantities alone, on a given state (guards not needed). */
int cbdiso_b200_reduce(
    const cbd_grid_t *grid, const cbd_epilogue_t *epilogue, const double *primitive,
    double *scratch, double *result, void *stream);

/* Test hook (no counterpart in the reference): evaluates the correctly
 * rounded arithmetic the EXACT stencil is built from, on device arrays of n
 * elements: out[4i] = a/b, out[4i+1] = a^-1.5, out[4i+2] = a^4,
 * out[4i+3] = PLM slope of (a, b, a + b) with theta 1.5. */
int cbdiso_b200_eval_primitives(long n, const double *a, const double *b, double *out, void *stream);

/* ------------------------------------------------------------------------
 * 3. the gamma-law sibling, cbdgam_2d (sailfish/solvers/cbdgam_2d.c)
 *
 * Arrays: C-contiguous (ni + 4, nj + 4, 4) float64, fields (Sigma, vx, vy,
 * pressure) or (Sigma, Sigma vx, Sigma vy, energy). Arithmetic is the
 * reference's, operation for operation and without FMA contraction; results
 * differ from a CPU build only where CUDA's pow / exp round differently.
 * ---------------------------------------------------------------------- */

/* Drop-in kernels: the reference's symbol names and positional arguments,
 * DEVICE pointers, the library's current stream, an int status. */

/* replaces cbdgam_2d_advance_rk, sailfish/solvers/cbdgam_2d.c:439-683
 * (writes the interior of primitive_wr; theta from cbdgam_b200_set_plm_theta) */
int cbdgam_2d_advance_rk(int ni, int nj, double patch_xl, double patch_xr, double patch_yl, double patch_yr,
                         double *conserved_rk, double *primitive_rd, double *primitive_wr, double gamma_law_index,
                         double buffer_surface_density, double buffer_surface_pressure, double buffer_central_mass,
                         double buffer_driving_rate, double buffer_outer_radius, double buffer_onset_width,
                         int buffer_is_enabled, double x1, double y1, double vx1, double vy1, double mass1,
                         double softening_length1, double sink_rate1, double sink_radius1, int sink_model1, double x2,
                         double y2, double vx2, double vy2, double mass2, double softening_length2,
                         double sink_rate2, double sink_radius2, int sink_model2, double alpha, double a, double dt,
                         double velocity_ceiling, double cooling_coefficient, double mach_ceiling,
                         double density_floor, double pressure_floor, int constant_softening);

/* replaces cbdgam_2d_wavespeed, sailfish/solvers/cbdgam_2d.c:685-708 */
int cbdgam_2d_wavespeed(int ni, int nj, double *primitive, double *wavespeed, double gamma_law_index);

/* replaces cbdgam_2d_primitive_to_conserved, sailfish/solvers/cbdgam_2d.c:710-729 */
int cbdgam_2d_primitive_to_conserved(int ni, int nj, double *primitive, double *conserved, double gamma_law_index);

/* replaces cbdgam_2d_point_mass_source_term, sailfish/solvers/cbdgam_2d.c:731-784 */
int cbdgam_2d_point_mass_source_term(int ni, int nj, double patch_xl, double patch_xr, double patch_yl,
                                     double patch_yr, double x1, double y1, double vx1, double vy1, double mass1,
                                     double softening_length1, double sink_rate1, double sink_radius1,
                                     int sink_model1, double x2, double y2, double vx2, double vy2, double mass2,
                                     double softening_length2, double sink_rate2, double sink_radius2,
                                     int sink_model2, int which_mass, double *primitive, double *cons_rate,
                                     int constant_softening, double gamma_law_index);

/* PLM theta of the gamma-law drop-in kernels, in [1, 2]; default 1.5 as in
 * sailfish/solvers/cbdgam_2d.c:15. Process-wide. */
int cbdgam_b200_set_plm_theta(double theta);

/* Mesh, equation of state, physics and options of a gamma-law run
 * (cbdgam_2d.py:23-27 Options; the Physics fields it reads). */
typedef struct cbdgam_grid {
    int ni, nj;
    double xl, xr, yl, yr;  /* patch extent (vertex coordinates) */
    double plm_theta;
    double gamma_law_index;
    double alpha;
    double cooling_coefficient;
    double mach_ceiling;
    double velocity_ceiling;
    double density_floor;
    double pressure_floor;
    int constant_softening;
    int buffer_is_enabled;
    double buffer_surface_density;
    double buffer_surface_pressure;
    double buffer_driving_rate;
    double buffer_outer_radius;
    double buffer_onset_width;
} cbdgam_grid_t;

typedef struct cbdgam_stage {
    cbd_mass_t mass[2];          /* point masses at the stage's start time */
    double buffer_central_mass;  /* m1 + m2 */
    double a;                    /* RK weight of u_n */
    double dt;
} cbdgam_stage_t;

/* One RK stage of the product path (cbdgam_2d.c:439-683 with
 * cbdgam_2d.py:473-520): u_n is rebuilt in the kernel from primitive_n
 * (null when a = 0: u_n is then the state read, as in the reference's first
 * stage) and the zero-gradient guard zones of primitive_wr are written with
 * its edge zones. primitive_wr may be primitive_n (each zone reads only its
 * own u_n); it must not be primitive_rd. wavespeed_max (device, may be null):
 * the largest signal speed of the written state is max-ed into it, so the
 * caller zeroes it first; a NaN state leaves a NaN there. */
int cbdgam_b200_advance_stage(const cbdgam_grid_t *grid, const cbdgam_stage_t *stage, const double *primitive_rd,
                              const double *primitive_n, double *primitive_wr, double *wavespeed_max, void *stream);

/* cbdgam_b200_advance_stage with a face cache (no counterpart in the
 * reference, which recomputes these values in every stage,
 * cbdgam_2d.c:75-106 and :108-203). The scale heights' geometry at every face
 * and zone centre and, with constant softening, the zones' gravity factors
 * depend only on the mesh and the point masses. `role` 1 (writer; the caller
 * gives it to the stage at t0 + dt when its masses equal the end-of-step
 * masses) stores them with a key of their inputs; role 2 (reader; a step's
 * first stage) loads them after a fill pass that recomputes them when the key
 * does not match the stage's masses; role 0 neither. Bit-identical to
 * cbdgam_b200_advance_stage. `face_cache`: a caller-owned, 16-byte aligned
 * device buffer of cbdgam_b200_face_cache_bytes(grid) bytes for this grid
 * only, its first 256 bytes zeroed before the first use; calls on one cache
 * ordered on one stream. */
size_t cbdgam_b200_face_cache_bytes(const cbdgam_grid_t *grid);
int cbdgam_b200_advance_stage_cached(const cbdgam_grid_t *grid, const cbdgam_stage_t *stage,
                                     const double *primitive_rd, const double *primitive_n, double *primitive_wr,
                                     double *wavespeed_max, double *face_cache, int role, void *stream);

/* Writes the zero-gradient guard zones of a state from its edge zones
 * (cbdgam_2d.py:491-520 on one patch). */
int cbdgam_b200_fill_guards(const cbdgam_grid_t *grid, double *primitive, void *stream);

/* The CFL wavespeed maximum and up to 4 diagnostic sums (cbdgam_2d.py:
 * 341-447: mdot, torque, sigma_m1, eccentricity_vector, with radial cuts) on
 * a state, with point masses `masses[2]`. mdot and torque take the
 * accretion rates when the diagnostic's accretion flag is set, else the
 * gravity rates (the gravity flag must then be set). result[0] = max
 * wavespeed, result[1 + 2k], result[2 + 2k] = real and imaginary part of
 * sum_cells f_k (not multiplied by dx dy); the summation order is fixed.
 * scratch: cbdgam_b200_scratch_bytes(grid) bytes of device memory. */
size_t cbdgam_b200_scratch_bytes(const cbdgam_grid_t *grid);
int cbdgam_b200_reduce(const cbdgam_grid_t *grid, const cbd_mass_t *masses, const cbd_diag_t *diags, int num_diags,
                       const double *primitive, double *scratch, double *result, void *stream);

/* Measurement hook (no counterpart in the reference): the FP64 issue-rate
 * probe behind the stencil kernels' FP64 roofline. `blocks` CTAs of 256
 * threads each run eight independent FMA chains of `iterations` steps;
 * cbdiso_b200_fp64_probe_fmas gives the thread-FMA count of one launch, to be
 * divided by its device time. `out` (device, `blocks` doubles) is written
 * only to keep the chains live. */
int cbdiso_b200_fp64_probe(long iterations, int blocks, double *out, void *stream);
long cbdiso_b200_fp64_probe_fmas(long iterations, int blocks);

/* Host function (no device work): the gamma-law circumbinary disk's initial
 * primitives (sailfish/setups/circumbinary_disk.py:95-110) at n points, with
 * the C library's sqrt / pow / exp in the setup's operation order, which is
 * what Python's float arithmetic computes; primitive holds 4 n doubles. */
void cbdgam_b200_disk_primitive(long n, const double *x, const double *y, double softening_length,
                                double initial_sigma, double initial_pressure, double *primitive);

/* sizeof of cbdgam_grid_t and cbdgam_stage_t, for bindings to check. */
void cbdgam_b200_abi_sizes(size_t out[2]);

/* Test hook (no counterpart in the reference): the correctly rounded powers
 * the gamma-law kernels use, on device arrays of n elements: out[8i + 0..6]
 * = x^3, x^-2, x^-3, x^4, x^-1.5, (1 + x)^RN(-1/3), exp(-x); out[8i + 7] = 0. */
int cbdgam_b200_eval_powers(long n, const double *x, double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CBDISO_B200_H */
