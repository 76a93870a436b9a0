// Device-resident time stepping: the driver's CFL time step
// (sailfish/driver.py:508-510), the RK stage times (cbdiso_2d.py:239) and the
// binary's Kepler orbit (sailfish/physics/kepler.py:329-366, 414-421) computed
// on the device, so that a run of steps needs no host round trip and can be
// captured in a CUDA graph. One single-thread prologue kernel per step writes
// the stage records that the stage kernels read.
#include <cmath>
#include <cstring>

#include "cbd_internal.h"
#include "stepper.h"
#include "orbit.cuh"

namespace cbd {

namespace {

// One step's prologue for n independent grids (thread d: grid d). With
// `finalize`, only records the previous step's time-series row. Otherwise:
// record the previous row (if any), choose dt, write the stage records of
// this step, advance the clock.
__global__ void step_prologue_kernel(StepperDev *steppers, int n, const double *results, int result_stride,
                                     StageDev *records, double *series, int num_values, int finalize)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n)
        return;
    StepperDev *s = steppers + d;
    const double *result = results + (size_t)d * result_stride;
    if (s->status != CBD_OK)
        return;
    if (s->step > 0 && series && s->step - 1 < s->series_capacity) {
        double *row = series + ((size_t)d * s->series_capacity + (s->step - 1)) * (3 + num_values);
        row[0] = s->time;
        row[1] = s->dt;
        row[2] = result[0];
        for (int v = 0; v < num_values; ++v)
            row[3 + v] = result[1 + v];
    }
    if (finalize)
        return;
    if (s->dt_sequence && s->step >= s->dt_count) {
        s->status = CBD_ERR_ARGUMENT;
        return;
    }
    const double dt = s->dt_sequence ? s->dt_sequence[s->step]
                                     : (s->fixed_dt > 0.0 ? s->fixed_dt : s->min_spacing / result[0] * s->cfl);
    StageDev *rec = records + (size_t)d * s->num_stages;
    if (!(isfinite(dt) && dt > 0.0)) {
        // a NaN, infinite or zero wavespeed (or a bad dt sequence entry):
        // stop here, and make the stages of this and every later step of a
        // captured sequence leave the state as it is
        s->status = CBD_ERR_NONFINITE;
        for (int k = 0; k < s->num_stages; ++k)
            rec[k].halt = 1;
        return;
    }
    const double time0 = s->time;
    double t = time0;
    double times[3];
    for (int k = 0; k < s->num_stages; ++k) {
        times[k] = t;
        t = time0 * s->weights[k] + (t + dt) * (1.0 - s->weights[k]);
    }
    MassDev end[2];
    if (!orbit_masses(s->orbit, t, end)) {
        s->status = CBD_ERR_KEPLER;
        return;
    }
    for (int k = 0; k < s->num_stages; ++k) {
        StageDev &r = rec[k];
        if (!orbit_masses(s->orbit, times[k], r.m)) {
            s->status = CBD_ERR_KEPLER;
            return;
        }
        r.e[0] = end[0];
        r.e[1] = end[1];
        r.a = s->weights[k];
        r.one_minus_a = 1.0 - s->weights[k];
        r.dt = dt;
        r.buffer_mass = r.m[0].mass + r.m[1].mass;
        r.buffer_k = s->buffer_k;
        r.halt = 0;
        if (s->history && s->step < s->history_capacity)
            s->history[(size_t)s->step * s->num_stages + k] = r;
    }
    s->dt = dt;
    s->time = t;
    s->step += 1;
}

}  // namespace

cudaError_t launch_step_prologue(StepperDev *s, int n, const double *results, int result_stride,
                                 StageDev *records, double *series, int num_values, int finalize,
                                 cudaStream_t stream)
{
    step_prologue_kernel<<<(n + 63) / 64, 64, 0, stream>>>(s, n, results, result_stride, records, series,
                                                           num_values, finalize);
    return cudaGetLastError();
}

}  // namespace cbd

using namespace cbd;

extern "C" {

size_t cbdiso_b200_stepper_bytes(void) { return sizeof(StepperDev); }

int cbdiso_b200_stepper_init(const cbd_grid_t *grid, const cbd_orbit_t *orbit, int rk_order, double time,
                             double cfl, double min_spacing, double fixed_dt, int series_capacity, void *stepper)
{
    if (!grid || !orbit || !stepper || rk_order < 1 || rk_order > 3 || !(cfl > 0.0) || !(min_spacing > 0.0) ||
        series_capacity < 0)
        return CBD_ERR_ARGUMENT;
    if (!(orbit->semimajor_axis > 0.0) || !(orbit->total_mass > 0.0) || !(orbit->mass_ratio > 0.0) ||
        !(orbit->eccentricity >= 0.0 && orbit->eccentricity < 1.0))
        return CBD_ERR_ARGUMENT;
    StepperDev s;
    std::memset(&s, 0, sizeof(s));
    s.time = time;
    s.cfl = cfl;
    s.fixed_dt = fixed_dt;
    s.min_spacing = min_spacing;
    static const double w1[] = {0.0}, w2[] = {0.0, 0.5}, w3[] = {0.0, 0.75, 1.0 / 3.0};
    const double *w = rk_order == 1 ? w1 : (rk_order == 2 ? w2 : w3);
    s.num_stages = rk_order;
    for (int k = 0; k < rk_order; ++k)
        s.weights[k] = w[k];
    s.orbit = *orbit;
    const double m1 = orbit->total_mass / (1.0 + orbit->mass_ratio);
    const double central = m1 + (orbit->total_mass - m1);
    const double onset = grid->buffer_outer_radius - grid->buffer_onset_width;
    s.buffer_k = grid->buffer_is_enabled
                     ? grid->buffer_driving_rate * std::sqrt(central * std::pow(onset, -3.0))
                     : 0.0;
    s.series_capacity = series_capacity;
    s.status = CBD_OK;
    std::memcpy(stepper, &s, sizeof(s));
    return CBD_OK;
}

int cbdiso_b200_stepper_attach(void *stepper, const double *dt_sequence, int dt_count, void *history,
                               int history_capacity)
{
    if (!stepper || dt_count < 0 || history_capacity < 0 || (dt_sequence && dt_count == 0))
        return CBD_ERR_ARGUMENT;
    StepperDev s;
    std::memcpy(&s, stepper, sizeof(s));
    s.dt_sequence = dt_sequence;
    s.dt_count = dt_count;
    s.history = static_cast<StageDev *>(history);
    s.history_capacity = history ? history_capacity : 0;
    std::memcpy(stepper, &s, sizeof(s));
    return CBD_OK;
}

int cbdiso_b200_step_prologue(void *stepper_dev, const double *result, void *records_dev, double *series,
                              int num_values, int finalize, void *stream)
{
    if (!stepper_dev || !result || !records_dev || num_values < 0 || num_values > 2 * CBD_MAX_DIAG)
        return CBD_ERR_ARGUMENT;
    return launch_step_prologue(static_cast<StepperDev *>(stepper_dev), 1, result, 0,
                                static_cast<StageDev *>(records_dev), series, num_values, finalize,
                                static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? CBD_OK
               : CBD_ERR_CUDA;
}

}  // extern "C"
