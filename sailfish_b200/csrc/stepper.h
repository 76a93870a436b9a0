// Device-side state of the device-resident time stepper (stepper.cu).
#pragma once

#include "cbd_stencil.cuh"

namespace cbd {

struct StepperDev {
    double time;         // simulation time after the last step
    double dt;           // the last step's dt
    double min_spacing;  // min(dx, dy) of the mesh, as the driver uses it
    double cfl;
    double fixed_dt;     // > 0: use this dt every step instead of the CFL rule
    double buffer_k;     // buffer driving_rate * sqrt(M onset^-3), from the host libm
    double weights[3];   // RK weights of u_n per stage
    cbd_orbit_t orbit;
    int num_stages;
    int step;            // steps taken
    int status;          // CBD_OK; CBD_ERR_KEPLER once an orbit solve failed, CBD_ERR_NONFINITE once a
                         // step's dt was not finite and positive (then no further steps)
    int series_capacity; // rows available in the time-series buffer
    const double *dt_sequence;  // if set: dt of step n is dt_sequence[n] (n < dt_count)
    StageDev *history;          // if set: stage records of step n also go to history[n * num_stages ...]
    int dt_count;
    int history_capacity;       // steps the history holds
};

// Prologue of n grids' steps; grid d reads results + d * result_stride and
// writes records + d * num_stages and its series block (series_capacity rows).
cudaError_t launch_step_prologue(StepperDev *s, int n, const double *results, int result_stride,
                                 StageDev *records, double *series, int num_values, int finalize,
                                 cudaStream_t stream);

}  // namespace cbd
