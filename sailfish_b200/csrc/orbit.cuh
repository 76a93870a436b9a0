// The binary's Kepler orbit on the device (sailfish/physics/kepler.py:300-373,
// 414-421), in the reference's operation order, and the stage-kernel mass
// records built from it. Shared by the single-grid and batched steppers.
#pragma once

#include "cbd_stencil.cuh"

namespace cbd {

// Newton iteration of kepler.py:414-421 on E - e sin E = M: stop when
// |f| <= 1e-15, fail after more than 10 updates.
__device__ inline bool eccentric_anomaly(double mean_anomaly, double e, double *out)
{
    double k = mean_anomaly;
    int n = 0;
    double f = k - e * sin(k) - mean_anomaly;
    while (fabs(f) > 1e-15) {
        k -= f / (1.0 - e * cos(k));
        n += 1;
        if (n > 10)
            return false;
        f = k - e * sin(k) - mean_anomaly;
    }
    *out = k;
    return true;
}

__device__ inline MassDev mass_record(double mass, double x, double y, double vx, double vy, const cbd_orbit_t &o)
{
    MassDev m;
    m.x = x;
    m.y = y;
    m.vx = vx;
    m.vy = vy;
    m.mass = mass;
    m.soft2 = o.softening_length * o.softening_length;
    m.sink_rate = o.sink_rate;
    m.sink_radius = o.sink_radius;
    m.inv_sink_radius = 1.0 / o.sink_radius;
    m.sink_r4 = 4.0 * o.sink_radius;
    m.sink_hi2 = m.sink_r4 * m.sink_r4 * (1.0 + 1e-10);
    m.sink_model = o.sink_model;
    m._pad = 0;
    return m;
}

// Positions and velocities of the two components at time t
// (kepler.py:300-373), in the reference's operation order.
__device__ inline bool orbit_masses(const cbd_orbit_t &o, double t, MassDev *out)
{
    const double a = o.semimajor_axis, m = o.total_mass, q = o.mass_ratio, e = o.eccentricity;
    const double w = sqrt(1.0 * m / a / a / a);
    const double period = 2.0 * 3.141592653589793 / w;
    const double tt = t - period * floor(t / period);
    double E;
    if (!eccentric_anomaly(w * tt, e, &E))
        return false;
    const double m1 = m / (1.0 + q);
    const double m2 = m - m1;
    const double ck = cos(E);
    const double sk = sin(E);
    const double x1 = -a * q / (1.0 + q) * (e - ck);
    const double y1 = +a * q / (1.0 + q) * (sk) * sqrt(1.0 - e * e);
    const double x2 = -x1 / q;
    const double y2 = -y1 / q;
    const double vx1 = -a * q / (1.0 + q) * w / (1.0 - e * ck) * sk;
    const double vy1 = +a * q / (1.0 + q) * w / (1.0 - e * ck) * ck * sqrt(1.0 - e * e);
    const double vx2 = -vx1 / q;
    const double vy2 = -vy1 / q;
    const double dx = o.has_x_offset ? o.x_offset : 0.0;
    out[0] = mass_record(m1, o.has_x_offset ? x1 + dx : x1, y1, vx1, vy1, o);
    out[1] = mass_record(m2, o.has_x_offset ? x2 + dx : x2, y2, vx2, vy2, o);
    return true;
}

}  // namespace cbd
