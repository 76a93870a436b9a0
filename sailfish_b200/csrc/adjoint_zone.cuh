// Generic per-zone pieces of the stage (templated on double / Dual) and the
// hand-written vector-Jacobian products of the adjoint. Included only by
// adjoint.cu, which is built with -fmad=false.
#pragma once

#include "adjoint.cuh"

namespace cbd {

// Sink term of one mass (cbdiso_2d.c:118-174) as a function of the zone's
// sigma and velocity, the mass's position and velocity and the sink rate;
// used by the tangent and, direction by direction, by the adjoint.
template <class T>
__device__ __forceinline__ void sink_generic(const MassDev &b, const T &xp, const T &yp, const T &vxp,
                                             const T &vyp, const T &rate, double x, double y, double dt,
                                             const T &sigma, const T &vx, const T &vy, T *du)
{
    if (val(rate) == 0.0 || b.sink_model < 1 || b.sink_model > 3)
        return;
    const T dx = x - xp, dy = y - yp;
    const T r2 = dx * dx + dy * dy;
    if (!(val(r2) < b.sink_hi2))
        return;
    const T dr = g_sqrt(r2);
    if (!(val(dr) < b.sink_r4))
        return;
    const T s = rate * g_exp(-g_pow4(g_div(dr, T{} * 0.0 + b.sink_radius)));
    T mdot = T{} * 0.0;
    if (val(s) > 0.0)
        mdot = -s * sigma;
    else if (val(s) < 0.0)
        mdot = -s;
    if (val(mdot) == 0.0)
        return;
    if (b.sink_model == 1) {
        du[0] = du[0] + dt * mdot;
        du[1] = du[1] + dt * mdot * vx;
        du[2] = du[2] + dt * mdot * vy;
    } else if (b.sink_model == 2) {
        const T d = dr + 1e-12;
        const T ex = g_div(dx, d), ey = g_div(dy, d);
        const T dvr = (vx - vxp) * ex + (vy - vyp) * ey;
        du[0] = du[0] + dt * mdot;
        du[1] = du[1] + dt * mdot * (dvr * ex + vxp);
        du[2] = du[2] + dt * mdot * (dvr * ey + vyp);
    } else {
        du[0] = du[0] + dt * mdot;
    }
}

template <class T>
__device__ __forceinline__ void mass_source_generic(const MassT<T> &m, double x, double y, double dt, const T *p,
                                                    T *du)
{
    if (val(m.mass) != 0.0) {
        const T dx = x - m.x, dy = y - m.y;
        const T fnum = p[0] * m.mass * g_pow15(dx * dx + dy * dy + m.base->soft2);
        du[1] = du[1] + (-fnum * dx) * dt;
        du[2] = du[2] + (-fnum * dy) * dt;
    }
    sink_generic(*m.base, m.x, m.y, m.vx, m.vy, m.sink_rate, x, y, dt, p[0], p[1], p[2], du);
}

template <class T>
__device__ __forceinline__ void buffer_generic(const Consts &k, const StageDev &st, double x, double y, double dt,
                                               const T *u, T *du)
{
    if (!k.buffer_on)
        return;
    const double r2 = x * x + y * y;
    if (!(r2 > k.buf_lo2))
        return;
    const double rc = sqrt(r2);
    if (!(rc > k.buf_onset))
        return;
    const double vk = sqrt(div_rn<false>(st.buffer_mass, rc));
    const double t[3] = {k.buf_sigma, k.buf_sigma * div_rn<false>(-y, rc) * vk,
                         k.buf_sigma * div_rn<false>(+x, rc) * vk};
    const double rate = div_by<false>(st.buffer_k * (rc - k.buf_onset), k.buf_span, k.inv_buf_span);
    for (int q = 0; q < 3; ++q)
        du[q] = du[q] - (u[q] - t[q]) * rate * dt;
}

// buffer rate at a zone (0 outside the buffer), for the adjoint
__device__ __forceinline__ double buffer_rate(const Consts &k, const StageDev &st, double x, double y)
{
    if (!k.buffer_on)
        return 0.0;
    const double r2 = x * x + y * y;
    if (!(r2 > k.buf_lo2))
        return 0.0;
    const double rc = sqrt(r2);
    if (!(rc > k.buf_onset))
        return 0.0;
    return div_by<false>(st.buffer_k * (rc - k.buf_onset), k.buf_span, k.inv_buf_span);
}

template <class T>
__device__ __forceinline__ unsigned c2p_generic(const T *u, T *p, const Consts &k)
{
    unsigned flags = 0;
    T rho;
    if (val(u[0]) > k.rho_min) {
        rho = u[0];
    } else {
        rho = T{} * 0.0 + k.rho_min;
        flags |= BW_FLOOR;
    }
    p[0] = rho;
    for (int q = 1; q < 3; ++q) {
        const T v = g_div(u[q], rho);
        T a = g_abs(v);
        if (!(val(a) < k.vmax)) {
            a = T{} * 0.0 + k.vmax;
            flags |= q == 1 ? BW_CEIL_X : BW_CEIL_Y;
        }
        p[q] = signbit(val(u[q])) ? -a : a;
    }
    return flags;
}

// strain times density (sxx, sxy, syy) from the zone's slopes
template <class T>
__device__ __forceinline__ void rho_strain_generic(const T &rho, const T *gx, const T *gy, const Consts &k, T *rs)
{
    const T sxx = g_div(4.0 / 3.0 * gx[1], T{} * 0.0 + k.dx) - g_div(2.0 / 3.0 * gy[2], T{} * 0.0 + k.dy);
    const T syy = g_div(-2.0 / 3.0 * gx[1], T{} * 0.0 + k.dx) + g_div(4.0 / 3.0 * gy[2], T{} * 0.0 + k.dy);
    const T sxy = g_div(gx[2], T{} * 0.0 + k.dx) + g_div(gy[1], T{} * 0.0 + k.dy);
    rs[0] = rho * sxx;
    rs[1] = rho * sxy;
    rs[2] = rho * syy;
}

// One zone's stage update in the reference's structure (cbdiso_2d.c:447-603).
// P(di, dj, q) returns the input primitive at offset (di, dj) from the zone.
template <class T, class Load>
__device__ void zone_update_generic(const Consts &k, const StageDev &st, const MassT<T> *m, const T &nu, int i,
                                    int j, const Load &P, const T *un, T *out)
{
    const double dx = k.dx, dy = k.dy;
    const double xl = k.xl + (i + 0.0) * dx, xc = k.xl + (i + 0.5) * dx, xr = k.xl + (i + 1.0) * dx;
    const double yl = k.yl + (j + 0.0) * dy, yc = k.yl + (j + 0.5) * dy, yr = k.yl + (j + 1.0) * dy;
    T c[3], w1[3], e1[3], s1[3], n1[3], w2[3], e2[3], s2[3], n2[3], sw[3], nw[3], se[3], ne[3];
    for (int q = 0; q < 3; ++q) {
        c[q] = P(0, 0, q);
        w1[q] = P(-1, 0, q);
        e1[q] = P(1, 0, q);
        s1[q] = P(0, -1, q);
        n1[q] = P(0, 1, q);
        w2[q] = P(-2, 0, q);
        e2[q] = P(2, 0, q);
        s2[q] = P(0, -2, q);
        n2[q] = P(0, 2, q);
        sw[q] = P(-1, -1, q);
        nw[q] = P(-1, 1, q);
        se[q] = P(1, -1, q);
        ne[q] = P(1, 1, q);
    }
    const double th = k.theta;
    T gxw[3], gxc[3], gxe[3], gys[3], gyc[3], gyn[3], gyw[3], gye[3], gxs[3], gxn[3];
    for (int q = 0; q < 3; ++q) {
        gxw[q] = slope_generic(w2[q], w1[q], c[q], th);
        gxc[q] = slope_generic(w1[q], c[q], e1[q], th);
        gxe[q] = slope_generic(c[q], e1[q], e2[q], th);
        gys[q] = slope_generic(s2[q], s1[q], c[q], th);
        gyc[q] = slope_generic(s1[q], c[q], n1[q], th);
        gyn[q] = slope_generic(c[q], n1[q], n2[q], th);
        gyw[q] = slope_generic(sw[q], w1[q], nw[q], th);
        gye[q] = slope_generic(se[q], e1[q], ne[q], th);
        gxs[q] = slope_generic(sw[q], s1[q], se[q], th);
        gxn[q] = slope_generic(nw[q], n1[q], ne[q], th);
    }
    T wm[3], wp[3], em[3], ep[3], sm[3], sp[3], nm[3], np_[3];
    for (int q = 0; q < 3; ++q) {
        wm[q] = w1[q] + 0.5 * gxw[q];
        wp[q] = c[q] - 0.5 * gxc[q];
        em[q] = c[q] + 0.5 * gxc[q];
        ep[q] = e1[q] - 0.5 * gxe[q];
        sm[q] = s1[q] + 0.5 * gys[q];
        sp[q] = c[q] - 0.5 * gyc[q];
        nm[q] = c[q] + 0.5 * gyc[q];
        np_[q] = n1[q] - 0.5 * gyn[q];
    }
    const T zero = T{} * 0.0;
    T fw[3], fe[3], fs[3], fn[3];
    hlle_generic<T, 0>(wm, wp, cs2_generic(k, m, zero + xl, zero + yc), fw, nullptr);
    hlle_generic<T, 0>(em, ep, cs2_generic(k, m, zero + xr, zero + yc), fe, nullptr);
    hlle_generic<T, 1>(sm, sp, cs2_generic(k, m, zero + xc, zero + yl), fs, nullptr);
    hlle_generic<T, 1>(nm, np_, cs2_generic(k, m, zero + xc, zero + yr), fn, nullptr);
    if (val(nu) > 0.0) {
        T rsw[3], rse[3], rss[3], rsn[3], rsc[3];
        rho_strain_generic(w1[0], gxw, gyw, k, rsw);
        rho_strain_generic(e1[0], gxe, gye, k, rse);
        rho_strain_generic(s1[0], gxs, gys, k, rss);
        rho_strain_generic(n1[0], gxn, gyn, k, rsn);
        rho_strain_generic(c[0], gxc, gyc, k, rsc);
        const T hn = 0.5 * nu;
        fw[1] = fw[1] - hn * (rsw[0] + rsc[0]);
        fw[2] = fw[2] - hn * (rsw[1] + rsc[1]);
        fe[1] = fe[1] - hn * (rsc[0] + rse[0]);
        fe[2] = fe[2] - hn * (rsc[1] + rse[1]);
        fs[1] = fs[1] - hn * (rss[1] + rsc[1]);
        fs[2] = fs[2] - hn * (rss[2] + rsc[2]);
        fn[1] = fn[1] - hn * (rsc[1] + rsn[1]);
        fn[2] = fn[2] - hn * (rsc[2] + rsn[2]);
    }
    T u[3] = {c[0], c[1] * c[0], c[2] * c[0]};
    T du[3] = {zero, zero, zero};
    const double dt = st.dt;
    buffer_generic(k, st, xc, yc, dt, u, du);
    mass_source_generic(m[0], xc, yc, dt, c, du);
    mass_source_generic(m[1], xc, yc, dt, c, du);
    for (int q = 0; q < 3; ++q)
        du[q] = du[q] - (g_div(fe[q] - fw[q], zero + dx) + g_div(fn[q] - fs[q], zero + dy)) * dt;
    T uu[3];
    for (int q = 0; q < 3; ++q)
        uu[q] = st.one_minus_a * (u[q] + du[q]) + st.a * un[q];
    c2p_generic(uu, out, k);
}

}  // namespace cbd
