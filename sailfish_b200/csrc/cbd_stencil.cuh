// Fused RK-stage stencil of the isothermal circumbinary-disk solver for sm_100a.
//
// Design (one kernel per RK stage):
//  * A CTA owns a strip of BJ columns (j, the contiguous axis) and marches down
//    a segment of rows (i) with one barrier per row. Each iteration stages one
//    new row of primitives in a five-row shared-memory ring with coalesced
//    loads, so every zone is read from HBM once per stage (plus a two-row and
//    two-column halo per CTA).
//  * Every quantity that the reference recomputes per zone (cbdiso_2d.c:447-603)
//    is computed once and shared: each PLM slope, each x- and y-face HLLE flux
//    with its viscous term, each zone's rho * strain. The shared values are
//    bit-identical to the per-zone values of the reference, because the same
//    operations run on the same operands.
//  * Boundary conditions are fused: the writer of an edge zone also writes its
//    zero-gradient guard zones, so the next stage reads valid guards.
//  * The final stage can fold in the next step's CFL wavespeed and up to
//    CBD_MAX_FUSED diagnostic sums, reduced deterministically (fixed-order warp
//    and block trees, then a last-CTA pass over per-CTA partials).
//
// PREC selects the arithmetic (CBD_PRECISION_*). EXACT and FMA run identical
// source (the EXACT translation unit is compiled with -fmad=false) and return
// the reference's values: every divide, square root and power is correctly
// rounded, as in the reference's CPU build, but computed cheaply --
//   * a / b as a Markstein-corrected product with y = RN(1/b), hoisted to the
//     host when b is a constant (dx, dy, mach^2, ...);
//   * (r^2 + s^2)^-1.5 and q^4 in double-double arithmetic, rounded once;
//   * sqrt only where a threshold test on the squared radius is undecided.
// Only the sign of an exact zero may differ from the reference, which no
// nonzero value depends on. FAST replaces these by uncorrected reciprocal
// multiplies and rsqrt, staying within about an ulp per operation.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/cbdiso_b200.h"
#include "cr_math.cuh"

namespace cbd {

constexpr int NG = 2;   // guard zones per side
constexpr int NQ = 3;   // fields
constexpr int MAX_FUSED = 4;
constexpr int PARTIAL_STRIDE = 1 + 2 * MAX_FUSED;  // doubles per CTA partial

// ---------------------------------------------------------------------------
// constants and per-stage parameters as the kernels see them
// ---------------------------------------------------------------------------

struct Consts {
    int ni, nj;
    int rows_per_cta;
    int un_kind;        // 0: u_n = cons(centre of primitive_rd); 1: from primitive_n; 2: from a conserved array
    int write_guards;
    int eos;
    int buffer_on;
    int want_ws;
    int num_diag;       // diagnostics fused into this launch (<= MAX_FUSED)
    int spacing_pow2;   // dx and dy are powers of two: inv_dx, inv_dy are exact
    double xl, yl, dx, dy, inv_dx, inv_dy;
    double theta;
    double cs2, mach2, inv_mach2, neg_inv_mach2;
    double nu, half_nu;
    double vmax, rho_min;
    double buf_sigma, buf_onset, buf_lo2, buf_span, inv_buf_span;
    int need_rates;     // epilogue: bit p gravity rates of mass p, bit 2 + p accretion rates
    int rates_only;     // epilogue: every diagnostic is a source rate of the masses, without a radial cut
    cbd_diag_t diag[CBD_MAX_DIAG];
};

struct MassDev {
    double x, y, vx, vy;
    double mass;
    double soft2;            // softening_length^2
    double sink_rate;
    double sink_radius;
    double inv_sink_radius;  // RN(1 / sink_radius)
    double sink_r4;          // 4 * sink_radius
    double sink_hi2;         // (4 sink_radius)^2 (1 + 1e-10): beyond it a zone is outside the sink
    int sink_model;
    int _pad;
};

struct StageDev {
    MassDev m[2];       // masses at the stage time
    MassDev e[2];       // masses at the end-of-step time (epilogue)
    double a, one_minus_a, dt;
    double buffer_mass, buffer_k;  // central mass, driving_rate * omega_outer
    int halt;           // set by a device stepper that stopped: the stage leaves every array untouched
    int _pad;
};

// ---------------------------------------------------------------------------
// scalar helpers with the reference's semantics (cbdiso_2d.c:16-21)
// ---------------------------------------------------------------------------

__device__ __forceinline__ double lesser(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double greater(double a, double b) { return a > b ? a : b; }
// the maximum of the wavespeed reductions: keeps a NaN operand, as numpy's
// max over the reference's wavespeed array does (cbdiso_2d.py:174)
__device__ __forceinline__ double max_nan(double a, double b) { return (a > b || a != a) ? a : b; }

// a / b rounded to nearest, given y = RN(1/b): the remainder a - q b of
// q = RN(a y) is exact under FMA, and one correction q + (a - q b) y rounds
// to RN(a / b) for operands in the normal range (Markstein's theorem).
template <bool FAST>
__device__ __forceinline__ double div_by(double a, double b, double y)
{
    const double q = a * y;
    if (FAST)
        return q;
    return fma(fma(-q, b, a), y, q);
}

template <bool FAST>
__device__ __forceinline__ double div_rn(double a, double b)
{
    return div_by<FAST>(a, b, __drcp_rn(b));
}

// correctly rounded powers (cr_math.cuh)
using crm::pow4_rn;
using crm::pow_m15_rn;

// s^-1.5 for the gravity term
template <bool FAST>
__device__ __forceinline__ double inv_pow15(double s2)
{
    if (FAST) {
        const double rs = rsqrt(s2);
        return rs * rs * rs;
    }
    return (s2 > 0.0 && s2 < 1e300) ? pow_m15_rn(s2) : pow(s2, -1.5);
}

// Generalised minmod, cbdiso_2d.c:23-29. Returns exactly the value of
// 0.25 |sgn a + sgn b| (sgn a + sgn c) min(|a|, |b|, |c|), signed zeros
// included, with the sign logic done on integer sign bits.
__device__ __forceinline__ double limited_slope(double yl, double y0, double yr, double theta)
{
    double a = (y0 - yl) * theta;
    double b = (yr - yl) * 0.5;
    double c = (yr - y0) * theta;
    double m = lesser(fabs(a), lesser(fabs(b), fabs(c)));
    unsigned sa = (unsigned)__double2hiint(a) >> 31;
    unsigned sb = (unsigned)__double2hiint(b) >> 31;
    unsigned sc = (unsigned)__double2hiint(c) >> 31;
    if ((sa == sb) & (sa == sc))
        return sa ? -m : m;
    return (sa & sc & (sa ^ sb)) ? -0.0 : 0.0;
}

// softened potential of the masses with positive mass, cbdiso_2d.c:70-95
template <bool FAST>
__device__ __forceinline__ double potential(const MassDev *m, double x, double y)
{
    // both terms evaluated unconditionally (two independent chains), the
    // massless ones then left out
    double term[2];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        double dx = x - m[p].x;
        double dy = y - m[p].y;
        double r2 = dx * dx + dy * dy;
        double s2 = r2 + m[p].soft2;
        term[p] = FAST ? m[p].mass * rsqrt(s2) : div_rn<false>(m[p].mass, sqrt(s2));
    }
    double phi = 0.0;
#pragma unroll
    for (int p = 0; p < 2; ++p)
        phi = m[p].mass > 0.0 ? phi - term[p] : phi;
    return phi;
}

// cbdiso_2d.c:194-211
template <bool FAST>
__device__ __forceinline__ double sound_speed2(const Consts &k, const MassDev *m, double x, double y)
{
    if (k.eos == 1)
        return k.cs2;
    if (k.eos == 2)
        return FAST ? potential<FAST>(m, x, y) * k.neg_inv_mach2
                    : div_by<false>(-potential<FAST>(m, x, y), k.mach2, k.inv_mach2);
    return 1.0;
}

// HLLE flux across a face with normal DIR (0: x, 1: y), cbdiso_2d.c:352-380
// cs = sqrt(cs2): computed here, or with CS_GIVEN taken from the caller (a
// face-cache value); the caller receives it either way.
template <bool FAST, int DIR, bool CS_GIVEN = false>
__device__ __forceinline__ void hlle(const double *pl, const double *pr, double cs2, double &cs, double *f)
{
    const double ul0 = pl[0], ul1 = pl[1] * pl[0], ul2 = pl[2] * pl[0];
    const double ur0 = pr[0], ur1 = pr[1] * pr[0], ur2 = pr[2] * pr[0];
    const double vl = DIR == 0 ? pl[1] : pl[2];
    const double vr = DIR == 0 ? pr[1] : pr[2];
    const double gl = pl[0] * cs2;
    const double gr = pr[0] * cs2;
    // the pressure enters only the normal-momentum flux (adding the
    // reference's `pressure * 0` to the other components changes no value)
    const double fl0 = vl * ul0, fr0 = vr * ur0;
    const double fl1 = DIR == 0 ? vl * ul1 + gl : vl * ul1;
    const double fl2 = DIR == 1 ? vl * ul2 + gl : vl * ul2;
    const double fr1 = DIR == 0 ? vr * ur1 + gr : vr * ur1;
    const double fr2 = DIR == 1 ? vr * ur2 + gr : vr * ur2;
    if (!CS_GIVEN)
        cs = sqrt(cs2);
    const double am = lesser(0.0, lesser(vl - cs, vr - cs));
    const double ap = greater(0.0, greater(vl + cs, vr + cs));
    const double den = ap - am;
    const double y = FAST ? 1.0 / den : __drcp_rn(den);
    if (FAST) {
        const double apam = ap * am;
        f[0] = (fl0 * ap - fr0 * am - (ul0 - ur0) * apam) * y;
        f[1] = (fl1 * ap - fr1 * am - (ul1 - ur1) * apam) * y;
        f[2] = (fl2 * ap - fr2 * am - (ul2 - ur2) * apam) * y;
    } else {
        f[0] = div_by<false>(fl0 * ap - fr0 * am - (ul0 - ur0) * ap * am, den, y);
        f[1] = div_by<false>(fl1 * ap - fr1 * am - (ul1 - ur1) * ap * am, den, y);
        f[2] = div_by<false>(fl2 * ap - fr2 * am - (ul2 - ur2) * ap * am, den, y);
    }
}

// rho times the trace-free strain (sxx, sxy, syy), cbdiso_2d.c:248-263; the
// viscous face terms of cbdiso_2d.c:579-586 combine two of these.
template <bool FAST, bool P2 = false>
__device__ __forceinline__ void rho_strain(double rho, const double *gx, const double *gy, const Consts &k,
                                           double *rs)
{
    double sxx, syy, sxy;
    if (FAST) {
        const double ax = gx[1] * k.inv_dx, by = gy[2] * k.inv_dy;
        sxx = (4.0 / 3.0) * ax - (2.0 / 3.0) * by;
        syy = (4.0 / 3.0) * by - (2.0 / 3.0) * ax;
        sxy = gx[2] * k.inv_dx + gy[1] * k.inv_dy;
    } else {
        // 4.0 / 3.0 * gx[1] / dx - 2.0 / 3.0 * gy[2] / dy, and so on, with
        // each quotient correctly rounded from the hoisted 1 / dx, 1 / dy
        // (with P2 these are exact powers of two and the product alone is
        // the correctly rounded quotient)
        const double ix = k.inv_dx, iy = k.inv_dy;
        sxx = div_by<P2>(4.0 / 3.0 * gx[1], k.dx, ix) - div_by<P2>(2.0 / 3.0 * gy[2], k.dy, iy);
        syy = div_by<P2>(-2.0 / 3.0 * gx[1], k.dx, ix) + div_by<P2>(4.0 / 3.0 * gy[2], k.dy, iy);
        sxy = div_by<P2>(gx[2], k.dx, ix) + div_by<P2>(gy[1], k.dy, iy);
    }
    rs[0] = rho * sxx;
    rs[1] = rho * sxy;
    rs[2] = rho * syy;
}

template <bool FAST>
__device__ __forceinline__ double fourth_power(double q)
{
    if (FAST) {
        const double h = q * q;
        return h * h;
    }
    return pow4_rn(q);
}

// Gravity and sink terms of one mass, added into du (cbdiso_2d.c:97-175).
// Terms that are exactly zero (no mass, or a zone outside 4 sink radii) are
// skipped: adding them changes no value. The gravity factor
// (r^2 + s^2)^-1.5 is taken from *g_in when given (a face-cache value), and
// stored to *g_out when given. GRAV and SINK select the two parts (both
// for the stage; the diagnostics take one at a time, as the reference's
// switches do, cbdiso_2d.py:105-137).
template <bool FAST, bool GRAV = true, bool SINK = true>
__device__ __forceinline__ void mass_source(const MassDev &m, double x, double y, double dt, const double *p,
                                            double *du, const double *g_in = nullptr, double *g_out = nullptr)
{
    const double sigma = p[0];
    const double dx = x - m.x;
    const double dy = y - m.y;
    const double r2 = dx * dx + dy * dy;
    if (GRAV && m.mass != 0.0) {
        const double g = g_in ? *g_in : inv_pow15<FAST>(r2 + m.soft2);
        if (g_out)
            *g_out = g;
        const double fnum = sigma * m.mass * g;
        const double fx = -fnum * dx;
        const double fy = -fnum * dy;
        du[1] += fx * dt;
        du[2] += fy * dt;
    }
    if (!SINK || m.sink_rate == 0.0 || m.sink_model < 1 || m.sink_model > 3 || !(r2 < m.sink_hi2))
        return;
    const double dr = sqrt(r2);
    if (!(dr < m.sink_r4))
        return;
    // CUDA's exp here: a correctly rounded one (crm::exp_rn) changed no zone
    // of the reference fixtures but cost the stage 3 % in register pressure
    const double s = m.sink_rate * exp(-fourth_power<FAST>(div_by<FAST>(dr, m.sink_radius, m.inv_sink_radius)));
    double mdot = 0.0;
    if (s > 0.0)
        mdot = -s * sigma;
    else if (s < 0.0)
        mdot = -s;
    if (mdot == 0.0)
        return;
    switch (m.sink_model) {
    case 1:
        du[0] += dt * mdot;
        du[1] += dt * mdot * p[1];
        du[2] += dt * mdot * p[2];
        break;
    case 2: {
        const double d = dr + 1e-12;
        const double yd = FAST ? 1.0 / d : __drcp_rn(d);
        const double ex = div_by<FAST>(dx, d, yd);
        const double ey = div_by<FAST>(dy, d, yd);
        const double dvr = (p[1] - m.vx) * ex + (p[2] - m.vy) * ey;
        const double vxs = dvr * ex + m.vx;
        const double vys = dvr * ey + m.vy;
        du[0] += dt * mdot;
        du[1] += dt * mdot * vxs;
        du[2] += dt * mdot * vys;
        break;
    }
    default:
        du[0] += dt * mdot;
        break;
    }
}

// Keplerian buffer relaxation, cbdiso_2d.c:213-246
template <bool FAST>
__device__ __forceinline__ void buffer_source(const Consts &k, const StageDev &st, double x, double y, double dt,
                                              const double *u, double *du)
{
    if (!k.buffer_on)
        return;
    const double r2 = x * x + y * y;
    if (!(r2 > k.buf_lo2))
        return;
    const double rc = sqrt(r2);
    if (!(rc > k.buf_onset))
        return;
    const double yr = FAST ? 1.0 / rc : __drcp_rn(rc);
    const double vk = sqrt(div_by<FAST>(st.buffer_mass, rc, yr));
    const double t1 = k.buf_sigma * div_by<FAST>(-y, rc, yr) * vk;
    const double t2 = k.buf_sigma * div_by<FAST>(+x, rc, yr) * vk;
    const double rate = div_by<FAST>(st.buffer_k * (rc - k.buf_onset), k.buf_span, k.inv_buf_span);
    du[0] -= (u[0] - k.buf_sigma) * rate * dt;
    du[1] -= (u[1] - t1) * rate * dt;
    du[2] -= (u[2] - t2) * rate * dt;
}

// cbdiso_2d.c:268-283
template <bool FAST>
__device__ __forceinline__ void cons_to_prim(const double *u, double *p, const Consts &k)
{
    const double rho = greater(u[0], k.rho_min);
    p[0] = rho;
    const double y = FAST ? 1.0 / rho : __drcp_rn(rho);
    p[1] = copysign(lesser(fabs(div_by<FAST>(u[1], rho, y)), k.vmax), u[1]);
    p[2] = copysign(lesser(fabs(div_by<FAST>(u[2], rho, y)), k.vmax), u[2]);
}

// max |v +- cs| over both directions, cbdiso_2d.c:340-350
__device__ __forceinline__ double max_wavespeed(const double *p, double cs2)
{
    const double cs = sqrt(cs2);
    const double ax = greater(fabs(p[1] - cs), fabs(p[1] + cs));
    const double ay = greater(fabs(p[2] - cs), fabs(p[2] + cs));
    return greater(ax, ay);
}

// Source rates of both masses at the end-of-step time with dt = 1 and the
// reference's on/off switches (cbdiso_2d.py:105-137, cbdiso_2d.c:626-664):
// rg[p] with gravity only, ra[p] with accretion only, each (mdot, fx, fy).
// `need` selects which are evaluated (bit p: rg[p], bit 2 + p: ra[p]).
template <bool FAST>
__device__ __forceinline__ void end_rates(const MassDev *e, int need, double x, double y, const double *p,
                                          double (&rg)[2][3], double (&ra)[2][3])
{
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        rg[q][0] = rg[q][1] = rg[q][2] = 0.0;
        ra[q][0] = ra[q][1] = ra[q][2] = 0.0;
        if (need & (1 << q)) {
            // the gravity rates only enter sums whose own rounding (their
            // summation order) is far above an ulp per zone: rsqrt-based
            // arithmetic, not the correctly rounded power
            mass_source<true, true, false>(e[q], x, y, 1.0, p, rg[q]);
        }
        if (need & (4 << q))
            mass_source<FAST, false, true>(e[q], x, y, 1.0, p, ra[q]);
    }
}

// Per-zone value of one diagnostic (cbdiso_2d.py:383-471): out = (re, im).
// RATES: the caller knows that d is a source rate (mdot, fx, fy, torque,
// power) without a radial cut, so only that code is compiled (w = 1 then,
// the same values).
template <bool FAST, bool RATES = false>
__device__ __forceinline__ void diag_value(const cbd_diag_t &d, const MassDev *e, double x, double y,
                                           const double *p, const double (&rg)[2][3], const double (&ra)[2][3],
                                           double *out)
{
    double w = 1.0, r = 0.0;
    const bool polar = !RATES && (d.quantity == CBD_Q_SIGMA_M1 || d.quantity == CBD_Q_ECCENTRICITY_VECTOR);
    if (!RATES && (d.has_cut || polar)) {
        r = sqrt(x * x + y * y);
        if (d.has_cut)
            w = ((d.r0 < r) & (r < d.r1)) ? 1.0 : 0.0;
    }
    out[0] = 0.0;
    out[1] = 0.0;
    switch (RATES ? CBD_Q_MDOT : d.quantity) {
    case CBD_Q_MDOT:
    case CBD_Q_FX:
    case CBD_Q_FY:
    case CBD_Q_TORQUE:
    case CBD_Q_POWER: {
        // the reference takes the accretion rates when both flags are set
        const bool acc = d.accretion != 0;
        double r1[3], r2[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            r1[c] = acc ? ra[0][c] : rg[0][c];
            r2[c] = acc ? ra[1][c] : rg[1][c];
        }
        double f[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
            f[c] = d.which_mass == 3 ? r1[c] + r2[c] : (d.which_mass == 2 ? r2[c] : r1[c]);
        if (d.quantity == CBD_Q_MDOT)
            out[0] = f[0] * w;
        else if (d.quantity == CBD_Q_FX)
            out[0] = f[1] * w;
        else if (d.quantity == CBD_Q_FY)
            out[0] = f[2] * w;
        else if (d.quantity == CBD_Q_TORQUE)
            out[0] = x * (f[2] * w) - y * (f[1] * w);
        else {
            const MassDev &mv = e[d.which_mass == 2 ? 1 : 0];
            out[0] = mv.vx * (f[1] * w) + mv.vy * (f[2] * w);
        }
        break;
    }
    case CBD_Q_SIGMA_M1:
        out[0] = p[0] * w * (x / r);
        out[1] = p[0] * w * (y / r);
        break;
    case CBD_Q_ECCENTRICITY_VECTOR: {
        const double s = p[0] * w, vx = p[1] * w, vy = p[2] * w;
        const double vv = vx * vx + vy * vy;
        const double vr = vx * x + vy * y;
        out[0] = s * ((vv * x - vr * vx) / 1.0 - x / r);
        out[1] = s * ((vv * y - vr * vy) / 1.0 - y / r);
        break;
    }
    case CBD_Q_ANGULAR_MOMENTUM: {
        const double s = p[0] * w, vx = p[1] * w, vy = p[2] * w;
        out[0] = s * (x * vy - y * vx);
        break;
    }
    case CBD_Q_MASS:
        out[0] = p[0] * w;
        break;
    default:
        break;
    }
}

// The end-of-step quantities of one zone, accumulated into acc: slot 0 the
// CFL wavespeed maximum, slots 1 + 2d, 2 + 2d the diagnostics (RATES: all of
// them source rates without a radial cut, k.rates_only).
template <bool FAST, bool RATES = false>
__device__ __forceinline__ void accumulate_zone(const Consts &k, const MassDev *e, double x, double y,
                                                const double *p, double (&acc)[PARTIAL_STRIDE])
{
    if (k.want_ws)
        acc[0] = max_nan(acc[0], max_wavespeed(p, sound_speed2<FAST>(k, e, x, y)));
    if (k.num_diag > 0) {
        double rg[2][3], ra[2][3];
        end_rates<FAST>(e, k.need_rates, x, y, p, rg, ra);
#pragma unroll
        for (int d = 0; d < MAX_FUSED; ++d) {
            if (d < k.num_diag) {
                double v[2];
                diag_value<FAST, RATES>(k.diag[d], e, x, y, p, rg, ra, v);
                acc[1 + 2 * d] += v[0];
                acc[2 + 2 * d] += v[1];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// deterministic block and grid reductions
// ---------------------------------------------------------------------------

// Reduces PARTIAL_STRIDE per-thread values over the block in a fixed order:
// slot 0 by max, the others by sum. Thread 0 receives the results in `out`.
// All indices are compile-time constants so the values stay in registers.
template <int BJ>
__device__ __forceinline__ void block_reduce(const double (&vals)[PARTIAL_STRIDE], double *smem,
                                             double (&out)[PARTIAL_STRIDE])
{
    constexpr int NW = BJ / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < PARTIAL_STRIDE; ++v) {
        double x = vals[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            x = v == 0 ? max_nan(x, y) : x + y;
        }
        if (lane == 0)
            smem[v * NW + warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < PARTIAL_STRIDE; ++v) {
            double x = smem[v * NW];
            for (int w = 1; w < NW; ++w)
                x = v == 0 ? max_nan(x, smem[v * NW + w]) : x + smem[v * NW + w];
            out[v] = x;
        }
    }
    __syncthreads();
}

// Writes this CTA's partials; the last CTA to finish reduces all partials
// in CTA order, writes value 0 to out0 (if non-null) and values 1 .. n-1 to
// out_rest, and re-arms the counter. `scratch` holds a 64-byte counter word
// followed by num_ctas * PARTIAL_STRIDE doubles.
template <int BJ>
__device__ void grid_finish(const double (&mine)[PARTIAL_STRIDE], int n, double *scratch, double *out0,
                            double *out_rest, double *smem)
{
    unsigned int *counter = reinterpret_cast<unsigned int *>(scratch);
    double *partials = scratch + 8;
    const unsigned int nblocks = gridDim.x * gridDim.y;
    const unsigned int bid = blockIdx.y * gridDim.x + blockIdx.x;
    __shared__ unsigned int ticket;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < PARTIAL_STRIDE; ++v)
            partials[(size_t)bid * PARTIAL_STRIDE + v] = mine[v];
        __threadfence();
        ticket = atomicAdd(counter, 1u);
    }
    __syncthreads();
    if (ticket != nblocks - 1)
        return;
    __threadfence();
    // Each thread folds a strided, ordered subset; then a fixed-order tree.
    double acc[PARTIAL_STRIDE];
#pragma unroll
    for (int v = 0; v < PARTIAL_STRIDE; ++v)
        acc[v] = 0.0;
    for (unsigned int b = threadIdx.x; b < nblocks; b += BJ) {
        const volatile double *src = partials + (size_t)b * PARTIAL_STRIDE;
#pragma unroll
        for (int v = 0; v < PARTIAL_STRIDE; ++v) {
            const double x = src[v];
            acc[v] = v == 0 ? max_nan(acc[v], x) : acc[v] + x;
        }
    }
    double red[PARTIAL_STRIDE];
    block_reduce<BJ>(acc, smem, red);
    if (threadIdx.x == 0) {
        if (out0)
            *out0 = red[0];
#pragma unroll
        for (int v = 1; v < PARTIAL_STRIDE; ++v)
            if (v < n)
                out_rest[v - 1] = red[v];
        *counter = 0u;
        __threadfence();
    }
}

// ---------------------------------------------------------------------------
// asynchronous global -> shared copies (cp.async), used to fetch the next row
// of the march one iteration ahead of its use
// ---------------------------------------------------------------------------

__device__ __forceinline__ void async_copy8(void *smem, const void *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

__device__ __forceinline__ void async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// the fused stage kernel
// ---------------------------------------------------------------------------

struct StageArgs {
    const double *prd;   // primitive state read by the stencil (guards valid)
    const double *un;    // primitive_n (un_kind 1) or conserved_rk (un_kind 2)
    double *pwr;         // output primitive state
    const StageDev *stage_dev;  // optional device copy of the stage parameters
    double *scratch;     // reductions scratch (epilogue only)
    double *result;      // reductions result (epilogue only)
    double *fcache;      // optional face cache (face_cache_doubles), null: none
};

// ---------------------------------------------------------------------------
// face cache
//
// The face sound speeds (cs^2, cs) at every x- and y-face centre and the
// gravity factors (r^2 + s^2)^-1.5 of both masses at every zone centre depend
// only on the mesh, the EOS constants and the point masses' positions, masses
// and softenings, not on the fluid state. A step's last stage usually runs
// with the masses of the step's end time, which are the next step's
// first-stage masses (RK2's second stage at t0 + dt, the next step at
// t0 / 2 + (t0 + 2 dt) / 2, equal in all but about 1 step in 5000). The host
// gives each stage launch a role:
//  * ROLE_WRITER (RK2's second stage, RK3's second): computes the values in
//    its stencil as usual and, when its masses equal its record's
//    end-of-step masses, also stores them with a key of everything they
//    depend on (written by one thread).
//  * ROLE_READER (a step's first stage): a fill kernel runs first; when the
//    key does not match the stage's masses (a solver's first step, a reset,
//    the rare time mismatch) it computes every value for them. The stage
//    loads them and then records the key.
//  * ROLE_NONE: neither.
// Evaluating the values inline in the writer costs less than a separate
// fill pass every step (measured on both the single-grid and the batched
// path); the fill kernel serves the mismatches.
// The values are the same bits as recomputing them. Each role is its own
// kernel, so that each keeps its own register allocation. Launches on one
// cache must be stream-ordered.
//
// Layout (doubles): a 32-double header holding the key, then
//   x-faces (ni + 1) x nj pairs (cs^2, cs): pair [i][j] is the face between
//     rows i - 1 and i in column j;
//   y-faces ni x (nj + 1) pairs: [i][j] is the face between columns j - 1 and
//     j in row i;
//   zones ni x nj pairs (g_1, g_2).
// ---------------------------------------------------------------------------

enum { ROLE_NONE = 0, ROLE_WRITER = 1, ROLE_READER = 2 };
// what one march (march_tile's COP) does with the cache, by role
enum { CACHE_NONE = 0, CACHE_WRITE = 1, CACHE_READ = 2 };
constexpr int CACHE_HEADER = 32;  // doubles
constexpr int CACHE_KEY = 20;     // doubles of the header holding the key

__host__ __device__ inline size_t face_cache_doubles(int ni, int nj)
{
    return CACHE_HEADER + 2 * ((size_t)(ni + 1) * nj + (size_t)ni * (nj + 1) + (size_t)ni * nj);
}

// the three arrays of a cache
struct CacheArrays {
    double *xf, *yf, *grav;
};

__host__ __device__ inline CacheArrays cache_arrays(double *fc, int ni, int nj)
{
    CacheArrays c;
    c.xf = fc + CACHE_HEADER;
    c.yf = c.xf + 2 * (size_t)(ni + 1) * nj;
    c.grav = c.yf + 2 * (size_t)ni * (nj + 1);
    return c;
}

// The key: a format tag, the precision, then every input of the cached values.
template <int PREC>
__device__ __forceinline__ double cache_key_value(const Consts &k, const MassDev *m, int v)
{
    switch (v) {
    case 0: return 20261204.5;
    case 1: return (double)PREC;
    case 2: return (double)k.eos;
    case 3: return (double)k.ni;
    case 4: return (double)k.nj;
    case 5: return k.xl;
    case 6: return k.yl;
    case 7: return k.dx;
    case 8: return k.dy;
    case 9: return k.cs2;
    case 10: return k.mach2;
    case 11: return k.inv_mach2;
    default: {
        const MassDev &q = m[(v - 12) >> 2];
        switch ((v - 12) & 3) {
        case 0: return q.x;
        case 1: return q.y;
        case 2: return q.mass;
        default: return q.soft2;
        }
    }
    }
}

__device__ __forceinline__ bool same_bits(double a, double b)
{
    return __double_as_longlong(a) == __double_as_longlong(b);
}

template <int PREC>
__device__ bool cache_key_matches(const Consts &k, const StageDev &st, const double *fc)
{
    for (int v = 0; v < CACHE_KEY; ++v)
        if (!same_bits(fc[v], cache_key_value<PREC>(k, st.m, v)))
            return false;
    return true;
}

template <int PREC>
__device__ void cache_write_key(const Consts &k, const StageDev &st, double *fc)
{
    for (int v = 0; v < CACHE_KEY; ++v)
        fc[v] = cache_key_value<PREC>(k, st.m, v);
}

// The cached values depend on these fields of the masses only (the same
// answer in every thread).
__device__ __forceinline__ bool same_cached_inputs(const StageDev &st)
{
    bool same = true;
#pragma unroll
    for (int p = 0; p < 2; ++p)
        same = same && same_bits(st.m[p].x, st.e[p].x) && same_bits(st.m[p].y, st.e[p].y) &&
               same_bits(st.m[p].mass, st.e[p].mass) && same_bits(st.m[p].soft2, st.e[p].soft2);
    return same;
}

// A writer stores the values when its masses are the end-of-step masses (the
// same answer in every thread); `key_writer` (one thread) then writes the key.
template <int PREC>
__device__ bool cache_write_check(const Consts &k, const StageDev &st, double *fc, bool key_writer)
{
    const bool end_masses = same_cached_inputs(st);
    if (end_masses && key_writer)
        cache_write_key<PREC>(k, st, fc);
    return end_masses;
}

__device__ __forceinline__ double2 cache_load(const double *p)
{
    return __ldcs(reinterpret_cast<const double2 *>(p));
}

__device__ __forceinline__ void cache_store(double *p, double a, double b)
{
    __stcs(reinterpret_cast<double2 *>(p), make_double2(a, b));
}

// Shared memory of the march, one instance per kernel whichever copies of
// march_tile it holds. ONE_SYNC selects the march with one barrier per row
// (march_tile).
template <int BJ, bool ONE_SYNC>
struct StageSmem {
    static constexpr int RING = ONE_SYNC ? 5 : 4;
    double sp[RING][NQ][BJ + 4];             // primitive rows ring, columns c0-2 .. c0+BJ+1
    double sgy[2][NQ][BJ + 2];               // y-slopes ring, columns c0-1 .. c0+BJ
    double srs[2][NQ][BJ + 2];               // rho * strain ring, same columns
    double sg[ONE_SYNC ? 2 : 1][NQ][BJ + 1];  // y-face fluxes (by row parity with ONE_SYNC)
    double sun[ONE_SYNC ? 1 : 2][NQ][ONE_SYNC ? 1 : BJ];  // u_n zones a row ahead (two-barrier march)
};

// A static allocation may take up to 48 KB; the march of a 256-column strip
// (68 KB) takes its shared memory from the launch's dynamic allocation,
// whose size the launch gives (march_dynamic_smem).
constexpr size_t STATIC_SMEM_LIMIT = 48 * 1024;

template <int BJ, bool ONE_SYNC>
__device__ __forceinline__ StageSmem<BJ, ONE_SYNC> &stage_smem()
{
    if constexpr (sizeof(StageSmem<BJ, ONE_SYNC>) > STATIC_SMEM_LIMIT) {
        extern __shared__ __align__(16) unsigned char stage_dynamic_smem[];
        return *reinterpret_cast<StageSmem<BJ, ONE_SYNC> *>(stage_dynamic_smem);
    } else {
        __shared__ StageSmem<BJ, ONE_SYNC> m;
        return m;
    }
}

// dynamic shared memory bytes a stage kernel of BJ columns is launched with
template <int BJ>
constexpr size_t march_dynamic_smem()
{
    return sizeof(StageSmem<BJ, true>) > STATIC_SMEM_LIMIT ? sizeof(StageSmem<BJ, true>) : 0;
}

// One tile of the march: columns c0 .. c0 + width - 1 (width <= BJ) and rows
// r0 .. r0 + k.rows_per_cta - 1 of one grid. `st` must live in shared memory
// and be visible after the first barrier; epilogue values of the updated
// zones are accumulated into `acc` when EPI (the launch has an epilogue;
// without, its code is left out). `COP` (CACHE_*) says what the tile does
// with args.fcache: CACHE_WRITE stores the face and gravity values if
// `store`, CACHE_READ loads them. ONE_SYNC marches with one barrier per row
// (five-row ring, u_n in registers), otherwise with two (four-row ring, u_n
// through shared memory), which needs fewer registers: the persistent
// batched kernel keeps it. All threads of the block must call it.
template <int BJ, bool FAST, int COP = CACHE_NONE, bool EPI = true, bool ONE_SYNC = true, bool P2 = false,
          bool RATES = false>
__device__ __forceinline__ void march_tile(const Consts &k, const StageDev &st, const StageArgs &args, int c0,
                                           int width, int r0, double (&acc)[PARTIAL_STRIDE], bool store = false)
{
    constexpr int cop = COP;
    StageSmem<BJ, ONE_SYNC> &sm = stage_smem<BJ, ONE_SYNC>();
    auto &sp = sm.sp;
    auto &sgy = sm.sgy;
    auto &srs = sm.srs;
    auto &sg = sm.sg;
    auto &sun = sm.sun;

    const int t = threadIdx.x;
    const int ni = k.ni, nj = k.nj;
    const int W = min(width, nj - c0);
    const int r1 = min(r0 + k.rows_per_cta, ni);
    const bool active = t < W;
    const int j = c0 + t;
    const size_t row_stride = (size_t)(nj + 2 * NG) * NQ;
    const bool viscous = k.nu > 0.0;

    // face-cache arrays (pairs of doubles), used when cop != CACHE_NONE
    const CacheArrays cache = cache_arrays(cop != CACHE_NONE ? args.fcache : nullptr, ni, nj);
    double *const cfx = cop != CACHE_NONE ? cache.xf : nullptr;
    double *const cfy = cop != CACHE_NONE ? cache.yf : nullptr;
    double *const cfz = cop != CACHE_NONE ? cache.grav : nullptr;

    auto zone = [&](const double *base, int i, int jj) -> const double * {
        return base + (size_t)(i + NG) * row_stride + (size_t)(jj + NG) * NQ;
    };
    // Row i (zones c0-2 .. c0+W+1) into ring slot `slot`, as asynchronous
    // copies into the field-major shared layout: thread t copies the three
    // fields of column t (a warp's copies of one field together cover its
    // columns' contiguous AoS bytes), and threads 0..3 also the last four
    // columns when the strip is full.
    auto fetch_row = [&](int slot, int i) {
        const double *src = args.prd + (size_t)(i + NG) * row_stride + (size_t)c0 * NQ;
        for (int kk = t; kk < W + 4; kk += BJ) {
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                async_copy8(&sp[slot][q][kk], src + NQ * kk + q);
        }
    };
    // The zone (i, j) of the u_n source array, for this thread's own update:
    // into registers at the top of row i's iteration (ONE_SYNC), or into
    // shared memory a row ahead. In the in-place final stage this array is
    // also written, by the same thread and only after the zone has been
    // consumed (so a plain load, not the read-only path).
    auto load_un = [&](int i, double *z3) {
        if (k.un_kind != 0 && active && i >= r0 && i < r1) {
            const double *z = zone(args.un, i, j);
            z3[0] = z[0];
            z3[1] = z[1];
            z3[2] = z[2];
        }
    };
    auto fetch_un = [&](int i) {
        if (k.un_kind != 0 && active) {
            const double *z = zone(args.un, i, j);
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                async_copy8(&sun[ONE_SYNC ? 0 : i & 1][q][ONE_SYNC ? 0 : t], z + q);
        }
    };
    // Lanes that do the strip's extra work, spread over different warps: the
    // slopes of the two halo columns, and the last y-face of the row.
    constexpr int HALO_LANE = BJ >= 64 ? 32 : 0;
    constexpr int FACE_LANE = BJ >= 128 ? 64 : (BJ >= 64 ? 0 : 2);

    // own-column carried state: x-slope and rho*strain of row r, x-face flux F(r - 1/2)
    double gx0[NQ] = {0.0, 0.0, 0.0}, rs0[NQ] = {0.0, 0.0, 0.0}, f0[NQ] = {0.0, 0.0, 0.0};

    // ONE_SYNC: one barrier per row. Rows sit in a five-slot ring (slot of
    // row i: (i - r0 + 2) mod 5). Row r + 4 is fetched right after iteration
    // r's barrier into the slot of row r - 1 (last read before that
    // barrier), and each thread waits for its copies of row r + 3 before the
    // barrier, so the rows r + 1 .. r + 3 that iteration r + 1 reads are
    // resident and visible. The y-face fluxes alternate between two buffers
    // by row parity, so iteration r + 1 may write its own while a slower warp
    // still reads iteration r's.
    // Otherwise two barriers per row: at the top of iteration r (rows r ..
    // r + 2 and the u_n zone of row r fetched one iteration ago have landed;
    // the slot of row r - 1 is free for row r + 3), and between the y-faces
    // and the zone update. Ring slot of row i: i mod 4.
    int s0;  // ring slot of row r
    if constexpr (ONE_SYNC) {
        fetch_row(0, r0 - 2);
        fetch_row(1, r0 - 1);
        fetch_row(2, r0);
        async_commit();
        async_wait_all();
        __syncthreads();
        if (r0 + 1 <= r1 + 1)
            fetch_row(3, r0 + 1);
        async_commit();
        s0 = 0;
    } else {
        fetch_row((r0 - 2) & 3, r0 - 2);
        fetch_row((r0 - 1) & 3, r0 - 1);
        fetch_row(r0 & 3, r0);
        async_commit();
        s0 = (r0 - 2) & 3;
    }

    for (int r = r0 - 2; r < r1; ++r) {
        if constexpr (!ONE_SYNC) {
            async_wait_all();
            __syncthreads();
            if (r + 3 <= r1 + 1)
                fetch_row((r + 3) & 3, r + 3);
            if (r + 1 >= r0 && r + 1 < r1)
                fetch_un(r + 1);
            async_commit();
        }
        constexpr int RING = StageSmem<BJ, ONE_SYNC>::RING;
        const int s1 = s0 == RING - 1 ? 0 : s0 + 1, s2 = s1 == RING - 1 ? 0 : s1 + 1;
        const int g1 = (r + 1) & 1, g0 = r & 1;
        const int gf = ONE_SYNC ? g0 : 0;  // y-face flux buffer of row r
        double un_cur[NQ] = {0.0, 0.0, 0.0};
        if (ONE_SYNC)
            load_un(r, un_cur);

        // cached face sound speeds and gravity factors of this row, loaded
        // ahead of the slopes so that their latency overlaps them
        double2 c_xf = make_double2(0.0, 0.0), c_yf = c_xf, c_ye = c_xf, c_z = c_xf;
        if (cop == CACHE_READ) {
            if (r >= r0 - 1 && active)
                c_xf = cache_load(cfx + 2 * ((size_t)(r + 1) * nj + j));
            if (r >= r0) {
                if (active) {
                    c_yf = cache_load(cfy + 2 * ((size_t)r * (nj + 1) + j));
                    c_z = cache_load(cfz + 2 * ((size_t)r * nj + j));
                }
                if (t == FACE_LANE)
                    c_ye = cache_load(cfy + 2 * ((size_t)r * (nj + 1) + c0 + W));
            }
        }

        // (1) slopes and rho * strain at row r + 1: own column, plus the two
        //     halo columns (c0 - 1 and c0 + W) handled by two lanes of one warp.
        double gx1[NQ] = {0.0, 0.0, 0.0}, rs1[NQ] = {0.0, 0.0, 0.0};
        {
            const bool halo = t == HALO_LANE || t == HALO_LANE + 1;
            const int passes = halo ? 2 : 1;
            for (int pass = 0; pass < passes; ++pass) {
                int kk;  // sp column index
                if (pass == 0) {
                    if (!active)
                        continue;
                    kk = t + 2;
                } else {
                    kk = (t == HALO_LANE) ? 1 : W + 2;
                }
                double gx[NQ], gy[NQ], rs[NQ] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    gx[q] = limited_slope(sp[s0][q][kk], sp[s1][q][kk], sp[s2][q][kk], k.theta);
                    gy[q] = limited_slope(sp[s1][q][kk - 1], sp[s1][q][kk], sp[s1][q][kk + 1], k.theta);
                }
                if (viscous)
                    rho_strain<FAST, P2>(sp[s1][0][kk], gx, gy, k, rs);
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    sgy[g1][q][kk - 1] = gy[q];
                    srs[g1][q][kk - 1] = rs[q];
                }
                if (pass == 0) {
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        gx1[q] = gx[q];
                        rs1[q] = rs[q];
                    }
                }
            }
        }

        // (2) x-face flux F(r + 1/2), own column
        double f1[NQ] = {0.0, 0.0, 0.0};
        if (r >= r0 - 1 && active) {
            const int kk = t + 2;
            double pl[NQ], pr[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                // one FMA each: halving a normal number is exact, so this rounds
                // as the reference's multiply then add
                pl[q] = fma(0.5, gx0[q], sp[s0][q][kk]);
                pr[q] = fma(-0.5, gx1[q], sp[s1][q][kk]);
            }
            if (cop == CACHE_READ) {
                double cs = c_xf.y;
                hlle<FAST, 0, true>(pl, pr, c_xf.x, cs, f1);
            } else {
                const double xf = k.xl + (double)(r + 1) * k.dx;
                const double yc = k.yl + ((double)j + 0.5) * k.dy;
                const double cs2 = sound_speed2<FAST>(k, st.m, xf, yc);
                double cs;
                hlle<FAST, 0>(pl, pr, cs2, cs, f1);
                // face r + 1/2 is stored by the tile below it, except the first
                if (cop == CACHE_WRITE && store && (r >= r0 || r0 == 0))
                    cache_store(cfx + 2 * ((size_t)(r + 1) * nj + j), cs2, cs);
            }
            if (viscous) {
                f1[1] -= k.half_nu * (rs0[0] + rs1[0]);
                f1[2] -= k.half_nu * (rs0[1] + rs1[1]);
            }
        }

        // (3) y-face fluxes of row r: face c0 + f - 1/2 for f = t, plus f = W
        if (r >= r0) {
            const int passes = (t == FACE_LANE) ? 2 : 1;
            for (int pass = 0; pass < passes; ++pass) {
                int fidx;
                if (pass == 0) {
                    if (!active)
                        continue;
                    fidx = t;
                } else {
                    fidx = W;
                }
                // zones on either side: sp columns fidx + 1 (minus side) and fidx + 2 (plus side)
                double pl[NQ], pr[NQ], g[NQ];
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    pl[q] = fma(0.5, sgy[g0][q][fidx], sp[s0][q][fidx + 1]);
                    pr[q] = fma(-0.5, sgy[g0][q][fidx + 1], sp[s0][q][fidx + 2]);
                }
                if (cop == CACHE_READ) {
                    double cs = pass == 0 ? c_yf.y : c_ye.y;
                    hlle<FAST, 1, true>(pl, pr, pass == 0 ? c_yf.x : c_ye.x, cs, g);
                } else {
                    const double xc = k.xl + ((double)r + 0.5) * k.dx;
                    const double yf = k.yl + (double)(c0 + fidx) * k.dy;
                    const double cs2 = sound_speed2<FAST>(k, st.m, xc, yf);
                    double cs;
                    hlle<FAST, 1>(pl, pr, cs2, cs, g);
                    // the strip's last face is stored by the next strip, except the last
                    if (cop == CACHE_WRITE && store && (pass == 0 || c0 + W == nj))
                        cache_store(cfy + 2 * ((size_t)r * (nj + 1) + c0 + fidx), cs2, cs);
                }
                if (viscous) {
                    g[1] -= k.half_nu * (srs[g0][1][fidx] + srs[g0][1][fidx + 1]);
                    g[2] -= k.half_nu * (srs[g0][2][fidx] + srs[g0][2][fidx + 1]);
                }
#pragma unroll
                for (int q = 0; q < NQ; ++q)
                    sg[gf][q][fidx] = g[q];
            }
        }
        if constexpr (ONE_SYNC) {
            // row r + 3 has landed for this thread; after the barrier for
            // all, and the slot of row r - 1 is free for row r + 4
            async_wait_all();
            __syncthreads();
            if (r + 4 <= r1 + 1) {
                const int s4 = s2 >= 3 ? s2 - 3 : s2 + 2;  // (s0 + 4) mod 5
                fetch_row(s4, r + 4);
            }
            async_commit();
        } else {
            __syncthreads();
        }

        // (4) update zone (r, j)
        if (r >= r0 && active) {
            const int kk = t + 2;
            const double xc = k.xl + ((double)r + 0.5) * k.dx;
            const double yc = k.yl + ((double)j + 0.5) * k.dy;
            double pc[NQ], u[NQ], un[NQ], du[NQ] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                pc[q] = sp[s0][q][kk];
            u[0] = pc[0];
            u[1] = pc[1] * pc[0];
            u[2] = pc[2] * pc[0];
            if (k.un_kind == 0) {
                un[0] = u[0];
                un[1] = u[1];
                un[2] = u[2];
            } else {
                const int ub = ONE_SYNC ? 0 : r & 1, uc = ONE_SYNC ? 0 : t;
                const double z0 = ONE_SYNC ? un_cur[0] : sun[ub][0][uc];
                const double z1 = ONE_SYNC ? un_cur[1] : sun[ub][1][uc];
                const double z2 = ONE_SYNC ? un_cur[2] : sun[ub][2][uc];
                if (k.un_kind == 1) {
                    un[0] = z0;
                    un[1] = z1 * z0;
                    un[2] = z2 * z0;
                } else {
                    un[0] = z0;
                    un[1] = z1;
                    un[2] = z2;
                }
            }
            const double dt = st.dt;
            buffer_source<FAST>(k, st, xc, yc, dt, u, du);
            if (cop == CACHE_READ) {
                mass_source<FAST>(st.m[0], xc, yc, dt, pc, du, &c_z.x);
                mass_source<FAST>(st.m[1], xc, yc, dt, pc, du, &c_z.y);
            } else {
                // both gravity factors first (two independent chains), the
                // terms then as with cached values; a massless mass has no
                // gravity term and caches 0
                double g[2];
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const double dx = xc - st.m[p].x, dy = yc - st.m[p].y;
                    const double s2 = dx * dx + dy * dy + st.m[p].soft2;
                    const double gp = inv_pow15<FAST>(s2);
                    g[p] = st.m[p].mass != 0.0 ? gp : 0.0;
                }
                mass_source<FAST>(st.m[0], xc, yc, dt, pc, du, &g[0]);
                mass_source<FAST>(st.m[1], xc, yc, dt, pc, du, &g[1]);
                if (cop == CACHE_WRITE && store)
                    cache_store(cfz + 2 * ((size_t)r * nj + j), g[0], g[1]);
            }
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const double gn = sg[gf][q][t + 1], gs = sg[gf][q][t];
                du[q] -= (div_by<FAST || P2>(f1[q] - f0[q], k.dx, k.inv_dx) +
                          div_by<FAST || P2>(gn - gs, k.dy, k.inv_dy)) *
                         dt;
            }
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                u[q] += du[q];
                u[q] = st.one_minus_a * u[q] + st.a * un[q];
            }
            double pn[NQ];
            cons_to_prim<FAST>(u, pn, k);

            // store the zone and, on the edges, its zero-gradient guard images
            const bool edge = k.write_guards && (r == 0 || r == ni - 1 || j == 0 || j == nj - 1);
            if (!edge) {
                double *z = args.pwr + (size_t)(r + NG) * row_stride + (size_t)(j + NG) * NQ;
                z[0] = pn[0];
                z[1] = pn[1];
                z[2] = pn[2];
            } else {
                const int ilo = r == 0 ? -2 : r;
                const int ihi = r == ni - 1 ? ni + 1 : r;
                const int jlo = j == 0 ? -2 : j;
                const int jhi = j == nj - 1 ? nj + 1 : j;
                for (int ii = ilo; ii <= ihi; ++ii) {
                    for (int jj = jlo; jj <= jhi; ++jj) {
                        double *z = args.pwr + (size_t)(ii + NG) * row_stride + (size_t)(jj + NG) * NQ;
                        z[0] = pn[0];
                        z[1] = pn[1];
                        z[2] = pn[2];
                    }
                }
            }

            if (EPI)
                accumulate_zone<FAST, RATES>(k, st.e, xc, yc, pn, acc);
        }

#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            gx0[q] = gx1[q];
            rs0[q] = rs1[q];
            f0[q] = f1[q];
        }
        s0 = s1;
    }

    // leave the shared buffers free for the block's next tile
    __syncthreads();
}

// One RK stage on one grid: CTA (x, y) marches strip x, segment y. ROLE
// (ROLE_*) is what the launch does with args.fcache; EPI whether it has an
// epilogue (k.want_ws or k.num_diag); P2 that k.spacing_pow2 is set (the
// divisions by dx and dy are then the products with their exact
// reciprocals).
template <int BJ, int MINB, int PREC, int ROLE = ROLE_NONE, bool EPI = true, bool P2 = false>
__global__ void __launch_bounds__(BJ, MINB) stage_kernel(const Consts k, const StageDev st_param, StageArgs args)
{
    constexpr bool FAST = PREC == CBD_PRECISION_FAST;
    __shared__ StageDev st;
    __shared__ double sred[PARTIAL_STRIDE * (BJ / 32)];
    if (threadIdx.x == 0)
        st = args.stage_dev ? *args.stage_dev : st_param;
    double acc[PARTIAL_STRIDE];
#pragma unroll
    for (int v = 0; v < PARTIAL_STRIDE; ++v)
        acc[v] = 0.0;
    const int c0 = blockIdx.x * BJ, r0 = blockIdx.y * k.rows_per_cta;
    __syncthreads();
    if (st.halt)
        return;
    if (ROLE == ROLE_WRITER) {
        const bool store = cache_write_check<PREC>(k, st, args.fcache,
                                                   threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0);
        march_tile<BJ, FAST, CACHE_WRITE, EPI, true, P2>(k, st, args, c0, BJ, r0, acc, store);
    } else if (ROLE == ROLE_READER) {
        march_tile<BJ, FAST, CACHE_READ, EPI, true, P2>(k, st, args, c0, BJ, r0, acc);
        // the fill kernel before this launch made the values valid for these
        // masses; say so for the next fill (no one reads the key meanwhile)
        if (threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0)
            cache_write_key<PREC>(k, st, args.fcache);
    } else {
        march_tile<BJ, FAST, CACHE_NONE, EPI, true, P2>(k, st, args, c0, BJ, r0, acc);
    }
    if (EPI) {
        double red[PARTIAL_STRIDE];
        block_reduce<BJ>(acc, sred, red);
        grid_finish<BJ>(red, 1 + 2 * k.num_diag, args.scratch, k.want_ws ? args.result : nullptr, args.result + 1,
                        sred);
    }
}

// resident 128-thread CTAs per SM the rates-only epilogue is built for
constexpr int EPI_RATES_MINB = 4;

// The epilogue of one tile after its stage has written it: thread t adds up
// the zones of column c0 + t, rows r0 .. r0 + k.rows_per_cta - 1, of the new
// state `p` in row order, exactly as the fused march accumulates them.
template <bool FAST, bool RATES = false>
__device__ __forceinline__ void epilogue_tile(const Consts &k, const StageDev &st, const double *p, int c0,
                                              int width, int r0, double (&acc)[PARTIAL_STRIDE])
{
    const int t = threadIdx.x;
    const int W = min(width, k.nj - c0);
    const int r1 = min(r0 + k.rows_per_cta, k.ni);
    if (t >= W)
        return;
    const int j = c0 + t;
    const size_t row_stride = (size_t)(k.nj + 2 * NG) * NQ;
    const double yc = k.yl + ((double)j + 0.5) * k.dy;
    const double *z = p + (size_t)(r0 + NG) * row_stride + (size_t)(j + NG) * NQ;
    if (r0 >= r1)
        return;
    double nx[NQ] = {z[0], z[1], z[2]};
    for (int r = r0; r < r1; ++r) {
        const double pn[NQ] = {nx[0], nx[1], nx[2]};
        z += row_stride;
        if (r + 1 < r1) {
            nx[0] = z[0];
            nx[1] = z[1];
            nx[2] = z[2];
        }
        const double xc = k.xl + ((double)r + 0.5) * k.dx;
        accumulate_zone<FAST, RATES>(k, st.e, xc, yc, pn, acc);
    }
}

// A stage's epilogue as its own launch, after a stage kernel launched
// without it (EPI = false) on the same grid: the same CTA tiles, per-thread
// order, block tree and CTA order, so the same bits as the fused epilogue.
// Reading the new state back (24 B per zone) costs less than carrying the
// epilogue's registers and code through the stencil's march. (As two
// launches, the wavespeed maximum and the diagnostic sums each with its own
// register budget, it measured slower.) RATES: the form for k.rates_only,
// with fewer registers.
template <int BJ, int PREC, bool RATES = false>
__global__ void __launch_bounds__(BJ, (RATES ? EPI_RATES_MINB : 4) * 128 / BJ)
    stage_epilogue_kernel(const Consts k, const StageDev st_param, StageArgs args)
{
    constexpr bool FAST = PREC == CBD_PRECISION_FAST;
    __shared__ StageDev st;
    __shared__ double sred[PARTIAL_STRIDE * (BJ / 32)];
    if (threadIdx.x == 0)
        st = args.stage_dev ? *args.stage_dev : st_param;
    __syncthreads();
    if (st.halt)
        return;
    double acc[PARTIAL_STRIDE];
#pragma unroll
    for (int v = 0; v < PARTIAL_STRIDE; ++v)
        acc[v] = 0.0;
    epilogue_tile<FAST, RATES>(k, st, args.pwr, blockIdx.x * BJ, BJ, blockIdx.y * k.rows_per_cta, acc);
    double red[PARTIAL_STRIDE];
    block_reduce<BJ>(acc, sred, red);
    grid_finish<BJ>(red, 1 + 2 * k.num_diag, args.scratch, k.want_ws ? args.result : nullptr, args.result + 1, sred);
}

// Every cached value at mesh point (i, j), 0 <= i <= ni, 0 <= j <= nj, for
// the masses m, with the stage kernel's own expressions: the x-face pair
// (i, j) when j < nj, the y-face pair when i < ni, and the zone's gravity
// factors when both are inside.
template <bool FAST>
__device__ __forceinline__ void face_cache_fill_point(const Consts &k, const MassDev *m, const CacheArrays &c,
                                                      int i, int j)
{
    const int ni = k.ni, nj = k.nj;
    const double xf = k.xl + (double)i * k.dx;
    const double xc = k.xl + ((double)i + 0.5) * k.dx;
    const double yf = k.yl + (double)j * k.dy;
    const double yc = k.yl + ((double)j + 0.5) * k.dy;
    if (j < nj) {
        const double cs2 = sound_speed2<FAST>(k, m, xf, yc);
        cache_store(c.xf + 2 * ((size_t)i * nj + j), cs2, sqrt(cs2));
    }
    if (i < ni) {
        const double cs2 = sound_speed2<FAST>(k, m, xc, yf);
        cache_store(c.yf + 2 * ((size_t)i * (nj + 1) + j), cs2, sqrt(cs2));
    }
    if (i < ni && j < nj) {
        double g[2] = {0.0, 0.0};
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            if (m[p].mass != 0.0) {
                const double dx = xc - m[p].x;
                const double dy = yc - m[p].y;
                g[p] = inv_pow15<FAST>(dx * dx + dy * dy + m[p].soft2);
            }
        }
        cache_store(c.grav + 2 * ((size_t)i * nj + j), g[0], g[1]);
    }
}

// The points of one tile of a grid: columns c0 .. c0 + width - 1 and rows
// r0 .. r0 + rows - 1, plus column nj in the last strip and row ni in the
// last segment. All threads of the block take part.
template <int BJ, bool FAST>
__device__ __forceinline__ void face_cache_fill_tile(const Consts &k, const MassDev *m, double *fc, int c0,
                                                     int width, int r0, int rows)
{
    const CacheArrays c = cache_arrays(fc, k.ni, k.nj);
    const int W = min(width, k.nj - c0);
    const int wext = c0 + W == k.nj ? W + 1 : W;
    const int r1 = min(r0 + rows, k.ni);
    const int rext = r1 == k.ni ? r1 + 1 : r1;
    for (int i = r0; i < rext; ++i)
        for (int t = threadIdx.x; t < wext; t += BJ)
            face_cache_fill_point<FAST>(k, m, c, i, c0 + t);
}

// Makes the face cache valid for a reader stage: when its key does not match
// the stage's masses, the CTAs fill the stage's tiles (`strips` x `tiles /
// strips` of BJ columns x k.rows_per_cta rows), CTA b taking tiles b,
// b + gridDim.x, ..., with the values for those masses (the reader stage then
// writes the key). A grid of a few CTAs per SM keeps the common case, a
// matching key, to one check per CTA. A halted record (a stopped device
// stepper) fills nothing. The evaluation is long chains of dependent
// operations: many warps per SM, registers capped to allow them.
constexpr int FILL_WARPS_PER_SM = 24;

template <int BJ, int PREC>
__global__ void __launch_bounds__(BJ, FILL_WARPS_PER_SM * 32 / BJ)
    face_cache_fill_kernel(const Consts k, const StageDev st_param, const StageDev *stage_dev, double *fc, int strips,
                           int tiles)
{
    __shared__ StageDev st;
    __shared__ int fill;
    if (threadIdx.x == 0) {
        st = stage_dev ? *stage_dev : st_param;
        fill = !st.halt && !cache_key_matches<PREC>(k, st, fc);
    }
    __syncthreads();
    if (!fill)
        return;
    for (int u = blockIdx.x; u < tiles; u += gridDim.x)
        face_cache_fill_tile<BJ, PREC == CBD_PRECISION_FAST>(k, st.m, fc, (u % strips) * BJ, BJ,
                                                             (u / strips) * k.rows_per_cta, k.rows_per_cta);
}

}  // namespace cbd
