// The gamma-law circumbinary-disk stage (cbdgam_2d): the reference's
// energy-equation sibling of cbdiso_2d (sailfish/solvers/cbdgam_2d.c), with
// four fields (sigma, vx, vy, pressure), alpha viscosity with the disk's
// scale height, softening that may follow the scale height, cooling, a
// pressure floor and a Mach ceiling.
//
// Built with -fmad=false: every +, -, *, / and sqrt gives the IEEE result the
// reference's CPU build computes, in the reference's order, and every power
// and exponential is correctly rounded (cr_math.cuh), so results differ from
// the reference only where glibc's pow / exp are not (about one call in a
// thousand for the non-integer exponents).
//
// A CTA of 256 threads over a tile of 16 x 32 zones (two rows of zones per
// thread). The tile's primitives (with a two-zone halo) are staged in shared
// memory; a first phase computes the per-zone quantities every neighbouring
// update needs (slopes, p / Sigma, sound speed, strain) and the scale
// heights' face geometry, a second the zone updates. The reference's face
// fluxes are not shareable between the two zones of a face (each zone takes
// the sound speed of the neighbour across the face, cbdgam_2d.c:608-611, and
// the viscous flux the neighbour's scale height), so each zone computes its
// four faces, as the reference does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#include "cbdiso_b200.h"
#include "cr_math.cuh"

namespace cbd {
cudaStream_t drop_in_stream();  // capi.cu: the stream set by cbdiso_b200_set_stream
}

namespace gam {

constexpr int NF = 4;
constexpr int NG = 2;
constexpr int TI = 16, TJ = 32;  // CTA tile (rows i, columns j)
constexpr int RPT = 2;            // tile rows per thread: zone rows ty and ty + TI / RPT
constexpr int NT = TI * TJ / RPT; // threads per CTA, a (TJ, TI / RPT) block
constexpr int HI = TI + 2 * NG, HJ = TJ + 2 * NG;
constexpr int STAGE_MIN_BLOCKS = 2;  // resident CTAs per SM the stage kernel is built for

struct Mass {
    double x, y, vx, vy, mass, soft, rate, radius;
    int model;
};

struct Consts {
    int ni, nj;
    double xl, yl, dx, dy;
    double theta, gamma, alpha, cooling, mach_ceiling, vmax, rho_floor, p_floor;
    int constant_softening;
    int buffer_on;
    double buf_sigma, buf_pressure, buf_rate, buf_outer, buf_width;
    double buf_onset_m3;  // pow(buf_outer - buf_width, -3.0), glibc's on the host
    double mach_m2;       // pow(mach_ceiling, -2.0), glibc's on the host
    double inv_dx, inv_dy, gm1, inv_gm1, inv_gamma;  // RN(1 / dx), ..., gamma - 1, RN(1 / (gamma - 1)), RN(1 / gamma)
};

struct Stage {
    Mass m[2];
    double buf_mass, a, dt;
    int massless;  // both masses have zero mass: every scale height is 1
    int write_guards;
    int un_from_primitive;  // u_n = cons(primitive_n) in-kernel (else: a conserved array)
};

// Powers and the exponential are correctly rounded (cr_math.cuh): in a
// near-vacuum zone an ulp in the energy update is amplified by the
// cancellation between total and kinetic energy, so matching glibc's
// correctly rounded results matters here.
using crm::cube_rn;
using crm::exp_rn;
using crm::fourth_rn;
using crm::inv_cube_rn;
using crm::inv_pow15_rn;
using crm::inv_square_rn;
using crm::pow_m13_rn;

__device__ __forceinline__ double lesser(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double greater(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double sign_of(double x) { return copysign(1.0, x); }
__device__ __forceinline__ size_t at(int i, int j, int nj) { return ((size_t)(i + NG) * (nj + 2 * NG) + (j + NG)) * NF; }

// cbdgam_2d.c:27-33: 0.25 |sgn a + sgn b| (sgn a + sgn c) min(|a|, |b|, |c|),
// returned exactly (signed zeros included) with the sign logic done on the
// sign bits: it is m, -m, +0 or -0.
__device__ __forceinline__ double slope(double yl, double y0, double yr, double theta)
{
    const double a = (y0 - yl) * theta;
    const double b = (yr - yl) * 0.5;
    const double c = (yr - y0) * theta;
    const double m = lesser(fabs(a), lesser(fabs(b), fabs(c)));
    const unsigned sa = (unsigned)__double2hiint(a) >> 31;
    const unsigned sb = (unsigned)__double2hiint(b) >> 31;
    const unsigned sc = (unsigned)__double2hiint(c) >> 31;
    if ((sa == sb) & (sa == sc))
        return sa ? -m : m;
    return (sa & sc & (sa ^ sb)) ? -0.0 : 0.0;
}

template <class V>
__device__ __forceinline__ double cs2_of(double gamma, const V &p) { return p[3] / p[0] * gamma; }

// cbdgam_2d.c:238-276
__device__ __forceinline__ void buffer_source(const Consts &k, double buf_mass, double x, double y, double dt,
                                              double *u)
{
    if (!k.buffer_on)
        return;
    const double rc = sqrt(x * x + y * y);
    const double onset = k.buf_outer - k.buf_width;
    if (rc > onset) {
        const double pf = k.buf_sigma * sqrt(buf_mass / rc);
        const double px = pf * (-y / rc), py = pf * (x / rc);
        const double ek = 0.5 * (px * px + py * py) / k.buf_sigma;
        const double target[NF] = {k.buf_sigma, px, py, k.buf_pressure / (k.gamma - 1.0) + ek};
        const double omega = sqrt(buf_mass * k.buf_onset_m3);  // pow(onset, -3.0), from the host
        const double rate = k.buf_rate * omega * (rc - onset) / (k.buf_outer - onset);
#pragma unroll
        for (int q = 0; q < NF; ++q)
            u[q] -= (u[q] - target[q]) * rate * dt;
    }
}

// cbdgam_2d.c:347-362
template <class V>
__device__ __forceinline__ void prim_to_cons(const V &p, double *u, double gamma)
{
    const double rho = p[0], vx = p[1], vy = p[2], pres = p[3];
    u[0] = rho;
    u[1] = vx * rho;
    u[2] = vy * rho;
    u[3] = pres / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy);
}

// cbdgam_2d.c:401-409
template <class V>
__device__ __forceinline__ double max_wavespeed(const V &p, double cs2)
{
    const double cs = sqrt(cs2);
    const double ax = greater(fabs(p[1] - cs), fabs(p[1] + cs));
    const double ay = greater(fabs(p[2] - cs), fabs(p[2] + cs));
    return greater(ax, ay);
}

// ---------------------------------------------------------------------------
// The stage kernel. The reference evaluates every quantity of a neighbour
// inside each zone's update (cbdgam_2d.c:499-682): the x and y slopes of five
// zones, four sound speeds, five scale heights and strain tensors. All of
// these except the scale heights' geometry are per-zone values, and the
// geometry is shared by the two zones of a face, so the kernel computes them
// once per zone (per face) into shared memory in a first phase and the zone
// updates read them in a second. Every value is computed by the same
// operations in the same order as in the reference, so the split changes no
// bit. Divisions by a constant (dx, dy, gamma - 1) or by one value several
// times (the HLLE denominator, Sigma in the primitive recovery) use a
// reciprocal rounded to nearest and a Markstein correction, which returns
// the correctly rounded quotient.
// ---------------------------------------------------------------------------

// a / b rounded to nearest from y = RN(1 / b): the remainder a - q b of
// q = RN(a y) is exact under FMA and one correction rounds to RN(a / b)
__device__ __forceinline__ double div_by(double a, double b, double y)
{
    const double q = a * y;
    return fma(fma(-q, b, a), y, q);
}

constexpr int ZI = TI + 2, ZJ = TJ + 2;  // zones with shared quantities: the tile and a ring of one
// per-zone quantities: x and y slopes, p / Sigma, sound speed, sqrt(p / Sigma), strain xx, xy, yy
enum { Q_GX = 0, Q_GY = 4, Q_T = 8, Q_CS = 9, Q_SQ = 10, Q_SXX = 11, Q_SXY = 12, Q_SYY = 13, NZQ = 14 };

struct StageSmem {
    double prim[NF][HI][HJ];
    double z[NZQ][ZI][ZJ];
    double fx[TI + 1][TJ];  // sqrt(sum_m M_m r^-3) at the x-faces (x_l of zone i0 + a, y_c of zone j0 + b)
    double fy[TI][TJ + 1];  // the same at the y-faces (x_c of zone i0 + a, y_l of zone j0 + b)
    double warp_max[NT / 32];
};

// sqrt(w2) of the scale height (cbdgam_2d.c:75-106) at (x, y)
__device__ __forceinline__ double root_w2(const Mass *m, double x, double y)
{
    double w2 = 0.0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (m[k].mass > 0.0) {
            const double dx = x - m[k].x, dy = y - m[k].y;
            const double r = sqrt(dx * dx + dy * dy + 1e-12);
            w2 += m[k].mass * inv_cube_rn(r);
        }
    }
    return sqrt(w2);
}

// cbdgam_2d.c:347-362 with the constant divisor gamma - 1
template <class V>
__device__ __forceinline__ void p2c_fast(const Consts &k, const V &p, double *u)
{
    const double rho = p[0], vx = p[1], vy = p[2], pres = p[3];
    u[0] = rho;
    u[1] = vx * rho;
    u[2] = vy * rho;
    u[3] = div_by(pres, k.gm1, k.inv_gm1) + 0.5 * rho * (vx * vx + vy * vy);
}

// cbdgam_2d.c:411-434 given the neighbour's sound speed cs = sqrt(cs2)
template <int DIR>
__device__ __forceinline__ void hlle_fast(const Consts &k, const double *pl, const double *pr, double cs, double *f)
{
    double ul[NF], ur[NF];
    p2c_fast(k, pl, ul);
    p2c_fast(k, pr, ur);
    const double vl = DIR == 0 ? pl[1] : pl[2], vr = DIR == 0 ? pr[1] : pr[2];
    const double fl[NF] = {vl * ul[0], vl * ul[1] + pl[3] * (double)(DIR == 0), vl * ul[2] + pl[3] * (double)(DIR == 1),
                           vl * (ul[3] + pl[3])};
    const double fr[NF] = {vr * ur[0], vr * ur[1] + pr[3] * (double)(DIR == 0), vr * ur[2] + pr[3] * (double)(DIR == 1),
                           vr * (ur[3] + pr[3])};
    const double am = lesser(0.0, lesser(vl - cs, vr - cs));
    const double ap = greater(0.0, greater(vl + cs, vr + cs));
    const double den = ap - am, y = __drcp_rn(den);
#pragma unroll
    for (int q = 0; q < NF; ++q)
        f[q] = div_by(fl[q] * ap - fr[q] * am - (ul[q] - ur[q]) * ap * am, den, y);
}

// cbdgam_2d.c:108-203: gravity, sink and their work on the gas for one mass,
// given T = p / Sigma, the disk height h and gamma - 1 with its reciprocal
template <class V>
__device__ __forceinline__ void mass_source(const Mass &m, double x, double y, double dt, const V &p, double T,
                                            double h, int constant_softening, double gm1, double inv_gm1, double *du,
                                            const double *g_in = nullptr, double *g_out = nullptr)
{
    const double sigma = p[0];
    const double eps = div_by(T, gm1, inv_gm1);
    const double dx = x - m.x, dy = y - m.y;
    const double r2 = dx * dx + dy * dy;
    const double dr = sqrt(r2);
    const double rs = m.radius;
    double soft;
    if (constant_softening) {
        soft = m.soft;
    } else if (dr > rs) {
        soft = 0.5 * h;
    } else {
        const double q = dr / rs;
        const double w = (1.0 - q * q) * (1.0 - q * q);  // pow(., 2.0) is the correctly rounded square
        soft = w * rs + (1.0 - w) * 0.5 * h;
    }
    const double rate = (dr < 4.0 * rs) ? m.rate * exp_rn(-fourth_rn(dr / rs)) : 0.0;
    // the gravity factor: from the face cache (constant softening), or computed
    const double g = g_in ? *g_in : inv_pow15_rn(r2 + soft * soft);
    if (g_out)
        *g_out = g;
    const double fnum = sigma * m.mass * g;
    const double fx = -fnum * dx, fy = -fnum * dy;
    const double mdot = sigma * rate * -1.0;
    const double vx = p[1], vy = p[2];
    if (m.model == 1) {
        du[0] = dt * mdot;
        du[1] = dt * mdot * p[1] + dt * fx;
        du[2] = dt * mdot * p[2] + dt * fy;
        du[3] = dt * (mdot * eps + 0.5 * mdot * (vx * vx + vy * vy)) + dt * (fx * vx + fy * vy);
    } else if (m.model == 2) {
        const double den = dr + 1e-12, yd = __drcp_rn(den);
        const double ex = div_by(dx, den, yd), ey = div_by(dy, den, yd);
        const double dvr = (vx - m.vx) * ex + (vy - m.vy) * ey;
        const double wx = dvr * ex + m.vx, wy = dvr * ey + m.vy;
        du[0] = dt * mdot;
        du[1] = dt * mdot * wx + dt * fx;
        du[2] = dt * mdot * wy + dt * fy;
        du[3] = dt * (mdot * eps + 0.5 * mdot * (wx * wx + wy * wy)) + dt * (fx * vx + fy * vy);
    } else if (m.model == 3) {
        du[0] = dt * mdot;
        du[1] = dt * fx;
        du[2] = dt * fy;
        du[3] = dt * (fx * vx + fy * vy);
    } else {
        du[0] = du[1] = du[2] = du[3] = 0.0;
    }
}

// cbdgam_2d.c:298-317 with T = p / Sigma given
template <class V>
__device__ __forceinline__ void cooling_fast(const Consts &k, double dt, const V &p, double T, double *u)
{
    const double sigma = p[0];
    const double eps = div_by(T, k.gm1, k.inv_gm1);
    // without cooling the power's argument is exactly 1 and so is the power
    // (for finite Sigma^-2 eps^3, which the floors keep)
    double cooled = k.cooling == 0.0
                        ? eps
                        : eps * pow_m13_rn(1.0 + 3.0 * k.cooling * inv_square_rn(sigma) * cube_rn(eps) * dt);
    const double ek = 0.5 * (p[1] * p[1] + p[2] * p[2]);
    cooled = greater(cooled, div_by(div_by(2.0 * ek, k.gamma, k.inv_gamma), k.gm1, k.inv_gm1) * k.mach_m2);
    u[3] += sigma * (cooled - eps);
}

// cbdgam_2d.c:319-345 with one reciprocal of Sigma
__device__ __forceinline__ void c2p_fast(const Consts &k, const double *u, double *p)
{
    const double y = __drcp_rn(u[0]);
    double pres = greater(k.p_floor, (u[3] - div_by(0.5 * (u[1] * u[1] + u[2] * u[2]), u[0], y)) * k.gm1);
    double vx = sign_of(u[1]) * lesser(fabs(div_by(u[1], u[0], y)), k.vmax);
    double vy = sign_of(u[2]) * lesser(fabs(div_by(u[2], u[0], y)), k.vmax);
    double rho = u[0];
    if (u[0] < k.rho_floor) {
        rho = k.rho_floor;
        vx = 0.0;
        vy = 0.0;
        pres = k.p_floor;
    }
    p[0] = rho;
    p[1] = vx;
    p[2] = vy;
    p[3] = pres;
}

// a maximum that keeps a NaN operand, so that a NaN wavespeed reaches the host
__device__ __forceinline__ double max_nan(double a, double b) { return (a > b || a != a) ? a : b; }

// ---------------------------------------------------------------------------
// Face cache. The scale heights' geometry sqrt(sum_m M_m r^-3) at every x- and
// y-face and zone centre, and (with constant softening) the gravity factors
// (r^2 + s^2)^-1.5 of both masses at every zone, depend only on the mesh and
// the point masses. RK2's second stage runs at t0 + dt, which is the next
// step's start time in all but about 1 step in 5000 (cbdgam_2d.py's time
// update), so the host makes that stage a writer when its masses equal the
// end-of-step masses (it stores the values with a key of their inputs) and
// the next step's first stage a reader (it loads them, after a fill kernel
// that recomputes them when the key does not match). The same bits either
// way; each role is its own kernel.
//
// Layout (doubles): a 32-double header holding the key, then the zones'
// (sqrt(w2), g_1) pairs ni x nj, the zones' g_2 ni x nj, the x-faces
// (ni + 1) x nj ([i][j]: between rows i - 1 and i) and the y-faces
// ni x (nj + 1) ([i][j]: between columns j - 1 and j).
// ---------------------------------------------------------------------------

enum { ROLE_NONE = 0, ROLE_WRITER = 1, ROLE_READER = 2 };
constexpr int CACHE_HEADER = 32;
constexpr int CACHE_KEY = 16;

struct CacheView {
    double *zp, *zg2, *xf, *yf;
};

__host__ __device__ inline size_t cache_doubles(int ni, int nj)
{
    return CACHE_HEADER + 3 * (size_t)ni * nj + (size_t)(ni + 1) * nj + (size_t)ni * (nj + 1);
}

__device__ __forceinline__ CacheView cache_view(const Consts &k, double *fc)
{
    CacheView v;
    v.zp = fc + CACHE_HEADER;
    v.zg2 = v.zp + 2 * (size_t)k.ni * k.nj;
    v.xf = v.zg2 + (size_t)k.ni * k.nj;
    v.yf = v.xf + (size_t)(k.ni + 1) * k.nj;
    return v;
}

// the key: a format tag, then every input of the cached values
__device__ __forceinline__ double cache_key_value(const Consts &k, const Mass *m, int v)
{
    switch (v) {
    case 0: return 20260102.5;
    case 1: return (double)k.ni;
    case 2: return (double)k.nj;
    case 3: return k.xl;
    case 4: return k.yl;
    case 5: return k.dx;
    case 6: return k.dy;
    case 7: return (double)k.constant_softening;
    default: {
        const Mass &q = m[(v - 8) >> 2];
        switch ((v - 8) & 3) {
        case 0: return q.x;
        case 1: return q.y;
        case 2: return q.mass;
        default: return q.soft;
        }
    }
    }
}

__device__ bool cache_key_matches(const Consts &k, const Mass *m, const double *fc)
{
    for (int v = 0; v < CACHE_KEY; ++v)
        if (__double_as_longlong(fc[v]) != __double_as_longlong(cache_key_value(k, m, v)))
            return false;
    return true;
}

// Phase 1: the per-zone quantities of zone (i0 - 1 + a, j0 - 1 + b) and the
// face geometry of the tile.
template <int ROLE>
__device__ __forceinline__ void stage_phase1(const Consts &k, const Stage &st, StageSmem &sm, int i0, int j0, int tid,
                                             const CacheView &cv)
{
    // one pool of work items for the whole CTA: the zones of the tile and its
    // ring, then (with viscosity) the x-faces and the y-faces, so that the
    // last pass over the pool is the only partly idle one
    constexpr int NZI = ZI * ZJ, NFX = (TI + 1) * TJ, NFY = TI * (TJ + 1);
    const bool faces = k.alpha > 0.0 && !st.massless;
    const int total = NZI + (faces ? NFX + NFY : 0);
    const double theta = k.theta;
    for (int s = tid; s < total; s += NT) {
        if (s >= NZI + NFX) {
            const int f = s - NZI - NFX, a = f / (TJ + 1), b = f % (TJ + 1);
            const int i = i0 + a, j = j0 + b;
            const bool in = i < k.ni && j <= k.nj;
            double w = 0.0;
            if (ROLE == ROLE_READER) {
                if (in)
                    w = cv.yf[(size_t)i * (k.nj + 1) + j];
            } else {
                w = root_w2(st.m, k.xl + (i + 0.5) * k.dx, k.yl + (j + 0.0) * k.dy);
                // a tile's last face column is stored by the next tile, except the last
                if (ROLE == ROLE_WRITER && in && (b < TJ || j == k.nj))
                    cv.yf[(size_t)i * (k.nj + 1) + j] = w;
            }
            sm.fy[a][b] = w;
            continue;
        }
        if (s >= NZI) {
            const int f = s - NZI, a = f / TJ, b = f % TJ;
            const int i = i0 + a, j = j0 + b;
            const bool in = i <= k.ni && j < k.nj;
            double w = 0.0;
            if (ROLE == ROLE_READER) {
                if (in)
                    w = cv.xf[(size_t)i * k.nj + j];
            } else {
                w = root_w2(st.m, k.xl + (i + 0.0) * k.dx, k.yl + (j + 0.5) * k.dy);
                // a tile's last face row is stored by the next tile, except the last
                if (ROLE == ROLE_WRITER && in && (a < TI || i == k.ni))
                    cv.xf[(size_t)i * k.nj + j] = w;
            }
            sm.fx[a][b] = w;
            continue;
        }
        const int a = s / ZJ, b = s % ZJ;
        if (i0 - 1 + a > k.ni || j0 - 1 + b > k.nj)
            continue;  // beyond the guard zones of the last tile: never read
        double gx[NF], gy[NF];
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            gx[q] = slope(sm.prim[q][a][b + 1], sm.prim[q][a + 1][b + 1], sm.prim[q][a + 2][b + 1], theta);
            gy[q] = slope(sm.prim[q][a + 1][b], sm.prim[q][a + 1][b + 1], sm.prim[q][a + 1][b + 2], theta);
            sm.z[Q_GX + q][a][b] = gx[q];
            sm.z[Q_GY + q][a][b] = gy[q];
        }
        const double T = sm.prim[3][a + 1][b + 1] / sm.prim[0][a + 1][b + 1];
        sm.z[Q_T][a][b] = T;
        sm.z[Q_CS][a][b] = sqrt(T * k.gamma);  // sqrt(cs2), cs2 = p / Sigma * gamma (cbdgam_2d.c:231-236)
        sm.z[Q_SQ][a][b] = sqrt(T);
        // strain (cbdgam_2d.c:278-294): (4/3 gx_vx) / dx - (2/3 gy_vy) / dy, ...
        sm.z[Q_SXX][a][b] = div_by(4.0 / 3.0 * gx[1], k.dx, k.inv_dx) - div_by(2.0 / 3.0 * gy[2], k.dy, k.inv_dy);
        sm.z[Q_SXY][a][b] = div_by(gx[2], k.dx, k.inv_dx) + div_by(gy[1], k.dy, k.inv_dy);
        sm.z[Q_SYY][a][b] = div_by(-2.0 / 3.0 * gx[1], k.dx, k.inv_dx) + div_by(4.0 / 3.0 * gy[2], k.dy, k.inv_dy);
    }
}

// Phase 2: zone (i, j) = (i0 + ty, j0 + tx); returns its new primitives.
template <int ROLE>
__device__ __forceinline__ void stage_phase2(const Consts &k, const Stage &st, const StageSmem &sm, int ty, int tx,
                                             const double *un, double *out, const CacheView &cv)
{
    const int i = blockIdx.y * TI + ty, j = blockIdx.x * TJ + tx;
    const double dt = st.dt;
    const double xc = k.xl + (i + 0.5) * k.dx, yc = k.yl + (j + 0.5) * k.dy;
    // primitives and per-zone quantities of the zone and its four neighbours
    auto P = [&](int di, int dj, int q) { return sm.prim[q][ty + NG + di][tx + NG + dj]; };
    auto Z = [&](int di, int dj, int q) { return sm.z[q][ty + 1 + di][tx + 1 + dj]; };
    double c[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q)
        c[q] = P(0, 0, q);

    // p +- g / 2 and f - S / 2 below are single FMAs: halving a normal number
    // is exact, so the fused operation rounds as the reference's multiply
    // then add
    double fw[NF], fe[NF], fs[NF], fn[NF];
    {
        double lo[NF], hi[NF];
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            lo[q] = fma(0.5, Z(-1, 0, Q_GX + q), P(-1, 0, q));
            hi[q] = fma(-0.5, Z(0, 0, Q_GX + q), c[q]);
        }
        hlle_fast<0>(k, lo, hi, Z(-1, 0, Q_CS), fw);
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            lo[q] = fma(0.5, Z(0, 0, Q_GX + q), c[q]);
            hi[q] = fma(-0.5, Z(1, 0, Q_GX + q), P(1, 0, q));
        }
        hlle_fast<0>(k, lo, hi, Z(1, 0, Q_CS), fe);
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            lo[q] = fma(0.5, Z(0, -1, Q_GY + q), P(0, -1, q));
            hi[q] = fma(-0.5, Z(0, 0, Q_GY + q), c[q]);
        }
        hlle_fast<1>(k, lo, hi, Z(0, -1, Q_CS), fs);
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            lo[q] = fma(0.5, Z(0, 0, Q_GY + q), c[q]);
            hi[q] = fma(-0.5, Z(0, 1, Q_GY + q), P(0, 1, q));
        }
        hlle_fast<1>(k, lo, hi, Z(0, 1, Q_CS), fn);
    }

    const size_t zc = (size_t)i * k.nj + j;
    double wc = 1.0, gz[2] = {0.0, 0.0};
    if (ROLE == ROLE_READER) {
        const double2 v = *reinterpret_cast<const double2 *>(cv.zp + 2 * zc);
        wc = v.x;
        gz[0] = v.y;
        gz[1] = cv.zg2[zc];
    } else if (!st.massless) {
        wc = root_w2(st.m, xc, yc);
    }
    const double hc = st.massless ? 1.0 : Z(0, 0, Q_SQ) / wc;

    if (k.alpha > 0.0) {
        const double hw = st.massless ? 1.0 : Z(-1, 0, Q_SQ) / sm.fx[ty][tx];
        const double he = st.massless ? 1.0 : Z(1, 0, Q_SQ) / sm.fx[ty + 1][tx];
        const double hs = st.massless ? 1.0 : Z(0, -1, Q_SQ) / sm.fy[ty][tx];
        const double hn = st.massless ? 1.0 : Z(0, 1, Q_SQ) / sm.fy[ty][tx + 1];
        const double nuc = k.alpha * hc * Z(0, 0, Q_CS);
        const double nuw = k.alpha * hw * Z(-1, 0, Q_CS), nue = k.alpha * he * Z(1, 0, Q_CS);
        const double nus = k.alpha * hs * Z(0, -1, Q_CS), nun = k.alpha * hn * Z(0, 1, Q_CS);
        const double w0 = P(-1, 0, 0), e0 = P(1, 0, 0), s0 = P(0, -1, 0), n0 = P(0, 1, 0);
        // strain tensors (xx, xy, yx = xy, yy) of the zone and its neighbours
        const double tc0 = Z(0, 0, Q_SXX), tc1 = Z(0, 0, Q_SXY), tc3 = Z(0, 0, Q_SYY);
        const double tw0 = Z(-1, 0, Q_SXX), tw1 = Z(-1, 0, Q_SXY);
        const double te0 = Z(1, 0, Q_SXX), te1 = Z(1, 0, Q_SXY);
        const double ts2 = Z(0, -1, Q_SXY), ts3 = Z(0, -1, Q_SYY);
        const double tn2 = Z(0, 1, Q_SXY), tn3 = Z(0, 1, Q_SYY);
        const double tc2 = tc1;

        fw[1] = fma(-0.5, nuw * w0 * tw0 + nuc * c[0] * tc0, fw[1]);
        fw[2] = fma(-0.5, nuw * w0 * tw1 + nuc * c[0] * tc1, fw[2]);
        fe[1] = fma(-0.5, nuc * c[0] * tc0 + nue * e0 * te0, fe[1]);
        fe[2] = fma(-0.5, nuc * c[0] * tc1 + nue * e0 * te1, fe[2]);
        fs[1] = fma(-0.5, nus * s0 * ts2 + nuc * c[0] * tc2, fs[1]);
        fs[2] = fma(-0.5, nus * s0 * ts3 + nuc * c[0] * tc3, fs[2]);
        fn[1] = fma(-0.5, nuc * c[0] * tc2 + nun * n0 * tn2, fn[1]);
        fn[2] = fma(-0.5, nuc * c[0] * tc3 + nun * n0 * tn3, fn[2]);

        fw[3] = fma(-0.5, nuw * w0 * tw0 * P(-1, 0, 1) + nuc * c[0] * tc0 * c[1], fw[3]);
        fe[3] = fma(-0.5, nuc * c[0] * tc0 * c[1] + nue * e0 * te0 * P(1, 0, 1), fe[3]);
        fw[3] = fma(-0.5, nuw * w0 * tw1 * P(-1, 0, 2) + nuc * c[0] * tc1 * c[2], fw[3]);
        fe[3] = fma(-0.5, nuc * c[0] * tc1 * c[2] + nue * e0 * te1 * P(1, 0, 2), fe[3]);
        fs[3] = fma(-0.5, nus * s0 * ts2 * P(0, -1, 1) + nuc * c[0] * tc2 * c[1], fs[3]);
        fn[3] = fma(-0.5, nuc * c[0] * tc2 * c[1] + nun * n0 * tn2 * P(0, 1, 1), fn[3]);
        fs[3] = fma(-0.5, nus * s0 * ts3 * P(0, -1, 2) + nuc * c[0] * tc3 * c[2], fs[3]);
        fn[3] = fma(-0.5, nuc * c[0] * tc3 * c[2] + nun * n0 * tn3 * P(0, 1, 2), fn[3]);
    }

    const double T = Z(0, 0, Q_T);
    double u[NF];
    p2c_fast(k, c, u);
    buffer_source(k, st.buf_mass, xc, yc, dt, u);
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        double du[NF];
        const bool cached_g = ROLE == ROLE_READER && k.constant_softening;
        mass_source(st.m[m], xc, yc, dt, c, T, hc, k.constant_softening, k.gm1, k.inv_gm1, du,
                    cached_g ? &gz[m] : nullptr, ROLE == ROLE_WRITER ? &gz[m] : nullptr);
#pragma unroll
        for (int q = 0; q < NF; ++q)
            u[q] += du[q];
    }
    if (ROLE == ROLE_WRITER) {
        *reinterpret_cast<double2 *>(cv.zp + 2 * zc) = make_double2(wc, gz[0]);
        cv.zg2[zc] = gz[1];
    }
    cooling_fast(k, dt, c, T, u);
#pragma unroll
    for (int q = 0; q < NF; ++q) {
        u[q] -= (div_by(fe[q] - fw[q], k.dx, k.inv_dx) + div_by(fn[q] - fs[q], k.dy, k.inv_dy)) * dt;
        u[q] = (1.0 - st.a) * u[q] + st.a * un[q];
    }
    c2p_fast(k, u, out);
}

// One RK stage. primitive_n supplies u_n (cons of it, rebuilt in the kernel)
// or un_all does (the reference's conserved_rk array). With ws_max set, the
// largest wavespeed of the written zones is max-ed into it (non-negative
// doubles order as their bit patterns do).
// ROLE (ROLE_*) is what the stage does with the face cache `fc`.
template <int ROLE>
__global__ void __launch_bounds__(NT, STAGE_MIN_BLOCKS) stage_kernel(Consts k, Stage st,
                                                                          const double *__restrict__ prd,
                                                                          const double *pn,
                                                                          const double *__restrict__ un_all,
                                                                          double *pwr, unsigned long long *ws_max,
                                                                          double *fc)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StageSmem &sm = *reinterpret_cast<StageSmem *>(smem_raw);
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const int ni = k.ni, nj = k.nj;
    const int tid = threadIdx.y * TJ + threadIdx.x;
    for (int s = tid; s < HI * HJ; s += NT) {
        const int ii = i0 - NG + s / HJ, jj = j0 - NG + s % HJ;
        if (ii <= ni + 1 && jj <= nj + 1) {
            const double *src = prd + at(ii, jj, nj);
#pragma unroll
            for (int q = 0; q < NF; ++q)
                sm.prim[q][s / HJ][s % HJ] = src[q];
        }
    }
    __syncthreads();
    CacheView cv = {};
    if (ROLE != ROLE_NONE) {
        cv = cache_view(k, fc);
        if (ROLE == ROLE_WRITER && blockIdx.x == 0 && blockIdx.y == 0 && tid < CACHE_KEY)
            fc[tid] = cache_key_value(k, st.m, tid);
    }
    stage_phase1<ROLE>(k, st, sm, i0, j0, tid, cv);
    __syncthreads();
    double ws = 0.0;
#pragma unroll 1
    for (int h = 0; h < RPT; ++h) {
        const int ty = threadIdx.y + h * (TI / RPT);
        const int i = i0 + ty, j = j0 + threadIdx.x;
        if (i >= ni || j >= nj)
            continue;
        // u_n enters as (1 - a) u + a u_n even when a = 0, as in the reference
        double un[NF];
        if (st.un_from_primitive) {
            double pn_z[NF];
#pragma unroll
            for (int q = 0; q < NF; ++q)
                pn_z[q] = pn[at(i, j, nj) + q];
            p2c_fast(k, pn_z, un);
        } else {
#pragma unroll
            for (int q = 0; q < NF; ++q)
                un[q] = un_all[at(i, j, nj) + q];
        }
        double out[NF];
        stage_phase2<ROLE>(k, st, sm, ty, threadIdx.x, un, out, cv);
        // the zone and, on the edges, its zero-gradient guard images
        const int ilo = (st.write_guards && i == 0) ? -NG : i, ihi = (st.write_guards && i == ni - 1) ? ni + 1 : i;
        const int jlo = (st.write_guards && j == 0) ? -NG : j, jhi = (st.write_guards && j == nj - 1) ? nj + 1 : j;
        for (int ii = ilo; ii <= ihi; ++ii)
            for (int jj = jlo; jj <= jhi; ++jj) {
                double *dst = pwr + at(ii, jj, nj);
#pragma unroll
                for (int q = 0; q < NF; ++q)
                    dst[q] = out[q];
            }
        if (ws_max)
            ws = max_nan(ws, max_wavespeed(out, cs2_of(k.gamma, out)));
    }
    if (ws_max) {  // uniform over the block
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            ws = max_nan(ws, __shfl_xor_sync(0xffffffffu, ws, o));
        if ((tid & 31) == 0)
            sm.warp_max[tid >> 5] = ws;
        __syncthreads();
        if (tid == 0) {
            double m = sm.warp_max[0];
            for (int w = 1; w < NT / 32; ++w)
                m = max_nan(m, sm.warp_max[w]);
            atomicMax(ws_max, (unsigned long long)__double_as_longlong(m));
        }
    }
}

// Makes the face cache valid for a reader stage: when the key does not match
// the stage's masses, marks it invalid (no later key check passes on what
// follows) and computes every value for those masses with the stage kernel's
// own expressions. CTAs take rows i = blockIdx.x, blockIdx.x + gridDim.x, ...
__global__ void __launch_bounds__(128) cache_fill_kernel(Consts k, Stage st, double *fc)
{
    __shared__ int fill;
    if (threadIdx.x == 0) {
        fill = cache_key_matches(k, st.m, fc) ? 0 : 1;
        if (fill)
            fc[0] = 0.0;
    }
    __syncthreads();
    if (!fill)
        return;
    const CacheView cv = cache_view(k, fc);
    const int ni = k.ni, nj = k.nj;
    for (int i = blockIdx.x; i <= ni; i += gridDim.x) {
        for (int j = threadIdx.x; j <= nj; j += blockDim.x) {
            if (j < nj)
                cv.xf[(size_t)i * nj + j] = root_w2(st.m, k.xl + (i + 0.0) * k.dx, k.yl + (j + 0.5) * k.dy);
            if (i < ni)
                cv.yf[(size_t)i * (nj + 1) + j] = root_w2(st.m, k.xl + (i + 0.5) * k.dx, k.yl + (j + 0.0) * k.dy);
            if (i < ni && j < nj) {
                const double xc = k.xl + (i + 0.5) * k.dx, yc = k.yl + (j + 0.5) * k.dy;
                double g[2];
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const double dx = xc - st.m[p].x, dy = yc - st.m[p].y;
                    const double r2 = dx * dx + dy * dy;
                    g[p] = inv_pow15_rn(r2 + st.m[p].soft * st.m[p].soft);
                }
                const size_t z = (size_t)i * nj + j;
                *reinterpret_cast<double2 *>(cv.zp + 2 * z) = make_double2(root_w2(st.m, xc, yc), g[0]);
                cv.zg2[z] = g[1];
            }
        }
    }
}

__global__ void p2c_kernel(int ni, int nj, double gamma, const double *prim, double *cons)
{
    const long n = (long)ni * nj;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < n; z += (long)gridDim.x * blockDim.x) {
        const int i = (int)(z / nj), j = (int)(z % nj);
        prim_to_cons(prim + at(i, j, nj), cons + at(i, j, nj), gamma);
    }
}

__global__ void wavespeed_kernel(int ni, int nj, double gamma, const double *prim, double *ws)
{
    const long n = (long)ni * nj;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < n; z += (long)gridDim.x * blockDim.x) {
        const int i = (int)(z / nj), j = (int)(z % nj);
        const double *p = prim + at(i, j, nj);
        ws[(size_t)(i + NG) * (nj + 2 * NG) + (j + NG)] = max_wavespeed(p, cs2_of(gamma, p));
    }
}

__global__ void source_kernel(int ni, int nj, double xl, double yl, double dx, double dy, Mass m1, Mass m2,
                              int which, int constant_softening, double gm1, double inv_gm1, const double *prim,
                              double *rate)
{
    const Mass ms[2] = {m1, m2};
    const bool massless = m1.mass == 0.0 && m2.mass == 0.0;
    const long n = (long)ni * nj;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < n; z += (long)gridDim.x * blockDim.x) {
        const int i = (int)(z / nj), j = (int)(z % nj);
        const double xc = xl + (i + 0.5) * dx, yc = yl + (j + 0.5) * dy;
        const double *p = prim + at(i, j, nj);
        const double T = p[3] / p[0];
        const double h = massless ? 1.0 : sqrt(T) / root_w2(ms, xc, yc);  // cbdgam_2d.c:75-106
        mass_source(ms[which - 1], xc, yc, 1.0, p, T, h, constant_softening, gm1, inv_gm1, rate + at(i, j, nj));
    }
}

// zero-gradient guard images of a state (the reference's outflow set_bc)
__global__ void guards_kernel(int ni, int nj, double *a)
{
    const long wi = ni + 2 * NG, wj = nj + 2 * NG;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < wi * wj; z += (long)gridDim.x * blockDim.x) {
        const int ii = (int)(z / wj) - NG, jj = (int)(z % wj) - NG;
        if (ii >= 0 && ii < ni && jj >= 0 && jj < nj)
            continue;
        const int ci = ii < 0 ? 0 : (ii >= ni ? ni - 1 : ii);
        const int cj = jj < 0 ? 0 : (jj >= nj ? nj - 1 : jj);
#pragma unroll
        for (int q = 0; q < NF; ++q)
            a[at(ii, jj, nj) + q] = a[at(ci, cj, nj) + q];
    }
}

// ---------------------------------------------------------------------------
// reductions: the CFL wavespeed maximum and the diagnostic sums
// ---------------------------------------------------------------------------

constexpr int RED_THREADS = 256;
constexpr int MAX_DIAG = 4;
constexpr int RED_VALUES = 1 + 2 * MAX_DIAG;

struct Diag {
    int quantity, which_mass, gravity, accretion, has_cut;
    double r0, r1;
};

struct RedArgs {
    Consts k;
    Mass m[2];
    Diag d[MAX_DIAG];
    int nd;
};

// a mass's source rates (dt = 1) for a diagnostic: the accretion rates
// (masses zero) when its accretion flag is set, else the gravity rates
// (sink rates zero), as the reference's reductions pass mass * gravity and
// sink_rate * accretion (cbdgam_2d.py:104-139, 346-349, 397-402)
__device__ __forceinline__ void diag_rates(const RedArgs &r, const Diag &d, int which, double xc, double yc,
                                           const double *p, double *rate)
{
    Mass ms[2] = {r.m[0], r.m[1]};
    const double gravity = d.accretion ? 0.0 : 1.0, accretion = d.accretion ? 1.0 : 0.0;
    for (int k = 0; k < 2; ++k) {
        ms[k].mass = ms[k].mass * gravity;
        ms[k].rate = ms[k].rate * accretion;
    }
    const double T = p[3] / p[0];
    const bool massless = ms[0].mass == 0.0 && ms[1].mass == 0.0;
    const double h = massless ? 1.0 : sqrt(T) / root_w2(ms, xc, yc);  // cbdgam_2d.c:75-106
    mass_source(ms[which - 1], xc, yc, 1.0, p, T, h, r.k.constant_softening, r.k.gm1, r.k.inv_gm1, rate);
}

__device__ __forceinline__ void diag_value(const RedArgs &r, const Diag &d, double x, double y, const double *p,
                                           double *re, double *im)
{
    const double rr = sqrt(x * x + y * y);
    const double cut = d.has_cut ? (double)((d.r0 < rr) * (rr < d.r1)) : 1.0;
    *im = 0.0;
    if (d.quantity == CBD_Q_SIGMA_M1) {
        const double s = p[0] * cut;
        *re = s * (x / rr);
        *im = s * (y / rr);
        return;
    }
    if (d.quantity == CBD_Q_ECCENTRICITY_VECTOR) {
        const double s = p[0] * cut, vx = p[1] * cut, vy = p[2] * cut;
        const double vv = vx * vx + vy * vy, vr = vx * x + vy * y;
        *re = s * ((vv * x - vr * vx) / 1.0 - x / rr);
        *im = s * ((vv * y - vr * vy) / 1.0 - y / rr);
        return;
    }
    double f[3] = {0.0, 0.0, 0.0};
    for (int which = 1; which <= 2; ++which) {
        if (d.which_mass != 3 && d.which_mass != which)
            continue;
        double rate[NF];
        diag_rates(r, d, which, x, y, p, rate);
        for (int q = 0; q < 3; ++q)
            f[q] += rate[q];
    }
    if (d.quantity == CBD_Q_MDOT)
        *re = f[0] * cut;
    else  // torque
        *re = x * (f[2] * cut) - y * (f[1] * cut);
}

// per-block partial sums in a fixed tree order; the wavespeed maximum
__global__ void __launch_bounds__(RED_THREADS) reduce_kernel(RedArgs r, const double *prim, double *partials)
{
    __shared__ double sm[RED_VALUES][RED_THREADS];
    const Consts &k = r.k;
    double v[RED_VALUES];
    for (int q = 0; q < RED_VALUES; ++q)
        v[q] = 0.0;
    const long n = (long)k.ni * k.nj;
    for (long z = blockIdx.x * (long)RED_THREADS + threadIdx.x; z < n; z += (long)gridDim.x * RED_THREADS) {
        const int i = (int)(z / k.nj), j = (int)(z % k.nj);
        const double *p = prim + at(i, j, k.nj);
        v[0] = max_nan(v[0], max_wavespeed(p, cs2_of(k.gamma, p)));
        const double x = k.xl + (i + 0.5) * k.dx, y = k.yl + (j + 0.5) * k.dy;
        for (int d = 0; d < r.nd; ++d) {
            double re, im;
            diag_value(r, r.d[d], x, y, p, &re, &im);
            v[1 + 2 * d] += re;
            v[2 + 2 * d] += im;
        }
    }
    for (int q = 0; q < RED_VALUES; ++q)
        sm[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sm[0][threadIdx.x] = max_nan(sm[0][threadIdx.x], sm[0][threadIdx.x + w]);
            for (int q = 1; q < RED_VALUES; ++q)
                sm[q][threadIdx.x] += sm[q][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x < RED_VALUES)
        partials[(size_t)blockIdx.x * RED_VALUES + threadIdx.x] = sm[threadIdx.x][0];
}

__global__ void finish_kernel(const double *partials, int nblocks, double *result)
{
    const int q = threadIdx.x;
    if (q >= RED_VALUES)
        return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        const double x = partials[(size_t)b * RED_VALUES + q];
        s = q == 0 ? max_nan(s, x) : s + x;
    }
    result[q] = s;
}

// the correctly rounded helpers on device arrays (a test hook)
__global__ void eval_powers_kernel(long n, const double *x, double *out)
{
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const double v = x[t];
        double *o = out + 8 * t;
        o[0] = cube_rn(v);
        o[1] = inv_square_rn(v);
        o[2] = inv_cube_rn(v);
        o[3] = fourth_rn(v);
        o[4] = inv_pow15_rn(v);
        o[5] = pow_m13_rn(1.0 + v);
        o[6] = exp_rn(-v);
        o[7] = 0.0;
    }
}

constexpr int RED_BLOCKS = 592;  // 4 per SM on a B200; fixed so the summation order is too

double g_theta = 1.5;  // the drop-in kernels' PLM theta (the reference fixes 1.5)

bool grid_ok(const cbdgam_grid_t *g)
{
    return g && g->ni > 0 && g->nj > 0 && g->xr > g->xl && g->yr > g->yl && g->gamma_law_index != 1.0;
}

Consts consts_of(const cbdgam_grid_t *g)
{
    Consts k;
    std::memset(&k, 0, sizeof(k));
    k.ni = g->ni;
    k.nj = g->nj;
    k.xl = g->xl;
    k.yl = g->yl;
    k.dx = (g->xr - g->xl) / g->ni;
    k.dy = (g->yr - g->yl) / g->nj;
    k.theta = g->plm_theta;
    k.gamma = g->gamma_law_index;
    k.alpha = g->alpha;
    k.cooling = g->cooling_coefficient;
    k.mach_ceiling = g->mach_ceiling;
    k.vmax = g->velocity_ceiling;
    k.rho_floor = g->density_floor;
    k.p_floor = g->pressure_floor;
    k.constant_softening = g->constant_softening;
    k.buffer_on = g->buffer_is_enabled;
    k.buf_sigma = g->buffer_surface_density;
    k.buf_pressure = g->buffer_surface_pressure;
    k.buf_rate = g->buffer_driving_rate;
    k.buf_outer = g->buffer_outer_radius;
    k.buf_width = g->buffer_onset_width;
    k.buf_onset_m3 = std::pow(g->buffer_outer_radius - g->buffer_onset_width, -3.0);
    k.mach_m2 = std::pow(g->mach_ceiling, -2.0);
    k.inv_dx = 1.0 / k.dx;
    k.inv_dy = 1.0 / k.dy;
    k.gm1 = k.gamma - 1.0;
    k.inv_gm1 = 1.0 / k.gm1;
    k.inv_gamma = 1.0 / k.gamma;
    return k;
}

Mass mass_of(const cbd_mass_t &m)
{
    return Mass{m.x, m.y, m.vx, m.vy, m.mass, m.softening_length, m.sink_rate, m.sink_radius, m.sink_model};
}

Mass mass_args(double x, double y, double vx, double vy, double mass, double soft, double rate, double radius,
               int model)
{
    return Mass{x, y, vx, vy, mass, soft, rate, radius, model};
}

int status_of(cudaError_t e) { return e == cudaSuccess ? CBD_OK : CBD_ERR_CUDA; }

template <int ROLE>
int launch_role(const Consts &k, const Stage &st, const double *prd, const double *pn, const double *un,
                double *pwr, double *ws_max, double *fc, cudaStream_t s)
{
    // the dynamic shared memory limit is a per-device attribute of the kernel
    static bool ready[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return CBD_ERR_CUDA;
    if (!ready[dev]) {
        if (cudaFuncSetAttribute(stage_kernel<ROLE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(StageSmem)) != cudaSuccess)
            return CBD_ERR_CUDA;
        ready[dev] = true;
    }
    if (ROLE == ROLE_READER) {
        const int rows = k.ni + 1 < 148 * 4 ? k.ni + 1 : 148 * 4;
        cache_fill_kernel<<<rows, 128, 0, s>>>(k, st, fc);
    }
    const dim3 grid((k.nj + TJ - 1) / TJ, (k.ni + TI - 1) / TI), block(TJ, TI / RPT);
    stage_kernel<ROLE><<<grid, block, sizeof(StageSmem), s>>>(k, st, prd, pn, un, pwr,
                                                              reinterpret_cast<unsigned long long *>(ws_max), fc);
    return status_of(cudaGetLastError());
}

int launch_stage(const Consts &k, const Stage &st, const double *prd, const double *pn, const double *un,
                 double *pwr, double *ws_max, cudaStream_t s, double *fc = nullptr, int role = ROLE_NONE)
{
    Stage s2 = st;
    s2.massless = st.m[0].mass == 0.0 && st.m[1].mass == 0.0;
    switch (role) {
    case ROLE_WRITER:
        return launch_role<ROLE_WRITER>(k, s2, prd, pn, un, pwr, ws_max, fc, s);
    case ROLE_READER:
        return launch_role<ROLE_READER>(k, s2, prd, pn, un, pwr, ws_max, fc, s);
    default:
        return launch_role<ROLE_NONE>(k, s2, prd, pn, un, pwr, ws_max, nullptr, s);
    }
}

int blocks_for(long n, int t)
{
    const long b = (n + t - 1) / t;
    return (int)(b < 2048 ? (b > 0 ? b : 1) : 2048);
}

}  // namespace gam

using namespace gam;

extern "C" {

int cbdgam_b200_eval_powers(long n, const double *x, double *out, void *stream)
{
    if (n < 0 || (n > 0 && (!x || !out)))
        return CBD_ERR_ARGUMENT;
    if (n == 0)
        return CBD_OK;
    eval_powers_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, x, out);
    return status_of(cudaGetLastError());
}

void cbdgam_b200_disk_primitive(long n, const double *x, const double *y, double softening_length,
                                double initial_sigma, double initial_pressure, double *primitive)
{
    // host code: the C library's sqrt / pow / exp, as Python's math and float
    // power call them, in the setup's operation order
    for (long k = 0; k < n; ++k) {
        const double xk = x[k], yk = y[k];
        const double r = std::sqrt(xk * xk + yk * yk);
        const double rs = std::sqrt(xk * xk + yk * yk + softening_length * softening_length);
        const double rmax = 1e-12 > r ? 1e-12 : r;
        const double phx = -yk / rmax, phy = +xk / rmax;
        const double taper = 0.0001 + 0.9999 * std::exp(-std::pow(1.0 / rs, 30.0));
        double *p = primitive + 4 * k;
        p[0] = initial_sigma * std::pow(rs, -3.0 / 5.0) * taper;
        p[1] = std::sqrt(1.0 / rs) * phx;
        p[2] = std::sqrt(1.0 / rs) * phy;
        p[3] = initial_pressure * std::pow(rs, -3.0 / 2.0) * taper;
    }
}

void cbdgam_b200_abi_sizes(size_t out[2])
{
    out[0] = sizeof(cbdgam_grid_t);
    out[1] = sizeof(cbdgam_stage_t);
}

int cbdgam_b200_set_plm_theta(double theta)
{
    if (!(theta >= 1.0 && theta <= 2.0))
        return CBD_ERR_ARGUMENT;
    g_theta = theta;
    return CBD_OK;
}

int cbdgam_2d_advance_rk(int ni, int nj, double xl, double xr, double yl, double yr, double *conserved_rk,
                         double *primitive_rd, double *primitive_wr, double gamma_law_index,
                         double buffer_surface_density, double buffer_surface_pressure, double buffer_central_mass,
                         double buffer_driving_rate, double buffer_outer_radius, double buffer_onset_width,
                         int buffer_is_enabled, double x1, double y1, double vx1, double vy1, double mass1,
                         double softening_length1, double sink_rate1, double sink_radius1, int sink_model1, double x2,
                         double y2, double vx2, double vy2, double mass2, double softening_length2,
                         double sink_rate2, double sink_radius2, int sink_model2, double alpha, double a, double dt,
                         double velocity_ceiling, double cooling_coefficient, double mach_ceiling,
                         double density_floor, double pressure_floor, int constant_softening)
{
    if (ni <= 0 || nj <= 0 || !conserved_rk || !primitive_rd || !primitive_wr)
        return CBD_ERR_ARGUMENT;
    cbdgam_grid_t g;
    std::memset(&g, 0, sizeof(g));
    g.ni = ni;
    g.nj = nj;
    g.xl = xl;
    g.xr = xr;
    g.yl = yl;
    g.yr = yr;
    g.plm_theta = g_theta;
    g.gamma_law_index = gamma_law_index;
    g.alpha = alpha;
    g.cooling_coefficient = cooling_coefficient;
    g.mach_ceiling = mach_ceiling;
    g.velocity_ceiling = velocity_ceiling;
    g.density_floor = density_floor;
    g.pressure_floor = pressure_floor;
    g.constant_softening = constant_softening;
    g.buffer_is_enabled = buffer_is_enabled;
    g.buffer_surface_density = buffer_surface_density;
    g.buffer_surface_pressure = buffer_surface_pressure;
    g.buffer_driving_rate = buffer_driving_rate;
    g.buffer_outer_radius = buffer_outer_radius;
    g.buffer_onset_width = buffer_onset_width;
    Stage st;
    std::memset(&st, 0, sizeof(st));
    st.m[0] = mass_args(x1, y1, vx1, vy1, mass1, softening_length1, sink_rate1, sink_radius1, sink_model1);
    st.m[1] = mass_args(x2, y2, vx2, vy2, mass2, softening_length2, sink_rate2, sink_radius2, sink_model2);
    st.buf_mass = buffer_central_mass;
    st.a = a;
    st.dt = dt;
    st.write_guards = 0;
    st.un_from_primitive = 0;
    return launch_stage(consts_of(&g), st, primitive_rd, nullptr, conserved_rk, primitive_wr, nullptr,
                        cbd::drop_in_stream());
}

int cbdgam_2d_wavespeed(int ni, int nj, double *primitive, double *wavespeed, double gamma_law_index)
{
    if (ni <= 0 || nj <= 0 || !primitive || !wavespeed)
        return CBD_ERR_ARGUMENT;
    wavespeed_kernel<<<blocks_for((long)ni * nj, 256), 256, 0,
                       cbd::drop_in_stream()>>>(ni, nj, gamma_law_index,
                                                                                   primitive, wavespeed);
    return status_of(cudaGetLastError());
}

int cbdgam_2d_primitive_to_conserved(int ni, int nj, double *primitive, double *conserved, double gamma_law_index)
{
    if (ni <= 0 || nj <= 0 || !primitive || !conserved)
        return CBD_ERR_ARGUMENT;
    p2c_kernel<<<blocks_for((long)ni * nj, 256), 256, 0, cbd::drop_in_stream()>>>(
        ni, nj, gamma_law_index, primitive, conserved);
    return status_of(cudaGetLastError());
}

int cbdgam_2d_point_mass_source_term(int ni, int nj, double xl, double xr, double yl, double yr, double x1,
                                     double y1, double vx1, double vy1, double mass1, double softening_length1,
                                     double sink_rate1, double sink_radius1, int sink_model1, double x2, double y2,
                                     double vx2, double vy2, double mass2, double softening_length2,
                                     double sink_rate2, double sink_radius2, int sink_model2, int which_mass,
                                     double *primitive, double *cons_rate, int constant_softening,
                                     double gamma_law_index)
{
    if (ni <= 0 || nj <= 0 || !primitive || !cons_rate || (which_mass != 1 && which_mass != 2))
        return CBD_ERR_ARGUMENT;
    const Mass m1 = mass_args(x1, y1, vx1, vy1, mass1, softening_length1, sink_rate1, sink_radius1, sink_model1);
    const Mass m2 = mass_args(x2, y2, vx2, vy2, mass2, softening_length2, sink_rate2, sink_radius2, sink_model2);
    source_kernel<<<blocks_for((long)ni * nj, 256), 256, 0,
                    cbd::drop_in_stream()>>>(
        ni, nj, xl, yl, (xr - xl) / ni, (yr - yl) / nj, m1, m2, which_mass, constant_softening, gamma_law_index - 1.0,
        1.0 / (gamma_law_index - 1.0), primitive, cons_rate);
    return status_of(cudaGetLastError());
}

}  // extern "C"

namespace {

int advance_stage(const cbdgam_grid_t *grid, const cbdgam_stage_t *stage, const double *primitive_rd,
                  const double *primitive_n, double *primitive_wr, double *wavespeed_max, double *face_cache,
                  int role, void *stream)
{
    if (!grid_ok(grid) || !stage || !primitive_rd || !primitive_wr || primitive_wr == primitive_rd)
        return CBD_ERR_ARGUMENT;
    if (!primitive_n) {
        if (stage->a != 0.0)
            return CBD_ERR_ARGUMENT;
        primitive_n = primitive_rd;  // the first stage's u_n is the state it reads
    }
    Stage st;
    std::memset(&st, 0, sizeof(st));
    st.m[0] = mass_of(stage->mass[0]);
    st.m[1] = mass_of(stage->mass[1]);
    st.buf_mass = stage->buffer_central_mass;
    st.a = stage->a;
    st.dt = stage->dt;
    st.write_guards = 1;
    st.un_from_primitive = 1;
    return launch_stage(consts_of(grid), st, primitive_rd, primitive_n, nullptr, primitive_wr, wavespeed_max,
                        static_cast<cudaStream_t>(stream), face_cache, role);
}

}  // namespace

extern "C" {

int cbdgam_b200_advance_stage(const cbdgam_grid_t *grid, const cbdgam_stage_t *stage, const double *primitive_rd,
                              const double *primitive_n, double *primitive_wr, double *wavespeed_max, void *stream)
{
    return advance_stage(grid, stage, primitive_rd, primitive_n, primitive_wr, wavespeed_max, nullptr, ROLE_NONE,
                         stream);
}

size_t cbdgam_b200_face_cache_bytes(const cbdgam_grid_t *grid)
{
    if (!grid_ok(grid))
        return 0;
    return cache_doubles(grid->ni, grid->nj) * sizeof(double);
}

int cbdgam_b200_advance_stage_cached(const cbdgam_grid_t *grid, const cbdgam_stage_t *stage,
                                     const double *primitive_rd, const double *primitive_n, double *primitive_wr,
                                     double *wavespeed_max, double *face_cache, int role, void *stream)
{
    // the zone pairs are moved as 16-byte vectors
    if (!face_cache || (reinterpret_cast<uintptr_t>(face_cache) & 15) != 0 || role < ROLE_NONE ||
        role > ROLE_READER)
        return CBD_ERR_ARGUMENT;
    return advance_stage(grid, stage, primitive_rd, primitive_n, primitive_wr, wavespeed_max, face_cache, role,
                         stream);
}

int cbdgam_b200_fill_guards(const cbdgam_grid_t *grid, double *primitive, void *stream)
{
    if (!grid_ok(grid) || !primitive)
        return CBD_ERR_ARGUMENT;
    const long n = (long)(grid->ni + 4) * (grid->nj + 4);
    guards_kernel<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(grid->ni, grid->nj,
                                                                                      primitive);
    return status_of(cudaGetLastError());
}

size_t cbdgam_b200_scratch_bytes(const cbdgam_grid_t *grid)
{
    if (!grid_ok(grid))
        return 0;
    return (size_t)RED_BLOCKS * RED_VALUES * sizeof(double);
}

int cbdgam_b200_reduce(const cbdgam_grid_t *grid, const cbd_mass_t *masses, const cbd_diag_t *diags, int num_diags,
                       const double *primitive, double *scratch, double *result, void *stream)
{
    if (!grid_ok(grid) || !masses || !primitive || !scratch || !result || num_diags < 0 ||
        num_diags > MAX_DIAG || (num_diags > 0 && !diags))
        return CBD_ERR_ARGUMENT;
    RedArgs r;
    std::memset(&r, 0, sizeof(r));
    r.k = consts_of(grid);
    r.m[0] = mass_of(masses[0]);
    r.m[1] = mass_of(masses[1]);
    for (int d = 0; d < num_diags; ++d) {
        const cbd_diag_t &src = diags[d];
        if (src.quantity != CBD_Q_MDOT && src.quantity != CBD_Q_TORQUE && src.quantity != CBD_Q_SIGMA_M1 &&
            src.quantity != CBD_Q_ECCENTRICITY_VECTOR)
            return CBD_ERR_ARGUMENT;
        const bool rates = src.quantity == CBD_Q_MDOT || src.quantity == CBD_Q_TORQUE;
        if (rates && ((!src.accretion && !src.gravity) || src.which_mass < 1 || src.which_mass > 3))
            return CBD_ERR_ARGUMENT;
        r.d[d] = Diag{src.quantity, src.which_mass, src.gravity, src.accretion, src.has_cut, src.r0, src.r1};
    }
    r.nd = num_diags;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    reduce_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(r, primitive, scratch);
    finish_kernel<<<1, 32, 0, s>>>(scratch, RED_BLOCKS, result);
    return status_of(cudaGetLastError());
}

}  // extern "C"
