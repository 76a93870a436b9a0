// Differentiation of the RK stage: a generic per-zone formulation of the
// stencil (the reference's structure, cbdiso_2d.c:447-603) templated on the
// scalar type, used
//   * with T = Dual for the forward-mode tangent kernel, and
//   * with T = double for the branch record that the adjoint replays,
// plus the data layout of the recorded branch words.
//
// Values are computed with the same correctly rounded operations as the EXACT
// stencil, so every branch taken here is the branch the stage kernel took.
#pragma once

#include "cbd_stencil.cuh"

namespace cbd {

// ---------------------------------------------------------------------------
// dual numbers (value, directional derivative)
// ---------------------------------------------------------------------------

struct Dual {
    double v, d;
};

__device__ __forceinline__ Dual dual(double v, double d = 0.0) { return Dual{v, d}; }
__device__ __forceinline__ double val(double x) { return x; }
__device__ __forceinline__ double val(const Dual &x) { return x.v; }

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = div_rn<false>(a.v, b.v);
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {div_rn<false>(a.v, b), a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b)
{
    const double q = div_rn<false>(a, b.v);
    return {q, -q * b.d / b.v};
}

// scalar functions on both types
__device__ __forceinline__ double g_div(double a, double b) { return div_rn<false>(a, b); }
__device__ __forceinline__ Dual g_div(Dual a, Dual b) { return a / b; }
__device__ __forceinline__ double g_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ Dual g_sqrt(Dual x)
{
    const double s = sqrt(x.v);
    return {s, x.d / (2.0 * s)};
}
__device__ __forceinline__ double g_exp(double x) { return exp(x); }
__device__ __forceinline__ Dual g_exp(Dual x)
{
    const double e = exp(x.v);
    return {e, e * x.d};
}
__device__ __forceinline__ double g_pow15(double x) { return inv_pow15<false>(x); }
__device__ __forceinline__ Dual g_pow15(Dual x)
{
    const double p = inv_pow15<false>(x.v);
    return {p, -1.5 * p / x.v * x.d};
}
__device__ __forceinline__ double g_pow4(double q) { return pow4_rn(q); }
__device__ __forceinline__ Dual g_pow4(Dual q) { return {pow4_rn(q.v), 4.0 * q.v * q.v * q.v * q.d}; }
__device__ __forceinline__ double g_abs(double x) { return fabs(x); }
__device__ __forceinline__ Dual g_abs(Dual x) { return x.v < 0.0 || (x.v == 0.0 && signbit(x.v)) ? -x : x; }
template <class T>
__device__ __forceinline__ T g_lesser(const T &a, const T &b) { return val(a) < val(b) ? a : b; }
template <class T>
__device__ __forceinline__ T g_greater(const T &a, const T &b) { return val(a) > val(b) ? a : b; }

// ---------------------------------------------------------------------------
// recorded branch word of a zone (bit fields)
// ---------------------------------------------------------------------------
//   bits  0..11 : limiter selection of the zone's slopes gx[q] (2q) and gy[q] (6 + 2q)
//                 0 = zero (signs disagree), 1 = a = theta (y0 - yl), 2 = b = (yr - yl) / 2,
//                 3 = c = theta (yr - y0)
//   bits 12..15 : HLLE of the zone's east x-face (i + 1/2): am (12-13), ap (14-15);
//                 0 = zero, 1 = the left state's wave, 2 = the right state's
//   bits 16..19 : HLLE of the zone's south y-face (j - 1/2): am (16-17), ap (18-19)
//   bit  20     : density floor applied in the zone's update
//   bits 21, 22 : velocity ceiling applied to vx, vy
constexpr int BW_XFACE = 12;
constexpr int BW_YFACE = 16;
constexpr unsigned BW_FLOOR = 1u << 20;
constexpr unsigned BW_CEIL_X = 1u << 21;
constexpr unsigned BW_CEIL_Y = 1u << 22;

// Selection of the generalised minmod (limited_slope): which candidate the
// value equals, with the reference's tie rules (min2(a, b) = a < b ? a : b).
__device__ __forceinline__ unsigned slope_select(double yl, double y0, double yr, double theta)
{
    const double a = (y0 - yl) * theta;
    const double b = (yr - yl) * 0.5;
    const double c = (yr - y0) * theta;
    const unsigned sa = (unsigned)__double2hiint(a) >> 31;
    const unsigned sb = (unsigned)__double2hiint(b) >> 31;
    const unsigned sc = (unsigned)__double2hiint(c) >> 31;
    if (!((sa == sb) & (sa == sc)))
        return 0;
    const double fa = fabs(a), fb = fabs(b), fc = fabs(c);
    const unsigned inner = fb < fc ? 2u : 3u;
    const double mi = fb < fc ? fb : fc;
    return fa < mi ? 1u : inner;
}

template <class T>
__device__ __forceinline__ T slope_generic(const T &yl, const T &y0, const T &yr, double theta)
{
    switch (slope_select(val(yl), val(y0), val(yr), theta)) {
    case 1:
        return (y0 - yl) * theta;
    case 2:
        return (yr - yl) * 0.5;
    case 3:
        return (yr - y0) * theta;
    default:
        return T{} * 0.0;
    }
}

// ---------------------------------------------------------------------------
// point-mass parameters of a stage, with derivatives for the tangent
// ---------------------------------------------------------------------------

template <class T>
struct MassT {
    T x, y, vx, vy, mass;
    T sink_rate;
    const MassDev *base;  // the non-differentiated fields (softening, sink radius, model)
};

template <class T>
__device__ __forceinline__ T potential_generic(const MassT<T> *m, const T &x, const T &y)
{
    T phi = T{} * 0.0;
    for (int p = 0; p < 2; ++p) {
        if (val(m[p].mass) > 0.0) {
            const T dx = x - m[p].x;
            const T dy = y - m[p].y;
            const T r2 = dx * dx + dy * dy;
            phi = phi - g_div(m[p].mass, g_sqrt(r2 + m[p].base->soft2));
        }
    }
    return phi;
}

template <class T>
__device__ __forceinline__ T cs2_generic(const Consts &k, const MassT<T> *m, const T &x, const T &y)
{
    if (k.eos == 1)
        return T{} * 0.0 + k.cs2;
    if (k.eos == 2)
        return g_div(-potential_generic(m, x, y), T{} * 0.0 + k.mach2);
    return T{} * 0.0 + 1.0;
}

// The HLLE wave choice (cbdiso_2d.c:370-373) from the face velocities and the
// sound speed: am in bits 0-1, ap in bits 2-3 (0 = zero, 1 = the left
// state's wave, 2 = the right state's).
__device__ __forceinline__ unsigned hlle_select(double vl, double vr, double cs)
{
    const double lm = vl - cs, rm = vr - cs, lp = vl + cs, rp = vr + cs;
    const unsigned s_in_m = lm < rm ? 1u : 2u;
    const double in_m = lm < rm ? lm : rm;
    const unsigned s_in_p = lp > rp ? 1u : 2u;
    const double in_p = lp > rp ? lp : rp;
    return (0.0 < in_m ? 0u : s_in_m) | ((0.0 > in_p ? 0u : s_in_p) << 2);
}

// HLLE flux (cbdiso_2d.c:352-380); sel receives am (bits 0-1) and ap (2-3).
template <class T, int DIR>
__device__ __forceinline__ void hlle_generic(const T *pl, const T *pr, const T &cs2, T *f, unsigned *sel)
{
    const T ul[3] = {pl[0], pl[1] * pl[0], pl[2] * pl[0]};
    const T ur[3] = {pr[0], pr[1] * pr[0], pr[2] * pr[0]};
    const T vl = DIR == 0 ? pl[1] : pl[2];
    const T vr = DIR == 0 ? pr[1] : pr[2];
    const T gl = pl[0] * cs2, gr = pr[0] * cs2;
    T fl[3] = {vl * ul[0], vl * ul[1], vl * ul[2]};
    T fr[3] = {vr * ur[0], vr * ur[1], vr * ur[2]};
    fl[1 + DIR] = fl[1 + DIR] + gl;
    fr[1 + DIR] = fr[1 + DIR] + gr;
    const T cs = g_sqrt(cs2);
    const T lm = vl - cs, rm = vr - cs, lp = vl + cs, rp = vr + cs;
    const unsigned s_in_m = val(lm) < val(rm) ? 1u : 2u;
    const T in_m = val(lm) < val(rm) ? lm : rm;
    const unsigned s_am = 0.0 < val(in_m) ? 0u : s_in_m;
    const T am = 0.0 < val(in_m) ? T{} * 0.0 : in_m;
    const unsigned s_in_p = val(lp) > val(rp) ? 1u : 2u;
    const T in_p = val(lp) > val(rp) ? lp : rp;
    const unsigned s_ap = 0.0 > val(in_p) ? 0u : s_in_p;
    const T ap = 0.0 > val(in_p) ? T{} * 0.0 : in_p;
    for (int q = 0; q < 3; ++q)
        f[q] = g_div(fl[q] * ap - fr[q] * am - (ul[q] - ur[q]) * ap * am, ap - am);
    if (sel)
        *sel = s_am | (s_ap << 2);
}

}  // namespace cbd
