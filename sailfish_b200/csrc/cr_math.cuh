// Correctly rounded powers and exponential in double-double arithmetic,
// shared by the isothermal and gamma-law kernels.
//
// The reference's CPU build takes these from glibc, whose results are the
// correctly rounded ones in all but rare cases near a rounding midpoint;
// CUDA's pow / exp may be an ulp off. Each function here computes its power
// as a double-double value (error-free products via FMA, Dekker / Knuth) and
// rounds it once, which gives the correctly rounded result except within
// about 2^-100 of a midpoint. The unguarded forms (pow_m15_rn, pow4_rn) take
// positive normal arguments away from overflow; the others fall back to
// pow / exp outside a safe range.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace crm {

// RN(x^-1.5) for positive normal x. 1/x and then its square root are carried
// as double-double pairs (error-free products via FMA, one Newton correction
// of the square root), and their product is rounded once.
__device__ __forceinline__ double pow_m15_rn(double x)
{
    const double u = __drcp_rn(x);
    const double u_lo = u * fma(-u, x, 1.0);
    const double w = sqrt(u);
    const double w_lo = (fma(-w, w, u) + u_lo) * (0.5 * w * x);
    const double h = u * w;
    const double h_lo = fma(u, w, -h) + (u * w_lo + u_lo * w);
    return h + h_lo;
}

// RN(q^4): q^2 as an exact double-double pair, squared, rounded once.
__device__ __forceinline__ double pow4_rn(double q)
{
    const double h = q * q;
    const double h_lo = fma(q, q, -h);
    const double r = h * h;
    const double r_lo = fma(h, h, -r) + 2.0 * h * h_lo;
    return r + r_lo;
}

__device__ __forceinline__ bool in_range(double x) { return x > 1e-90 && x < 1e90; }

// RN(x^3): x^2 = h + l exactly, x^3 = h x + l x with h x an exact pair
__device__ __forceinline__ double cube_rn(double x)
{
    if (!in_range(fabs(x)))
        return pow(x, 3.0);
    const double h = x * x, l = fma(x, x, -h);
    const double p = h * x, e = fma(h, x, -p);
    return p + (e + l * x);
}

// RN(1 / (h + l)) for a double-double h + l: q = RN(1 / h) leaves the exact
// residual 1 - q h, and one correction step rounds once
__device__ __forceinline__ double recip_dd_rn(double h, double l)
{
    const double q = 1.0 / h;
    const double r = fma(-q, h, 1.0) - q * l;
    return q + q * r;
}

// RN(x^-2)
__device__ __forceinline__ double inv_square_rn(double x)
{
    if (!in_range(fabs(x)))
        return pow(x, -2.0);
    const double h = x * x, l = fma(x, x, -h);
    return recip_dd_rn(h, l);
}

// RN(x^-3)
__device__ __forceinline__ double inv_cube_rn(double x)
{
    if (!in_range(fabs(x)))
        return pow(x, -3.0);
    const double h = x * x, l = fma(x, x, -h);
    const double p = h * x, e = fma(h, x, -p) + l * x;
    return recip_dd_rn(p, e);
}

// RN(pow(x, RN(-1/3))) for x >= 1. The exponent -1/3 rounded to a double is
// -1/3 + d with d = 2^-54 / 3, so the power is x^(-1/3) (1 + d ln x) to far
// below an ulp. x^(-1/3) comes from one Newton step y + y (1 - x y^3) / 3 on
// rcbrt(x), with the residual 1 - x y^3 in double-double.
__device__ __forceinline__ double pow_m13_rn(double x)
{
    if (!(x >= 1.0 && x < 1e90))
        return pow(x, -1.0 / 3.0);
    const double y = rcbrt(x);
    const double h = y * y, l = fma(y, y, -h);
    const double p = h * y, e = fma(h, y, -p) + l * y;  // y^3 = p + e
    const double s = x * p, s_lo = fma(x, p, -s) + x * e;  // x y^3 = s + s_lo
    const double resid = (1.0 - s) - s_lo;  // 1 - s is exact: s is within an ulp or so of 1
    const double d = 0x1.5555555555555p-56;
    return y + y * (resid / 3.0 + d * log(x));
}

// RN(exp(x)) for -745 < x <= 0: x = k ln2 + r with r carried as a
// double-double (ln 2 = LN2_HI + LN2_LO), exp(r) by its Taylor series to
// degree 23 in double-double Horner form (|r| <= 0.35: truncation below
// 2^-103), scaled by 2^k.
__device__ __forceinline__ double exp_rn(double x)
{
    if (!(x > -700.0 && x <= 0.0))
        return exp(x);
    constexpr double LN2_HI = 0x1.62e42fefa39efp-1, LN2_LO = 0x1.abc9e3b39803fp-56;
    const double k = rint(x * 0x1.71547652b82fep+0);
    const double t = k * LN2_HI, t_lo = fma(k, LN2_HI, -t);  // k LN2_HI exactly
    const double a = x - t;  // exact: x and t agree to within a factor of two, or k = 0
    const double b = -t_lo - k * LN2_LO;
    double r = a + b;
    double r_lo = b - (r - a);  // r + r_lo = a + b (Fast2Sum, |a| >= |b|)
    // Horner: s <- 1 + s r / n for n = 23 .. 1, s as a double-double
    double sh = 1.0, sl = 0.0;
    for (int n = 23; n >= 1; --n) {
        // (sh + sl)(r + r_lo)
        const double m = sh * r;
        const double m_lo = fma(sh, r, -m) + (sh * r_lo + sl * r);
        // divided by n: q = RN(m / n), exact remainder m - q n
        const double q = m / n;
        const double q_lo = (fma(-q, (double)n, m) + m_lo) / n;
        // 1 + q + q_lo
        const double u = 1.0 + q;
        const double u_lo = (1.0 - u) + q + q_lo;  // |q| < 1: Fast2Sum
        sh = u + u_lo;
        sl = u_lo - (sh - u);
    }
    return ldexp(sh + sl, (int)k);
}

// guarded forms of the two above
__device__ __forceinline__ double fourth_rn(double x) { return in_range(fabs(x)) ? pow4_rn(x) : pow(x, 4.0); }
__device__ __forceinline__ double inv_pow15_rn(double x) { return in_range(x) ? pow_m15_rn(x) : pow(x, -1.5); }

}  // namespace crm
