// Tangent (forward-mode) and discrete adjoint (reverse-mode) of one RK stage
// and of the end-of-step objective, plus the branch record the adjoint
// replays. Built with -fmad=false.
//
// Adjoint of a stage, as passes over zones and faces (all arrays in the
// padded (ni + 4, nj + 4) layout):
//   S  zone:  slopes and rho * strain of the input, once per zone.
//   B  face:  lambda of each face flux from the two adjacent zones (the
//             conserved-to-primitive adjoint with the recorded floor / ceiling
//             flags, inline); HLLE and viscous-term products with the
//             recorded am / ap choices; face sound-speed terms to the
//             point-mass parameters.
//   C  zone:  gather the four faces: direct and slope contributions,
//             rho * strain products, point-mass and buffer sources, the u_n
//             adjoint.
//   D  zone:  per interior zone, the slope products of every zone it feeds
//             (recorded limiter choices), its guard images folded in
//             (zero-gradient boundary).
// Parameter derivatives (per mass x, y, vx, vy, mass; nu; sink rate) are
// summed per block in a fixed order, then either reduced per stage (12
// values) or chained through the stage's d(mass parameters)/d(q, e) and
// accumulated per block over the whole reverse sweep (4 values per block).
#include <cstring>

#include "adjoint_zone.cuh"
#include "cbd_internal.h"

namespace cbd {

constexpr int NPAR = 12;  // m1 (x, y, vx, vy, mass), m2 (...), nu, sink rate

namespace {

__device__ __forceinline__ size_t zi(int i, int j, int nj) { return (size_t)(i + NG) * (nj + 2 * NG) + (j + NG); }

struct TangentParams {
    double dm[2][5];  // d(x, y, vx, vy, mass) of both masses
    double dnu, drate;
};

template <class T>
__device__ __forceinline__ void masses_t(const StageDev &st, const TangentParams *tp, MassT<T> *m);

template <>
__device__ __forceinline__ void masses_t<Dual>(const StageDev &st, const TangentParams *tp, MassT<Dual> *m)
{
    for (int p = 0; p < 2; ++p) {
        const MassDev &b = st.m[p];
        m[p].x = dual(b.x, tp->dm[p][0]);
        m[p].y = dual(b.y, tp->dm[p][1]);
        m[p].vx = dual(b.vx, tp->dm[p][2]);
        m[p].vy = dual(b.vy, tp->dm[p][3]);
        m[p].mass = dual(b.mass, tp->dm[p][4]);
        m[p].sink_rate = dual(b.sink_rate, tp->drate);
        m[p].base = &st.m[p];
    }
}

template <>
__device__ __forceinline__ void masses_t<double>(const StageDev &st, const TangentParams *, MassT<double> *m)
{
    for (int p = 0; p < 2; ++p) {
        const MassDev &b = st.m[p];
        m[p] = MassT<double>{b.x, b.y, b.vx, b.vy, b.mass, b.sink_rate, &st.m[p]};
    }
}

// ---------------------------------------------------------------------------
// tangent of a stage: thread per interior zone
// ---------------------------------------------------------------------------

__global__ void stage_tangent_kernel(Consts k, const StageDev *stp, TangentParams tp, const double *p,
                                     const double *dp, const double *pun, const double *dpun, double *out,
                                     double *dout)
{
    __shared__ StageDev st;
    if (threadIdx.x == 0)
        st = *stp;
    __syncthreads();
    const long n = (long)k.ni * k.nj;
    const long z = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (z >= n)
        return;
    const int i = (int)(z / k.nj), j = (int)(z - (long)i * k.nj);
    const int nj = k.nj;
    MassT<Dual> m[2];
    masses_t<Dual>(st, &tp, m);
    auto P = [&](int di, int dj, int q) {
        const size_t o = zi(i + di, j + dj, nj) * 3 + q;
        return dual(p[o], dp[o]);
    };
    Dual un[3];
    const size_t oc = zi(i, j, nj) * 3;
    if (pun) {
        const Dual r = dual(pun[oc], dpun[oc]);
        un[0] = r;
        un[1] = dual(pun[oc + 1], dpun[oc + 1]) * r;
        un[2] = dual(pun[oc + 2], dpun[oc + 2]) * r;
    } else {
        const Dual r = P(0, 0, 0);
        un[0] = r;
        un[1] = P(0, 0, 1) * r;
        un[2] = P(0, 0, 2) * r;
    }
    Dual o[3];
    zone_update_generic<Dual>(k, st, m, dual(k.nu, tp.dnu), i, j, P, un, o);
    for (int q = 0; q < 3; ++q) {
        out[oc + q] = o[q].v;
        dout[oc + q] = o[q].d;
    }
}

// zero-gradient guard images of a tangent (same rule as the state's guards)
__global__ void guards_kernel(int ni, int nj, double *a)
{
    const long wi = ni + 2 * NG, wj = nj + 2 * NG;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < wi * wj; z += (long)gridDim.x * blockDim.x) {
        const int ii = (int)(z / wj) - NG, jj = (int)(z % wj) - NG;
        if (ii >= 0 && ii < ni && jj >= 0 && jj < nj)
            continue;
        const int ci = ii < 0 ? 0 : (ii >= ni ? ni - 1 : ii);
        const int cj = jj < 0 ? 0 : (jj >= nj ? nj - 1 : jj);
        for (int q = 0; q < 3; ++q)
            a[zi(ii, jj, nj) * 3 + q] = a[zi(ci, cj, nj) * 3 + q];
    }
}

// ---------------------------------------------------------------------------
// branch record: thread per zone of [-1, ni] x [-1, nj]
// ---------------------------------------------------------------------------

__device__ __forceinline__ void slopes_at(const Consts &k, const double *p, int i, int j, double *gx, double *gy,
                                          unsigned *bits)
{
    const int nj = k.nj;
    unsigned b = 0;
    for (int q = 0; q < 3; ++q) {
        const double xm = p[zi(i - 1, j, nj) * 3 + q], x0 = p[zi(i, j, nj) * 3 + q], xp = p[zi(i + 1, j, nj) * 3 + q];
        const double ym = p[zi(i, j - 1, nj) * 3 + q], yp = p[zi(i, j + 1, nj) * 3 + q];
        const unsigned sx = slope_select(xm, x0, xp, k.theta);
        const unsigned sy = slope_select(ym, x0, yp, k.theta);
        gx[q] = slope_generic(xm, x0, xp, k.theta);
        gy[q] = slope_generic(ym, x0, yp, k.theta);
        b |= sx << (2 * q);
        b |= sy << (6 + 2 * q);
    }
    if (bits)
        *bits = b;
}

__global__ void record_kernel(Consts k, const StageDev *stp, const double *p, const double *pout,
                              unsigned *words)
{
    __shared__ StageDev st;
    if (threadIdx.x == 0)
        st = *stp;
    __syncthreads();
    const int ni = k.ni, nj = k.nj;
    const long wi = ni + 2, wj = nj + 2;
    const long z = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (z >= wi * wj)
        return;
    const int i = (int)(z / wj) - 1, j = (int)(z % wj) - 1;
    MassT<double> m[2];
    masses_t<double>(st, nullptr, m);
    double gx[3], gy[3];
    unsigned w = 0;
    slopes_at(k, p, i, j, gx, gy, &w);
    if (i <= ni - 1 && j >= 0 && j < nj) {  // east x-face (i + 1/2)
        double gx1[3], gy1[3];
        slopes_at(k, p, i + 1, j, gx1, gy1, nullptr);
        double pl[3], pr[3], f[3];
        for (int q = 0; q < 3; ++q) {
            pl[q] = p[zi(i, j, nj) * 3 + q] + 0.5 * gx[q];
            pr[q] = p[zi(i + 1, j, nj) * 3 + q] - 0.5 * gx1[q];
        }
        unsigned sel;
        hlle_generic<double, 0>(pl, pr, cs2_generic(k, m, k.xl + (i + 1.0) * k.dx, k.yl + (j + 0.5) * k.dy),
                                f, &sel);
        w |= sel << BW_XFACE;
    }
    if (i >= 0 && i < ni && j <= nj) {  // south y-face (j - 1/2)
        double gx0[3], gy0[3];
        slopes_at(k, p, i, j - 1, gx0, gy0, nullptr);
        double pl[3], pr[3], f[3];
        for (int q = 0; q < 3; ++q) {
            pl[q] = p[zi(i, j - 1, nj) * 3 + q] + 0.5 * gy0[q];
            pr[q] = p[zi(i, j, nj) * 3 + q] - 0.5 * gy[q];
        }
        unsigned sel;
        hlle_generic<double, 1>(pl, pr, cs2_generic(k, m, k.xl + (i + 0.5) * k.dx, k.yl + (j + 0.0) * k.dy),
                                f, &sel);
        w |= sel << BW_YFACE;
    }
    if (i >= 0 && i < ni && j >= 0 && j < nj) {
        const double *o = pout + zi(i, j, nj) * 3;
        if (!(o[0] > k.rho_min))
            w |= BW_FLOOR;
        if (!(fabs(o[1]) < k.vmax))
            w |= BW_CEIL_X;
        if (!(fabs(o[2]) < k.vmax))
            w |= BW_CEIL_Y;
    }
    words[zi(i, j, nj)] = w;
}

// ---------------------------------------------------------------------------
// adjoint building blocks
// ---------------------------------------------------------------------------

// Derivative values need no correct rounding (the branches they follow are
// fixed): the vector-Jacobian products below use reciprocal square roots and
// reciprocals.

// Parameter-derivative accumulator of one thread. Indices: 5 p + (x, y, vx,
// vy, mass) of mass p, 10 = nu, 11 = sink rate. The per-stage form keeps the
// 12 sums; the chained form contracts the mass part with the stage's Kepler
// Jacobian (shared memory) as it goes and keeps 4: d/dq, d/de, d/dnu, d/drate.
template <bool CHAIN>
struct ParAcc;

template <>
struct ParAcc<false> {
    static constexpr int N = NPAR;
    double v[NPAR];
    __device__ explicit ParAcc(const double *)
    {
        for (int r = 0; r < NPAR; ++r)
            v[r] = 0.0;
    }
    __device__ __forceinline__ void add(int r, double x) { v[r] += x; }
};

template <>
struct ParAcc<true> {
    static constexpr int N = 4;
    double v[4];
    const double *jac;
    __device__ explicit ParAcc(const double *j) : jac(j)
    {
        for (int r = 0; r < 4; ++r)
            v[r] = 0.0;
    }
    __device__ __forceinline__ void add(int r, double x)
    {
        if (r < 10) {
            v[0] += x * jac[2 * r];
            v[1] += x * jac[2 * r + 1];
        } else {
            v[r - 8] += x;
        }
    }
};

// An accumulator that counts only when `on` (halo work recomputed by a
// neighbouring CTA must not be counted twice).
template <class Acc>
struct GatedAcc {
    Acc &acc;
    bool on;
    __device__ __forceinline__ void add(int r, double x)
    {
        if (on)
            acc.add(r, x);
    }
};

// d(cs^2)/d(mass parameters) at (x, y), times lam, into the accumulator
template <class Acc>
__device__ __forceinline__ void cs2_param_vjp(const Consts &k, const StageDev &st, double x, double y, double lam,
                                              Acc &par)
{
    if (k.eos != 2 || lam == 0.0)
        return;
    const double l = lam * k.inv_mach2;
    for (int p = 0; p < 2; ++p) {
        const MassDev &m = st.m[p];
        if (!(m.mass > 0.0))
            continue;
        const double dx = x - m.x, dy = y - m.y;
        const double s12 = rsqrt(dx * dx + dy * dy + m.soft2);
        const double w = l * m.mass * s12 * s12 * s12;
        par.add(5 * p + 0, w * dx);
        par.add(5 * p + 1, w * dy);
        par.add(5 * p + 4, l * s12);
    }
}

// HLLE vector-Jacobian product for the recorded am / ap choice `sel`.
template <int DIR>
__device__ __forceinline__ void hlle_vjp(const double *pl, const double *pr, double cs2, double cs, unsigned sel,
                                         const double *lf, double *lpl, double *lpr, double *lcs2)
{
    const double ul[3] = {pl[0], pl[1] * pl[0], pl[2] * pl[0]};
    const double ur[3] = {pr[0], pr[1] * pr[0], pr[2] * pr[0]};
    const double vl = DIR == 0 ? pl[1] : pl[2];
    const double vr = DIR == 0 ? pr[1] : pr[2];
    double fl[3] = {vl * ul[0], vl * ul[1], vl * ul[2]};
    double fr[3] = {vr * ur[0], vr * ur[1], vr * ur[2]};
    fl[1 + DIR] += pl[0] * cs2;
    fr[1 + DIR] += pr[0] * cs2;
    const unsigned s_am = sel & 3u, s_ap = (sel >> 2) & 3u;
    const double am = s_am == 0 ? 0.0 : (s_am == 1 ? vl - cs : vr - cs);
    const double ap = s_ap == 0 ? 0.0 : (s_ap == 1 ? vl + cs : vr + cs);
    const double inv_d = 1.0 / (ap - am);
    double lfl[3], lfr[3], lul[3], lur[3], lap = 0.0, lam = 0.0;
    for (int q = 0; q < 3; ++q) {
        const double F = (fl[q] * ap - fr[q] * am - (ul[q] - ur[q]) * ap * am) * inv_d;
        const double w = lf[q] * inv_d;
        lfl[q] = w * ap;
        lfr[q] = -w * am;
        lul[q] = -w * ap * am;
        lur[q] = w * ap * am;
        lap += w * (fl[q] - (ul[q] - ur[q]) * am - F);
        lam += w * (F - fr[q] - (ul[q] - ur[q]) * ap);
    }
    double lvl = 0.0, lvr = 0.0, lcs = 0.0;
    if (s_am == 1) {
        lvl += lam;
        lcs -= lam;
    } else if (s_am == 2) {
        lvr += lam;
        lcs -= lam;
    }
    if (s_ap == 1) {
        lvl += lap;
        lcs += lap;
    } else if (s_ap == 2) {
        lvr += lap;
        lcs += lap;
    }
    if (cs > 0.0)
        *lcs2 += lcs * (0.5 / cs);
    // fluxes: f0 = v u0, f1 = v u1 (+ rho cs2 if DIR == 0), f2 = v u2 (+ rho cs2 if DIR == 1)
    lvl += lfl[0] * ul[0] + lfl[1] * ul[1] + lfl[2] * ul[2];
    lvr += lfr[0] * ur[0] + lfr[1] * ur[1] + lfr[2] * ur[2];
    double lrl = lfl[1 + DIR] * cs2, lrr = lfr[1 + DIR] * cs2;
    *lcs2 += lfl[1 + DIR] * pl[0] + lfr[1 + DIR] * pr[0];
    for (int q = 0; q < 3; ++q) {
        lul[q] += lfl[q] * vl;
        lur[q] += lfr[q] * vr;
    }
    // conserved states u = (rho, vx rho, vy rho)
    lrl += lul[0] + lul[1] * pl[1] + lul[2] * pl[2];
    lrr += lur[0] + lur[1] * pr[1] + lur[2] * pr[2];
    double lvxl = lul[1] * pl[0], lvyl = lul[2] * pl[0];
    double lvxr = lur[1] * pr[0], lvyr = lur[2] * pr[0];
    if (DIR == 0) {
        lvxl += lvl;
        lvxr += lvr;
    } else {
        lvyl += lvl;
        lvyr += lvr;
    }
    lpl[0] += lrl;
    lpl[1] += lvxl;
    lpl[2] += lvyl;
    lpr[0] += lrr;
    lpr[1] += lvxr;
    lpr[2] += lvyr;
}

// Gravity of mass p: d(du)/d(sigma) and d(du)/d(mass parameters).
template <class Acc>
__device__ __forceinline__ void gravity_vjp(const MassDev &m, int p, double x, double y, double dt, const double *pc,
                                            const double *ld, double *lp, Acc &par)
{
    if (m.mass == 0.0)
        return;
    const double dx = x - m.x, dy = y - m.y;
    const double r = rsqrt(dx * dx + dy * dy + m.soft2);
    const double g = r * r * r;
    const double h = g * r * r;
    const double sig = pc[0];
    const double a = ld[1] * dx + ld[2] * dy;
    lp[0] += -m.mass * g * a * dt;
    par.add(5 * p + 4, -sig * g * a * dt);
    par.add(5 * p + 0, -sig * m.mass * dt * (ld[1] * (3.0 * dx * dx * h - g) + ld[2] * (3.0 * dx * dy * h)));
    par.add(5 * p + 1, -sig * m.mass * dt * (ld[1] * (3.0 * dx * dy * h) + ld[2] * (3.0 * dy * dy * h - g)));
}

// ---------------------------------------------------------------------------
// adjoint passes
// ---------------------------------------------------------------------------

struct AdjArgs {
    const StageDev *st;
    const double *p;        // stage input (read by the stencil)
    const double *pn;       // u_n source (null for a = 0)
    const double *pout;     // stage output
    unsigned *words;        // branch words (read; written by the recording slope pass)
    const double *lam_out;  // adjoint of the output (interior)
    double *lam_rd;         // += adjoint of the input (interior, guards folded)
    double *lam_n;          // += adjoint of the u_n source (interior)
    double *sl;             // per zone: gx (3), gy (3), rho * strain (3)
    double *fx, *fy;        // per face: see adj_faces
    double *lg, *lp;        // per zone: slope adjoints (6), direct adjoints (3)
    double *par;            // per block: 12 parameter partials, or 4 chained sums (accumulated)
    const double *jac;      // d(mass parameters)/d(q, e) of this stage, 10 x 2 (chained form)
};

// lambda of the RK sum u' of a zone from its output primitives o and their
// adjoint l: the conserved-to-primitive VJP with the floor / ceiling flags
// the stage took (decided from the output as the branch record does).
__device__ __forceinline__ void lam_rk_zone(const Consts &k, const double *o, const double *l, double *lu)
{
    const bool floor = !(o[0] > k.rho_min);
    const bool ceil_x = !(fabs(o[1]) < k.vmax), ceil_y = !(fabs(o[2]) < k.vmax);
    const double inv_rho = 1.0 / o[0];
    const double lvx = ceil_x ? 0.0 : l[1];
    const double lvy = ceil_y ? 0.0 : l[2];
    lu[1] = lvx * inv_rho;
    lu[2] = lvy * inv_rho;
    lu[0] = floor ? 0.0 : l[0] - (o[1] * lvx + o[2] * lvy) * inv_rho;
}

// lambda of the RK sum u' of zone (i, j); zero outside the interior.
__device__ __forceinline__ bool lam_rk(const Consts &k, const AdjArgs &a, int i, int j, double *lu)
{
    if (i < 0 || i >= k.ni || j < 0 || j >= k.nj) {
        lu[0] = lu[1] = lu[2] = 0.0;
        return false;
    }
    const size_t c = zi(i, j, k.nj);
    lam_rk_zone(k, a.pout + c * 3, a.lam_out + c * 3, lu);
    return true;
}

// The stage record in shared memory, and in the chained form the stage's
// Kepler Jacobian (10 x 2).
struct StageShared {
    StageDev st;
    double jac[20];
};

template <bool CHAIN>
__device__ __forceinline__ void load_stage(const AdjArgs &a, StageShared &sh)
{
    if (threadIdx.x == 0)
        sh.st = *a.st;
    if (CHAIN && threadIdx.x >= 32 && threadIdx.x < 52)
        sh.jac[threadIdx.x - 32] = a.jac[threadIdx.x - 32];
    __syncthreads();
}

// Block sum of the accumulators, in a fixed order: the per-stage form stores
// the block's 12 sums as its row; the chained form adds its 4 sums to its row.
template <int NT, bool CHAIN>
__device__ __forceinline__ void store_params(const AdjArgs &a, const ParAcc<CHAIN> &acc, int row = -1)
{
    if (row < 0)
        row = blockIdx.x;
    constexpr int NV = ParAcc<CHAIN>::N;
    constexpr int NW = NT / 32;
    __shared__ double sm[NV * NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = 0; r < NV; ++r) {
        double x = acc.v[r];
        for (int o = 16; o > 0; o >>= 1)
            x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0)
            sm[r * NW + warp] = x;
    }
    __syncthreads();
    if ((int)threadIdx.x < NV) {
        double x = 0.0;
        for (int w = 0; w < NW; ++w)
            x += sm[threadIdx.x * NW + w];
        double *out = a.par + (size_t)row * NV + threadIdx.x;
        if (CHAIN)
            *out += x;
        else
            *out = x;
    }
}

__device__ __forceinline__ long grid_start(int nt) { return blockIdx.x * (long)nt + threadIdx.x; }
__device__ __forceinline__ long grid_step(int nt) { return (long)gridDim.x * nt; }

constexpr int ADJ_THREADS = 128;
constexpr int ADJ_MIN_BLOCKS = 5;  // resident blocks per SM the register budget allows

// rho * strain (xx, xy, yy) of a zone from its slopes gx, gy (shear_strain,
// cbdiso_2d.c:248-263, with the constant divisors as reciprocals: derivative
// arithmetic needs no correct rounding)
__device__ __forceinline__ void rho_strain_of(const Consts &k, double rho, const double *gx, const double *gy,
                                              double *rs)
{
    const double sxx = 4.0 / 3.0 * gx[1] * k.inv_dx - 2.0 / 3.0 * gy[2] * k.inv_dy;
    const double syy = -2.0 / 3.0 * gx[1] * k.inv_dx + 4.0 / 3.0 * gy[2] * k.inv_dy;
    const double sxy = gx[2] * k.inv_dx + gy[1] * k.inv_dy;
    rs[0] = rho * sxx;
    rs[1] = rho * sxy;
    rs[2] = rho * syy;
}

// The adjoint of one face. L / R: primitives, slopes along the face normal,
// the two rho * strain components of the viscous flux (x: xx, xy; y: xy,
// yy), and the adjoint of the zones' RK sums. Out, 8 doubles: lambda of
// the minus-side face state (3), of the plus-side state (3), and of the
// viscous flux's two rho * strain sums (2, the same for both sides).
template <int DIR, class Acc>
__device__ __forceinline__ void face_vjp(const Consts &k, const StageDev &st, const MassT<double> *m,
                                         const double *pL, const double *pR, const double *gL, const double *gR,
                                         const double *rL, const double *rR, const double *lul, const double *lur,
                                         double xf, double yf, Acc &par, double *o)
{
    const double hn = 0.5 * k.nu, b = st.one_minus_a;
    const double cf = b * st.dt * (DIR ? k.inv_dy : k.inv_dx);
    double pl[3], pr[3], lf[3];
    for (int q = 0; q < 3; ++q) {
        pl[q] = pL[q] + 0.5 * gL[q];
        pr[q] = pR[q] - 0.5 * gR[q];
        lf[q] = (lur[q] - lul[q]) * cf;
    }
    const double cs2 = cs2_generic(k, m, xf, yf), cs = sqrt(cs2);
    double lpl[3] = {0, 0, 0}, lpr[3] = {0, 0, 0}, lcs2 = 0.0;
    hlle_vjp<DIR>(pl, pr, cs2, cs, hlle_select(pl[1 + DIR], pr[1 + DIR], cs), lf, lpl, lpr, &lcs2);
    cs2_param_vjp(k, st, xf, yf, lcs2, par);
    for (int q = 0; q < 3; ++q) {
        o[q] = lpl[q];
        o[3 + q] = lpr[q];
    }
    if (k.nu > 0.0) {
        o[6] = -hn * lf[1];
        o[7] = -hn * lf[2];
        par.add(10, -0.5 * (rL[0] + rR[0]) * lf[1] - 0.5 * (rL[1] + rR[1]) * lf[2]);
    } else {
        o[6] = o[7] = 0.0;
    }
}

// The adjoint gathered at one zone of [-1, ni] x [-1, nj] from its four
// faces (8-double records; a face that does not exist reads as zeros): the
// direct adjoint lp, the slope adjoints lgx, lgy, the rho * strain products,
// and for interior zones the gravity and buffer sources and the u_n term.
// Out: g[0..2] = lgx, g[3..5] = lgy, g[6..8] = lp.
template <class Acc>
__device__ __forceinline__ void zone_gather(const Consts &k, const StageDev &st, int i, int j, const double *xe,
                                            const double *xw, const double *ys, const double *yn, const double *gx,
                                            const double *gy, const double *pc, const double *lu, bool interior,
                                            const double *pn, double *lam_n, Acc &par, double *g)
{
    double lp[3], lgx[3], lgy[3];
    for (int q = 0; q < 3; ++q) {
        lp[q] = xe[q] + xw[3 + q] + yn[q] + ys[3 + q];
        lgx[q] = 0.5 * xe[q] - 0.5 * xw[3 + q];
        lgy[q] = 0.5 * yn[q] - 0.5 * ys[3 + q];
    }
    if (k.nu > 0.0) {
        const double lxx = xe[6] + xw[6];
        const double lxy = xe[7] + xw[7] + yn[6] + ys[6];
        const double lyy = yn[7] + ys[7];
        const double rho = pc[0];
        double s[3];
        rho_strain_of(k, 1.0, gx, gy, s);
        lp[0] += s[0] * lxx + s[1] * lxy + s[2] * lyy;
        lgx[1] += rho * (4.0 / 3.0 * lxx - 2.0 / 3.0 * lyy) * k.inv_dx;
        lgy[2] += rho * (-2.0 / 3.0 * lxx + 4.0 / 3.0 * lyy) * k.inv_dy;
        lgx[2] += rho * lxy * k.inv_dx;
        lgy[1] += rho * lxy * k.inv_dy;
    }
    if (interior) {
        double ld[3];
        for (int q = 0; q < 3; ++q)
            ld[q] = st.one_minus_a * lu[q];
        const double xc = k.xl + (i + 0.5) * k.dx, yc = k.yl + (j + 0.5) * k.dy;
        const double dt = st.dt;
        const double rate = buffer_rate(k, st, xc, yc);
        double luu[3];
        for (int q = 0; q < 3; ++q)
            luu[q] = ld[q] * (1.0 - rate * dt);
        for (int q = 0; q < 2; ++q)
            gravity_vjp(st.m[q], q, xc, yc, dt, pc, ld, lp, par);
        lp[0] += luu[0] + luu[1] * pc[1] + luu[2] * pc[2];
        lp[1] += luu[1] * pc[0];
        lp[2] += luu[2] * pc[0];
        if (pn && st.a != 0.0) {
            const double l0 = st.a * lu[0], l1 = st.a * lu[1], l2 = st.a * lu[2];
            lam_n[0] += l0 + l1 * pn[1] + l2 * pn[2];
            lam_n[1] += l1 * pn[0];
            lam_n[2] += l2 * pn[0];
        }
    }
    for (int q = 0; q < 3; ++q) {
        g[q] = lgx[q];
        g[3 + q] = lgy[q];
        g[6 + q] = lp[q];
    }
}

// S: slopes and rho * strain of the zones of [-1, ni] x [-1, nj]; with
// RECORD also the branch word (limiter choices; floor and ceiling flags of
// interior zones) that cbdiso_b200_stage_record_branches would write, less
// the HLLE choices, which pass B recomputes.
template <bool RECORD>
__global__ void __launch_bounds__(ADJ_THREADS, ADJ_MIN_BLOCKS) adj_slopes(Consts k, AdjArgs a)
{
    const long wi = k.ni + 2, wj = k.nj + 2;
    const long z = grid_start(ADJ_THREADS);
    if (z < wi * wj) {
        const int i = (int)(z / wj) - 1, j = (int)(z % wj) - 1;
        const size_t c = zi(i, j, k.nj);
        double *o = a.sl + c * 9;
        unsigned w = 0;
        slopes_at(k, a.p, i, j, o, o + 3, RECORD ? &w : nullptr);
        if (k.nu > 0.0)
            rho_strain_of(k, a.p[c * 3], o, o + 3, o + 6);
        else
            o[6] = o[7] = o[8] = 0.0;
        if (RECORD) {
            if (i >= 0 && i < k.ni && j >= 0 && j < k.nj) {
                const double *q = a.pout + c * 3;
                if (!(q[0] > k.rho_min))
                    w |= BW_FLOOR;
                if (!(fabs(q[1]) < k.vmax))
                    w |= BW_CEIL_X;
                if (!(fabs(q[2]) < k.vmax))
                    w |= BW_CEIL_Y;
            }
            a.words[c] = w;
        }
    }
}

// B: faces, one per thread: items [0, n) are the x-faces, [n, 2 n) the
// y-faces, n = (ni + 2)(nj + 2). fx[c] is the x-face i + 1/2 of zone
// c = (i, j), fy[c] the y-face j - 1/2, 8 doubles each (face_vjp). The HLLE
// wave choice is recomputed with the stage's own (correctly rounded) face
// sound speed.
template <bool CHAIN>
__global__ void __launch_bounds__(ADJ_THREADS, ADJ_MIN_BLOCKS) adj_faces(Consts k, AdjArgs a)
{
    __shared__ StageShared sh;
    load_stage<CHAIN>(a, sh);
    const StageDev &st = sh.st;
    const int ni = k.ni, nj = k.nj;
    const long wi = ni + 2, wj = nj + 2, n = wi * wj;
    ParAcc<CHAIN> par(sh.jac);
    MassT<double> m[2];
    masses_t<double>(st, nullptr, m);
    const long f = grid_start(ADJ_THREADS);
    const bool ydir = f >= n;
    const long z = ydir ? f - n : f;
    const int i = (int)(z / wj) - 1, j = (int)(z % wj) - 1;
    // x-face i + 1/2: L = (i, j), R = (i + 1, j); y-face j - 1/2: L = (i, j - 1), R = (i, j)
    const bool live = f < 2 * n &&
                      (ydir ? (i >= 0 && i < ni && j >= 0 && j <= nj) : (i <= ni - 1 && j >= 0 && j < nj));
    if (live) {
        const int il = i, jl = ydir ? j - 1 : j, ir = ydir ? i : i + 1, jr = j;
        const size_t cl = zi(il, jl, nj), cr = zi(ir, jr, nj);
        double lul[3], lur[3];
        lam_rk(k, a, il, jl, lul);
        lam_rk(k, a, ir, jr, lur);
        const double *sl = a.sl + cl * 9, *sr = a.sl + cr * 9;
        double *o = (ydir ? a.fy : a.fx) + zi(i, j, nj) * 8;
        if (ydir)
            face_vjp<1>(k, st, m, a.p + cl * 3, a.p + cr * 3, sl + 3, sr + 3, sl + 7, sr + 7, lul, lur,
                        k.xl + (i + 0.5) * k.dx, k.yl + (j + 0.0) * k.dy, par, o);
        else
            face_vjp<0>(k, st, m, a.p + cl * 3, a.p + cr * 3, sl, sr, sl + 6, sr + 6, lul, lur,
                        k.xl + (i + 1.0) * k.dx, k.yl + (j + 0.5) * k.dy, par, o);
    }
    store_params<ADJ_THREADS, CHAIN>(a, par);
}

__constant__ double kZeroFace[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

// C: zones of [-1, ni] x [-1, nj]: zone_gather of the four faces pass B wrote
// (sinks: adj_sinks).
template <bool CHAIN>
__global__ void __launch_bounds__(ADJ_THREADS, ADJ_MIN_BLOCKS) adj_zones(Consts k, AdjArgs a)
{
    __shared__ StageShared sh;
    load_stage<CHAIN>(a, sh);
    const StageDev &st = sh.st;
    const int ni = k.ni, nj = k.nj;
    const long wi = ni + 2, wj = nj + 2;
    ParAcc<CHAIN> par(sh.jac);
    const long z = grid_start(ADJ_THREADS);
    if (z < wi * wj) {
        const int i = (int)(z / wj) - 1, j = (int)(z % wj) - 1;
        const size_t c = zi(i, j, nj);
        const bool row = j >= 0 && j < nj, col = i >= 0 && i < ni;
        const double *xe = row && i < ni ? a.fx + c * 8 : kZeroFace;
        const double *xw = row && i >= 0 ? a.fx + zi(i - 1, j, nj) * 8 : kZeroFace;
        const double *ys = col && j >= 0 ? a.fy + c * 8 : kZeroFace;
        const double *yn = col && j < nj ? a.fy + zi(i, j + 1, nj) * 8 : kZeroFace;
        double lu[3];
        const bool interior = lam_rk(k, a, i, j, lu);
        const double *sl = a.sl + c * 9;
        double g[9];
        zone_gather(k, st, i, j, xe, xw, ys, yn, sl, sl + 3, a.p + c * 3, lu, interior,
                    a.pn ? a.pn + c * 3 : nullptr, a.lam_n ? a.lam_n + c * 3 : nullptr, par, g);
        for (int q = 0; q < 3; ++q) {
            a.lg[c * 6 + q] = g[q];
            a.lg[c * 6 + 3 + q] = g[3 + q];
            a.lp[c * 3 + q] = g[6 + q];
        }
    }
    store_params<ADJ_THREADS, CHAIN>(a, par);
}

// Interior zones near a mass that its sink can reach: an index box around
// the mass, one zone wider than the sink's reach on each side.
__device__ __forceinline__ void sink_box(const Consts &k, const MassDev &m, int *i0, int *i1, int *j0, int *j1)
{
    const double reach = m.sink_r4 * 1.0000001;
    *i0 = max(0, (int)floor((m.x - reach - k.xl) * k.inv_dx) - 1);
    *i1 = min(k.ni - 1, (int)floor((m.x + reach - k.xl) * k.inv_dx) + 1);
    *j0 = max(0, (int)floor((m.y - reach - k.yl) * k.inv_dy) - 1);
    *j1 = min(k.nj - 1, (int)floor((m.y + reach - k.yl) * k.inv_dy) + 1);
}

// One directional derivative of a mass's sink term at a zone: direction
// dir of (sigma, vx, vy, x_p, y_p, vx_p, vy_p, rate), weighted by ld.
__device__ __forceinline__ double sink_direction(const MassDev &m, double x, double y, double dt, const double *pc,
                                                 const double *ld, int dir)
{
    Dual du[3] = {dual(0.0), dual(0.0), dual(0.0)};
    sink_generic<Dual>(m, dual(m.x, dir == 3), dual(m.y, dir == 4), dual(m.vx, dir == 5), dual(m.vy, dir == 6),
                       dual(m.sink_rate, dir == 7), x, y, dt, dual(pc[0], dir == 0), dual(pc[1], dir == 1),
                       dual(pc[2], dir == 2), du);
    return ld[0] * du[0].d + ld[1] * du[1].d + ld[2] * du[2].d;
}

__device__ __forceinline__ bool in_box(int i, int j, int i0, int i1, int j0, int j1)
{
    return i >= i0 && i <= i1 && j >= j0 && j <= j1;
}

// Sinks of the stage, after the input pass: their adjoint goes straight into
// lambda_rd (sink zones are interior zones, which no guard image reaches),
// one thread per (zone, direction) of the union of the masses' sink boxes;
// a zone in both boxes adds mass 1's term to mass 0's before the store, so
// no two threads write one element.
template <bool CHAIN>
__global__ void __launch_bounds__(ADJ_THREADS) adj_sinks(Consts k, AdjArgs a)
{
    __shared__ StageShared sh;
    load_stage<CHAIN>(a, sh);
    const StageDev &st = sh.st;
    ParAcc<CHAIN> par(sh.jac);
    int box[2][4];
    bool on[2];
    for (int q = 0; q < 2; ++q) {
        const MassDev &m = st.m[q];
        on[q] = !(m.sink_rate == 0.0 || m.sink_model < 1 || m.sink_model > 3);
        if (on[q]) {
            sink_box(k, m, &box[q][0], &box[q][1], &box[q][2], &box[q][3]);
            on[q] = box[q][1] >= box[q][0] && box[q][3] >= box[q][2];
        }
    }
    for (int q = 0; q < 2; ++q) {
        if (!on[q])
            continue;
        const int i0 = box[q][0], j0 = box[q][2];
        const long bw = box[q][3] - j0 + 1, n = (long)(box[q][1] - i0 + 1) * bw * 8;
        for (long t = grid_start(ADJ_THREADS); t < n; t += grid_step(ADJ_THREADS)) {
            const long z = t >> 3;
            const int dir = (int)(t & 7);
            const int i = i0 + (int)(z / bw), j = j0 + (int)(z % bw);
            if (q == 1 && on[0] && in_box(i, j, box[0][0], box[0][1], box[0][2], box[0][3]))
                continue;  // done with mass 0's box
            const double x = k.xl + (i + 0.5) * k.dx, y = k.yl + (j + 0.5) * k.dy;
            const size_t c = zi(i, j, k.nj);
            double lu[3];
            lam_rk(k, a, i, j, lu);
            const double ld[3] = {st.one_minus_a * lu[0], st.one_minus_a * lu[1], st.one_minus_a * lu[2]};
            double vsum = 0.0;
            bool any = false;
            for (int p = q; p < 2; ++p) {
                const MassDev &m = st.m[p];
                if (!on[p] || !in_box(i, j, box[p][0], box[p][1], box[p][2], box[p][3]))
                    continue;
                const double dx = x - m.x, dy = y - m.y;
                if (!(dx * dx + dy * dy < m.sink_hi2))
                    continue;
                const double v = sink_direction(m, x, y, st.dt, a.p + c * 3, ld, dir);
                if (dir < 3) {
                    vsum = any ? vsum + v : v;
                    any = true;
                } else {
                    par.add(dir < 7 ? 5 * p + dir - 3 : 11, v);
                }
            }
            if (dir < 3 && any)
                a.lam_rd[c * 3 + dir] += vsum;
        }
    }
    store_params<ADJ_THREADS, CHAIN>(a, par);
}

__device__ __forceinline__ void slope_weights(unsigned sel, double theta, double *w)
{
    // d g / d(y_minus, y_0, y_plus)
    w[0] = w[1] = w[2] = 0.0;
    if (sel == 1) {
        w[0] = -theta;
        w[1] = theta;
    } else if (sel == 2) {
        w[0] = -0.5;
        w[2] = 0.5;
    } else if (sel == 3) {
        w[1] = -theta;
        w[2] = theta;
    }
}

// the full input adjoint at padded position (i, j): its direct part plus its
// share of the slopes of its x- and y-neighbours (slopes live on [-1, ni] x [-1, nj])
__device__ __forceinline__ void input_adjoint_at(const Consts &k, const AdjArgs &a, int i, int j, double *acc)
{
    const int ni = k.ni, nj = k.nj;
    const size_t c = zi(i, j, nj);
    const bool in_range = i >= -1 && i <= ni && j >= -1 && j <= nj;
    for (int q = 0; q < 3; ++q)
        acc[q] = in_range ? a.lp[c * 3 + q] : 0.0;
    for (int d = -1; d <= 1; ++d) {
        const int ii = i + d;
        if (ii < -1 || ii > ni || j < -1 || j > nj)
            continue;
        const size_t o = zi(ii, j, nj);
        const unsigned w = a.words[o];
        for (int q = 0; q < 3; ++q) {
            double wt[3];
            slope_weights((w >> (2 * q)) & 3u, k.theta, wt);
            acc[q] += wt[1 - d] * a.lg[o * 6 + q];
        }
    }
    for (int d = -1; d <= 1; ++d) {
        const int jj = j + d;
        if (jj < -1 || jj > nj || i < -1 || i > ni)
            continue;
        const size_t o = zi(i, jj, nj);
        const unsigned w = a.words[o];
        for (int q = 0; q < 3; ++q) {
            double wt[3];
            slope_weights((w >> (6 + 2 * q)) & 3u, k.theta, wt);
            acc[q] += wt[1 - d] * a.lg[o * 6 + 3 + q];
        }
    }
}

// D: interior zones: slope products and the guard images folded into the
// zones they copy (zero-gradient boundary)
__global__ void __launch_bounds__(ADJ_THREADS, ADJ_MIN_BLOCKS) adj_inputs(Consts k, AdjArgs a)
{
    const int ni = k.ni, nj = k.nj;
    const long z = grid_start(ADJ_THREADS);
    if (z < (long)ni * nj) {
        const int i = (int)(z / nj), j = (int)(z - (long)i * nj);
        const int ilo = i == 0 ? -2 : i, ihi = i == ni - 1 ? ni + 1 : i;
        const int jlo = j == 0 ? -2 : j, jhi = j == nj - 1 ? nj + 1 : j;
        // row sums of the folded images first, then the rows in order
        double tot[3] = {0.0, 0.0, 0.0};
        for (int ii = ilo; ii <= ihi; ++ii) {
            double row[3] = {0.0, 0.0, 0.0};
            for (int jj = jlo; jj <= jhi; ++jj) {
                double v[3];
                input_adjoint_at(k, a, ii, jj, v);
                for (int q = 0; q < 3; ++q)
                    row[q] += v[q];
            }
            for (int q = 0; q < 3; ++q)
                tot[q] += row[q];
        }
        for (int q = 0; q < 3; ++q)
            a.lam_rd[zi(i, j, nj) * 3 + q] += tot[q];
    }
}

// ---------------------------------------------------------------------------
// fused adjoint stage: one row-marching pass (the passes S, B, C and D above
// in one kernel, their intermediate results kept in shared-memory rings)
// ---------------------------------------------------------------------------
//
// A CTA of AM_NT threads owns AM_BJ output columns [j0, j0 + AM_BJ) and a
// segment of output rows, and marches down the rows. At iteration r it
//   1. stages row r + 3 of the input primitives and the RK-sum adjoint of
//      row r + 2 (prefetched into registers one iteration ahead),
//   2. computes the slopes, rho * strain and limiter choices of row r + 2,
//   3. the x-face adjoint between rows r + 1 and r + 2 (one per column, kept
//      in registers) and the y-face adjoints of row r + 1,
//   4. the zone gather of row r + 1,
//   5. the input adjoint of row r (slope products of rows r - 1 .. r + 1,
//      guard images folded in) and adds it to lambda_rd.
// Each quantity is computed once per zone or face with the same functions
// and operation order as the separate passes, so the two agree bit for bit
// in lambda_rd and lambda_n. Column spans relative to j0: primitives
// [j0 - 3, j0 + BJ + 2], slopes and RK-sum adjoints [j0 - 2, j0 + BJ + 1],
// gathers [j0 - 1, j0 + BJ], y-faces j - 1/2 for j in [j0 - 1, j0 + BJ + 1].

constexpr int AM_NT = 128;
constexpr int AM_BJ = AM_NT - 8;
constexpr int AM_NP = AM_BJ + 6, AM_NS = AM_BJ + 4, AM_NG = AM_BJ + 2, AM_NY = AM_BJ + 3;

struct MarchSmem {
    double p[4][AM_NP][3];   // rows mod 4
    double sl[2][AM_NS][9];  // rows mod 2: gx (3), gy (3), rho * strain (3)
    double lr[2][AM_NS][3];  // RK-sum adjoint, rows mod 2
    double yf[AM_NY][8];     // y-faces of the gathered row
    double lg[3][AM_NG][9];  // rows mod 3: lgx (3), lgy (3), lp (3)
    unsigned wd[4][AM_NS];   // limiter choices, rows mod 4
};

__device__ __forceinline__ int mod(int r, int m) { return ((r % m) + m) % m; }

// input_adjoint_at on the shared rings (row r must be in [r0 - 1 ..] of the
// rings; c any padded column the strip covers)
__device__ __forceinline__ void march_input_adjoint(const Consts &k, const MarchSmem &sm, int r, int c, int j0,
                                                    double *acc)
{
    const int ni = k.ni, nj = k.nj;
    const bool in_range = r >= -1 && r <= ni && c >= -1 && c <= nj;
    const int cg = c - (j0 - 1), cs = c - (j0 - 2);
    for (int q = 0; q < 3; ++q)
        acc[q] = in_range ? sm.lg[mod(r, 3)][cg][6 + q] : 0.0;
    for (int d = -1; d <= 1; ++d) {
        const int ii = r + d;
        if (ii < -1 || ii > ni || c < -1 || c > nj)
            continue;
        const unsigned w = sm.wd[mod(ii, 4)][cs];
        for (int q = 0; q < 3; ++q) {
            double wt[3];
            slope_weights((w >> (2 * q)) & 3u, k.theta, wt);
            acc[q] += wt[1 - d] * sm.lg[mod(ii, 3)][cg][q];
        }
    }
    for (int d = -1; d <= 1; ++d) {
        const int jj = c + d;
        if (jj < -1 || jj > nj || r < -1 || r > ni)
            continue;
        const unsigned w = sm.wd[mod(r, 4)][cs + d];
        for (int q = 0; q < 3; ++q) {
            double wt[3];
            slope_weights((w >> (6 + 2 * q)) & 3u, k.theta, wt);
            acc[q] += wt[1 - d] * sm.lg[mod(r, 3)][cg + d][3 + q];
        }
    }
}

template <bool CHAIN>
__global__ void __launch_bounds__(AM_NT, 3) adj_march(Consts k, AdjArgs a, int seg_rows)
{
    extern __shared__ __align__(16) unsigned char am_raw[];
    MarchSmem &sm = *reinterpret_cast<MarchSmem *>(am_raw);
    __shared__ StageShared sh;
    load_stage<CHAIN>(a, sh);
    const StageDev &st = sh.st;
    ParAcc<CHAIN> par(sh.jac);
    MassT<double> m[2];
    masses_t<double>(st, nullptr, m);

    const int ni = k.ni, nj = k.nj, t = threadIdx.x;
    const int j0 = blockIdx.x * AM_BJ;
    const int R0 = blockIdx.y * seg_rows, R1 = min(R0 + seg_rows, ni);
    // output rows, with the guard rows that fold into the edge rows
    const int r_first = R0 == 0 ? -2 : R0, r_last = R1 == ni ? ni + 1 : R1 - 1;

    // own columns of each span
    const int cP = j0 - 3 + t, cS = j0 - 2 + t, cG = j0 - 1 + t, cY = j0 - 1 + t, cO = j0 + t;
    const bool onP = t < AM_NP && cP >= -2 && cP <= nj + 1;
    const bool onS = t < AM_NS && cS >= -2 && cS <= nj + 1;
    const bool onG = t < AM_NG && cG >= -1 && cG <= nj;
    const bool onY = t < AM_NY;
    const bool onO = t < AM_BJ && cO < nj;

    // registers: prefetched row, the previous x-face's plus side, output sums
    double pre_p[3] = {0.0, 0.0, 0.0}, pre_o[3] = {0.0, 0.0, 0.0}, pre_l[3] = {0.0, 0.0, 0.0};
    double xprev[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double acc[3] = {0.0, 0.0, 0.0};

    auto fetch = [&](int r) {
        // primitives of row r + 3, output and its adjoint of row r + 2
        const int L = r + 3, R = r + 2;
        if (onP && L >= -2 && L <= ni + 1 && L >= r_first - 3 && L <= r_last + 3) {
            const double *src = a.p + zi(L, cP, nj) * 3;
            pre_p[0] = src[0];
            pre_p[1] = src[1];
            pre_p[2] = src[2];
        }
        if (onS && R >= 0 && R < ni && cS >= 0 && cS < nj && R >= r_first - 2 && R <= r_last + 2) {
            const size_t c = zi(R, cS, nj) * 3;
            for (int q = 0; q < 3; ++q) {
                pre_o[q] = a.pout[c + q];
                pre_l[q] = a.lam_out[c + q];
            }
        }
    };

    fetch(r_first - 6);
    for (int r = r_first - 6; r <= r_last; ++r) {
        // 1. stage the prefetched row, prefetch the next
        {
            const int L = r + 3, R = r + 2;
            if (t < AM_NP) {
                double *d = sm.p[mod(L, 4)][t];
                const bool live = onP && L >= -2 && L <= ni + 1;
                d[0] = live ? pre_p[0] : 0.0;
                d[1] = live ? pre_p[1] : 0.0;
                d[2] = live ? pre_p[2] : 0.0;
            }
            if (t < AM_NS) {
                double *d = sm.lr[mod(R, 2)][t];
                if (onS && R >= 0 && R < ni && cS >= 0 && cS < nj && R >= r_first - 2) {
                    lam_rk_zone(k, pre_o, pre_l, d);
                } else {
                    d[0] = d[1] = d[2] = 0.0;
                }
            }
        }
        if (r < r_last)
            fetch(r + 1);
        __syncthreads();

        // 2. slopes, rho * strain and limiter choices of row r + 2
        {
            const int R = r + 2;
            if (t < AM_NS && R >= -1 && R <= ni && R >= r_first - 2) {
                double *o = sm.sl[mod(R, 2)][t];
                unsigned w = 0;
                if (onS && cS >= -1 && cS <= nj) {
                    const double *pm = sm.p[mod(R - 1, 4)][t + 1], *p0 = sm.p[mod(R, 4)][t + 1];
                    const double *pp = sm.p[mod(R + 1, 4)][t + 1];
                    const double *pw = sm.p[mod(R, 4)][t], *pe = sm.p[mod(R, 4)][t + 2];
                    for (int q = 0; q < 3; ++q) {
                        const unsigned sx = slope_select(pm[q], p0[q], pp[q], k.theta);
                        const unsigned sy = slope_select(pw[q], p0[q], pe[q], k.theta);
                        o[q] = slope_generic(pm[q], p0[q], pp[q], k.theta);
                        o[3 + q] = slope_generic(pw[q], p0[q], pe[q], k.theta);
                        w |= sx << (2 * q);
                        w |= sy << (6 + 2 * q);
                    }
                    if (k.nu > 0.0)
                        rho_strain_of(k, p0[0], o, o + 3, o + 6);
                    else
                        o[6] = o[7] = o[8] = 0.0;
                } else {
                    for (int q = 0; q < 9; ++q)
                        o[q] = 0.0;
                }
                sm.wd[mod(R, 4)][t] = w;
            }
        }
        __syncthreads();

        // 3. x-face (r + 1) + 1/2 in registers, y-faces of row r + 1
        double xnew[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        {
            const int A = r + 1;
            if (onG && A >= -1 && A <= ni - 1 && A >= r_first - 2 && cG >= 0 && cG < nj) {
                const int s = t + 1, pc = t + 2;  // this column in the S and P spans
                const double *sA = sm.sl[mod(A, 2)][s], *sB = sm.sl[mod(A + 1, 2)][s];
                // the face A + 1/2 belongs to the CTA owning row min(A + 1, ni - 1) and its column
                const int orow = A + 1 < ni ? A + 1 : ni - 1;
                GatedAcc<ParAcc<CHAIN>> gp{par, orow >= R0 && orow < R1 && cG >= j0 && cG < j0 + AM_BJ};
                face_vjp<0>(k, st, m, sm.p[mod(A, 4)][pc], sm.p[mod(A + 1, 4)][pc], sA, sB, sA + 6, sB + 6,
                            sm.lr[mod(A, 2)][s], sm.lr[mod(A + 1, 2)][s], k.xl + (A + 1.0) * k.dx,
                            k.yl + (cG + 0.5) * k.dy, gp, xnew);
            }
            if (onY) {
                double *o = sm.yf[t];
                const int j = cY;  // face j - 1/2: L = (A, j - 1), R = (A, j)
                if (A >= 0 && A < ni && j >= 0 && j <= nj && A >= r_first - 1 && A <= r_last + 1) {
                    const int sl_ = t, sr_ = t + 1;  // S-span indices of j - 1 and j
                    const double *gL = sm.sl[mod(A, 2)][sl_], *gR = sm.sl[mod(A, 2)][sr_];
                    // the face j - 1/2 belongs to the CTA owning row A and column min(j, nj - 1)
                    const int ocol = j < nj ? j : nj - 1;
                    GatedAcc<ParAcc<CHAIN>> gp{par, A >= R0 && A < R1 && ocol >= j0 && ocol < j0 + AM_BJ};
                    face_vjp<1>(k, st, m, sm.p[mod(A, 4)][t + 1], sm.p[mod(A, 4)][t + 2], gL + 3, gR + 3, gL + 7,
                                gR + 7, sm.lr[mod(A, 2)][sl_], sm.lr[mod(A, 2)][sr_], k.xl + (A + 0.5) * k.dx,
                                k.yl + (j + 0.0) * k.dy, gp, o);
                } else {
                    for (int q = 0; q < 8; ++q)
                        o[q] = 0.0;
                }
            }
        }
        __syncthreads();

        // 4. zone gather of row r + 1
        {
            const int A = r + 1;
            if (t < AM_NG && A >= -1 && A <= ni && A >= r_first - 1) {
                double *g = sm.lg[mod(A, 3)][t];
                if (onG) {
                    const bool interior = A >= 0 && A < ni && cG >= 0 && cG < nj;
                    // sources and the u_n term count once: in the CTA owning the zone
                    const bool own = interior && A >= R0 && A < R1 && cG >= j0 && cG < j0 + AM_BJ;
                    const size_t c = zi(A, cG, nj);
                    const double *sl = sm.sl[mod(A, 2)][t + 1];
                    GatedAcc<ParAcc<CHAIN>> gp{par, own};
                    zone_gather(k, st, A, cG, xnew, xprev, sm.yf[t], sm.yf[t + 1], sl, sl + 3,
                                sm.p[mod(A, 4)][t + 2], sm.lr[mod(A, 2)][t + 1], interior,
                                own && a.pn ? a.pn + c * 3 : nullptr, own && a.lam_n ? a.lam_n + c * 3 : nullptr,
                                gp, g);
                } else {
                    for (int q = 0; q < 9; ++q)
                        g[q] = 0.0;
                }
            }
            for (int q = 0; q < 8; ++q)
                xprev[q] = xnew[q];
        }
        __syncthreads();

        // 5. input adjoint of row r, guard images folded into the edge zones
        if (onO && r >= r_first) {
            double row[3] = {0.0, 0.0, 0.0}, v[3];
            const int clo = cO == 0 ? -2 : cO, chi = cO == nj - 1 ? nj + 1 : cO;
            for (int c = clo; c <= chi; ++c) {
                march_input_adjoint(k, sm, r, c, j0, v);
                for (int q = 0; q < 3; ++q)
                    row[q] += v[q];
            }
            const int z = r < 0 ? 0 : (r >= ni ? ni - 1 : r);
            const int start = z == 0 ? -2 : z, end = z == ni - 1 ? ni + 1 : z;
            if (r == start)
                acc[0] = acc[1] = acc[2] = 0.0;
            for (int q = 0; q < 3; ++q)
                acc[q] += row[q];
            if (r == end) {
                double *dst = a.lam_rd + zi(z, cO, nj) * 3;
                for (int q = 0; q < 3; ++q)
                    dst[q] += acc[q];
            }
        }
        __syncthreads();
    }
    store_params<AM_NT, CHAIN>(a, par, blockIdx.y * gridDim.x + blockIdx.x);
}

// Fixed-order sum of block partials into one parameter row: warp v sums
// column v, lane l the rows l, l + 32, ... in order, then the lanes in a
// fixed shuffle tree (deterministic, independent of timing).
__global__ void sum_params(const double *blocks, int nblocks, int width, double *out)
{
    const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (v >= width)
        return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32)
        s += blocks[(size_t)b * width + v];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0)
        out[v] += s;
}

// ---------------------------------------------------------------------------
// objective: F = w_mdot * (-(mdot_1 + mdot_2)) + w_torque * torque, per zone,
// with the end-of-step masses; dA and the time weight are folded into the
// weights by the caller
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T objective_zone(const StageDev &st, const MassT<T> *m, double x, double y, const T *p,
                                            double wm, double wt)
{
    T mdot = T{} * 0.0, tq = T{} * 0.0;
    for (int q = 0; q < 2; ++q) {
        // accretion rates: mass off, sink on (cbdiso_2d.py:129-131)
        T du[3] = {T{} * 0.0, T{} * 0.0, T{} * 0.0};
        sink_generic(*m[q].base, m[q].x, m[q].y, m[q].vx, m[q].vy, m[q].sink_rate, x, y, 1.0, p[0], p[1], p[2], du);
        mdot = mdot + du[0];
        // gravity rates: torque = x fy - y fx
        if (val(m[q].mass) != 0.0) {
            const T dx = x - m[q].x, dy = y - m[q].y;
            const T fnum = p[0] * m[q].mass * g_pow15(dx * dx + dy * dy + m[q].base->soft2);
            tq = tq + x * (-fnum * dy) - y * (-fnum * dx);
        }
    }
    return -mdot * wm + tq * wt;
}

__global__ void objective_tangent_kernel(Consts k, const StageDev *stp, TangentParams tp, const double *p,
                                         const double *dp, double wm, double wt, double *partial)
{
    __shared__ StageDev st;
    __shared__ double sm[8];
    if (threadIdx.x == 0)
        st = *stp;
    __syncthreads();
    // objective masses are the end-of-step ones
    MassT<Dual> m[2];
    for (int q = 0; q < 2; ++q) {
        const MassDev &b = st.e[q];
        m[q].x = dual(b.x, tp.dm[q][0]);
        m[q].y = dual(b.y, tp.dm[q][1]);
        m[q].vx = dual(b.vx, tp.dm[q][2]);
        m[q].vy = dual(b.vy, tp.dm[q][3]);
        m[q].mass = dual(b.mass, tp.dm[q][4]);
        m[q].sink_rate = dual(b.sink_rate, tp.drate);
        m[q].base = &st.e[q];
    }
    const long n = (long)k.ni * k.nj;
    double acc = 0.0;
    for (long z = blockIdx.x * (long)blockDim.x + threadIdx.x; z < n; z += (long)gridDim.x * blockDim.x) {
        const int i = (int)(z / k.nj), j = (int)(z - (long)i * k.nj);
        const size_t c = zi(i, j, k.nj) * 3;
        const Dual pz[3] = {dual(p[c], dp[c]), dual(p[c + 1], dp[c + 1]), dual(p[c + 2], dp[c + 2])};
        acc += objective_zone<Dual>(st, m, k.xl + (i + 0.5) * k.dx, k.yl + (j + 0.5) * k.dy, pz, wm, wt).d;
    }
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
        sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w)
            s += sm[w];
        partial[blockIdx.x] = s;
    }
}

// lambda_p += dF/dp per zone (torque part); parameter derivatives to blocks.
// With per_time the weight is multiplied by the record's dt.
template <bool CHAIN>
__global__ void __launch_bounds__(ADJ_THREADS, ADJ_MIN_BLOCKS) objective_adjoint_kernel(Consts k, AdjArgs args, double wt,
                                                                        bool per_time)
{
    __shared__ StageShared sh;
    load_stage<CHAIN>(args, sh);
    const StageDev &st = sh.st;
    const double *p = args.p;
    double *lam = args.lam_rd;
    ParAcc<CHAIN> par(sh.jac);
    const double w = per_time ? wt * st.dt : wt;
    const long n = w != 0.0 ? (long)k.ni * k.nj : 0;
    const long z = grid_start(ADJ_THREADS);
    if (z < n) {
        const int i = (int)(z / k.nj), j = (int)(z - (long)i * k.nj);
        const size_t c = zi(i, j, k.nj) * 3;
        const double x = k.xl + (i + 0.5) * k.dx, y = k.yl + (j + 0.5) * k.dy;
        const double sig = p[c];
        for (int q = 0; q < 2; ++q) {
            const MassDev &b = st.e[q];
            // T = -sigma m g (x dy - y dx)
            if (b.mass != 0.0) {
                const double dx = x - b.x, dy = y - b.y;
                const double r = rsqrt(dx * dx + dy * dy + b.soft2);
                const double g = r * r * r, h = g * r * r;
                const double cr = x * dy - y * dx;
                lam[c] += w * (-b.mass * g * cr);
                par.add(5 * q + 4, w * (-sig * g * cr));
                par.add(5 * q + 0, w * (-sig * b.mass) * (3.0 * dx * h * cr + g * y));
                par.add(5 * q + 1, w * (-sig * b.mass) * (3.0 * dy * h * cr - g * x));
            }
        }
    }
    store_params<ADJ_THREADS, CHAIN>(args, par);
}

// accretion part of the objective (-mdot), through the dual sink, over the
// sink boxes of the end-of-step masses, one thread per (zone, direction)
template <bool CHAIN>
__global__ void __launch_bounds__(ADJ_THREADS) objective_sinks(Consts k, AdjArgs args, double wm, bool per_time)
{
    __shared__ StageShared sh;
    load_stage<CHAIN>(args, sh);
    const StageDev &st = sh.st;
    const double *p = args.p;
    double *lam = args.lam_rd;
    ParAcc<CHAIN> par(sh.jac);
    const double w = per_time ? wm * st.dt : wm;
    const double ld[3] = {-w, 0.0, 0.0};
    for (int q = 0; q < 2 && w != 0.0; ++q) {
        const MassDev &b = st.e[q];
        if (b.sink_rate == 0.0 || b.sink_model < 1 || b.sink_model > 3)
            continue;
        int i0, i1, j0, j1;
        sink_box(k, b, &i0, &i1, &j0, &j1);
        if (i1 < i0 || j1 < j0)
            continue;
        const long bw = j1 - j0 + 1, n = (long)(i1 - i0 + 1) * bw * 8;
        for (long t = grid_start(ADJ_THREADS); t < n; t += grid_step(ADJ_THREADS)) {
            const long z = t >> 3;
            const int dir = (int)(t & 7);
            const int i = i0 + (int)(z / bw), j = j0 + (int)(z % bw);
            const size_t c = zi(i, j, k.nj) * 3;
            const double x = k.xl + (i + 0.5) * k.dx, y = k.yl + (j + 0.5) * k.dy;
            const double dx = x - b.x, dy = y - b.y;
            if (!(dx * dx + dy * dy < b.sink_hi2))
                continue;
            const double v = sink_direction(b, x, y, 1.0, p + c, ld, dir);
            if (dir < 3)
                lam[c + dir] += v;
            else
                par.add(dir < 7 ? 5 * q + dir - 3 : 11, v);
        }
    }
    store_params<ADJ_THREADS, CHAIN>(args, par);
}

inline int nblocks(long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

}  // namespace cbd

using namespace cbd;

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------

namespace {

// per zone: slopes and rho * strain (9), x-face (8), y-face (8), slope
// adjoints (6), direct adjoints (3), the branch word (one slot)
constexpr size_t WS_PER_ZONE = 9 + 8 + 8 + 6 + 3 + 1;

bool grid_ok(const cbd_grid_t *g)
{
    return g && g->ni > 0 && g->nj > 0 && g->xr > g->xl && g->yr > g->yl && (g->eos_type == 1 || g->eos_type == 2);
}

AdjArgs adj_args(const cbd_grid_t *grid, const void *stage_dev, void *workspace, const double *jac)
{
    AdjArgs a;
    std::memset(&a, 0, sizeof(a));
    a.st = static_cast<const StageDev *>(stage_dev);
    const size_t zones = (size_t)(grid->ni + 4) * (grid->nj + 4);
    double *ws = static_cast<double *>(workspace);
    a.sl = ws;
    a.fx = a.sl + zones * 9;
    a.fy = a.fx + zones * 8;
    a.lg = a.fy + zones * 8;
    a.lp = a.lg + zones * 6;
    a.words = reinterpret_cast<unsigned *>(a.lp + zones * 3);
    a.par = ws + zones * WS_PER_ZONE;  // per-block partials of the per-stage form
    a.jac = jac;
    return a;
}

// Blocks of the adjoint passes: one item (zone or face) per thread; the face
// pass is the widest. Rows of the chained accumulator and of the per-block
// partials.
// shortest segment of the fused kernel's march
constexpr int AM_MIN_ROWS = 4;

int adj_rows(const cbd_grid_t *grid)
{
    const long faces = 2L * (grid->ni + 2) * (grid->nj + 2);
    const long pass = (faces + ADJ_THREADS - 1) / ADJ_THREADS;
    // the fused kernel's CTAs at its shortest segments
    const long march = (long)((grid->nj + AM_BJ - 1) / AM_BJ) * ((grid->ni + AM_MIN_ROWS - 1) / AM_MIN_ROWS);
    return (int)(pass > march ? pass : march);
}

int pass_blocks(long items) { return items > 0 ? (int)((items + ADJ_THREADS - 1) / ADJ_THREADS) : 1; }

// grid-stride over the sink boxes' (zone, direction) items: about one pass at
// 2048^2 (a box of ~3k zones per mass); never more than the accumulator rows
constexpr int SINK_PASS_BLOCKS = 148;

// the fused row-marching stage adjoint (default) or the separate passes
int g_fused_adjoint = 1;
// the fused kernel's segment length: 0 = by the wave rule of march_grid
int g_march_rows = 0;

// Strips of AM_BJ columns x segments of rows. A CTA marches its rows plus six
// (the pipeline's lead rows), and CTAs run in waves of three per SM: the
// segment length (4 .. 32 rows) minimises waves x (rows + 6), the longer
// segment on a tie.
dim3 march_grid(int ni, int nj)
{
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                   cudaSuccess)
        cudaGetLastError();
    const int strips = (nj + AM_BJ - 1) / AM_BJ;
    if (g_march_rows > 0)
        return dim3(strips, (ni + g_march_rows - 1) / g_march_rows, 1);
    const long slots = 3L * sms;
    int best = 32;
    long best_cost = -1;
    for (int rows = 32; rows >= AM_MIN_ROWS; --rows) {
        const long ctas = (long)strips * ((ni + rows - 1) / rows);
        const long cost = (ctas + slots - 1) / slots * (rows + 6);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = rows;
        }
    }
    return dim3(strips, (ni + best - 1) / best, 1);
}

template <bool CHAIN>
bool march_ready()
{
    static int ok = -1;
    if (ok < 0)
        ok = cudaFuncSetAttribute(adj_march<CHAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(MarchSmem)) == cudaSuccess;
    return ok == 1;
}

// With `jac` null: `words` is the recorded branch record and the 12
// parameter derivatives of this stage are ADDED into params_out. Otherwise
// the branch words are recorded here (into the workspace) and the chained
// (q, e, nu, rate) sums are accumulated per block into params_out
// (adj_rows() x 4), reduced by cbdiso_b200_adjoint_chain_finish.
int stage_adjoint_impl(const cbd_grid_t *grid, const void *stage_dev, const double *primitive_rd,
                       const double *primitive_n, const double *primitive_out, const unsigned int *words,
                       const double *lam_out, double *lam_rd, double *lam_n, const double *jac, double *params_out,
                       void *workspace, void *stream)
{
    if (!grid_ok(grid) || !stage_dev || !primitive_rd || !primitive_out || (!jac && !words) || !lam_out ||
        !lam_rd || !params_out || !workspace || (primitive_n && !lam_n))
        return CBD_ERR_ARGUMENT;
    const Consts k = consts_from_grid(grid);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int ni = grid->ni, nj = grid->nj;
    AdjArgs a = adj_args(grid, stage_dev, workspace, jac);
    a.p = primitive_rd;
    a.pn = primitive_n;
    a.pout = primitive_out;
    if (!jac)
        a.words = const_cast<unsigned *>(words);  // read only: RECORD is off
    a.lam_out = lam_out;
    a.lam_rd = lam_rd;
    a.lam_n = lam_n;
    double *parts = a.par;
    if (jac)
        a.par = params_out;
    const long wide = (long)(ni + 2) * (nj + 2);
    const int bw = pass_blocks(wide), bf = pass_blocks(2 * wide), bi = pass_blocks((long)ni * nj);
    const int bs = adj_rows(grid) < SINK_PASS_BLOCKS ? adj_rows(grid) : SINK_PASS_BLOCKS;
    constexpr int T = ADJ_THREADS;
    if (g_fused_adjoint) {
        const dim3 grid = march_grid(ni, nj);
        const int seg = (ni + (int)grid.y - 1) / (int)grid.y;
        const size_t smem = sizeof(MarchSmem);
        if (jac) {
            if (!march_ready<true>())
                return CBD_ERR_CUDA;
            adj_march<true><<<grid, AM_NT, smem, s>>>(k, a, seg);
            adj_sinks<true><<<bs, T, 0, s>>>(k, a);
        } else {
            if (!march_ready<false>())
                return CBD_ERR_CUDA;
            adj_march<false><<<grid, AM_NT, smem, s>>>(k, a, seg);
            sum_params<<<1, 32 * NPAR, 0, s>>>(parts, (int)(grid.x * grid.y), NPAR, params_out);
            adj_sinks<false><<<bs, T, 0, s>>>(k, a);
            sum_params<<<1, 32 * NPAR, 0, s>>>(parts, bs, NPAR, params_out);
        }
        return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
    }
    if (jac) {
        adj_slopes<true><<<bw, T, 0, s>>>(k, a);
        adj_faces<true><<<bf, T, 0, s>>>(k, a);
        adj_zones<true><<<bw, T, 0, s>>>(k, a);
        adj_inputs<<<bi, T, 0, s>>>(k, a);
        adj_sinks<true><<<bs, T, 0, s>>>(k, a);
    } else {
        adj_slopes<false><<<bw, T, 0, s>>>(k, a);
        adj_faces<false><<<bf, T, 0, s>>>(k, a);
        sum_params<<<1, 32 * NPAR, 0, s>>>(parts, bf, NPAR, params_out);
        adj_zones<false><<<bw, T, 0, s>>>(k, a);
        sum_params<<<1, 32 * NPAR, 0, s>>>(parts, bw, NPAR, params_out);
        adj_inputs<<<bi, T, 0, s>>>(k, a);
        adj_sinks<false><<<bs, T, 0, s>>>(k, a);
        sum_params<<<1, 32 * NPAR, 0, s>>>(parts, bs, NPAR, params_out);
    }
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

int objective_adjoint_impl(const cbd_grid_t *grid, const void *stage_dev, const double *primitive, double w_mdot,
                           double w_torque, double *lam, const double *jac, double *params_out, void *workspace,
                           void *stream)
{
    if (!grid_ok(grid) || !stage_dev || !primitive || !lam || !params_out || !workspace)
        return CBD_ERR_ARGUMENT;
    const Consts k = consts_from_grid(grid);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    AdjArgs a = adj_args(grid, stage_dev, workspace, jac);
    a.p = primitive;
    a.lam_rd = lam;
    double *parts = a.par;
    const int bz = pass_blocks((long)grid->ni * grid->nj);
    const int bs = adj_rows(grid) < SINK_PASS_BLOCKS ? adj_rows(grid) : SINK_PASS_BLOCKS;
    constexpr int T = ADJ_THREADS;
    if (jac) {
        a.par = params_out;
        objective_adjoint_kernel<true><<<bz, T, 0, s>>>(k, a, w_torque, true);
        objective_sinks<true><<<bs, T, 0, s>>>(k, a, w_mdot, true);
    } else {
        objective_adjoint_kernel<false><<<bz, T, 0, s>>>(k, a, w_torque, false);
        sum_params<<<1, 32 * NPAR, 0, s>>>(parts, bz, NPAR, params_out);
        objective_sinks<false><<<bs, T, 0, s>>>(k, a, w_mdot, false);
        sum_params<<<1, 32 * NPAR, 0, s>>>(parts, bs, NPAR, params_out);
    }
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

}  // namespace

extern "C" {

size_t cbdiso_b200_adjoint_workspace_bytes(const cbd_grid_t *grid)
{
    if (!grid_ok(grid))
        return 0;
    const size_t zones = (size_t)(grid->ni + 4) * (grid->nj + 4);
    // WS_PER_ZONE doubles per zone, then the block partials
    return zones * WS_PER_ZONE * sizeof(double) + (size_t)adj_rows(grid) * NPAR * sizeof(double) + 256;
}

int cbdiso_b200_stage_record_branches(const cbd_grid_t *grid, const void *stage_dev, const double *primitive_rd,
                                      const double *primitive_out, unsigned int *words, void *stream)
{
    if (!grid_ok(grid) || !stage_dev || !primitive_rd || !primitive_out || !words)
        return CBD_ERR_ARGUMENT;
    const Consts k = consts_from_grid(grid);
    const long n = (long)(grid->ni + 2) * (grid->nj + 2);
    record_kernel<<<nblocks(n, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        k, static_cast<const StageDev *>(stage_dev), primitive_rd, primitive_out, words);
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

int cbdiso_b200_stage_tangent(const cbd_grid_t *grid, const void *stage_dev, const double *dmass, double dnu,
                              double drate, const double *primitive_rd, const double *dprimitive_rd,
                              const double *primitive_n, const double *dprimitive_n, double *primitive_out,
                              double *dprimitive_out, void *stream)
{
    if (!grid_ok(grid) || !stage_dev || !primitive_rd || !dprimitive_rd || !primitive_out || !dprimitive_out ||
        (primitive_n && !dprimitive_n))
        return CBD_ERR_ARGUMENT;
    const Consts k = consts_from_grid(grid);
    TangentParams tp;
    std::memset(&tp, 0, sizeof(tp));
    if (dmass)
        for (int p = 0; p < 2; ++p)
            for (int v = 0; v < 5; ++v)
                tp.dm[p][v] = dmass[5 * p + v];
    tp.dnu = dnu;
    tp.drate = drate;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long n = (long)grid->ni * grid->nj;
    stage_tangent_kernel<<<nblocks(n, 128), 128, 0, s>>>(k, static_cast<const StageDev *>(stage_dev), tp,
                                                         primitive_rd, dprimitive_rd, primitive_n, dprimitive_n,
                                                         primitive_out, dprimitive_out);
    const long ng = (long)(grid->ni + 4) * (grid->nj + 4);
    guards_kernel<<<nblocks(ng, 256) < 2048 ? nblocks(ng, 256) : 2048, 256, 0, s>>>(grid->ni, grid->nj,
                                                                                     primitive_out);
    guards_kernel<<<nblocks(ng, 256) < 2048 ? nblocks(ng, 256) : 2048, 256, 0, s>>>(grid->ni, grid->nj,
                                                                                     dprimitive_out);
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

int cbdiso_b200_stage_adjoint(const cbd_grid_t *grid, const void *stage_dev, const double *primitive_rd,
                              const double *primitive_n, const double *primitive_out, const unsigned int *words,
                              const double *lam_out, double *lam_rd, double *lam_n, double *params_out,
                              void *workspace, void *stream)
{
    return stage_adjoint_impl(grid, stage_dev, primitive_rd, primitive_n, primitive_out, words, lam_out, lam_rd,
                              lam_n, nullptr, params_out, workspace, stream);
}

int cbdiso_b200_stage_adjoint_chained(const cbd_grid_t *grid, const void *stage_dev, const double *primitive_rd,
                                      const double *primitive_n, const double *primitive_out, const double *lam_out,
                                      double *lam_rd, double *lam_n, const double *jacobian, double *chain_acc,
                                      void *workspace, void *stream)
{
    if (!jacobian || !chain_acc)
        return CBD_ERR_ARGUMENT;
    return stage_adjoint_impl(grid, stage_dev, primitive_rd, primitive_n, primitive_out, nullptr, lam_out, lam_rd,
                              lam_n, jacobian, chain_acc, workspace, stream);
}

int cbdiso_b200_set_adjoint_variant(int fused)
{
    if (fused != 0 && fused != 1)
        return CBD_ERR_ARGUMENT;
    g_fused_adjoint = fused;
    return CBD_OK;
}

int cbdiso_b200_set_adjoint_segment_rows(int rows)
{
    if (rows != 0 && (rows < AM_MIN_ROWS || rows > 32))
        return CBD_ERR_ARGUMENT;
    g_march_rows = rows;
    return CBD_OK;
}

size_t cbdiso_b200_adjoint_chain_blocks(const cbd_grid_t *grid)
{
    if (!grid_ok(grid))
        return 0;
    return (size_t)adj_rows(grid);
}

int cbdiso_b200_adjoint_chain_finish(const double *chain_acc, int num_blocks, double *out4, void *stream)
{
    if (!chain_acc || num_blocks <= 0 || !out4)
        return CBD_ERR_ARGUMENT;
    sum_params<<<1, 32 * 4, 0, static_cast<cudaStream_t>(stream)>>>(chain_acc, num_blocks, 4, out4);
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

int cbdiso_b200_objective_tangent(const cbd_grid_t *grid, const void *stage_dev, const double *dmass,
                                  double drate, const double *primitive, const double *dprimitive, double w_mdot,
                                  double w_torque, double *partials, int num_partials, void *stream)
{
    if (!grid_ok(grid) || !stage_dev || !primitive || !dprimitive || !partials || num_partials < 1)
        return CBD_ERR_ARGUMENT;
    const Consts k = consts_from_grid(grid);
    TangentParams tp;
    std::memset(&tp, 0, sizeof(tp));
    if (dmass)
        for (int p = 0; p < 2; ++p)
            for (int v = 0; v < 5; ++v)
                tp.dm[p][v] = dmass[5 * p + v];
    tp.drate = drate;
    objective_tangent_kernel<<<num_partials, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        k, static_cast<const StageDev *>(stage_dev), tp, primitive, dprimitive, w_mdot, w_torque, partials);
    return cudaGetLastError() == cudaSuccess ? CBD_OK : CBD_ERR_CUDA;
}

int cbdiso_b200_objective_adjoint(const cbd_grid_t *grid, const void *stage_dev, const double *primitive,
                                  double w_mdot, double w_torque, double *lam, double *params_out, void *workspace,
                                  void *stream)
{
    return objective_adjoint_impl(grid, stage_dev, primitive, w_mdot, w_torque, lam, nullptr, params_out,
                                  workspace, stream);
}

int cbdiso_b200_objective_adjoint_chained(const cbd_grid_t *grid, const void *stage_dev, const double *primitive,
                                          double w_mdot, double w_torque, double *lam, const double *jacobian,
                                          double *chain_acc, void *workspace, void *stream)
{
    if (!jacobian || !chain_acc)
        return CBD_ERR_ARGUMENT;
    return objective_adjoint_impl(grid, stage_dev, primitive, w_mdot, w_torque, lam, jacobian, chain_acc,
                                  workspace, stream);
}

}  // extern "C"
