/*
 * CPU oracle for the isothermal circumbinary-disk solver (cbdiso_2d).
 *
 * TEST INFRASTRUCTURE ONLY. This file is a plain-C restatement of the
 * reference kernels in sailfish/solvers/cbdiso_2d.c. It exists so that the
 * CUDA product (sailfish_b200/csrc) can be checked against an independent CPU
 * implementation. Nothing in the product imports, links or calls it; only
 * tests/, the smoke check and the CPU-baseline leg of bench.py do.
 *
 * Arithmetic follows the reference expression by expression (same operand
 * order, same divisions, same libm calls), so that a gcc -O2 build of this
 * file reproduces the reference build bit for bit. The one deliberate
 * difference: the PLM limiter parameter theta is a runtime argument here,
 * whereas the reference fixes it with `#define PLM_THETA 1.8`
 * (cbdiso_2d.c:11).
 *
 * Array layout is the reference layout: C-contiguous (ni + 4, nj + 4, 3)
 * float64 with two guard zones on every side, j fastest, then the field.
 */
#include <math.h>

#define NQ 3
#define NG 2

/* cbdiso_2d.c:16-21 */
#define LESSER(a, b) ((a) < (b) ? (a) : (b))
#define GREATER(a, b) ((a) > (b) ? (a) : (b))
#define SIGN_OF(x) copysign(1.0, x)

typedef struct {
    double x, y, vx, vy, mass, softening_length, sink_rate, sink_radius;
    int sink_model;
} oracle_mass_t;

typedef struct {
    double surface_density, central_mass, driving_rate, outer_radius, onset_width;
    int is_enabled;
} oracle_buffer_t;

/* cbdiso_2d.c:23-29: generalised minmod with parameter theta. */
static double limited_slope(double yl, double y0, double yr, double theta)
{
    double a = (y0 - yl) * theta;
    double b = (yr - yl) * 0.5;
    double c = (yr - y0) * theta;
    double m = LESSER(fabs(a), LESSER(fabs(b), fabs(c)));
    return 0.25 * fabs(SIGN_OF(a) + SIGN_OF(b)) * (SIGN_OF(a) + SIGN_OF(c)) * m;
}

/* cbdiso_2d.c:31-37 */
static void limited_slopes(const double *yl, const double *y0, const double *yr, double theta, double *g)
{
    for (int q = 0; q < NQ; ++q)
        g[q] = limited_slope(yl[q], y0[q], yr[q], theta);
}

/* cbdiso_2d.c:70-95: softened potential of the masses with positive mass. */
static double potential_at(const oracle_mass_t *m, double x, double y)
{
    double phi = 0.0;
    for (int p = 0; p < 2; ++p) {
        if (m[p].mass > 0.0) {
            double dx = x - m[p].x;
            double dy = y - m[p].y;
            double r2 = dx * dx + dy * dy;
            double s2 = r2 + m[p].softening_length * m[p].softening_length;
            phi -= m[p].mass / sqrt(s2);
        }
    }
    return phi;
}

/* cbdiso_2d.c:97-175: gravity and sink terms of one mass, added to du. */
static void mass_source(const oracle_mass_t *m, double x, double y, double dt, const double *p, double *du)
{
    double sigma = p[0];
    double dx = x - m->x;
    double dy = y - m->y;
    double r2 = dx * dx + dy * dy;
    double dr = sqrt(r2);
    double rsink = m->sink_radius;
    double rsoft = m->softening_length;
    double fnum = sigma * m->mass * pow(r2 + rsoft * rsoft, -1.5);
    double fx = -fnum * dx;
    double fy = -fnum * dy;
    double s = (dr < 4.0 * rsink) ? m->sink_rate * exp(-pow(dr / rsink, 4.0)) : 0.0;
    double mdot = 0.0;

    if (s > 0.0)
        mdot = -s * sigma;
    else if (s < 0.0)
        mdot = -s;

    du[0] += 0.0;
    du[1] += fx * dt;
    du[2] += fy * dt;

    if (m->sink_model == 1) {
        du[0] += dt * mdot;
        du[1] += dt * mdot * p[1];
        du[2] += dt * mdot * p[2];
    } else if (m->sink_model == 2) {
        double ex = dx / (dr + 1e-12);
        double ey = dy / (dr + 1e-12);
        double dvr = (p[1] - m->vx) * ex + (p[2] - m->vy) * ey;
        double vxs = dvr * ex + m->vx;
        double vys = dvr * ey + m->vy;
        du[0] += dt * mdot;
        du[1] += dt * mdot * vxs;
        du[2] += dt * mdot * vys;
    } else if (m->sink_model == 3) {
        du[0] += dt * mdot;
        du[1] += 0.0;
        du[2] += 0.0;
    } else {
        du[0] += 0.0;
        du[1] += 0.0;
        du[2] += 0.0;
    }
}

/* cbdiso_2d.c:194-211 */
static double sound_speed2(double cs2, double mach2, int eos, double x, double y, const oracle_mass_t *m)
{
    if (eos == 1)
        return cs2;
    if (eos == 2)
        return -potential_at(m, x, y) / mach2;
    return 1.0;
}

/* cbdiso_2d.c:213-246: relaxation toward a Keplerian state beyond onset. */
static void buffer_source(const oracle_buffer_t *b, double x, double y, double dt, const double *u, double *du)
{
    if (!b->is_enabled)
        return;
    double rc = sqrt(x * x + y * y);
    double onset = b->outer_radius - b->onset_width;
    if (rc > onset) {
        double vk = sqrt(b->central_mass / rc);
        double target[NQ] = {
            b->surface_density,
            b->surface_density * (-y / rc) * vk,
            b->surface_density * (+x / rc) * vk,
        };
        double omega = sqrt(b->central_mass * pow(onset, -3.0));
        double rate = b->driving_rate * omega * (rc - onset) / (b->outer_radius - onset);
        for (int q = 0; q < NQ; ++q)
            du[q] -= (u[q] - target[q]) * rate * dt;
    }
}

/* cbdiso_2d.c:248-263: s = (sxx, sxy, syx, syy). */
static void strain(const double *gx, const double *gy, double dx, double dy, double *s)
{
    double sxx = 4.0 / 3.0 * gx[1] / dx - 2.0 / 3.0 * gy[2] / dy;
    double syy = -2.0 / 3.0 * gx[1] / dx + 4.0 / 3.0 * gy[2] / dy;
    double sxy = 1.0 / 1.0 * gx[2] / dx + 1.0 / 1.0 * gy[1] / dy;
    s[0] = sxx;
    s[1] = sxy;
    s[2] = sxy;
    s[3] = syy;
}

/* cbdiso_2d.c:268-283 */
static void cons_to_prim(const double *u, double *p, double vmax, double rho_min)
{
    double rho = GREATER(u[0], rho_min);
    double px = u[1];
    double py = u[2];
    p[0] = rho;
    p[1] = SIGN_OF(px) * LESSER(fabs(px / rho), vmax);
    p[2] = SIGN_OF(py) * LESSER(fabs(py / rho), vmax);
}

/* cbdiso_2d.c:285-298 */
static void prim_to_cons(const double *p, double *u)
{
    u[0] = p[0];
    u[1] = p[1] * p[0];
    u[2] = p[2] * p[0];
}

/* cbdiso_2d.c:312-326 */
static void prim_flux(const double *p, const double *u, double cs2, int dir, double *f)
{
    double vn = dir == 0 ? p[1] : p[2];
    double pg = p[0] * cs2;
    f[0] = vn * u[0];
    f[1] = vn * u[1] + pg * (double)(dir == 0);
    f[2] = vn * u[2] + pg * (double)(dir == 1);
}

/* cbdiso_2d.c:352-380 */
static void hlle(const double *pl, const double *pr, double cs2, int dir, double *f)
{
    double ul[NQ], ur[NQ], fl[NQ], fr[NQ];
    prim_to_cons(pl, ul);
    prim_to_cons(pr, ur);
    prim_flux(pl, ul, cs2, dir, fl);
    prim_flux(pr, ur, cs2, dir, fr);
    double cs = sqrt(cs2);
    double vl = dir == 0 ? pl[1] : pl[2];
    double vr = dir == 0 ? pr[1] : pr[2];
    double am = LESSER(0.0, LESSER(vl - cs, vr - cs));
    double ap = GREATER(0.0, GREATER(vl + cs, vr + cs));
    for (int q = 0; q < NQ; ++q)
        f[q] = (fl[q] * ap - fr[q] * am - (ul[q] - ur[q]) * ap * am) / (ap - am);
}

static void pack_masses(oracle_mass_t *m,
    double x1, double y1, double vx1, double vy1, double mass1, double soft1, double rate1, double rsink1, int model1,
    double x2, double y2, double vx2, double vy2, double mass2, double soft2, double rate2, double rsink2, int model2)
{
    oracle_mass_t a = {x1, y1, vx1, vy1, mass1, soft1, rate1, rsink1, model1};
    oracle_mass_t b = {x2, y2, vx2, vy2, mass2, soft2, rate2, rsink2, model2};
    m[0] = a;
    m[1] = b;
}

/*
 * cbdiso_2d.c:385-604. Same argument order as the reference kernel, plus the
 * limiter parameter theta as the final argument.
 */
void oracle_cbdiso_2d_advance_rk(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    const double *conserved_rk, const double *primitive_rd, double *primitive_wr,
    double buffer_surface_density, double buffer_central_mass, double buffer_driving_rate,
    double buffer_outer_radius, double buffer_onset_width, int buffer_is_enabled,
    double x1, double y1, double vx1, double vy1, double mass1, double soft1, double rate1, double rsink1, int model1,
    double x2, double y2, double vx2, double vy2, double mass2, double soft2, double rate2, double rsink2, int model2,
    double cs2, double mach2, int eos, double nu, double a, double dt,
    double velocity_ceiling, double density_floor, double theta)
{
    oracle_buffer_t buf = {buffer_surface_density, buffer_central_mass, buffer_driving_rate,
                           buffer_outer_radius, buffer_onset_width, buffer_is_enabled};
    oracle_mass_t ms[2];
    pack_masses(ms, x1, y1, vx1, vy1, mass1, soft1, rate1, rsink1, model1,
                x2, y2, vx2, vy2, mass2, soft2, rate2, rsink2, model2);

    double dx = (patch_xr - patch_xl) / ni;
    double dy = (patch_yr - patch_yl) / nj;
    long si = (long)NQ * (nj + 2 * NG);
    long sj = NQ;

#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i) {
        for (int j = 0; j < nj; ++j) {
            double xl = patch_xl + (i + 0.0) * dx;
            double xc = patch_xl + (i + 0.5) * dx;
            double xr = patch_xl + (i + 1.0) * dx;
            double yl = patch_yl + (j + 0.0) * dy;
            double yc = patch_yl + (j + 0.5) * dy;
            double yr = patch_yl + (j + 1.0) * dy;

#define AT(di, dj) (primitive_rd + (i + (di) + NG) * si + (j + (dj) + NG) * sj)
            const double *c = AT(0, 0);
            const double *w1 = AT(-1, 0), *e1 = AT(1, 0), *s1 = AT(0, -1), *n1 = AT(0, 1);
            const double *w2 = AT(-2, 0), *e2 = AT(2, 0), *s2 = AT(0, -2), *n2 = AT(0, 2);
            const double *sw = AT(-1, -1), *nw = AT(-1, 1), *se = AT(1, -1), *ne = AT(1, 1);
#undef AT
            const double *un = conserved_rk + (i + NG) * si + (j + NG) * sj;

            /* x- and y-slopes at the centre and the four edge neighbours */
            double gx_w[NQ], gx_c[NQ], gx_e[NQ], gy_s[NQ], gy_c[NQ], gy_n[NQ];
            double gy_w[NQ], gy_e[NQ], gx_s[NQ], gx_n[NQ];
            limited_slopes(w2, w1, c, theta, gx_w);
            limited_slopes(w1, c, e1, theta, gx_c);
            limited_slopes(c, e1, e2, theta, gx_e);
            limited_slopes(s2, s1, c, theta, gy_s);
            limited_slopes(s1, c, n1, theta, gy_c);
            limited_slopes(c, n1, n2, theta, gy_n);
            limited_slopes(sw, w1, nw, theta, gy_w);
            limited_slopes(se, e1, ne, theta, gy_e);
            limited_slopes(sw, s1, se, theta, gx_s);
            limited_slopes(nw, n1, ne, theta, gx_n);

            /* face states: m = minus side of the face, p = plus side */
            double wm[NQ], wp[NQ], em[NQ], ep[NQ], sm[NQ], sp[NQ], nm[NQ], np_[NQ];
            for (int q = 0; q < NQ; ++q) {
                wm[q] = w1[q] + 0.5 * gx_w[q];
                wp[q] = c[q] - 0.5 * gx_c[q];
                em[q] = c[q] + 0.5 * gx_c[q];
                ep[q] = e1[q] - 0.5 * gx_e[q];
                sm[q] = s1[q] + 0.5 * gy_s[q];
                sp[q] = c[q] - 0.5 * gy_c[q];
                nm[q] = c[q] + 0.5 * gy_c[q];
                np_[q] = n1[q] - 0.5 * gy_n[q];
            }

            double cs2_w = sound_speed2(cs2, mach2, eos, xl, yc, ms);
            double cs2_e = sound_speed2(cs2, mach2, eos, xr, yc, ms);
            double cs2_s = sound_speed2(cs2, mach2, eos, xc, yl, ms);
            double cs2_n = sound_speed2(cs2, mach2, eos, xc, yr, ms);

            double fw[NQ], fe[NQ], fs[NQ], fn[NQ];
            hlle(wm, wp, cs2_w, 0, fw);
            hlle(em, ep, cs2_e, 0, fe);
            hlle(sm, sp, cs2_s, 1, fs);
            hlle(nm, np_, cs2_n, 1, fn);

            if (nu > 0.0) {
                double st_w[4], st_e[4], st_s[4], st_n[4], st_c[4];
                strain(gx_w, gy_w, dx, dy, st_w);
                strain(gx_e, gy_e, dx, dy, st_e);
                strain(gx_s, gy_s, dx, dy, st_s);
                strain(gx_n, gy_n, dx, dy, st_n);
                strain(gx_c, gy_c, dx, dy, st_c);
                fw[1] -= 0.5 * nu * (w1[0] * st_w[0] + c[0] * st_c[0]);
                fw[2] -= 0.5 * nu * (w1[0] * st_w[1] + c[0] * st_c[1]);
                fe[1] -= 0.5 * nu * (c[0] * st_c[0] + e1[0] * st_e[0]);
                fe[2] -= 0.5 * nu * (c[0] * st_c[1] + e1[0] * st_e[1]);
                fs[1] -= 0.5 * nu * (s1[0] * st_s[2] + c[0] * st_c[2]);
                fs[2] -= 0.5 * nu * (s1[0] * st_s[3] + c[0] * st_c[3]);
                fn[1] -= 0.5 * nu * (c[0] * st_c[2] + n1[0] * st_n[2]);
                fn[2] -= 0.5 * nu * (c[0] * st_c[3] + n1[0] * st_n[3]);
            }

            double du[NQ] = {0.0, 0.0, 0.0};
            double uc[NQ];
            prim_to_cons(c, uc);
            buffer_source(&buf, xc, yc, dt, uc, du);
            mass_source(&ms[0], xc, yc, dt, c, du);
            mass_source(&ms[1], xc, yc, dt, c, du);

            for (int q = 0; q < NQ; ++q)
                du[q] -= ((fe[q] - fw[q]) / dx + (fn[q] - fs[q]) / dy) * dt;
            for (int q = 0; q < NQ; ++q) {
                uc[q] += du[q];
                uc[q] = (1.0 - a) * uc[q] + a * un[q];
            }
            cons_to_prim(uc, primitive_wr + (i + NG) * si + (j + NG) * sj, velocity_ceiling, density_floor);
        }
    }
}

/* cbdiso_2d.c:606-624 */
void oracle_cbdiso_2d_primitive_to_conserved(int ni, int nj, const double *primitive, double *conserved)
{
    long si = (long)NQ * (nj + 2 * NG);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) {
            long n = (i + NG) * si + (long)(j + NG) * NQ;
            prim_to_cons(primitive + n, conserved + n);
        }
}

/* cbdiso_2d.c:626-664: source rate (dt = 1) of one mass, added into cons_rate. */
void oracle_cbdiso_2d_point_mass_source_term(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    double x1, double y1, double vx1, double vy1, double mass1, double soft1, double rate1, double rsink1, int model1,
    const double *primitive, double *cons_rate)
{
    oracle_mass_t m = {x1, y1, vx1, vy1, mass1, soft1, rate1, rsink1, model1};
    long si = (long)NQ * (nj + 2 * NG);
    double dx = (patch_xr - patch_xl) / ni;
    double dy = (patch_yr - patch_yl) / nj;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) {
            long n = (i + NG) * si + (long)(j + NG) * NQ;
            double xc = patch_xl + (i + 0.5) * dx;
            double yc = patch_yl + (j + 0.5) * dy;
            mass_source(&m, xc, yc, 1.0, primitive + n, cons_rate + n);
        }
}

/* cbdiso_2d.c:666-722: per-zone max |v +- cs| into an (ni + 4, nj + 4) array. */
void oracle_cbdiso_2d_wavespeed(
    int ni, int nj,
    double patch_xl, double patch_xr, double patch_yl, double patch_yr,
    double soundspeed2, double mach2, int eos,
    double x1, double y1, double vx1, double vy1, double mass1, double soft1, double rate1, double rsink1, int model1,
    double x2, double y2, double vx2, double vy2, double mass2, double soft2, double rate2, double rsink2, int model2,
    const double *primitive, double *wavespeed)
{
    oracle_mass_t ms[2];
    pack_masses(ms, x1, y1, vx1, vy1, mass1, soft1, rate1, rsink1, model1,
                x2, y2, vx2, vy2, mass2, soft2, rate2, rsink2, model2);
    long si = (long)NQ * (nj + 2 * NG);
    long ti = nj + 2 * NG;
    double dx = (patch_xr - patch_xl) / ni;
    double dy = (patch_yr - patch_yl) / nj;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) {
            const double *p = primitive + (i + NG) * si + (long)(j + NG) * NQ;
            double x = patch_xl + (i + 0.5) * dx;
            double y = patch_yl + (j + 0.5) * dy;
            double c2 = sound_speed2(soundspeed2, mach2, eos, x, y, ms);
            double cs = sqrt(c2);
            double ax = GREATER(fabs(p[1] - cs), fabs(p[1] + cs));
            double ay = GREATER(fabs(p[2] - cs), fabs(p[2] + cs));
            wavespeed[(i + NG) * ti + (j + NG)] = GREATER(ax, ay);
        }
}
