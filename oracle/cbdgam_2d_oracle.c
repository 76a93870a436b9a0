/*
 * CPU oracle for the gamma-law circumbinary-disk solver (cbdgam_2d).
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference kernels in
 * sailfish/solvers/cbdgam_2d.c, used to check the CUDA product against an
 * independent CPU implementation. Nothing in the product imports, links or
 * calls it; only tests/, the smoke check and bench.py's CPU leg do.
 *
 * The arithmetic follows the reference expression by expression (operand
 * order, divisions, libm calls), so that a gcc -O2 build reproduces the
 * reference build bit for bit. The one deliberate difference: the PLM
 * limiter parameter theta is a runtime argument (the reference fixes it with
 * `#define PLM_THETA 1.5`, cbdgam_2d.c:15).
 *
 * Layout: C-contiguous (ni + 4, nj + 4, 4) float64 (sigma, vx, vy, pressure)
 * with two guard zones on each side, j fastest, then the field.
 */
#include <math.h>
#include <stddef.h>

#define NF 4
#define NG 2

#define LESSER(a, b) ((a) < (b) ? (a) : (b))
#define GREATER(a, b) ((a) > (b) ? (a) : (b))
#define SIGN_OF(x) copysign(1.0, x)

typedef struct {
    double x, y, vx, vy, mass, softening_length, sink_rate, sink_radius;
    int sink_model;
} gam_mass_t;

typedef struct {
    double sigma, pressure, central_mass, driving_rate, outer_radius, onset_width;
    int on;
} gam_buffer_t;

/* cbdgam_2d.c:27-33 */
static double gam_slope(double yl, double y0, double yr, double theta)
{
    double a = (y0 - yl) * theta;
    double b = (yr - yl) * 0.5;
    double c = (yr - y0) * theta;
    double m = LESSER(fabs(a), LESSER(fabs(b), fabs(c)));
    return 0.25 * fabs(SIGN_OF(a) + SIGN_OF(b)) * (SIGN_OF(a) + SIGN_OF(c)) * m;
}

static void gam_slopes(const double *yl, const double *y0, const double *yr, double theta, double *g)
{
    for (int q = 0; q < NF; ++q)
        g[q] = gam_slope(yl[q], y0[q], yr[q], theta);
}

/* cbdgam_2d.c:75-106: the disk's scale height sqrt(p / sigma) / Omega~ */
static double scale_height(const gam_mass_t *m, double x, double y, const double *p)
{
    if (m[0].mass == 0.0 && m[1].mass == 0.0)
        return 1.0;
    double w2 = 0.0;
    for (int k = 0; k < 2; ++k) {
        if (m[k].mass > 0.0) {
            double dx = x - m[k].x;
            double dy = y - m[k].y;
            double r = sqrt(dx * dx + dy * dy + 1e-12);
            w2 += m[k].mass * pow(r, -3.0);
        }
    }
    return sqrt(p[3] / p[0]) / sqrt(w2);
}

/* cbdgam_2d.c:108-203: gravity, sink and their work on the gas for one mass */
static void gam_mass_source(const gam_mass_t *m, double x, double y, double dt, const double *p, double h,
                            int constant_softening, double gamma, double *du)
{
    double sigma = p[0];
    double eps = p[3] / sigma / (gamma - 1.0);
    double dx = x - m->x;
    double dy = y - m->y;
    double r2 = dx * dx + dy * dy;
    double dr = sqrt(r2);
    double rs = m->sink_radius;
    double soft;
    if (constant_softening) {
        soft = m->softening_length;
    } else if (dr > rs) {
        soft = 0.5 * h;
    } else {
        double w = pow(1.0 - pow(dr / rs, 2.0), 2.0);
        soft = w * rs + (1.0 - w) * 0.5 * h;
    }
    double rate = (dr < 4.0 * rs) ? m->sink_rate * exp(-pow(dr / rs, 4.0)) : 0.0;
    double fnum = sigma * m->mass * pow(r2 + soft * soft, -1.5);
    double fx = -fnum * dx;
    double fy = -fnum * dy;
    double mdot = sigma * rate * -1.0;
    double vx = p[1], vy = p[2];

    if (m->sink_model == 1) {
        du[0] = dt * mdot;
        du[1] = dt * mdot * p[1] + dt * fx;
        du[2] = dt * mdot * p[2] + dt * fy;
        du[3] = dt * (mdot * eps + 0.5 * mdot * (vx * vx + vy * vy)) + dt * (fx * vx + fy * vy);
    } else if (m->sink_model == 2) {
        double ex = dx / (dr + 1e-12);
        double ey = dy / (dr + 1e-12);
        double dvr = (vx - m->vx) * ex + (vy - m->vy) * ey;
        double wx = dvr * ex + m->vx;
        double wy = dvr * ey + m->vy;
        du[0] = dt * mdot;
        du[1] = dt * mdot * wx + dt * fx;
        du[2] = dt * mdot * wy + dt * fy;
        du[3] = dt * (mdot * eps + 0.5 * mdot * (wx * wx + wy * wy)) + dt * (fx * vx + fy * vy);
    } else if (m->sink_model == 3) {
        du[0] = dt * mdot;
        du[1] = dt * fx;
        du[2] = dt * fy;
        du[3] = dt * (fx * vx + fy * vy);
    } else {
        du[0] = du[1] = du[2] = du[3] = 0.0;
    }
}

/* cbdgam_2d.c:231-236 */
static double gam_cs2(double gamma, const double *p) { return p[3] / p[0] * gamma; }

/* cbdgam_2d.c:238-276: damping toward the Keplerian state beyond the onset radius */
static void gam_buffer(const gam_buffer_t *b, double x, double y, double dt, double *u, double gamma)
{
    if (!b->on)
        return;
    double rc = sqrt(x * x + y * y);
    double onset = b->outer_radius - b->onset_width;
    if (rc > onset) {
        double pf = b->sigma * sqrt(b->central_mass / rc);
        double px = pf * (-y / rc);
        double py = pf * (x / rc);
        double ek = 0.5 * (px * px + py * py) / b->sigma;
        double target[NF] = {b->sigma, px, py, b->pressure / (gamma - 1.0) + ek};
        double omega = sqrt(b->central_mass * pow(onset, -3.0));
        double rate = b->driving_rate * omega * (rc - onset) / (b->outer_radius - onset);
        for (int q = 0; q < NF; ++q)
            u[q] -= (u[q] - target[q]) * rate * dt;
    }
}

/* cbdgam_2d.c:278-294: xx, xy, yx, yy */
static void gam_strain(const double *gx, const double *gy, double dx, double dy, double *s)
{
    double sxx = 4.0 / 3.0 * gx[1] / dx - 2.0 / 3.0 * gy[2] / dy;
    double syy = -2.0 / 3.0 * gx[1] / dx + 4.0 / 3.0 * gy[2] / dy;
    double sxy = 1.0 / 1.0 * gx[2] / dx + 1.0 / 1.0 * gy[1] / dy;
    s[0] = sxx;
    s[1] = sxy;
    s[2] = sxy;
    s[3] = syy;
}

/* cbdgam_2d.c:298-317 */
static void gam_cooling(double coefficient, double mach_ceiling, double dt, const double *p, double *u, double gamma)
{
    double sigma = p[0];
    double eps = p[3] / p[0] / (gamma - 1.0);
    double cooled = eps * pow(1.0 + 3.0 * coefficient * pow(sigma, -2.0) * pow(eps, 3.0) * dt, -1.0 / 3.0);
    double ek = 0.5 * (p[1] * p[1] + p[2] * p[2]);
    cooled = GREATER(cooled, 2.0 * ek / gamma / (gamma - 1.0) * pow(mach_ceiling, -2.0));
    u[3] += sigma * (cooled - eps);
}

/* cbdgam_2d.c:319-345 */
static void gam_cons_to_prim(const double *u, double *p, double vmax, double rho_floor, double p_floor, double gamma)
{
    double pres = GREATER(p_floor, (u[3] - 0.5 * (u[1] * u[1] + u[2] * u[2]) / u[0]) * (gamma - 1.0));
    double vx = SIGN_OF(u[1]) * LESSER(fabs(u[1] / u[0]), vmax);
    double vy = SIGN_OF(u[2]) * LESSER(fabs(u[2] / u[0]), vmax);
    double rho = u[0];
    if (u[0] < rho_floor) {
        rho = rho_floor;
        vx = 0.0;
        vy = 0.0;
        pres = p_floor;
    }
    p[0] = rho;
    p[1] = vx;
    p[2] = vy;
    p[3] = pres;
}

/* cbdgam_2d.c:347-362 */
static void gam_prim_to_cons(const double *p, double *u, double gamma)
{
    double rho = p[0], vx = p[1], vy = p[2], pres = p[3];
    u[0] = rho;
    u[1] = vx * rho;
    u[2] = vy * rho;
    u[3] = pres / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy);
}

/* cbdgam_2d.c:374-387 */
static void gam_flux(const double *p, const double *u, double *f, int dir)
{
    double vn = dir == 0 ? p[1] : (dir == 1 ? p[2] : 0.0);
    double pres = p[3];
    f[0] = vn * u[0];
    f[1] = vn * u[1] + pres * (double)(dir == 0);
    f[2] = vn * u[2] + pres * (double)(dir == 1);
    f[3] = vn * (u[3] + pres);
}

/* cbdgam_2d.c:401-409 */
static double gam_max_wavespeed(const double *p, double cs2)
{
    double cs = sqrt(cs2);
    double ax = GREATER(fabs(p[1] - cs), fabs(p[1] + cs));
    double ay = GREATER(fabs(p[2] - cs), fabs(p[2] + cs));
    return GREATER(ax, ay);
}

/* cbdgam_2d.c:411-434 */
static void gam_hlle(const double *pl, const double *pr, double *f, double cs2, int dir, double gamma)
{
    double ul[NF], ur[NF], fl[NF], fr[NF];
    gam_prim_to_cons(pl, ul, gamma);
    gam_prim_to_cons(pr, ur, gamma);
    gam_flux(pl, ul, fl, dir);
    gam_flux(pr, ur, fr, dir);
    double cs = sqrt(cs2);
    double vl = dir == 0 ? pl[1] : pl[2];
    double vr = dir == 0 ? pr[1] : pr[2];
    double am = LESSER(0.0, LESSER(vl - cs, vr - cs));
    double ap = GREATER(0.0, GREATER(vl + cs, vr + cs));
    for (int q = 0; q < NF; ++q)
        f[q] = (fl[q] * ap - fr[q] * am - (ul[q] - ur[q]) * ap * am) / (ap - am);
}

static size_t at(int i, int j, int nj) { return ((size_t)(i + NG) * (nj + 2 * NG) + (j + NG)) * NF; }

/* cbdgam_2d.c:439-683: one RK stage over the interior */
void oracle_cbdgam_2d_advance_rk(int ni, int nj, double xl0, double xr0, double yl0, double yr0,
                                 const double *un_all, const double *prd, double *pwr, double gamma,
                                 double buf_sigma, double buf_pressure, double buf_mass, double buf_rate,
                                 double buf_outer, double buf_width, int buf_on, double x1, double y1, double vx1,
                                 double vy1, double mass1, double soft1, double rate1, double radius1, int model1,
                                 double x2, double y2, double vx2, double vy2, double mass2, double soft2,
                                 double rate2, double radius2, int model2, double alpha, double a, double dt,
                                 double vmax, double cooling, double mach_ceiling, double rho_floor, double p_floor,
                                 int constant_softening, double theta)
{
    const gam_buffer_t buf = {buf_sigma, buf_pressure, buf_mass, buf_rate, buf_outer, buf_width, buf_on};
    const gam_mass_t ms[2] = {{x1, y1, vx1, vy1, mass1, soft1, rate1, radius1, model1},
                              {x2, y2, vx2, vy2, mass2, soft2, rate2, radius2, model2}};
    const double dx = (xr0 - xl0) / ni;
    const double dy = (yr0 - yl0) / nj;
#pragma omp parallel for
    for (int i = 0; i < ni; ++i) {
        for (int j = 0; j < nj; ++j) {
            double xl = xl0 + (i + 0.0) * dx, xc = xl0 + (i + 0.5) * dx, xr = xl0 + (i + 1.0) * dx;
            double yl = yl0 + (j + 0.0) * dy, yc = yl0 + (j + 0.5) * dy, yr = yl0 + (j + 1.0) * dy;
            const double *un = un_all + at(i, j, nj);
            const double *c = prd + at(i, j, nj);
            const double *w1 = prd + at(i - 1, j, nj), *e1 = prd + at(i + 1, j, nj);
            const double *s1 = prd + at(i, j - 1, nj), *n1 = prd + at(i, j + 1, nj);
            const double *w2 = prd + at(i - 2, j, nj), *e2 = prd + at(i + 2, j, nj);
            const double *s2 = prd + at(i, j - 2, nj), *n2 = prd + at(i, j + 2, nj);
            const double *sw = prd + at(i - 1, j - 1, nj), *nw = prd + at(i - 1, j + 1, nj);
            const double *se = prd + at(i + 1, j - 1, nj), *ne = prd + at(i + 1, j + 1, nj);

            double gxw[NF], gxc[NF], gxe[NF], gys[NF], gyc[NF], gyn[NF], gyw[NF], gye[NF], gxs[NF], gxn[NF];
            gam_slopes(w2, w1, c, theta, gxw);
            gam_slopes(w1, c, e1, theta, gxc);
            gam_slopes(c, e1, e2, theta, gxe);
            gam_slopes(s2, s1, c, theta, gys);
            gam_slopes(s1, c, n1, theta, gyc);
            gam_slopes(c, n1, n2, theta, gyn);
            gam_slopes(sw, w1, nw, theta, gyw);
            gam_slopes(se, e1, ne, theta, gye);
            gam_slopes(sw, s1, se, theta, gxs);
            gam_slopes(nw, n1, ne, theta, gxn);

            double wm[NF], wp[NF], em[NF], ep[NF], sm[NF], sp[NF], nm[NF], np_[NF];
            for (int q = 0; q < NF; ++q) {
                wm[q] = w1[q] + 0.5 * gxw[q];
                wp[q] = c[q] - 0.5 * gxc[q];
                em[q] = c[q] + 0.5 * gxc[q];
                ep[q] = e1[q] - 0.5 * gxe[q];
                sm[q] = s1[q] + 0.5 * gys[q];
                sp[q] = c[q] - 0.5 * gyc[q];
                nm[q] = c[q] + 0.5 * gyc[q];
                np_[q] = n1[q] - 0.5 * gyn[q];
            }

            /* each face takes the sound speed of the neighbour across it */
            double cs2w = gam_cs2(gamma, w1), cs2e = gam_cs2(gamma, e1);
            double cs2s = gam_cs2(gamma, s1), cs2n = gam_cs2(gamma, n1);
            double hc = scale_height(ms, xc, yc, c);

            double fw[NF], fe[NF], fs[NF], fn[NF], u[NF];
            gam_hlle(wm, wp, fw, cs2w, 0, gamma);
            gam_hlle(em, ep, fe, cs2e, 0, gamma);
            gam_hlle(sm, sp, fs, cs2s, 1, gamma);
            gam_hlle(nm, np_, fn, cs2n, 1, gamma);

            if (alpha > 0.0) {
                double tw[4], te[4], ts[4], tn[4], tc[4];
                gam_strain(gxw, gyw, dx, dy, tw);
                gam_strain(gxe, gye, dx, dy, te);
                gam_strain(gxs, gys, dx, dy, ts);
                gam_strain(gxn, gyn, dx, dy, tn);
                gam_strain(gxc, gyc, dx, dy, tc);
                double cs2c = gam_cs2(gamma, c);
                double hw = scale_height(ms, xl, yc, w1);
                double he = scale_height(ms, xr, yc, e1);
                double hs = scale_height(ms, xc, yl, s1);
                double hn = scale_height(ms, xc, yr, n1);
                double nuc = alpha * hc * sqrt(cs2c);
                double nuw = alpha * hw * sqrt(cs2w);
                double nue = alpha * he * sqrt(cs2e);
                double nus = alpha * hs * sqrt(cs2s);
                double nun = alpha * hn * sqrt(cs2n);

                fw[1] -= 0.5 * (nuw * w1[0] * tw[0] + nuc * c[0] * tc[0]);
                fw[2] -= 0.5 * (nuw * w1[0] * tw[1] + nuc * c[0] * tc[1]);
                fe[1] -= 0.5 * (nuc * c[0] * tc[0] + nue * e1[0] * te[0]);
                fe[2] -= 0.5 * (nuc * c[0] * tc[1] + nue * e1[0] * te[1]);
                fs[1] -= 0.5 * (nus * s1[0] * ts[2] + nuc * c[0] * tc[2]);
                fs[2] -= 0.5 * (nus * s1[0] * ts[3] + nuc * c[0] * tc[3]);
                fn[1] -= 0.5 * (nuc * c[0] * tc[2] + nun * n1[0] * tn[2]);
                fn[2] -= 0.5 * (nuc * c[0] * tc[3] + nun * n1[0] * tn[3]);

                fw[3] -= 0.5 * (nuw * w1[0] * tw[0] * w1[1] + nuc * c[0] * tc[0] * c[1]);
                fe[3] -= 0.5 * (nuc * c[0] * tc[0] * c[1] + nue * e1[0] * te[0] * e1[1]);
                fw[3] -= 0.5 * (nuw * w1[0] * tw[1] * w1[2] + nuc * c[0] * tc[1] * c[2]);
                fe[3] -= 0.5 * (nuc * c[0] * tc[1] * c[2] + nue * e1[0] * te[1] * e1[2]);
                fs[3] -= 0.5 * (nus * s1[0] * ts[2] * s1[1] + nuc * c[0] * tc[2] * c[1]);
                fn[3] -= 0.5 * (nuc * c[0] * tc[2] * c[1] + nun * n1[0] * tn[2] * n1[1]);
                fs[3] -= 0.5 * (nus * s1[0] * ts[3] * s1[2] + nuc * c[0] * tc[3] * c[2]);
                fn[3] -= 0.5 * (nuc * c[0] * tc[3] * c[2] + nun * n1[0] * tn[3] * n1[2]);
            }

            gam_prim_to_cons(c, u, gamma);
            gam_buffer(&buf, xc, yc, dt, u, gamma);
            for (int k = 0; k < 2; ++k) {
                double du[NF];
                gam_mass_source(&ms[k], xc, yc, dt, c, hc, constant_softening, gamma, du);
                for (int q = 0; q < NF; ++q)
                    u[q] += du[q];
            }
            gam_cooling(cooling, mach_ceiling, dt, c, u, gamma);
            for (int q = 0; q < NF; ++q) {
                u[q] -= ((fe[q] - fw[q]) / dx + (fn[q] - fs[q]) / dy) * dt;
                u[q] = (1.0 - a) * u[q] + a * un[q];
            }
            gam_cons_to_prim(u, pwr + at(i, j, nj), vmax, rho_floor, p_floor, gamma);
        }
    }
}

/* cbdgam_2d.c:685-708 */
void oracle_cbdgam_2d_wavespeed(int ni, int nj, const double *prim, double *ws, double gamma)
{
#pragma omp parallel for
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) {
            const double *p = prim + at(i, j, nj);
            ws[(size_t)(i + NG) * (nj + 2 * NG) + (j + NG)] = gam_max_wavespeed(p, gam_cs2(gamma, p));
        }
}

/* cbdgam_2d.c:710-729 */
void oracle_cbdgam_2d_primitive_to_conserved(int ni, int nj, const double *prim, double *cons, double gamma)
{
#pragma omp parallel for
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j)
            gam_prim_to_cons(prim + at(i, j, nj), cons + at(i, j, nj), gamma);
}

/* cbdgam_2d.c:731-784: one mass's source terms with dt = 1 */
void oracle_cbdgam_2d_point_mass_source_term(int ni, int nj, double xl0, double xr0, double yl0, double yr0,
                                             double x1, double y1, double vx1, double vy1, double mass1,
                                             double soft1, double rate1, double radius1, int model1, double x2,
                                             double y2, double vx2, double vy2, double mass2, double soft2,
                                             double rate2, double radius2, int model2, int which_mass,
                                             const double *prim, double *rate_out, int constant_softening,
                                             double gamma)
{
    const gam_mass_t ms[2] = {{x1, y1, vx1, vy1, mass1, soft1, rate1, radius1, model1},
                              {x2, y2, vx2, vy2, mass2, soft2, rate2, radius2, model2}};
    const double dx = (xr0 - xl0) / ni;
    const double dy = (yr0 - yl0) / nj;
#pragma omp parallel for
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) {
            double xc = xl0 + (i + 0.5) * dx, yc = yl0 + (j + 0.5) * dy;
            const double *p = prim + at(i, j, nj);
            double h = scale_height(ms, xc, yc, p);
            gam_mass_source(&ms[which_mass - 1], xc, yc, 1.0, p, h, constant_softening, gamma,
                            rate_out + at(i, j, nj));
        }
}
