/*
 * grid.c -- oracle restatement of MACH-2D's grid generation and metrics.
 * TEST INFRASTRUCTURE ONLY (see m2d_oracle.h).  Parity unpinned.
 *   nozzle contour N01   src/user/internal_flow/mod_intflow_geometry.f90:29-225
 *   C01 cosine nozzle    new geometry (no counterpart in the reference): the
 *                        wall r(x') = 1 + (Rin-1)/2 (1-cos(pi x'/Lc)) on
 *                        [-Lc,0] and 1 + (Rout-1)/2 (1-cos(pi x'/Ld)) on
 *                        [0,Ld], with x = x' + Lc so that the inlet is x = 0
 *                        like N01 (the inlet boundary conditions of
 *                        mod_intflow.f90:244,907 measure distances from x = 0).
 *   kg = 1, 2            src/grid/mod_grid_procedures.f90:152-279, 349-420
 *   centroids, metrics,
 *   radius               src/grid/mod_grid.f90:237-723
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "m2d_oracle.h"

#define F(v, np) (v)[(size_t)(np) - 1]

/* x**n with an integer exponent: gfortran lowers it to libgcc's __powidf2
 * (square and multiply), not to pow(). */
static double powi(double x, int m)
{
    unsigned int n = m < 0 ? -(unsigned int)m : (unsigned int)m;
    double y = (n % 2) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

void orc_nozzle_boundary_c01(int nx, int ny, double Lc, double Ld, double Rin,
                             double Rout, double *x, double *y)
{
    const double pi = acos(-1.0);
    const double x0 = 0.0, x6 = Lc + Ld;
    for (int i = 1; i <= nx - 1; i++) {
        int np = nx * (ny - 2) + i;
        double xi = ((double)(i - 1) / (double)(nx - 2)) * (x6 - x0) + x0;
        double xq = xi - Lc, r;
        if (xq <= 0.0) r = 1.0 + 0.5 * (Rin - 1.0) * (1.0 - cos(pi * xq / Lc));
        else r = 1.0 + 0.5 * (Rout - 1.0) * (1.0 - cos(pi * xq / Ld));
        F(x, np) = xi;
        F(y, np) = r;
        F(x, i) = xi;
        F(y, i) = 0.0;
    }
}

static double nozzle01(double x, double x0, double x1, double x2, double x3,
    double x4, double x5, double x6, double y0, double y1, double y2, double y3,
    double y4, double y5, double y6, double Rc1, double Rc2, double Rc3)
{
    (void)y3; (void)y6;
    double y;
    if (x0 <= x && x <= x1) y = y0;
    else if (x1 <= x && x <= x2) y = y1 - Rc1 + sqrt(Rc1 * Rc1 - (x - x1) * (x - x1));
    else if (x2 <= x && x <= x3) y = y2 + (y3 - y2) / (x3 - x2) * (x - x2);
    else if (x3 <= x && x <= x4) y = y4 + Rc2 - sqrt(Rc2 * Rc2 - (x - x4) * (x - x4));
    else if (x4 <= x && x <= x5) y = y4 + Rc3 - sqrt(Rc3 * Rc3 - (x - x4) * (x - x4));
    else if (x5 <= x && x <= x6) y = y5 + (y6 - y5) / (x6 - x5) * (x - x5);
    else y = NAN;
    return y;
}

void orc_nozzle_boundary_n01(int nx, int ny, double Rth, double Rin, double Rout,
    double Rc1, double Rc2, double Rc3, double alf_deg, double bet_deg,
    double Lchamb, double *x, double *y)
{
    const double pi = acos(-1.0);
    double alf = alf_deg * pi / 180.0, bet = bet_deg * pi / 180.0;
    double x0, x1, x2, x3, x4, x5, x6, y0, y1, y2, y3, y4, y5, y6, ra, rb, la, lb;
    x0 = 0.0; y0 = Rin;
    x1 = Lchamb; y1 = Rin;
    x2 = x1 + Rc1 * sin(alf);
    y2 = y1 - Rc1 * (1.0 - cos(alf));
    y4 = Rth;
    y3 = y4 + Rc2 * (1.0 - cos(alf));
    ra = y2 - y3;
    la = ra / tan(alf);
    x3 = x2 + la;
    x4 = x3 + Rc2 * sin(alf);
    x5 = x4 + Rc3 * sin(bet);
    y5 = y4 + Rc3 * (1.0 - cos(bet));
    y6 = Rout;
    rb = y6 - y5;
    lb = rb / tan(bet);
    x6 = x5 + lb;
    for (int i = 1; i <= nx - 1; i++) {
        int np = nx * (ny - 2) + i;
        double xi = ((double)(i - 1) / (double)(nx - 2)) * (x6 - x0) + x0;
        F(x, np) = xi;
        F(y, np) = nozzle01(xi, x0, x1, x2, x3, x4, x5, x6, y0, y1, y2, y3, y4, y5, y6,
                            Rc1, Rc2, Rc3);
        F(x, i) = xi;
        F(y, i) = 0.0;
    }
}

/* mod_grid_procedures.f90:152-185 */
void orc_get_uniform_grid(int nx, int ny, double *x, double *y)
{
    for (int i = 1; i <= nx - 1; i++) {
        double xi = F(x, i), yi = F(y, i);
        int np = nx * (ny - 2) + i;
        double xf = F(x, np), yf = F(y, np);
        double dx = (xf - xi) / (ny - 2), dy = (yf - yi) / (ny - 2);
        for (int j = 2; j <= ny - 2; j++) {
            np = nx * (j - 1) + i;
            F(x, np) = F(x, np - nx) + dx;
            F(y, np) = F(y, np - nx) + dy;
        }
    }
}

/* mod_grid_procedures.f90:349-420 */
double orc_get_gp_ratio(int n, double r)
{
    int nit = 1000, i;
    double tol = 1.0e-15, qi, qf, qm = 0.0;
#define FQ(q) (powi((q), n) + r * (1.0 - (q)) - 1.0)
    if (r < n) { qi = 0.1; qf = 1.0 - 1.0e-15; }
    else { qi = 1.0 + 1.0e-15; qf = 10.0; }
    for (i = 1; i <= nit; i++) {
        qm = 0.5 * qi + 0.5 * qf;
        if (0.0 < FQ(qi) * FQ(qm)) qi = qm; else qf = qm;
        if (fabs(qf - qi) < tol) break;
    }
#undef FQ
    return qm;
}

/* mod_grid_procedures.f90:60-85,128-148 */
static void gp_distribution(int isReversed, int N, double r, double *t)
{
    double q = orc_get_gp_ratio(N - 1, r);
    t[0] = 0.0;
    for (int j = 2; j <= N - 1; j++) t[j - 1] = t[j - 2] + powi(q, j - 2) / r;
    t[N - 1] = 1.0;
    if (isReversed) {
        int n = N - 1;
        double *dt = (double *)malloc(sizeof(double) * (size_t)n);
        for (int i = 1; i <= n; i++) dt[n - i] = t[i] - t[i - 1];
        for (int i = 2; i <= n; i++) t[i - 1] = t[i - 2] + dt[i - 2];
        free(dt);
    }
}

/* mod_grid_procedures.f90:235-279 */
void orc_get_pg_grid(int isReversed, double a1, int nx, int ny, double *x, double *y)
{
    double *tv = (double *)malloc(sizeof(double) * (size_t)(ny - 1));
    for (int i = 1; i <= nx - 1; i++) {
        double xi = F(x, i), yi = F(y, i);
        int np = nx * (ny - 2) + i;
        double xf = F(x, np), yf = F(y, np);
        double r = sqrt((xf - xi) * (xf - xi) + (yf - yi) * (yf - yi)) / a1;
        gp_distribution(isReversed, ny - 1, r, tv);
        for (int j = 1; j <= ny - 3; j++) {
            int npn = nx * (j - 1) + i + nx;
            F(x, npn) = xi + (xf - xi) * tv[j];
            F(y, npn) = yi + (yf - yi) * tv[j];
        }
    }
    free(tv);
}

/* mod_grid.f90:237-300 */
void orc_get_real_centroids_xy(int opt, int nx, int ny, const double *x,
                               const double *y, double *xp, double *yp)
{
    size_t N = (size_t)nx * (size_t)ny;
    memset(xp, 0, N * sizeof(double));
    memset(yp, 0, N * sizeof(double));
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npw = np - 1, npsw = nps - 1;
            if (opt == 1) {
                F(xp, np) = (F(x, np) + F(x, npw) + F(x, npsw) + F(x, nps)) / 4.0;
                F(yp, np) = (F(y, np) + F(y, npw) + F(y, npsw) + F(y, nps)) / 4.0;
            } else {
                double A1 = 0.5 * (F(x, npsw) * (F(y, nps) - F(y, np))
                                   + F(x, nps) * (F(y, np) - F(y, npsw))
                                   + F(x, np) * (F(y, npsw) - F(y, nps)));
                double A2 = 0.5 * (F(x, npsw) * (F(y, np) - F(y, npw))
                                   + F(x, np) * (F(y, npw) - F(y, npsw))
                                   + F(x, npw) * (F(y, npsw) - F(y, np)));
                F(xp, np) = ((F(x, npsw) + F(x, nps) + F(x, np)) * A1
                             + (F(x, npsw) + F(x, np) + F(x, npw)) * A2) / (3.0 * (A1 + A2));
                F(yp, np) = ((F(y, npsw) + F(y, nps) + F(y, np)) * A1
                             + (F(y, npsw) + F(y, np) + F(y, npw)) * A2) / (3.0 * (A1 + A2));
            }
        }
}

/* mod_grid.f90:304-558 */
void orc_get_metrics(int nx, int ny, const double *x, const double *y,
    const double *xp, const double *yp, double *xe, double *ye, double *xen,
    double *yen, double *xk, double *yk, double *xke, double *yke, double *Jp,
    double *Je, double *Jn, double *alphae, double *gamman, double *betae,
    double *betan)
{
    size_t N = (size_t)nx * (size_t)ny;
    double *all[] = {xe, ye, xen, yen, xk, yk, xke, yke, Jp, Je, Jn, alphae, gamman, betae, betan};
    for (int k = 0; k < 15; k++) memset(all[k], 0, N * sizeof(double));
    int i, j, np, nps, npw, npe, npn, npsw;
    double fw, fe, fs, fn, xkp, xep, ykp, yep;
    for (j = 2; j <= ny - 1; j++)
        for (i = 1; i <= nx - 1; i++) {
            np = nx * (j - 1) + i; nps = np - nx;
            F(xe, np) = F(x, np) - F(x, nps);
            F(ye, np) = F(y, np) - F(y, nps);
            F(alphae, np) = F(xe, np) * F(xe, np) + F(ye, np) * F(ye, np);
        }
    for (j = 1; j <= ny - 1; j++)
        for (i = 2; i <= nx - 1; i++) {
            np = nx * (j - 1) + i; npw = np - 1;
            F(xk, np) = F(x, np) - F(x, npw);
            F(yk, np) = F(y, np) - F(y, npw);
            F(gamman, np) = F(xk, np) * F(xk, np) + F(yk, np) * F(yk, np);
        }
    for (j = 2; j <= ny - 1; j++)
        for (i = 2; i <= nx - 2; i++) {
            np = nx * (j - 1) + i; npe = np + 1;
            F(xke, np) = F(xp, npe) - F(xp, np);
            F(yke, np) = F(yp, npe) - F(yp, np);
        }
    i = 2;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; nps = np - nx; npw = np - 1; npsw = nps - 1;
        fw = (F(x, npw) + F(x, npsw)) / 2.0;
        fe = (F(x, np) + F(x, nps)) / 2.0;
        F(xke, npw) = -3.0 * fw + 4.0 * F(xp, np) - fe;
        fw = (F(y, npw) + F(y, npsw)) / 2.0;
        fe = (F(y, np) + F(y, nps)) / 2.0;
        F(yke, npw) = -3.0 * fw + 4.0 * F(yp, np) - fe;
    }
    i = nx - 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; nps = np - nx; npw = np - 1; npsw = nps - 1;
        fw = (F(x, npw) + F(x, npsw)) / 2.0;
        fe = (F(x, np) + F(x, nps)) / 2.0;
        F(xke, np) = fw - 4.0 * F(xp, np) + 3.0 * fe;
        fw = (F(y, npw) + F(y, npsw)) / 2.0;
        fe = (F(y, np) + F(y, nps)) / 2.0;
        F(yke, np) = fw - 4.0 * F(yp, np) + 3.0 * fe;
    }
    for (j = 2; j <= ny - 2; j++)
        for (i = 2; i <= nx - 1; i++) {
            np = nx * (j - 1) + i; npn = np + nx;
            F(xen, np) = F(xp, npn) - F(xp, np);
            F(yen, np) = F(yp, npn) - F(yp, np);
        }
    j = 2;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i; nps = np - nx; npw = np - 1; npsw = nps - 1;
        fs = (F(x, nps) + F(x, npsw)) / 2.0;
        fn = (F(x, np) + F(x, npw)) / 2.0;
        F(xen, nps) = -3.0 * fs + 4.0 * F(xp, np) - fn;
        fs = (F(y, nps) + F(y, npsw)) / 2.0;
        fn = (F(y, np) + F(y, npw)) / 2.0;
        F(yen, nps) = -3.0 * fs + 4.0 * F(yp, np) - fn;
    }
    j = ny - 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i; nps = np - nx; npw = np - 1; npsw = nps - 1;
        fs = (F(x, nps) + F(x, npsw)) / 2.0;
        fn = (F(x, np) + F(x, npw)) / 2.0;
        F(xen, np) = fs - 4.0 * F(xp, np) + 3.0 * fn;
        fs = (F(y, nps) + F(y, npsw)) / 2.0;
        fn = (F(y, np) + F(y, npw)) / 2.0;
        F(yen, np) = fs - 4.0 * F(yp, np) + 3.0 * fn;
    }
    for (j = 2; j <= ny - 1; j++)
        for (i = 1; i <= nx - 1; i++) {
            np = nx * (j - 1) + i;
            F(betae, np) = F(xke, np) * F(xe, np) + F(yke, np) * F(ye, np);
            F(Je, np) = 1.0 / (F(xke, np) * F(ye, np) - F(xe, np) * F(yke, np));
        }
    for (j = 1; j <= ny - 1; j++)
        for (i = 2; i <= nx - 1; i++) {
            np = nx * (j - 1) + i;
            F(betan, np) = F(xk, np) * F(xen, np) + F(yk, np) * F(yen, np);
            F(Jn, np) = 1.0 / (F(xk, np) * F(yen, np) - F(xen, np) * F(yk, np));
        }
    for (j = 2; j <= ny - 1; j++)
        for (i = 2; i <= nx - 1; i++) {
            np = nx * (j - 1) + i; nps = np - nx; npw = np - 1; npsw = nps - 1;
            fw = (F(x, npw) + F(x, npsw)) / 2.0;
            fe = (F(x, np) + F(x, nps)) / 2.0;
            fs = (F(x, nps) + F(x, npsw)) / 2.0;
            fn = (F(x, np) + F(x, npw)) / 2.0;
            xkp = fe - fw; xep = fn - fs;
            fw = (F(y, npw) + F(y, npsw)) / 2.0;
            fe = (F(y, np) + F(y, nps)) / 2.0;
            fs = (F(y, nps) + F(y, npsw)) / 2.0;
            fn = (F(y, np) + F(y, npw)) / 2.0;
            ykp = fe - fw; yep = fn - fs;
            F(Jp, np) = 1.0 / (xkp * yep - xep * ykp);
        }
    for (size_t k = 0; k < N; k++) { Je[k] = fabs(Je[k]); Jn[k] = fabs(Jn[k]); Jp[k] = fabs(Jp[k]); }
}

/* mod_grid.f90:562-723 */
void orc_get_radius(int coord, int nx, int ny, const double *y, const double *yp,
                    double *radius, double *re, double *rn, double *rp)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (size_t k = 0; k < N; k++) { radius[k] = 1.0; re[k] = 1.0; rn[k] = 1.0; rp[k] = 1.0; }
    if (coord != 1) return;
    int i, j, np;
    memcpy(radius, y, N * sizeof(double));
    for (i = 1; i <= nx - 1; i++)
        for (j = 2; j <= ny - 1; j++) { np = nx * (j - 1) + i; F(re, np) = (F(y, np) + F(y, np - nx)) / 2.0; }
    for (i = 2; i <= nx - 1; i++)
        for (j = 1; j <= ny - 1; j++) { np = nx * (j - 1) + i; F(rn, np) = (F(y, np) + F(y, np - 1)) / 2.0; }
    memcpy(rp, yp, N * sizeof(double));
    j = 1;
    for (i = 2; i <= nx - 1; i++) { np = i; F(rp, np) = F(rn, np) - F(rp, np + nx) + F(rn, np); }
    j = ny;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i; int nps = np - nx;
        F(rp, np) = F(rn, nps) - F(rp, nps) + F(rn, nps);
    }
    i = 1;
    for (j = 2; j <= ny - 1; j++) { np = nx * (j - 1) + i; F(rp, np) = F(re, np) - F(rp, np + 1) + F(re, np); }
    i = nx;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; int npw = np - 1;
        F(rp, np) = F(re, npw) - F(rp, npw) + F(re, npw);
    }
    np = 1;
    F(rp, np) = 4.0 * F(y, np) - F(rp, np + 1) - F(rp, np + nx) - F(rp, np + nx + 1);
    np = nx;
    F(rp, np) = 4.0 * F(y, np - 1) - F(rp, np - 1) - F(rp, np + nx) - F(rp, np + nx - 1);
    np = nx * (ny - 1) + 1;
    F(rp, np) = 4.0 * F(y, np - nx) - F(rp, np + 1) - F(rp, np - nx) - F(rp, np - nx + 1);
    np = nx * (ny - 1) + nx;
    F(rp, np) = 4.0 * F(y, np - nx - 1) - F(rp, np - 1) - F(rp, np - nx) - F(rp, np - nx - 1);
}
