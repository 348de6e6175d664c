/*
 * tstepper.c -- oracle restatement of MACH-2D's time steppers.
 * TEST INFRASTRUCTURE ONLY (see m2d_oracle.h).  Parity unpinned.
 *   SCARBOROUGH  src/tstepper/mod_tstepper_scarborough.f90:40-123, 260-320
 *   RAMP         src/tstepper/mod_tstepper_ramp.f90:41-54
 */
#include <math.h>
#include <stddef.h>
#include "m2d_oracle.h"

#define F(v, np) (v)[(size_t)(np) - 1]
#define A(np, k) a[((size_t)(k) - 1) * N + (size_t)(np) - 1]

double orc_tstepper_dt0_scarborough(int nx, int ny, const double *Jp,
                                    const double *u, const double *v)
{
    double dt = 1.0e10;
    for (int i = 2; i <= nx - 1; i++)
        for (int j = 2; j <= ny - 1; j++) {
            int np = nx * (j - 1) + i;
            double aux = 1.0 / sqrt(F(Jp, np) * (F(u, np) * F(u, np) + F(v, np) * F(v, np)));
            if (dt > aux) dt = aux;
        }
    return dt * 0.25;
}

/* sum(abs(a(np,1:4))) + sum(abs(a(np,6:9))), each sum sequential */
double orc_get_mean_cc_9d(int nx, int ny, const double *a)
{
    size_t N = (size_t)nx * (size_t)ny;
    double m = 0.0;
    for (int i = 2; i <= nx - 1; i++)
        for (int j = 2; j <= ny - 1; j++) {
            int np = nx * (j - 1) + i;
            double s1 = 0.0, s2 = 0.0;
            for (int k = 1; k <= 4; k++) s1 = s1 + fabs(A(np, k));
            for (int k = 6; k <= 9; k++) s2 = s2 + fabs(A(np, k));
            m = (s1 + s2) / fabs(A(np, 5)) + m;
        }
    return m / (double)((nx - 2) * (ny - 2));
}

double orc_get_mean_cc_5d(int nx, int ny, const double *a)
{
    size_t N = (size_t)nx * (size_t)ny;
    double m = 0.0;
    for (int i = 2; i <= nx - 1; i++)
        for (int j = 2; j <= ny - 1; j++) {
            int np = nx * (j - 1) + i;
            double s1 = 0.0, s2 = 0.0;
            for (int k = 1; k <= 2; k++) s1 = s1 + fabs(A(np, k));
            for (int k = 4; k <= 5; k++) s2 = s2 + fabs(A(np, k));
            m = (s1 + s2) / fabs(A(np, 3)) + m;
        }
    return m / (double)((nx - 2) * (ny - 2));
}

/* c = max(curef, cvref, ctref, cpref).  With constant properties and the Euler
 * model the T matrix is never assembled (at = 0), so ctref = 0/0 = NaN and the
 * result of max() depends on how the compiler orders the operands.
 * nan_policy 0 drops NaN operands; nan_policy 1 propagates them. */
static double max4(double a, double b, double c, double d, int nan_policy)
{
    double v[4] = {a, b, c, d};
    double m = NAN;
    if (nan_policy == 1) {
        for (int k = 0; k < 4; k++) if (isnan(v[k])) return NAN;
        m = a;
        for (int k = 1; k < 4; k++) if (v[k] > m) m = v[k];
        return m;
    }
    for (int k = 0; k < 4; k++) {
        if (isnan(v[k])) continue;
        if (isnan(m) || v[k] > m) m = v[k];
    }
    return m;
}

double orc_tstepper_dt_scarborough(int nx, int ny, double dt, const double *au,
    const double *av, const double *at, const double *ap, double h0, double mincc,
    double maxcc, int nan_policy)
{
    double curef = orc_get_mean_cc_9d(nx, ny, au);
    double cvref = orc_get_mean_cc_9d(nx, ny, av);
    double ctref = orc_get_mean_cc_9d(nx, ny, at);
    double cpref = orc_get_mean_cc_5d(nx, ny, ap);
    double c = max4(curef, cvref, ctref, cpref, nan_policy);
    double h;
    if (c < mincc) h = h0 * sqrt(1.0 - c / mincc);
    else if (maxcc < c) h = -(h0 * sqrt(c / maxcc - 1.0));
    else h = 0.0;
    return dt * (1.0 + h);
}

/* mod_tstepper_ramp.f90:41-54 */
double orc_tstepper_dt_ramp(int it, double dt1, double dt2, int it1, int it2)
{
    double dt = 0.0;
    if (it + 1 <= it1) dt = dt1;
    if (it + 1 > it1 && it + 1 < it2)
        dt = dt1 + (dt2 - dt1) * (double)(it + 1 - it1) / (double)(it2 - it1);
    if (it + 1 >= it2) dt = dt2;
    return dt;
}
