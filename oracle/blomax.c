/*
 * blomax.c -- Baldwin-Lomax eddy viscosity (src/equations/blomax.f90).
 * TEST INFRASTRUCTURE ONLY (see m2d_oracle.h).
 *
 * The reference computes mu_t column by column along the eta lines from the
 * north wall (j = ny-1 down to 2): wall shear stress from the first north
 * face, inner and outer eddy viscosities of the two-layer model, the outer
 * length scale from the maximum of F(y) refined by a three-point parabola,
 * and the switch at the first sign change of nu_outer - nu_inner.
 * Constant integer powers follow gfortran -O2's expansion (x**2 = x*x,
 * x**6 = (x*x*x)**2).
 */
#include <math.h>
#include "m2d_oracle.h"

/* model constants, blomax.f90:5-10 */
static double bl_kappa = 0.40, bl_Aop = 26.0, bl_alpha = 0.0168, bl_Ccp = 1.6, bl_Ckleb = 0.3,
              bl_Cwk = 1.0;

void orc_set_blomax_coefficients(double kappa, double Aop, double alpha, double Ccp, double Ckleb,
                                 double Cwk)
{   /* blomax.f90:25-43 */
    bl_kappa = kappa; bl_Aop = Aop; bl_alpha = alpha; bl_Ccp = Ccp; bl_Ckleb = Ckleb; bl_Cwk = Cwk;
}

#define IDX(i, j) ((long)nx * ((j) - 1) + (i) - 1)

/* vorticity at the real nodes from the corner coordinates, blomax.f90:83-148 */
static double omega_at(int nx, const double *x, const double *y, const double *Jp, const double *u,
                       const double *v, int i, int j)
{
    const long np = IDX(i, j), nps = np - nx, npw = np - 1, npsw = nps - 1, npn = np + nx, npe = np + 1;
    const double xkp = 0.5 * (x[np] + x[nps] - x[npw] - x[npsw]);
    const double ykp = 0.5 * (y[np] + y[nps] - y[npw] - y[npsw]);
    const double xep = 0.5 * (x[np] + x[npw] - x[nps] - x[npsw]);
    const double yep = 0.5 * (y[np] + y[npw] - y[nps] - y[npsw]);
    return 0.5 * Jp[np] * fabs((v[npe] - v[npw]) * yep - (v[npn] - v[nps]) * ykp
                               + (u[npe] - u[npw]) * xep - (u[npn] - u[nps]) * xkp);
}

/* parabola through three points: its maximum if it opens downwards and the
 * vertex lies in [x1, x3], else the largest sample, blomax.f90:244-283 */
static void get_maximum(const double *x, const double *y, double *xmax, double *ymax)
{
    const double a1 = (y[1] - y[0]) / (x[1] - x[0]);
    const double a2 = ((y[2] - y[1]) / (x[2] - x[1]) - a1) / (x[2] - x[0]);
    int k = 0;
    for (int m = 1; m < 3; m++) if (y[m] > y[k]) k = m;
    if (a2 < 0.0) {
        const double xm = 0.5 * (x[0] + x[1] - a1 / a2);
        if (x[0] <= xm && xm <= x[2]) {
            *xmax = xm;
            *ymax = y[0] + a1 * (xm - x[0]) + a2 * (xm - x[0]) * (xm - x[1]);
            return;
        }
    }
    *ymax = y[k];
    *xmax = x[k];
}

/* dimensionless eddy viscosity along one eta line, blomax.f90:151-240.
 * work holds 4n doubles. */
static void get_nut_plus(int n, double Udp, const double *yplus, const double *omgplus, double *nutplus,
                         double *work)
{
    double *f = work, *nutip = work + n, *nutop = work + 2 * n;
    double amax = 0.0;
    for (int k = 0; k < n; k++) {
        const double t = fabs(omgplus[k]);
        if (k == 0 || t > amax) amax = t;
    }
    if (amax < 1.0e-15) {
        for (int k = 0; k < n; k++) nutplus[k] = 0.0;
        return;
    }
    for (int k = 0; k < n; k++) {
        const double lmp = bl_kappa * yplus[k] * (1.0 - exp(-yplus[k] / bl_Aop));
        nutip[k] = lmp * lmp * fabs(omgplus[k]);
        f[k] = lmp * fabs(omgplus[k]) / bl_kappa;
    }
    int km = 0;                                   /* maxloc: first maximum */
    for (int k = 1; k < n; k++) if (f[k] > f[km]) km = k;
    const int k0 = (km == 0) ? 0 : (km == n - 1 ? n - 3 : km - 1);
    double ymaxp, Fmaxp;
    get_maximum(yplus + k0, f + k0, &ymaxp, &Fmaxp);
    const double w1 = ymaxp * Fmaxp, w2 = bl_Cwk * ymaxp * (Udp * Udp) / Fmaxp;
    const double Fwakep = (w2 < w1) ? w2 : w1;
    for (int k = 0; k < n; k++) {
        const double c = bl_Ckleb * yplus[k] / ymaxp;
        const double c3 = c * c * c;
        nutop[k] = bl_alpha * bl_Ccp * Fwakep / (1.0 + 5.5 * (c3 * c3));
        f[k] = nutop[k] - nutip[k];
    }
    for (int k = 1; k < n; k++) {
        if (f[k - 1] * f[k] <= 0.0) {
            for (int m = 0; m < k; m++) nutplus[m] = nutip[m];
            for (int m = k; m < n; m++) nutplus[m] = nutop[m];
            return;
        }
    }
    for (int k = 0; k < n; k++) nutplus[k] = nutip[k];
}

void orc_get_eddy_viscosity_blomax(int nx, int ny, const double *x, const double *y, const double *xp,
                                   const double *yp, const double *xk, const double *yk, const double *Jp,
                                   const double *Jn, const double *vln, const double *ro, const double *ron,
                                   const double *u, const double *v, double *vtp, double *work)
{   /* blomax.f90:285-395; work: 9 (ny-2) doubles */
    const int n = ny - 2;
    double *yplus = work, *omgplus = work + n, *nutplus = work + 2 * n, *sp = work + 3 * n,
           *scratch = work + 4 * n, *dw = work + 8 * n;
    (void)sp;
    const int j = ny - 1;
    for (int i = 2; i <= nx - 1; i++) {
        const long np = IDX(i, j), npw = np - 1;
        const double tauw = fabs(vln[np] * Jn[np] * 2.0 * (u[np] * xk[np] + v[np] * yk[np]));
        const double row = ron[np], vlw = vln[np];
        const double nuw = vlw / row;
        const double utau = sqrt(fabs(tauw / row));
        const double xw = 0.5 * (x[np] + x[npw]);
        const double yw = 0.5 * (y[np] + y[npw]);
        double Udif = 0.0;
        for (int k = ny - 1; k >= 2; k--) {      /* line index m = ny - k - 1, from the wall */
            const int m = ny - k - 1;
            const long npl = IDX(i, k);
            const double s = sqrt(u[npl] * u[npl] + v[npl] * v[npl]);
            if (m == 0 || s > Udif) Udif = s;
            const double dx = xp[npl] - xw, dy = yp[npl] - yw;
            dw[m] = sqrt(dx * dx + dy * dy);
            yplus[m] = dw[m] * utau / nuw;
            omgplus[m] = omega_at(nx, x, y, Jp, u, v, i, k) * nuw / (utau * utau);
        }
        get_nut_plus(n, Udif / utau, yplus, omgplus, nutplus, scratch);
        for (int k = ny - 1; k >= 2; k--) {
            const long npl = IDX(i, k);
            vtp[npl] = ro[npl] * nutplus[ny - k - 1] * nuw;
        }
    }
}

void orc_get_eddy_viscosity_fictitious(int nx, int ny, double *phi)
{   /* blomax.f90:397-490: copy the adjacent real value, corners diagonally */
    for (int i = 2; i <= nx - 1; i++) {
        phi[IDX(i, 1)] = phi[IDX(i, 2)];
        phi[IDX(i, ny)] = phi[IDX(i, ny - 1)];
    }
    for (int j = 2; j <= ny - 1; j++) {
        phi[IDX(1, j)] = phi[IDX(2, j)];
        phi[IDX(nx, j)] = phi[IDX(nx - 1, j)];
    }
    phi[IDX(1, 1)] = phi[IDX(2, 2)];
    phi[IDX(nx, 1)] = phi[IDX(nx - 1, 2)];
    phi[IDX(1, ny)] = phi[IDX(2, ny - 1)];
    phi[IDX(nx, ny)] = phi[IDX(nx - 1, ny - 1)];
}

/* Wiring of the eddy viscosity into the momentum and energy equations, which
 * the reference leaves out (it never calls get_eddy_viscosity_blomax; its
 * post-processing zeroes vtp, mod_intflow_postp.f90:57,63).  Effective
 * viscosity mu + mu_t and conductivity k + cp mu_t / Pr_t at the nodes; at
 * the east and north faces the arithmetic means of mu_t and of cp mu_t of the
 * two cells; the north faces of the last real row (the wall) and the faces
 * past the last column or row keep the laminar values. */
void orc_add_eddy_viscosity(int nx, int ny, int ktm, double mu, double kappa, double prt, const double *vtp,
                            const double *cp, double *vlp, double *vle, double *vln, double *kp, double *ke,
                            double *kn)
{
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            const long np = IDX(i, j);
            const double mp = ktm ? vlp[np] : mu, me = ktm ? vle[np] : mu, mn = ktm ? vln[np] : mu;
            const double kpl = ktm ? kp[np] : kappa, kel = ktm ? ke[np] : kappa, knl = ktm ? kn[np] : kappa;
            const double tp = cp[np] * vtp[np];
            vlp[np] = mp + vtp[np];
            kp[np] = kpl + tp / prt;
            if (i < nx) {
                const double te = cp[np + 1] * vtp[np + 1];
                vle[np] = me + 0.5 * (vtp[np] + vtp[np + 1]);
                ke[np] = kel + 0.5 * (tp + te) / prt;
            } else {
                vle[np] = me;
                ke[np] = kel;
            }
            if (j < ny - 1) {
                const double tn = cp[np + nx] * vtp[np + nx];
                vln[np] = mn + 0.5 * (vtp[np] + vtp[np + nx]);
                kn[np] = knl + 0.5 * (tp + tn) / prt;
            } else {
                vln[np] = mn;
                kn[np] = knl;
            }
        }
}
