/*
 * coef.c -- oracle restatement of MACH-2D's `module coefficients`
 * (src/equations/mach2d_coef.f90).  TEST INFRASTRUCTURE ONLY (see
 * m2d_oracle.h).  Parity unpinned.  Each routine follows the Fortran loop
 * by loop, in the same evaluation order; SIGN(0.5,x) is copysign, as gfortran
 * implements it.
 */
#include <math.h>
#include <string.h>
#include "m2d_oracle.h"

#define F(v, np) (v)[(size_t)(np) - 1]
#define A(np, k) a[((size_t)(k) - 1) * N + (size_t)(np) - 1]
#define AU(np, k) au[((size_t)(k) - 1) * N + (size_t)(np) - 1]
#define AV(np, k) av[((size_t)(k) - 1) * N + (size_t)(np) - 1]
#define SGN(x) copysign(0.5, (x))

/* mach2d_coef.f90:6-17 */
void orc_get_density_at_nodes(int nx, int ny, double Rg, const double *p,
                              const double *T, double *ro)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (size_t k = 0; k < N; k++) ro[k] = p[k] / (Rg * T[k]);
}

/* mach2d_coef.f90:20-60 */
void orc_get_density_at_faces(int nx, int ny, double beta, const double *ro,
                              const double *Uce, const double *Vcn, double *roe,
                              double *ron)
{
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, npe = np + 1;
            double ae = SGN(F(Uce, np));
            F(roe, np) = (0.5 + ae) * F(ro, np) + (0.5 - ae) * F(ro, npe)
                       + beta * ae * (F(ro, npe) - F(ro, np));
        }
    for (int j = 1; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, npn = np + nx;
            double an = SGN(F(Vcn, np));
            F(ron, np) = (0.5 + an) * F(ro, np) + (0.5 - an) * F(ro, npn)
                       + beta * an * (F(ro, npn) - F(ro, np));
        }
}

/* mach2d_coef.f90:63-218 */
void orc_get_u_coefficients(int nx, int ny, int modvis, double dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *Je,
    const double *Jn, const double *ye, const double *yk, const double *alphae,
    const double *betae, const double *betan, const double *gamman,
    const double *vle, const double *vln, const double *roe, const double *ron,
    const double *roa, const double *Uce, const double *Vcn, double *a)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npw = np - 1;
            double fme = F(roe, np) * F(re, np) * F(Uce, np);
            double fmw = F(roe, npw) * F(re, npw) * F(Uce, npw);
            double fmn = F(ron, np) * F(rn, np) * F(Vcn, np);
            double fms = F(ron, nps) * F(rn, nps) * F(Vcn, nps);
            double mpa = F(roa, np) * F(rp, np) / F(Jp, np);
            double as = SGN(F(Vcn, nps)), an = SGN(F(Vcn, np));
            double aw = SGN(F(Uce, npw)), ae = SGN(F(Uce, np));
            if (modvis == 0) {
                A(np, 1) = 0.0; A(np, 3) = 0.0; A(np, 7) = 0.0; A(np, 9) = 0.0;
                A(np, 2) = -fms * (0.5 + as);
                A(np, 4) = -fmw * (0.5 + aw);
                A(np, 6) = fme * (0.5 - ae);
                A(np, 8) = fmn * (0.5 - an);
                A(np, 5) = mpa / dt - (A(np, 8) + A(np, 2) + A(np, 4) + A(np, 6));
            } else {
                A(np, 1) = (F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          + F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)) / 4.0;
                A(np, 2) = -fms * (0.5 + as)
                         - F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(gamman, nps)
                         + (F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)) / 4.0;
                A(np, 3) = -(F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)
                           + F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)) / 4.0;
                A(np, 4) = -fmw * (0.5 + aw)
                         - F(vle, npw) * F(re, npw) * F(Je, npw) * F(alphae, npw)
                         + (F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)
                          - F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 6) = fme * (0.5 - ae)
                         - F(vle, np) * F(re, np) * F(Je, np) * F(alphae, np)
                         + (-F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)
                          + F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 7) = (-F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 8) = fmn * (0.5 - an)
                         - F(vln, np) * F(rn, np) * F(Jn, np) * F(gamman, np)
                         - (F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)) / 4.0;
                A(np, 9) = (F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)
                          + F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 5) = mpa / dt - (A(np, 8) + A(np, 2) + A(np, 4) + A(np, 6));
                double S1p = F(rp, np) * F(Je, np) * F(vle, np) * (F(ye, np) * F(ye, np)) / 3.0
                           + F(rp, np) * F(Je, npw) * F(vle, npw) * (F(ye, npw) * F(ye, npw)) / 3.0;
                double S2p = F(rp, np) * F(Jn, np) * F(vln, np) * (F(yk, np) * F(yk, np)) / 3.0
                           + F(rp, np) * F(Jn, nps) * F(vln, nps) * (F(yk, nps) * F(yk, nps)) / 3.0;
                A(np, 5) = A(np, 5) + S1p + S2p;
            }
        }
}

/* mach2d_coef.f90:221-451 */
void orc_get_u_source(int nx, int ny, int modvis, double beta, double dt,
    const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *Jp,
    const double *Je, const double *Jn, const double *roe, const double *ron,
    const double *roa, const double *p, const double *vle, const double *vln,
    const double *Uce, const double *Vcn, const double *ua, const double *u,
    const double *v, double *cup, double *sup, double *b)
{
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            double fme = F(roe, np) * F(re, np) * F(Uce, np);
            double fmw = F(roe, npw) * F(re, npw) * F(Uce, npw);
            double fmn = F(ron, np) * F(rn, np) * F(Vcn, np);
            double fms = F(ron, nps) * F(rn, nps) * F(Vcn, nps);
            double mpa = F(roa, np) * F(rp, np) / F(Jp, np);
            double as = SGN(F(Vcn, nps)), an = SGN(F(Vcn, np));
            double aw = SGN(F(Uce, npw)), ae = SGN(F(Uce, np));
            F(b, np) = mpa * F(ua, np) / dt;
            F(cup, np) = -(beta * (fme * ae * (F(u, npe) - F(u, np))
                                 - fmw * aw * (F(u, np) - F(u, npw))
                                 + fmn * an * (F(u, npn) - F(u, np))
                                 - fms * as * (F(u, np) - F(u, nps))));
            F(b, np) = F(b, np) + F(cup, np);
            F(b, np) = F(b, np) + 0.5 * F(rp, np) * (
                         +F(yk, np) * (F(p, npn) + F(p, np))
                         - F(yk, nps) * (F(p, nps) + F(p, np))
                         - F(ye, np) * (F(p, npe) + F(p, np))
                         + F(ye, npw) * (F(p, npw) + F(p, np)));
        }
    if (modvis != 1) return;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            int npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
            double S1, S2, S3, S4, S5, S6;
            S1 = F(rp, np) / 3.0 * (
                  +F(Je, np) * F(vle, np) *
                   ((F(ye, np) * F(ye, np)) * F(u, npe) - F(yke, np) * F(ye, np)
                    * (F(u, npn) + F(u, npne) - F(u, nps) - F(u, npse)) / 4.0)
                  - F(Je, npw) * F(vle, npw) *
                   (-(F(ye, npw) * F(ye, npw)) * F(u, npw) - F(yke, npw) * F(ye, npw)
                    * (F(u, npn) + F(u, npnw) - F(u, nps) - F(u, npsw)) / 4.0));
            S2 = F(rp, np) / 3.0 * (
                  +F(Jn, np) * F(vln, np) *
                   ((F(yk, np) * F(yk, np)) * F(u, npn) - F(yk, np) * F(yen, np)
                    * (F(u, npe) + F(u, npne) - F(u, npw) - F(u, npnw)) / 4.0)
                  - F(Jn, nps) * F(vln, nps) *
                   (-(F(yk, nps) * F(yk, nps)) * F(u, nps) - F(yk, nps) * F(yen, nps)
                    * (F(u, npe) + F(u, npse) - F(u, npw) - F(u, npsw)) / 4.0));
            S3 = F(Je, np) * F(re, np) * F(vle, np) * F(xe, np) *
                  (F(yke, np) * (F(v, npn) + F(v, npne) - F(v, nps) - F(v, npse)) / 4.0
                   - F(ye, np) * (F(v, npe) - F(v, np)))
               - F(Je, npw) * F(re, npw) * F(vle, npw) * F(xe, npw) *
                  (F(yke, npw) * (F(v, npn) + F(v, npnw) - F(v, nps) - F(v, npsw)) / 4.0
                   - F(ye, npw) * (F(v, np) - F(v, npw)));
            S4 = F(Jn, np) * F(rn, np) * F(vln, np) * F(xk, np) *
                  (F(yen, np) * (F(v, npne) + F(v, npe) - F(v, npnw) - F(v, npw)) / 4.0
                   - F(yk, np) * (F(v, npn) - F(v, np)))
               - F(Jn, nps) * F(rn, nps) * F(vln, nps) * F(xk, nps) *
                  (F(yen, nps) * (F(v, npse) + F(v, npe) - F(v, npsw) - F(v, npw)) / 4.0
                   - F(yk, nps) * (F(v, np) - F(v, nps)));
            if (fabs(F(re, npw)) < 1.0e-15) {
                S5 = -(2.0 * F(rp, np) / 3.0 * F(Je, np) * F(vle, np) / F(re, np) * F(ye, np) *
                       (F(xke, np) * (F(rp, npn) * F(v, npn) + F(rp, npne) * F(v, npne)
                                      - F(rp, nps) * F(v, nps) - F(rp, npse) * F(v, npse)) / 4.0
                        - F(xe, np) * (F(rp, npe) * F(v, npe) - F(rp, np) * F(v, np))));
            } else if (fabs(F(re, np)) < 1.0e-15) {
                S5 = +2.0 * F(rp, np) / 3.0 * F(Je, npw) * F(vle, npw) / F(re, npw) * F(ye, npw) *
                      (F(xke, npw) * (F(rp, npn) * F(v, npn) + F(rp, npnw) * F(v, npnw)
                                      - F(rp, nps) * F(v, nps) - F(rp, npsw) * F(v, npsw)) / 4.0
                       - F(xe, npw) * (F(rp, np) * F(v, np) - F(rp, npw) * F(v, npw)));
            } else {
                S5 = -(2.0 * F(rp, np) / 3.0 * F(Je, np) * F(vle, np) / F(re, np) * F(ye, np) *
                       (F(xke, np) * (F(rp, npn) * F(v, npn) + F(rp, npne) * F(v, npne)
                                      - F(rp, nps) * F(v, nps) - F(rp, npse) * F(v, npse)) / 4.0
                        - F(xe, np) * (F(rp, npe) * F(v, npe) - F(rp, np) * F(v, np))))
                   + 2.0 * F(rp, np) / 3.0 * F(Je, npw) * F(vle, npw) / F(re, npw) * F(ye, npw) *
                      (F(xke, npw) * (F(rp, npn) * F(v, npn) + F(rp, npnw) * F(v, npnw)
                                      - F(rp, nps) * F(v, nps) - F(rp, npsw) * F(v, npsw)) / 4.0
                       - F(xe, npw) * (F(rp, np) * F(v, np) - F(rp, npw) * F(v, npw)));
            }
            if (fabs(F(rn, nps)) < 1.0e-15) {
                S6 = -(2.0 * F(rp, np) / 3.0 * F(Jn, np) * F(vln, np) / F(rn, np) * F(yk, np) *
                       (F(xen, np) * (F(rp, npne) * F(v, npne) + F(rp, npe) * F(v, npe)
                                      - F(rp, npnw) * F(v, npnw) - F(rp, npw) * F(v, npw)) / 4.0
                        - F(xk, np) * (F(rp, npn) * F(v, npn) - F(rp, np) * F(v, np))));
            } else if (fabs(F(rn, np)) < 1.0e-15) {
                S6 = 2.0 * F(rp, np) / 3.0 * F(Jn, nps) * F(vln, nps) / F(rn, nps) * F(yk, nps) *
                     (F(xen, nps) * (F(rp, npe) * F(v, npe) + F(rp, npse) * F(v, npse)
                                     - F(rp, npw) * F(v, npw) - F(rp, npsw) * F(v, npsw)) / 4.0
                      - F(xk, nps) * (F(rp, np) * F(v, np) - F(rp, nps) * F(v, nps)));
            } else {
                S6 = -(2.0 * F(rp, np) / 3.0 * F(Jn, np) * F(vln, np) / F(rn, np) * F(yk, np) *
                       (F(xen, np) * (F(rp, npne) * F(v, npne) + F(rp, npe) * F(v, npe)
                                      - F(rp, npnw) * F(v, npnw) - F(rp, npw) * F(v, npw)) / 4.0
                        - F(xk, np) * (F(rp, npn) * F(v, npn) - F(rp, np) * F(v, np))))
                   + 2.0 * F(rp, np) / 3.0 * F(Jn, nps) * F(vln, nps) / F(rn, nps) * F(yk, nps) *
                     (F(xen, nps) * (F(rp, npe) * F(v, npe) + F(rp, npse) * F(v, npse)
                                     - F(rp, npw) * F(v, npw) - F(rp, npsw) * F(v, npsw)) / 4.0
                      - F(xk, nps) * (F(rp, np) * F(v, np) - F(rp, nps) * F(v, nps)));
            }
            F(sup, np) = S1 + S2 + S3 + S4 + S5 + S6;
            F(b, np) = F(b, np) + F(sup, np);
        }
}

/* mach2d_coef.f90:454-613 */
void orc_get_v_coefficients(int nx, int ny, int coord, int modvis, double dt,
    const double *rp, const double *re, const double *rn, const double *Jp,
    const double *Je, const double *Jn, const double *xe, const double *xk,
    const double *alphae, const double *betae, const double *betan,
    const double *gamman, const double *vle, const double *vln, const double *vlp,
    const double *roe, const double *ron, const double *roa, const double *Uce,
    const double *Vcn, double *a)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npw = np - 1;
            double fme = F(roe, np) * F(re, np) * F(Uce, np);
            double fmw = F(roe, npw) * F(re, npw) * F(Uce, npw);
            double fmn = F(ron, np) * F(rn, np) * F(Vcn, np);
            double fms = F(ron, nps) * F(rn, nps) * F(Vcn, nps);
            double mpa = F(roa, np) * F(rp, np) / F(Jp, np);
            double as = SGN(F(Vcn, nps)), an = SGN(F(Vcn, np));
            double aw = SGN(F(Uce, npw)), ae = SGN(F(Uce, np));
            if (modvis == 0) {
                A(np, 1) = 0.0; A(np, 3) = 0.0; A(np, 7) = 0.0; A(np, 9) = 0.0;
                A(np, 2) = -fms * (0.5 + as);
                A(np, 4) = -fmw * (0.5 + aw);
                A(np, 6) = fme * (0.5 - ae);
                A(np, 8) = fmn * (0.5 - an);
                A(np, 5) = mpa / dt - (A(np, 8) + A(np, 2) + A(np, 4) + A(np, 6));
            } else {
                A(np, 1) = (F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          + F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)) / 4.0;
                A(np, 2) = -fms * (0.5 + as)
                         - F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(gamman, nps)
                         + (F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)) / 4.0;
                A(np, 3) = -(F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)
                           + F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)) / 4.0;
                A(np, 4) = -fmw * (0.5 + aw)
                         - F(vle, npw) * F(re, npw) * F(Je, npw) * F(alphae, npw)
                         + (F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)
                          - F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 6) = fme * (0.5 - ae)
                         - F(vle, np) * F(re, np) * F(Je, np) * F(alphae, np)
                         + (-F(vln, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)
                          + F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 7) = (-F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 8) = fmn * (0.5 - an)
                         - F(vln, np) * F(rn, np) * F(Jn, np) * F(gamman, np)
                         - (F(vle, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)) / 4.0;
                A(np, 9) = (F(vle, np) * F(re, np) * F(Je, np) * F(betae, np)
                          + F(vln, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 5) = mpa / dt - (A(np, 8) + A(np, 2) + A(np, 4) + A(np, 6));
                double S1p = F(vle, np) * F(re, np) * F(Je, np) * (F(xe, np) * F(xe, np)) / 3.0
                           + F(vle, npw) * F(re, npw) * F(Je, npw) * (F(xe, npw) * F(xe, npw)) / 3.0;
                double S2p = F(vln, np) * F(rn, np) * F(Jn, np) * (F(xk, np) * F(xk, np)) / 3.0
                           + F(vln, nps) * F(rn, nps) * F(Jn, nps) * (F(xk, nps) * F(xk, nps)) / 3.0;
                double S7p = (double)coord * F(vlp, np) * 4.0 / (3.0 * F(rp, np) * F(Jp, np));
                A(np, 5) = A(np, 5) + S1p + S2p + S7p;
            }
        }
}

/* mach2d_coef.f90:616-783 */
void orc_get_v_source(int nx, int ny, int coord, int modvis, double beta, double dt,
    const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *Jp,
    const double *Je, const double *Jn, const double *roe, const double *ron,
    const double *roa, const double *p, const double *vle, const double *vln,
    const double *Uce, const double *Vcn, const double *va, const double *u,
    const double *v, double *cvp, double *svp, double *b)
{
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            double fme = F(roe, np) * F(re, np) * F(Uce, np);
            double fmw = F(roe, npw) * F(re, npw) * F(Uce, npw);
            double fmn = F(ron, np) * F(rn, np) * F(Vcn, np);
            double fms = F(ron, nps) * F(rn, nps) * F(Vcn, nps);
            double mpa = F(roa, np) * F(rp, np) / F(Jp, np);
            double as = SGN(F(Vcn, nps)), an = SGN(F(Vcn, np));
            double aw = SGN(F(Uce, npw)), ae = SGN(F(Uce, np));
            F(b, np) = mpa * F(va, np) / dt;
            F(cvp, np) = -(beta * (fme * ae * (F(v, npe) - F(v, np))
                                 - fmw * aw * (F(v, np) - F(v, npw))
                                 + fmn * an * (F(v, npn) - F(v, np))
                                 - fms * as * (F(v, np) - F(v, nps))));
            F(b, np) = F(b, np) + F(cvp, np);
            F(b, np) = F(b, np) + 0.5 * F(rp, np) * (
                         +F(xe, np) * (F(p, np) + F(p, npe))
                         - F(xe, npw) * (F(p, np) + F(p, npw))
                         - F(xk, np) * (F(p, np) + F(p, npn))
                         + F(xk, nps) * (F(p, np) + F(p, nps)));
        }
    if (modvis != 1) return;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            int npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
            double S1, S2, S3, S4, S5, S6, S8;
            S1 = F(vle, np) * F(re, np) * F(Je, np) / 3.0 *
                  ((F(xe, np) * F(xe, np)) * F(v, npe)
                   - F(xke, np) * F(xe, np) * (F(v, npn) + F(v, npne) - F(v, nps) - F(v, npse)) / 4.0)
               - F(vle, npw) * F(re, npw) * F(Je, npw) / 3.0 *
                  (-(F(xe, npw) * F(xe, npw)) * F(v, npw)
                   - F(xke, npw) * F(xe, npw) * (F(v, npn) + F(v, npnw) - F(v, nps) - F(v, npsw)) / 4.0);
            S2 = F(vln, np) * F(rn, np) * F(Jn, np) / 3.0 *
                  ((F(xk, np) * F(xk, np)) * F(v, npn)
                   - F(xk, np) * F(xen, np) * (F(v, npe) + F(v, npne) - F(v, npnw) - F(v, npw)) / 4.0)
               - F(vln, nps) * F(rn, nps) * F(Jn, nps) / 3.0 *
                  (-(F(xk, nps) * F(xk, nps)) * F(v, nps)
                   - F(xk, nps) * F(xen, nps) * (F(v, npe) + F(v, npse) - F(v, npsw) - F(v, npw)) / 4.0);
            S3 = F(rp, np) * F(vle, np) * F(Je, np) * F(ye, np) *
                  (+F(xke, np) * (F(u, npn) + F(u, npne) - F(u, nps) - F(u, npse)) / 4.0
                   - F(xe, np) * (F(u, npe) - F(u, np)))
               - F(rp, np) * F(vle, npw) * F(Je, npw) * F(ye, npw) *
                  (+F(xke, npw) * (F(u, npn) + F(u, npnw) - F(u, nps) - F(u, npsw)) / 4.0
                   - F(xe, npw) * (F(u, np) - F(u, npw)));
            S4 = F(rp, np) * F(vln, np) * F(Jn, np) * F(yk, np) *
                  (+F(xen, np) * (F(u, npne) + F(u, npe) - F(u, npnw) - F(u, npw)) / 4.0
                   - F(xk, np) * (F(u, npn) - F(u, np)))
               - F(rp, np) * F(vln, nps) * F(Jn, nps) * F(yk, nps) *
                  (+F(xen, nps) * (F(u, npse) + F(u, npe) - F(u, npsw) - F(u, npw)) / 4.0
                   - F(xk, nps) * (F(u, np) - F(u, nps)));
            S5 = -(2.0 / 3.0 * F(rp, np) * F(vle, np) * F(Je, np) * F(xe, np) *
                   (+F(yke, np) * (F(u, npn) + F(u, npne) - F(u, nps) - F(u, npse)) / 4.0
                    - F(ye, np) * (F(u, npe) - F(u, np))))
               + 2.0 / 3.0 * F(rp, np) * F(vle, npw) * F(Je, npw) * F(xe, npw) *
                  (+F(yke, npw) * (F(u, npn) + F(u, npnw) - F(u, nps) - F(u, npsw)) / 4.0
                   - F(ye, npw) * (F(u, np) - F(u, npw)));
            S6 = -(2.0 / 3.0 * F(rp, np) * F(vln, np) * F(Jn, np) * F(xk, np) *
                   (+F(yen, np) * (F(u, npe) + F(u, npne) - F(u, npw) - F(u, npnw)) / 4.0
                    - F(yk, np) * (F(u, npn) - F(u, np))))
               + 2.0 / 3.0 * F(rp, np) * F(vln, nps) * F(Jn, nps) * F(xk, nps) *
                  (+F(yen, nps) * (F(u, npe) + F(u, npse) - F(u, npw) - F(u, npsw)) / 4.0
                   - F(yk, nps) * (F(u, np) - F(u, nps)));
            S8 = 2.0 / 3.0 * (double)coord * F(v, np) *
                  (-F(vln, np) * F(xk, np) + F(vln, nps) * F(xk, nps)
                   + F(vle, np) * F(xe, np) - F(vle, npw) * F(xe, npw));
            F(svp, np) = S1 + S2 + S3 + S4 + S5 + S6 + S8;
            F(b, np) = F(b, np) + F(svp, np);
        }
}

/* mach2d_coef.f90:787-1203 */
void orc_get_T_coefficients_and_source(int nx, int ny, int modvis, double beta,
    double dt, const double *rp, const double *re, const double *rn,
    const double *xe, const double *ye, const double *xk, const double *yk,
    const double *xke, const double *yke, const double *xen, const double *yen,
    const double *alphae, const double *betae, const double *betan,
    const double *gamman, const double *Jp, const double *Je, const double *Jn,
    const double *roe, const double *ron, const double *ro, const double *roa,
    const double *p, const double *pa, const double *cp, const double *vle,
    const double *vln, const double *ke, const double *kn, const double *Uce,
    const double *Vcn, const double *u, const double *v, const double *ue,
    const double *ve, const double *un, const double *vn, const double *ua,
    const double *va, const double *T, const double *Ta, const double *fbe,
    const double *fbn, double *a, double *b)
{
    size_t N = (size_t)nx * (size_t)ny;
    const double eps = 2.220446049250313e-16;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            int npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
            double fme = F(roe, np) * F(re, np) * F(Uce, np);
            double fmw = F(roe, npw) * F(re, npw) * F(Uce, npw);
            double fmn = F(ron, np) * F(rn, np) * F(Vcn, np);
            double fms = F(ron, nps) * F(rn, nps) * F(Vcn, nps);
            double mpa = F(roa, np) * F(rp, np) / F(Jp, np);
            double as = SGN(F(Vcn, nps)), an = SGN(F(Vcn, np));
            double aw = SGN(F(Uce, npw)), ae = SGN(F(Uce, np));
            if (modvis == 0) {
                A(np, 1) = 0.0; A(np, 3) = 0.0; A(np, 7) = 0.0; A(np, 9) = 0.0;
                A(np, 2) = -fms * (0.5 + as) * F(cp, np);
                A(np, 4) = -fmw * (0.5 + aw) * F(cp, np);
                A(np, 6) = fme * (0.5 - ae) * F(cp, np);
                A(np, 8) = fmn * (0.5 - an) * F(cp, np);
            } else {
                A(np, 1) = (F(ke, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          + F(kn, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)) / 4.0;
                A(np, 2) = -fms * (0.5 + as) * F(cp, np)
                         - F(kn, nps) * F(rn, nps) * F(Jn, nps) * F(gamman, nps)
                         + (F(ke, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(ke, np) * F(re, np) * F(Je, np) * F(betae, np)) / 4.0;
                A(np, 3) = -(F(ke, np) * F(re, np) * F(Je, np) * F(betae, np)
                           + F(kn, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)) / 4.0;
                A(np, 4) = -fmw * (0.5 + aw) * F(cp, np)
                         - F(ke, npw) * F(re, npw) * F(Je, npw) * F(alphae, npw)
                         + (F(kn, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)
                          - F(kn, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 6) = fme * (0.5 - ae) * F(cp, np)
                         - F(ke, np) * F(re, np) * F(Je, np) * F(alphae, np)
                         + (-F(kn, nps) * F(rn, nps) * F(Jn, nps) * F(betan, nps)
                          + F(kn, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 7) = (-F(ke, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(kn, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
                A(np, 8) = fmn * (0.5 - an) * F(cp, np)
                         - F(kn, np) * F(rn, np) * F(Jn, np) * F(gamman, np)
                         - (F(ke, npw) * F(re, npw) * F(Je, npw) * F(betae, npw)
                          - F(ke, np) * F(re, np) * F(Je, np) * F(betae, np)) / 4.0;
                A(np, 9) = (F(ke, np) * F(re, np) * F(Je, np) * F(betae, np)
                          + F(kn, np) * F(rn, np) * F(Jn, np) * F(betan, np)) / 4.0;
            }
            A(np, 5) = mpa * F(cp, np) / dt - (A(np, 8) + A(np, 2) + A(np, 4) + A(np, 6));
            F(b, np) = mpa * F(Ta, np) * F(cp, np) / dt;
            F(b, np) = F(b, np) - beta * F(cp, np) *
                        (fme * ae * (F(T, npe) - F(T, np))
                         - fmw * aw * (F(T, np) - F(T, npw))
                         + fmn * an * (F(T, npn) - F(T, np))
                         - fms * as * (F(T, np) - F(T, nps)));
            double KpE = (F(u, npe) * F(u, npe) + F(v, npe) * F(v, npe)) / 2.0;
            double KpW = (F(u, npw) * F(u, npw) + F(v, npw) * F(v, npw)) / 2.0;
            double KpN = (F(u, npn) * F(u, npn) + F(v, npn) * F(v, npn)) / 2.0;
            double KpS = (F(u, nps) * F(u, nps) + F(v, nps) * F(v, nps)) / 2.0;
            double KpP = (F(u, np) * F(u, np) + F(v, np) * F(v, np)) / 2.0;
            double KpPa = (F(ua, np) * F(ua, np) + F(va, np) * F(va, np)) / 2.0;
            double Kfe = (0.5 + ae) * KpP + (0.5 - ae) * KpE + beta * ae * (KpE - KpP);
            double Kfw = (0.5 + aw) * KpW + (0.5 - aw) * KpP + beta * aw * (KpP - KpW);
            double Kfn = (0.5 + an) * KpP + (0.5 - an) * KpN + beta * an * (KpN - KpP);
            double Kfs = (0.5 + as) * KpS + (0.5 - as) * KpP + beta * as * (KpP - KpS);
            double Kfbe = (F(ue, np) * F(ue, np) + F(ve, np) * F(ve, np)) / 2.0;
            double Kfbw = (F(ue, npw) * F(ue, npw) + F(ve, npw) * F(ve, npw)) / 2.0;
            double Kfbn = (F(un, np) * F(un, np) + F(vn, np) * F(vn, np)) / 2.0;
            double Kfbs = (F(un, nps) * F(un, nps) + F(vn, nps) * F(vn, nps)) / 2.0;
            Kfe = Kfe * (1.0 - F(fbe, np)) + Kfbe * F(fbe, np);
            Kfw = Kfw * (1.0 - F(fbe, npw)) + Kfbw * F(fbe, npw);
            Kfn = Kfn * (1.0 - F(fbn, np)) + Kfbn * F(fbn, np);
            Kfs = Kfs * (1.0 - F(fbn, nps)) + Kfbs * F(fbn, nps);
            double raux = F(rp, np) / F(Jp, np) * (F(ro, np) * KpP - F(roa, np) * KpPa) / dt
                        + fme * Kfe - fmw * Kfw + fmn * Kfn - fms * Kfs;
            F(b, np) = F(b, np) + F(rp, np) / F(Jp, np) * (F(p, np) - F(pa, np)) / dt - raux;
            if (modvis == 0) continue;
            double dudk_e = F(u, npe) - F(u, np);
            double dudk_w = F(u, np) - F(u, npw);
            double dudk_n = (F(u, npne) + F(u, npe) - F(u, npnw) - F(u, npw)) / 4.0;
            double dudk_s = (F(u, npse) + F(u, npe) - F(u, npsw) - F(u, npw)) / 4.0;
            double dude_e = (F(u, npne) + F(u, npn) - F(u, npse) - F(u, nps)) / 4.0;
            double dude_w = (F(u, npnw) + F(u, npn) - F(u, npsw) - F(u, nps)) / 4.0;
            double dude_n = F(u, npn) - F(u, np);
            double dude_s = F(u, np) - F(u, nps);
            double dvdk_e = F(v, npe) - F(v, np);
            double dvdk_w = F(v, np) - F(v, npw);
            double dvdk_n = (F(v, npne) + F(v, npe) - F(v, npnw) - F(v, npw)) / 4.0;
            double dvdk_s = (F(v, npse) + F(v, npe) - F(v, npsw) - F(v, npw)) / 4.0;
            double dvde_e = (F(v, npne) + F(v, npn) - F(v, npse) - F(v, nps)) / 4.0;
            double dvde_w = (F(v, npnw) + F(v, npn) - F(v, npsw) - F(v, nps)) / 4.0;
            double dvde_n = F(v, npn) - F(v, np);
            double dvde_s = F(v, np) - F(v, nps);
            double dudx_e = F(Je, np) * (F(ye, np) * dudk_e - F(yke, np) * dude_e);
            double dudx_w = F(Je, npw) * (F(ye, npw) * dudk_w - F(yke, npw) * dude_w);
            double dudx_n = F(Jn, np) * (F(yen, np) * dudk_n - F(yk, np) * dude_n);
            double dudx_s = F(Jn, nps) * (F(yen, nps) * dudk_s - F(yk, nps) * dude_s);
            double dudy_e = F(Je, np) * (F(xke, np) * dude_e - F(xe, np) * dudk_e);
            double dudy_w = F(Je, npw) * (F(xke, npw) * dude_w - F(xe, npw) * dudk_w);
            double dudy_n = F(Jn, np) * (F(xk, np) * dude_n - F(xen, np) * dudk_n);
            double dudy_s = F(Jn, nps) * (F(xk, nps) * dude_s - F(xen, nps) * dudk_s);
            double dvdx_e = F(Je, np) * (F(ye, np) * dvdk_e - F(yke, np) * dvde_e);
            double dvdx_w = F(Je, npw) * (F(ye, npw) * dvdk_w - F(yke, npw) * dvde_w);
            double dvdx_n = F(Jn, np) * (F(yen, np) * dvdk_n - F(yk, np) * dvde_n);
            double dvdx_s = F(Jn, nps) * (F(yen, nps) * dvdk_s - F(yk, nps) * dvde_s);
            double dvdy_e = F(Je, np) * (F(xke, np) * dvde_e - F(xe, np) * dvdk_e);
            double dvdy_w = F(Je, npw) * (F(xke, npw) * dvde_w - F(xe, npw) * dvdk_w);
            double dvdy_n = F(Jn, np) * (F(xk, np) * dvde_n - F(xen, np) * dvdk_n);
            double dvdy_s = F(Jn, nps) * (F(xk, nps) * dvde_s - F(xen, nps) * dvdk_s);
            double divU_e = dudx_e + dvdy_e + F(ve, np) / (fabs(F(re, np)) + eps);
            double divU_w = dudx_w + dvdy_w + F(ve, npw) / (fabs(F(re, npw)) + eps);
            double divU_n = dudx_n + dvdy_n + F(vn, np) / (fabs(F(rn, np)) + eps);
            double divU_s = dudx_s + dvdy_s + F(vn, nps) / (fabs(F(rn, nps)) + eps);
            double Txx_e = -2.0 * F(vle, np) * dudx_e + 2.0 / 3.0 * F(vle, np) * divU_e;
            double Txx_w = -2.0 * F(vle, npw) * dudx_w + 2.0 / 3.0 * F(vle, npw) * divU_w;
            double Txx_n = -2.0 * F(vln, np) * dudx_n + 2.0 / 3.0 * F(vln, np) * divU_n;
            double Txx_s = -2.0 * F(vln, nps) * dudx_s + 2.0 / 3.0 * F(vln, nps) * divU_s;
            double Txy_e = -(F(vle, np) * (dvdx_e + dudy_e));
            double Txy_w = -(F(vle, npw) * (dvdx_w + dudy_w));
            double Txy_n = -(F(vln, np) * (dvdx_n + dudy_n));
            double Txy_s = -(F(vln, nps) * (dvdx_s + dudy_s));
            double Tyy_e = -2.0 * F(vle, np) * dvdy_e + 2.0 / 3.0 * F(vle, np) * divU_e;
            double Tyy_w = -2.0 * F(vle, npw) * dvdy_w + 2.0 / 3.0 * F(vle, npw) * divU_w;
            double Tyy_n = -2.0 * F(vln, np) * dvdy_n + 2.0 / 3.0 * F(vln, np) * divU_n;
            double Tyy_s = -2.0 * F(vln, nps) * dvdy_s + 2.0 / 3.0 * F(vln, nps) * divU_s;
            double Lbd_x_e = F(ve, np) * Txy_e + F(ue, np) * Txx_e;
            double Lbd_x_w = F(ve, npw) * Txy_w + F(ue, npw) * Txx_w;
            double Lbd_x_n = F(vn, np) * Txy_n + F(un, np) * Txx_n;
            double Lbd_x_s = F(vn, nps) * Txy_s + F(un, nps) * Txx_s;
            double Lbd_y_e = F(ve, np) * Tyy_e + F(ue, np) * Txy_e;
            double Lbd_y_w = F(ve, npw) * Tyy_w + F(ue, npw) * Txy_w;
            double Lbd_y_n = F(vn, np) * Tyy_n + F(un, np) * Txy_n;
            double Lbd_y_s = F(vn, nps) * Tyy_s + F(un, nps) * Txy_s;
            double Lbd_k_e = Lbd_x_e * F(ye, np) - Lbd_y_e * F(xe, np);
            double Lbd_k_w = Lbd_x_w * F(ye, npw) - Lbd_y_w * F(xe, npw);
            double Lbd_e_n = Lbd_y_n * F(xk, np) - Lbd_x_n * F(yk, np);
            double Lbd_e_s = Lbd_y_s * F(xk, nps) - Lbd_x_s * F(yk, nps);
            raux = F(re, np) * Lbd_k_e - F(re, npw) * Lbd_k_w
                 + F(rn, np) * Lbd_e_n - F(rn, nps) * Lbd_e_s;
            F(b, np) = F(b, np) - raux;
        }
}

/* mach2d_coef.f90:1207-1278 */
void orc_get_p_coefficients(int nx, int ny, double dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *Uce,
    const double *Vcn, const double *roe, const double *ron, const double *g,
    const double *de, const double *dn, double *a)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            double as = SGN(F(Vcn, nps)), an = SGN(F(Vcn, np));
            double aw = SGN(F(Uce, npw)), ae = SGN(F(Uce, np));
            double roem = F(roe, np), rowm = F(roe, npw), ronm = F(ron, np), rosm = F(ron, nps);
            A(np, 1) = -(F(rn, nps) * ((0.5 + as) * F(Vcn, nps) * F(g, nps) + rosm * F(dn, nps)));
            A(np, 2) = -(F(re, npw) * ((0.5 + aw) * F(Uce, npw) * F(g, npw) + rowm * F(de, npw)));
            A(np, 3) = F(g, np) * (F(rp, np) / (F(Jp, np) * dt)
                                   + (0.5 + ae) * F(re, np) * F(Uce, np)
                                   - (0.5 - aw) * F(re, npw) * F(Uce, npw)
                                   + (0.5 + an) * F(rn, np) * F(Vcn, np)
                                   - (0.5 - as) * F(rn, nps) * F(Vcn, nps))
                     + roem * F(re, np) * F(de, np)
                     + rowm * F(re, npw) * F(de, npw)
                     + ronm * F(rn, np) * F(dn, np)
                     + rosm * F(rn, nps) * F(dn, nps);
            A(np, 4) = F(re, np) * ((0.5 - ae) * F(Uce, np) * F(g, npe) - roem * F(de, np));
            A(np, 5) = F(rn, np) * ((0.5 - an) * F(Vcn, np) * F(g, npn) - ronm * F(dn, np));
        }
}

/* mach2d_coef.f90:1281-1348 */
void orc_get_p_source(int nx, int ny, double dt, const double *rp, const double *re,
    const double *rn, const double *Jp, const double *roe, const double *ron,
    const double *ro, const double *roa, const double *Uce, const double *Vcn,
    const double *de, const double *dn, const double *g, const double *pl,
    double *b)
{
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            double as = SGN(F(Vcn, nps)), an = SGN(F(Vcn, np));
            double aw = SGN(F(Uce, npw)), ae = SGN(F(Uce, np));
            double roel = F(g, np) * F(pl, np) * (0.5 + ae) + F(g, npe) * F(pl, npe) * (0.5 - ae);
            double rowl = F(g, npw) * F(pl, npw) * (0.5 + aw) + F(g, np) * F(pl, np) * (0.5 - aw);
            double ronl = F(g, np) * F(pl, np) * (0.5 + an) + F(g, npn) * F(pl, npn) * (0.5 - an);
            double rosl = F(g, nps) * F(pl, nps) * (0.5 + as) + F(g, np) * F(pl, np) * (0.5 - as);
            double Ucel = F(de, np) * (F(pl, np) - F(pl, npe));
            double Ucwl = F(de, npw) * (F(pl, npw) - F(pl, np));
            double Vcnl = F(dn, np) * (F(pl, np) - F(pl, npn));
            double Vcsl = F(dn, nps) * (F(pl, nps) - F(pl, np));
            F(b, np) = -F(rp, np) * (F(ro, np) - F(roa, np)) / (F(Jp, np) * dt)
                     - F(roe, np) * F(re, np) * F(Uce, np)
                     + F(roe, npw) * F(re, npw) * F(Uce, npw)
                     - F(ron, np) * F(rn, np) * F(Vcn, np)
                     + F(ron, nps) * F(rn, nps) * F(Vcn, nps)
                     - roel * F(re, np) * Ucel
                     + rowl * F(re, npw) * Ucwl
                     - ronl * F(rn, np) * Vcnl
                     + rosl * F(rn, nps) * Vcsl;
        }
}

/* mach2d_coef.f90:1350-1501 */
void orc_get_velocities_at_internal_faces(int nx, int ny, double dt,
    const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xen,
    const double *yen, const double *xke, const double *yke, const double *Jp,
    const double *cup, const double *cvp, const double *sup, const double *svp,
    const double *au, const double *av, const double *roa, const double *p,
    const double *u, const double *v, const double *uea, const double *vea,
    const double *una, const double *vna, double *ue, double *ve, double *un,
    double *vn, double *Uce, double *Vcn)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 2; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            int npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
            int npee = npe + 1, npsee = npse + 1, npnee = npne + 1;
            double mpa = F(roa, np) * F(rp, np) / F(Jp, np);
            double mea = F(roa, npe) * F(rp, npe) / F(Jp, npe);
            double sumup = AU(np, 1) * F(u, npsw) + AU(np, 2) * F(u, nps) + AU(np, 3) * F(u, npse)
                         + AU(np, 4) * F(u, npw) + AU(np, 6) * F(u, npe) + AU(np, 7) * F(u, npnw)
                         + AU(np, 8) * F(u, npn) + AU(np, 9) * F(u, npne);
            double sumue = AU(npe, 1) * F(u, nps) + AU(npe, 2) * F(u, npse) + AU(npe, 3) * F(u, npsee)
                         + AU(npe, 4) * F(u, np) + AU(npe, 6) * F(u, npee) + AU(npe, 7) * F(u, npn)
                         + AU(npe, 8) * F(u, npne) + AU(npe, 9) * F(u, npnee);
            double sumvp = AV(np, 1) * F(v, npsw) + AV(np, 2) * F(v, nps) + AV(np, 3) * F(v, npse)
                         + AV(np, 4) * F(v, npw) + AV(np, 6) * F(v, npe) + AV(np, 7) * F(v, npnw)
                         + AV(np, 8) * F(v, npn) + AV(np, 9) * F(v, npne);
            double sumve = AV(npe, 1) * F(v, nps) + AV(npe, 2) * F(v, npse) + AV(npe, 3) * F(v, npsee)
                         + AV(npe, 4) * F(v, np) + AV(npe, 6) * F(v, npee) + AV(npe, 7) * F(v, npn)
                         + AV(npe, 8) * F(v, npne) + AV(npe, 9) * F(v, npnee);
            double aux = (F(p, npn) + F(p, npne) - F(p, nps) - F(p, npse)) / 4.0;
            double pue = F(re, np) * (F(yke, np) * aux + F(ye, np) * (F(p, np) - F(p, npe)));
            double pve = F(re, np) * (-F(xke, np) * aux + F(xe, np) * (F(p, npe) - F(p, np)));
            F(ue, np) = ((mpa + mea) * F(uea, np) / dt + F(cup, np) + F(cup, npe) + F(sup, np)
                         + F(sup, npe) - sumup - sumue + 2.0 * pue) / (AU(np, 5) + AU(npe, 5));
            F(ve, np) = ((mpa + mea) * F(vea, np) / dt + F(cvp, np) + F(cvp, npe) + F(svp, np)
                         + F(svp, npe) - sumvp - sumve + 2.0 * pve) / (AV(np, 5) + AV(npe, 5));
            F(Uce, np) = F(ue, np) * F(ye, np) - F(ve, np) * F(xe, np);
        }
    for (int j = 2; j <= ny - 2; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            int npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
            int npnn = npn + nx, npnnw = npnn - 1, npnne = npnn + 1;
            double mpa = F(roa, np) * F(rp, np) / F(Jp, np);
            double mna = F(roa, npn) * F(rp, npn) / F(Jp, npn);
            double sumup = AU(np, 1) * F(u, npsw) + AU(np, 2) * F(u, nps) + AU(np, 3) * F(u, npse)
                         + AU(np, 4) * F(u, npw) + AU(np, 6) * F(u, npe) + AU(np, 7) * F(u, npnw)
                         + AU(np, 8) * F(u, npn) + AU(np, 9) * F(u, npne);
            double sumun = AU(npn, 1) * F(u, npw) + AU(npn, 2) * F(u, np) + AU(npn, 3) * F(u, npe)
                         + AU(npn, 4) * F(u, npnw) + AU(npn, 6) * F(u, npne) + AU(npn, 7) * F(u, npnnw)
                         + AU(npn, 8) * F(u, npnn) + AU(npn, 9) * F(u, npnne);
            double sumvp = AV(np, 1) * F(v, npsw) + AV(np, 2) * F(v, nps) + AV(np, 3) * F(v, npse)
                         + AV(np, 4) * F(v, npw) + AV(np, 6) * F(v, npe) + AV(np, 7) * F(v, npnw)
                         + AV(np, 8) * F(v, npn) + AV(np, 9) * F(v, npne);
            double sumvn = AV(npn, 1) * F(v, npw) + AV(npn, 2) * F(v, np) + AV(npn, 3) * F(v, npe)
                         + AV(npn, 4) * F(v, npnw) + AV(npn, 6) * F(v, npne) + AV(npn, 7) * F(v, npnnw)
                         + AV(npn, 8) * F(v, npnn) + AV(npn, 9) * F(v, npnne);
            double aux = (F(p, npne) + F(p, npe) - F(p, npnw) - F(p, npw)) / 4.0;
            double pun = F(rn, np) * (F(yk, np) * (F(p, npn) - F(p, np)) - F(yen, np) * aux);
            double pvn = F(rn, np) * (F(xk, np) * (F(p, np) - F(p, npn)) + F(xen, np) * aux);
            F(un, np) = ((mpa + mna) * F(una, np) / dt + F(cup, np) + F(cup, npn) + F(sup, np)
                         + F(sup, npn) - sumup - sumun + 2.0 * pun) / (AU(np, 5) + AU(npn, 5));
            F(vn, np) = ((mpa + mna) * F(vna, np) / dt + F(cvp, np) + F(cvp, npn) + F(svp, np)
                         + F(svp, npn) - sumvp - sumvn + 2.0 * pvn) / (AV(np, 5) + AV(npn, 5));
            F(Vcn, np) = F(vn, np) * F(xk, np) - F(un, np) * F(yk, np);
        }
}

/* Fortran sum(a(np,:)): sequential k = 1..9 */
static double sum9(const double *a, size_t N, int np)
{
    double s = 0.0;
    for (int k = 1; k <= 9; k++) s = s + A(np, k);
    return s;
}

/* mach2d_coef.f90:1504-1600 */
void orc_get_internal_simplec_coefficients(int nx, int ny, const double *re,
    const double *rn, const double *xe, const double *ye, const double *xk,
    const double *yk, const double *au, const double *av, double *due,
    double *dve, double *dun, double *dvn, double *de, double *dn)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 2; i++) {
            int np = nx * (j - 1) + i, npe = np + 1;
            double Lue = 2.0 * F(re, np) / (sum9(au, N, np) + sum9(au, N, npe));
            double Lve = 2.0 * F(re, np) / (sum9(av, N, np) + sum9(av, N, npe));
            F(due, np) = Lue * F(ye, np);
            F(dve, np) = Lve * F(xe, np);
            F(de, np) = F(ye, np) * F(due, np) + F(xe, np) * F(dve, np);
        }
    for (int j = 2; j <= ny - 2; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, npn = np + nx;
            double Lun = 2.0 * F(rn, np) / (sum9(au, N, np) + sum9(au, N, npn));
            double Lvn = 2.0 * F(rn, np) / (sum9(av, N, np) + sum9(av, N, npn));
            F(dun, np) = Lun * F(yk, np);
            F(dvn, np) = Lvn * F(xk, np);
            F(dn, np) = F(xk, np) * F(dvn, np) + F(yk, np) * F(dun, np);
        }
}

/* mach2d_coef.f90:1602-1624 */
void orc_get_pressure_correction_with_pl(int nx, int ny, const double *pl, double *p)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (size_t k = 0; k < N; k++) p[k] = p[k] + pl[k];
}

void orc_get_density_correction_with_pl(int nx, int ny, const double *pl,
                                        const double *g, double *ro)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (size_t k = 0; k < N; k++) ro[k] = ro[k] + pl[k] * g[k];
}

/* mach2d_coef.f90:1626-1675 */
void orc_get_u_v_at_real_nodes_with_pl(int nx, int ny, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *rp,
    const double *pl, const double *au, const double *av, double *u, double *v)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            double plup = 0.5 * F(rp, np) * (+F(yk, np) * (F(pl, npn) + F(pl, np))
                                             - F(yk, nps) * (F(pl, nps) + F(pl, np))
                                             - F(ye, np) * (F(pl, npe) + F(pl, np))
                                             + F(ye, npw) * (F(pl, npw) + F(pl, np)));
            double plvp = 0.5 * F(rp, np) * (+F(xe, np) * (F(pl, np) + F(pl, npe))
                                             - F(xe, npw) * (F(pl, np) + F(pl, npw))
                                             - F(xk, np) * (F(pl, np) + F(pl, npn))
                                             + F(xk, nps) * (F(pl, np) + F(pl, nps)));
            F(u, np) = F(u, np) + plup / sum9(au, N, np);
            F(v, np) = F(v, np) + plvp / sum9(av, N, np);
        }
}

/* mach2d_coef.f90:1679-1758 */
void orc_get_velocity_correction_at_faces_with_pl(int nx, int ny, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *due,
    const double *dve, const double *dun, const double *dvn, const double *de,
    const double *dn, const double *pl, double *ue, double *ve, double *un,
    double *vn, double *Uce, double *Vcn)
{
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, npe = np + 1;
            F(Uce, np) = F(ue, np) * F(ye, np) - F(ve, np) * F(xe, np)
                       + F(de, np) * (F(pl, np) - F(pl, npe));
            F(ue, np) = F(ue, np) + F(due, np) * (F(pl, np) - F(pl, npe));
            F(ve, np) = F(ve, np) + F(dve, np) * (F(pl, npe) - F(pl, np));
        }
    for (int j = 1; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, npn = np + nx;
            F(Vcn, np) = F(vn, np) * F(xk, np) - F(un, np) * F(yk, np)
                       + F(dn, np) * (F(pl, np) - F(pl, npn));
            F(un, np) = F(un, np) + F(dun, np) * (F(pl, npn) - F(pl, np));
            F(vn, np) = F(vn, np) + F(dvn, np) * (F(pl, np) - F(pl, npn));
        }
}

/* mach2d_coef.f90:1764-1828 */
void orc_initialize_boundary_faces_flags(int nx, int ny, double *fbe, double *fbn)
{
    size_t N = (size_t)nx * (size_t)ny;
    memset(fbe, 0, N * sizeof(double));
    for (int j = 2; j <= ny - 1; j++) F(fbe, nx * (j - 1) + 1) = 1.0;
    for (int j = 2; j <= ny - 1; j++) F(fbe, nx * (j - 1) + nx - 1) = 1.0;
    memset(fbn, 0, N * sizeof(double));
    for (int i = 2; i <= nx - 1; i++) F(fbn, nx * (ny - 2) + i) = 1.0;
    for (int i = 2; i <= nx - 1; i++) F(fbn, i) = 1.0;
}

/* mach2d_coef.f90:1833-1880 */
double orc_check_mass_conservation(int nx, int ny, double dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *ro,
    const double *roa, const double *ron, const double *roe, const double *Uce,
    const double *Vcn)
{
    double res = 0.0;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npw = np - 1;
            double fme = F(roe, np) * F(re, np) * F(Uce, np);
            double fmw = F(roe, npw) * F(re, npw) * F(Uce, npw);
            double fmn = F(ron, np) * F(rn, np) * F(Vcn, np);
            double fms = F(ron, nps) * F(rn, nps) * F(Vcn, nps);
            res = res + fabs((F(ro, np) - F(roa, np)) * F(rp, np) / (F(Jp, np) * dt)
                             + fme - fmw + fmn - fms);
        }
    return res;
}
