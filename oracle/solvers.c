/*
 * solvers.c -- oracle restatement of MACH-2D's linear solvers.
 * TEST INFRASTRUCTURE ONLY (see m2d_oracle.h).  Parity unpinned: no Fortran
 * compiler in this image and no golden vectors in the reference.
 *
 * Follows, statement by statement and in the same order:
 *   lu2d9 / fb2d9  src/solvers/msi2d9-v03.f90:277-432 / :42-262
 *   lu2d5 / fb2d5  src/solvers/msi2d5-v03.f90:247-330 / :42-233
 *   tdma2d9        src/solvers/tdma2d9.f90:38-322
 *   tdma2d5        src/solvers/tdma2d5.f90:38-241
 *   norms          src/solvers/mod_solvers.f90:91-277
 *   solve          src/solvers/mod_solver_msi.f90:79-133 (lu recomputed per call)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "m2d_oracle.h"

/* 1-based accessors for column-major a(nij,k) and vectors */
#define B(ip, k)  b[((size_t)(k) - 1) * (size_t)nij + (size_t)(ip) - 1]
#define DL(ip, k) dl[((size_t)(k) - 1) * (size_t)nij + (size_t)(ip) - 1]
#define DU(ip, k) du[((size_t)(k) - 1) * (size_t)nij + (size_t)(ip) - 1]
#define V(arr, ip) (arr)[(size_t)(ip) - 1]

/* residual r = A.var - rhs of fb2d9 (msi2d9-v03.f90:61-131, repeated 185-255) */
static void fb9_residual(const double *b, int ni, int nij, const double *var,
                         const double *rhs, double *r)
{
    int ip, isw, is, ise, iw, ie, inw, in, ine;
    ip = 1; ie = ip + 1; in = ip + ni; ine = in + 1;
    V(r, ip) = -V(rhs, ip) + B(ip, 5) * V(var, ip) + B(ip, 6) * V(var, ie)
             + B(ip, 8) * V(var, in) + B(ip, 9) * V(var, ine);
    for (ip = 2; ip <= ni - 1; ip++) {
        iw = ip - 1; ie = ip + 1; in = ip + ni; inw = in - 1; ine = in + 1;
        V(r, ip) = -V(rhs, ip) + B(ip, 4) * V(var, iw) + B(ip, 5) * V(var, ip)
                 + B(ip, 6) * V(var, ie) + B(ip, 7) * V(var, inw)
                 + B(ip, 8) * V(var, in) + B(ip, 9) * V(var, ine);
    }
    ip = ni; iw = ip - 1; in = ip + ni; inw = in - 1;
    V(r, ip) = -V(rhs, ip) + B(ip, 4) * V(var, iw) + B(ip, 5) * V(var, ip)
             + B(ip, 7) * V(var, inw) + B(ip, 8) * V(var, in);
    for (ip = ni + 1; ip <= nij - ni; ip++) {
        iw = ip - 1; ie = ip + 1; is = ip - ni; in = ip + ni;
        isw = is - 1; ise = is + 1; inw = in - 1; ine = in + 1;
        if (ip % ni == 1) {
            V(r, ip) = -V(rhs, ip) + B(ip, 2) * V(var, is) + B(ip, 3) * V(var, ise)
                     + B(ip, 5) * V(var, ip) + B(ip, 6) * V(var, ie)
                     + B(ip, 8) * V(var, in) + B(ip, 9) * V(var, ine);
        } else if (ip % ni == 0) {
            V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, isw) + B(ip, 2) * V(var, is)
                     + B(ip, 4) * V(var, iw) + B(ip, 5) * V(var, ip)
                     + B(ip, 7) * V(var, inw) + B(ip, 8) * V(var, in);
        } else {
            V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, isw) + B(ip, 2) * V(var, is)
                     + B(ip, 3) * V(var, ise) + B(ip, 4) * V(var, iw)
                     + B(ip, 5) * V(var, ip) + B(ip, 6) * V(var, ie)
                     + B(ip, 7) * V(var, inw) + B(ip, 8) * V(var, in)
                     + B(ip, 9) * V(var, ine);
        }
    }
    ip = nij - ni + 1; ie = ip + 1; is = ip - ni; ise = is + 1;
    V(r, ip) = -V(rhs, ip) + B(ip, 2) * V(var, is) + B(ip, 3) * V(var, ise)
             + B(ip, 5) * V(var, ip) + B(ip, 6) * V(var, ie);
    for (ip = nij - ni + 2; ip <= nij - 1; ip++) {
        iw = ip - 1; ie = ip + 1; is = ip - ni; isw = is - 1; ise = is + 1;
        V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, isw) + B(ip, 2) * V(var, is)
                 + B(ip, 3) * V(var, ise) + B(ip, 4) * V(var, iw)
                 + B(ip, 5) * V(var, ip) + B(ip, 6) * V(var, ie);
    }
    ip = nij; iw = ip - 1; is = ip - ni; isw = is - 1;
    V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, isw) + B(ip, 2) * V(var, is)
             + B(ip, 4) * V(var, iw) + B(ip, 5) * V(var, ip);
}

/* Fortran dot_product: sequential sum */
static double dot_seq(const double *r, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s = s + r[i] * r[i];
    return s;
}

int orc_fb2d9(const double *b, const double *dl, const double *du, int nj, int ni,
              int nij, double *var, double gamma, int nitm, const double *rhs)
{
    (void)nj;
    double *r = (double *)malloc(sizeof(double) * (size_t)nij);
    double *w = (double *)malloc(sizeof(double) * (size_t)nij);
    double *z = (double *)malloc(sizeof(double) * (size_t)nij);
    int ip, nit;
    fb9_residual(b, ni, nij, var, rhs, r);
    double gammarp = gamma * sqrt(dot_seq(r, nij));
    nit = 0;
    for (;;) {
        nit = nit + 1;
        /* Lw = -r (msi2d9-v03.f90:141-156) */
        ip = 1;
        V(w, ip) = -V(r, ip) / DL(ip, 1);
        for (ip = 2; ip <= ni - 1; ip++)
            V(w, ip) = -(V(r, ip) + DL(ip, 2) * V(w, ip - 1)) / DL(ip, 1);
        ip = ni;
        V(w, ip) = -(V(r, ip) + DL(ip, 2) * V(w, ip - 1) + DL(ip, 3) * V(w, ip - ni + 1)) / DL(ip, 1);
        ip = ni + 1;
        V(w, ip) = -(V(r, ip) + DL(ip, 2) * V(w, ip - 1) + DL(ip, 3) * V(w, ip - ni + 1)
                     + DL(ip, 4) * V(w, ip - ni)) / DL(ip, 1);
        for (ip = ni + 2; ip <= nij; ip++)
            V(w, ip) = -(V(r, ip) + DL(ip, 2) * V(w, ip - 1) + DL(ip, 3) * V(w, ip - ni + 1)
                         + DL(ip, 4) * V(w, ip - ni) + DL(ip, 5) * V(w, ip - ni - 1)) / DL(ip, 1);
        /* Uz = w (msi2d9-v03.f90:161-176) */
        ip = nij;
        V(z, ip) = V(w, ip);
        for (ip = nij - 1; ip >= nij - ni + 2; ip--)
            V(z, ip) = V(w, ip) - DU(ip, 1) * V(z, ip + 1);
        ip = nij - ni + 1;
        V(z, ip) = V(w, ip) - DU(ip, 1) * V(z, ip + 1) - DU(ip, 2) * V(z, ip + ni - 1);
        ip = nij - ni;
        V(z, ip) = V(w, ip) - DU(ip, 1) * V(z, ip + 1) - DU(ip, 2) * V(z, ip + ni - 1)
                 - DU(ip, 3) * V(z, ip + ni);
        for (ip = nij - ni - 1; ip >= 1; ip--)
            V(z, ip) = V(w, ip) - DU(ip, 1) * V(z, ip + 1) - DU(ip, 2) * V(z, ip + ni - 1)
                     - DU(ip, 3) * V(z, ip + ni) - DU(ip, 4) * V(z, ip + ni + 1);
        /* var = z + var */
        for (ip = 1; ip <= nij; ip++) V(var, ip) = V(z, ip) + V(var, ip);
        fb9_residual(b, ni, nij, var, rhs, r);
        if (sqrt(dot_seq(r, nij)) < gammarp) break;
        if (nit == nitm) break;
    }
    free(r); free(w); free(z);
    return nit;
}

void orc_lu2d9(const double *b, double *dl, double *du, int nij, int ni, int nj)
{
    (void)nj;
    int isw, is, ise, iw, ip;
    double alpha, phi1, phi2, phi3, phi4, alpha0;
    alpha0 = 0.5;
    alpha = alpha0;
    memset(du, 0, sizeof(double) * 4 * (size_t)nij);
    memset(dl, 0, sizeof(double) * 5 * (size_t)nij);

    ip = 1;
    DL(ip, 1) = B(ip, 5);
    DU(ip, 1) = B(ip, 6) / DL(ip, 1);
    DU(ip, 2) = B(ip, 7) / DL(ip, 1);
    DU(ip, 3) = B(ip, 8) / DL(ip, 1);
    DU(ip, 4) = B(ip, 9) / DL(ip, 1);

    for (ip = 2; ip <= ni - 1; ip++) {
        iw = ip - 1;
        DL(ip, 2) = B(ip, 4);
        DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1);
        DU(ip, 1) = B(ip, 6) / DL(ip, 1);
        DU(ip, 2) = (B(ip, 7) - DL(ip, 2) * DU(iw, 3)) / DL(ip, 1);
        DU(ip, 3) = (B(ip, 8) - DL(ip, 2) * DU(iw, 4)) / DL(ip, 1);
        DU(ip, 4) = B(ip, 9) / DL(ip, 1);
    }

    ip = ni;
    iw = ip - 1; is = ip - ni; ise = is + 1;
    DL(ip, 3) = B(ip, 3);
    DL(ip, 2) = B(ip, 4);
    DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2);
    DU(ip, 1) = (B(ip, 6) - DL(ip, 3) * DU(ise, 3)) / DL(ip, 1);
    DU(ip, 2) = (B(ip, 7) - DL(ip, 2) * DU(iw, 3)) / DL(ip, 1);
    DU(ip, 3) = (B(ip, 8) - DL(ip, 2) * DU(iw, 4)) / DL(ip, 1);
    DU(ip, 4) = B(ip, 9) / DL(ip, 1);

    ip = ni + 1;
    iw = ip - 1; is = ip - ni; ise = is + 1;
    DL(ip, 4) = B(ip, 2);
    DL(ip, 3) = B(ip, 3) - DL(ip, 4) * DU(is, 1);
    DL(ip, 2) = B(ip, 4) - DL(ip, 4) * DU(is, 2);
    DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2) - DL(ip, 4) * DU(is, 3);
    DU(ip, 1) = (B(ip, 6) - DL(ip, 3) * DU(ise, 3) - DL(ip, 4) * DU(is, 4)) / DL(ip, 1);
    DU(ip, 2) = (B(ip, 7) - DL(ip, 2) * DU(iw, 3)) / DL(ip, 1);
    DU(ip, 3) = (B(ip, 8) - DL(ip, 2) * DU(iw, 4)) / DL(ip, 1);
    DU(ip, 4) = B(ip, 9) / DL(ip, 1);

    alpha = alpha0;
    for (ip = ni + 2; ip <= nij - ni - 1; ip++) {
        if (ip % ni == 0 || ip % ni == 1) alpha = 0.0; else alpha = alpha0;
        iw = ip - 1; is = ip - ni; isw = is - 1; ise = is + 1;
        DL(ip, 5) = B(ip, 1);
        DL(ip, 4) = (B(ip, 2) - DL(ip, 5) * DU(isw, 1) - alpha * B(ip, 3) * DU(ise, 1))
                  / (1.0 - alpha * DU(is, 1) * DU(ise, 1));
        DL(ip, 3) = B(ip, 3) - DL(ip, 4) * DU(is, 1);
        DL(ip, 2) = (B(ip, 4) - DL(ip, 4) * DU(is, 2) - DL(ip, 5) * DU(isw, 3)
                     - 2.0 * alpha * DL(ip, 5) * DU(isw, 2))
                  / (1 + 2.0 * alpha * DU(iw, 2));
        phi1 = DL(ip, 3) * DU(ise, 1);
        phi2 = DL(ip, 5) * DU(isw, 2);
        phi3 = DL(ip, 3) * DU(ise, 4);
        phi4 = DL(ip, 2) * DU(iw, 2);
        DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2)
                  - DL(ip, 4) * DU(is, 3) - DL(ip, 5) * DU(isw, 4)
                  + alpha * (2.0 * phi1 + phi2 + phi3 + 2.0 * phi4);
        DU(ip, 1) = (B(ip, 6) - DL(ip, 3) * DU(ise, 3) - DL(ip, 4) * DU(is, 4)
                     - 2.0 * alpha * (phi1 + phi3)) / DL(ip, 1);
        DU(ip, 2) = (B(ip, 7) - DL(ip, 2) * DU(iw, 3)) / DL(ip, 1);
        DU(ip, 3) = (B(ip, 8) - DL(ip, 2) * DU(iw, 4) - alpha * phi4) / DL(ip, 1);
        DU(ip, 4) = B(ip, 9) / DL(ip, 1);
    }

    ip = nij - ni;
    iw = ip - 1; is = ip - ni; isw = is - 1; ise = is + 1;
    DL(ip, 5) = B(ip, 1);
    DL(ip, 4) = B(ip, 2) - DL(ip, 5) * DU(isw, 1);
    DL(ip, 3) = B(ip, 3) - DL(ip, 4) * DU(is, 1);
    DL(ip, 2) = B(ip, 4) - DL(ip, 4) * DU(is, 2) - DL(ip, 5) * DU(isw, 3);
    DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2)
              - DL(ip, 4) * DU(is, 3) - DL(ip, 5) * DU(isw, 4);
    DU(ip, 1) = (B(ip, 6) - DL(ip, 3) * DU(ise, 3) - DL(ip, 4) * DU(is, 4)) / DL(ip, 1);
    DU(ip, 2) = (B(ip, 7) - DL(ip, 2) * DU(iw, 3)) / DL(ip, 1);
    DU(ip, 3) = (B(ip, 8) - DL(ip, 2) * DU(iw, 4)) / DL(ip, 1);

    ip = nij - ni + 1;
    iw = ip - 1; is = ip - ni; isw = is - 1; ise = is + 1;
    DL(ip, 5) = B(ip, 1);
    DL(ip, 4) = B(ip, 2) - DL(ip, 5) * DU(isw, 1);
    DL(ip, 3) = B(ip, 3) - DL(ip, 4) * DU(is, 1);
    DL(ip, 2) = B(ip, 4) - DL(ip, 4) * DU(is, 2) - DL(ip, 5) * DU(isw, 3);
    DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2)
              - DL(ip, 4) * DU(is, 3) - DL(ip, 5) * DU(isw, 4);
    DU(ip, 1) = (B(ip, 6) - DL(ip, 3) * DU(ise, 3) - DL(ip, 4) * DU(is, 4)) / DL(ip, 1);
    DU(ip, 2) = (B(ip, 7) - DL(ip, 2) * DU(iw, 3)) / DL(ip, 1);

    for (ip = nij - ni + 2; ip <= nij - 1; ip++) {
        iw = ip - 1; is = ip - ni; isw = is - 1; ise = is + 1;
        DL(ip, 5) = B(ip, 1);
        DL(ip, 4) = B(ip, 2) - DL(ip, 5) * DU(isw, 1);
        DL(ip, 3) = B(ip, 3) - DL(ip, 4) * DU(is, 1);
        DL(ip, 2) = B(ip, 4) - DL(ip, 4) * DU(is, 2) - DL(ip, 5) * DU(isw, 3);
        DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2)
                  - DL(ip, 4) * DU(is, 3) - DL(ip, 5) * DU(isw, 4);
        DU(ip, 1) = (B(ip, 6) - DL(ip, 3) * DU(ise, 3) - DL(ip, 4) * DU(is, 4)) / DL(ip, 1);
    }

    ip = nij;
    iw = ip - 1; is = ip - ni; isw = is - 1; ise = is + 1;
    DL(ip, 5) = B(ip, 1);
    DL(ip, 4) = B(ip, 2) - DL(ip, 5) * DU(isw, 1);
    DL(ip, 3) = B(ip, 3) - DL(ip, 4) * DU(is, 1);
    DL(ip, 2) = B(ip, 4) - DL(ip, 4) * DU(is, 2) - DL(ip, 5) * DU(isw, 3);
    DL(ip, 1) = B(ip, 5) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2)
              - DL(ip, 4) * DU(is, 3) - DL(ip, 5) * DU(isw, 4);
}

/* residual of fb2d5 (msi2d5-v03.f90:61-119) */
static void fb5_residual(const double *b, int ni, int nij, const double *var,
                         const double *rhs, double *r)
{
    int ip, is, iw, ie, in;
    ip = 1; ie = ip + 1; in = ip + ni;
    V(r, ip) = -V(rhs, ip) + B(ip, 3) * V(var, ip) + B(ip, 4) * V(var, ie)
             + B(ip, 5) * V(var, in);
    for (ip = 2; ip <= ni - 1; ip++) {
        iw = ip - 1; ie = ip + 1; in = ip + ni;
        V(r, ip) = -V(rhs, ip) + B(ip, 2) * V(var, iw) + B(ip, 3) * V(var, ip)
                 + B(ip, 4) * V(var, ie) + B(ip, 5) * V(var, in);
    }
    ip = ni; iw = ip - 1; in = ip + ni;
    V(r, ip) = -V(rhs, ip) + B(ip, 2) * V(var, iw) + B(ip, 3) * V(var, ip)
             + B(ip, 5) * V(var, in);
    for (ip = ni + 1; ip <= nij - ni; ip++) {
        iw = ip - 1; ie = ip + 1; is = ip - ni; in = ip + ni;
        if (ip % ni == 0) {
            V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, is) + B(ip, 2) * V(var, iw)
                     + B(ip, 3) * V(var, ip) + B(ip, 5) * V(var, in);
        } else if (ip % ni == 1) {
            V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, is) + B(ip, 3) * V(var, ip)
                     + B(ip, 4) * V(var, ie) + B(ip, 5) * V(var, in);
        } else {
            V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, is) + B(ip, 2) * V(var, iw)
                     + B(ip, 3) * V(var, ip) + B(ip, 4) * V(var, ie)
                     + B(ip, 5) * V(var, in);
        }
    }
    ip = nij - ni + 1; ie = ip + 1; is = ip - ni;
    V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, is) + B(ip, 3) * V(var, ip)
             + B(ip, 4) * V(var, ie);
    for (ip = nij - ni + 2; ip <= nij - 1; ip++) {
        iw = ip - 1; ie = ip + 1; is = ip - ni;
        V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, is) + B(ip, 2) * V(var, iw)
                 + B(ip, 3) * V(var, ip) + B(ip, 4) * V(var, ie);
    }
    ip = nij; iw = ip - 1; is = ip - ni;
    V(r, ip) = -V(rhs, ip) + B(ip, 1) * V(var, is) + B(ip, 2) * V(var, iw)
             + B(ip, 3) * V(var, ip);
}

int orc_fb2d5(const double *b, const double *dl, const double *du, int nj, int ni,
              int nij, double *var, double gamma, int nitm, const double *rhs)
{
    (void)nj;
    double *r = (double *)malloc(sizeof(double) * (size_t)nij);
    double *w = (double *)malloc(sizeof(double) * (size_t)nij);
    double *z = (double *)malloc(sizeof(double) * (size_t)nij);
    int ip, nit;
    fb5_residual(b, ni, nij, var, rhs, r);
    double gammarp = gamma * sqrt(dot_seq(r, nij));
    nit = 0;
    for (;;) {
        nit = nit + 1;
        ip = 1;
        V(w, ip) = -V(r, ip) / DL(ip, 1);
        for (ip = 2; ip <= ni - 1; ip++)
            V(w, ip) = -(V(r, ip) + DL(ip, 2) * V(w, ip - 1)) / DL(ip, 1);
        ip = ni;
        V(w, ip) = -(V(r, ip) + DL(ip, 2) * V(w, ip - 1) + DL(ip, 3) * V(w, ip - ni + 1)) / DL(ip, 1);
        for (ip = ni + 1; ip <= nij; ip++)
            V(w, ip) = -(V(r, ip) + DL(ip, 2) * V(w, ip - 1) + DL(ip, 3) * V(w, ip - ni + 1)
                         + DL(ip, 4) * V(w, ip - ni)) / DL(ip, 1);
        ip = nij;
        V(z, ip) = V(w, ip);
        for (ip = nij - 1; ip >= nij - ni + 2; ip--)
            V(z, ip) = V(w, ip) - DU(ip, 1) * V(z, ip + 1);
        ip = nij - ni + 1;
        V(z, ip) = V(w, ip) - DU(ip, 1) * V(z, ip + 1) - DU(ip, 2) * V(z, ip + ni - 1);
        for (ip = nij - ni; ip >= 1; ip--)
            V(z, ip) = V(w, ip) - DU(ip, 1) * V(z, ip + 1) - DU(ip, 2) * V(z, ip + ni - 1)
                     - DU(ip, 3) * V(z, ip + ni);
        for (ip = 1; ip <= nij; ip++) V(var, ip) = V(z, ip) + V(var, ip);
        fb5_residual(b, ni, nij, var, rhs, r);
        if (sqrt(dot_seq(r, nij)) < gammarp) break;
        if (nit == nitm) break;
    }
    free(r); free(w); free(z);
    return nit;
}

void orc_lu2d5(const double *b, double *dl, double *du, int nij, int ni, int nj)
{
    (void)nj;
    int is, ise, iw, ip;
    double alpha, phi1, phi4, alpha0;
    alpha0 = 0.5;
    alpha = alpha0;
    memset(du, 0, sizeof(double) * 3 * (size_t)nij);
    memset(dl, 0, sizeof(double) * 4 * (size_t)nij);
    ip = 1;
    DL(ip, 1) = B(ip, 3);
    DU(ip, 1) = B(ip, 4) / DL(ip, 1);
    DU(ip, 3) = B(ip, 5) / DL(ip, 1);
    for (ip = 2; ip <= ni; ip++) {
        iw = ip - 1;
        DL(ip, 2) = B(ip, 2);
        DL(ip, 1) = B(ip, 3) - DL(ip, 2) * DU(iw, 1);
        DU(ip, 1) = B(ip, 4) / DL(ip, 1);
        DU(ip, 2) = -DL(ip, 2) * DU(iw, 3) / DL(ip, 1);
        DU(ip, 3) = B(ip, 5) / DL(ip, 1);
    }
    for (ip = ni + 1; ip <= nij - ni; ip++) {
        iw = ip - 1; is = ip - ni; ise = is + 1;
        if (ip % ni == 0 || ip % ni == 1) alpha = 0.0; else alpha = alpha0;
        DL(ip, 4) = B(ip, 1) / (1.0 - alpha * DU(is, 1) * DU(ise, 1));
        DL(ip, 3) = -DL(ip, 4) * DU(is, 1);
        DL(ip, 2) = (B(ip, 2) - DL(ip, 4) * DU(is, 2)) / (1.0 + 2.0 * alpha * DU(iw, 2));
        phi1 = DL(ip, 3) * DU(ise, 1);
        phi4 = DL(ip, 2) * DU(iw, 2);
        DL(ip, 1) = B(ip, 3) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2)
                  - DL(ip, 4) * DU(is, 3) + 2.0 * alpha * (phi1 + phi4);
        DU(ip, 1) = (B(ip, 4) - DL(ip, 3) * DU(ise, 3) - 2.0 * alpha * phi1) / DL(ip, 1);
        DU(ip, 2) = -DL(ip, 2) * DU(iw, 3) / DL(ip, 1);
        DU(ip, 3) = (B(ip, 5) - alpha * phi4) / DL(ip, 1);
    }
    ip = nij - ni + 1;
    iw = ip - 1; is = ip - ni; ise = is + 1;
    DL(ip, 4) = B(ip, 1);
    DL(ip, 3) = -DL(ip, 4) * DU(is, 1);
    DL(ip, 2) = (B(ip, 2) - DL(ip, 4) * DU(is, 2));
    DL(ip, 1) = B(ip, 3) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2) - DL(ip, 4) * DU(is, 3);
    DU(ip, 1) = (B(ip, 4) - DL(ip, 3) * DU(ise, 3)) / DL(ip, 1);
    DU(ip, 2) = -DL(ip, 2) * DU(iw, 3) / DL(ip, 1);
    for (ip = nij - ni + 2; ip <= nij - 1; ip++) {
        iw = ip - 1; is = ip - ni; ise = is + 1;
        DL(ip, 4) = B(ip, 1);
        DL(ip, 3) = -DL(ip, 4) * DU(is, 1);
        DL(ip, 2) = B(ip, 2) - DL(ip, 4) * DU(is, 2);
        DL(ip, 1) = B(ip, 3) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2) - DL(ip, 4) * DU(is, 3);
        DU(ip, 1) = (B(ip, 4) - DL(ip, 3) * DU(ise, 3)) / DL(ip, 1);
    }
    ip = nij;
    iw = ip - 1; is = ip - ni; ise = is + 1;
    DL(ip, 4) = B(ip, 1);
    DL(ip, 3) = -DL(ip, 4) * DU(is, 1);
    DL(ip, 2) = B(ip, 2) - DL(ip, 4) * DU(is, 2);
    DL(ip, 1) = B(ip, 3) - DL(ip, 2) * DU(iw, 1) - DL(ip, 3) * DU(ise, 2) - DL(ip, 4) * DU(is, 3);
}

int orc_msi9_solve(int nx, int ny, int nitm, double tol, const double *a,
                   const double *b, double *x)
{
    size_t N = (size_t)nx * (size_t)ny;
    double *dl = (double *)calloc(5 * N, sizeof(double));
    double *du = (double *)calloc(4 * N, sizeof(double));
    orc_lu2d9(a, dl, du, (int)N, nx, ny);
    int nit = orc_fb2d9(a, dl, du, ny, nx, (int)N, x, tol, nitm, b);
    free(dl); free(du);
    return nit;
}

int orc_msi5_solve(int nx, int ny, int nitm, double tol, const double *a,
                   const double *b, double *x)
{
    size_t N = (size_t)nx * (size_t)ny;
    double *dl = (double *)calloc(4 * N, sizeof(double));
    double *du = (double *)calloc(3 * N, sizeof(double));
    orc_lu2d5(a, dl, du, (int)N, nx, ny);
    int nit = orc_fb2d5(a, dl, du, ny, nx, (int)N, x, tol, nitm, b);
    free(dl); free(du);
    return nit;
}

/* ---- line TDMA ---------------------------------------------------------- */
#define A9(np, k) a[((size_t)(k) - 1) * N + (size_t)(np) - 1]
#define X(np) x[(size_t)(np) - 1]
#define BB(np) b[(size_t)(np) - 1]
#define PP(np) P[(size_t)(np) - 1]
#define QQ(np) Q[(size_t)(np) - 1]

void orc_tdma2d9(int nx, int ny, int nitm, const double *a, const double *b, double *x)
{
    size_t N = (size_t)nx * (size_t)ny;
    double *P = (double *)calloc(N, sizeof(double));
    double *Q = (double *)calloc(N, sizeof(double));
    int i, j, it, npsw, nps, npse, npw, np, npe, npnw, npn, npne;
    double D;
    for (it = 1; it <= nitm; it++) {
        /* x lines: src/solvers/tdma2d9.f90:80-172 */
        for (j = 1; j <= ny; j++) {
            i = 1;
            np = nx * (j - 1) + i; nps = np - nx; npn = np + nx; npse = nps + 1; npne = npn + 1;
            if (j == 1)
                D = BB(np) - A9(np, 8) * X(npn) - A9(np, 9) * X(npne);
            else if (j == ny)
                D = BB(np) - A9(np, 2) * X(nps) - A9(np, 3) * X(npse);
            else
                D = BB(np) - A9(np, 2) * X(nps) - A9(np, 3) * X(npse)
                  - A9(np, 8) * X(npn) - A9(np, 9) * X(npne);
            PP(np) = -A9(np, 6) / A9(np, 5);
            QQ(np) = D / A9(np, 5);
            for (i = 2; i <= nx - 1; i++) {
                np = nx * (j - 1) + i; nps = np - nx; npn = np + nx;
                npsw = nps - 1; npse = nps + 1; npnw = npn - 1; npne = npn + 1;
                if (j == 1)
                    D = BB(np) - A9(np, 7) * X(npnw) - A9(np, 8) * X(npn) - A9(np, 9) * X(npne);
                else if (j == ny)
                    D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 2) * X(nps) - A9(np, 3) * X(npse);
                else
                    D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 2) * X(nps) - A9(np, 3) * X(npse)
                      - A9(np, 7) * X(npnw) - A9(np, 8) * X(npn) - A9(np, 9) * X(npne);
                PP(np) = -A9(np, 6) / (A9(np, 5) + A9(np, 4) * PP(np - 1));
                QQ(np) = (D - A9(np, 4) * QQ(np - 1)) / (A9(np, 5) + A9(np, 4) * PP(np - 1));
            }
            i = nx;
            np = nx * (j - 1) + i; nps = np - nx; npn = np + nx; npsw = nps - 1; npnw = npn - 1;
            if (j == 1)
                D = BB(np) - A9(np, 7) * X(npnw) - A9(np, 8) * X(npn);
            else if (j == ny)
                D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 2) * X(nps);
            else
                D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 2) * X(nps)
                  - A9(np, 7) * X(npnw) - A9(np, 8) * X(npn);
            PP(np) = -A9(np, 6) / (A9(np, 5) + A9(np, 4) * PP(np - 1));
            QQ(np) = (D - A9(np, 4) * QQ(np - 1)) / (A9(np, 5) + A9(np, 4) * PP(np - 1));
        }
        for (j = 1; j <= ny; j++) {
            i = nx; np = nx * (j - 1) + i;
            X(np) = QQ(np);
            for (i = nx - 1; i >= 1; i--) {
                np = nx * (j - 1) + i;
                X(np) = PP(np) * X(np + 1) + QQ(np);
            }
        }
        /* y lines: src/solvers/tdma2d9.f90:201-315 */
        for (i = 1; i <= nx; i++) {
            j = 1;
            np = nx * (j - 1) + i; npn = np + nx; npw = np - 1; npe = np + 1;
            npnw = npn - 1; npne = npn + 1;
            if (i == 1)
                D = BB(np) - A9(np, 6) * X(npe) - A9(np, 9) * X(npne);
            else if (i == nx)
                D = BB(np) - A9(np, 4) * X(npw) - A9(np, 7) * X(npnw);
            else
                D = BB(np) - A9(np, 4) * X(npw) - A9(np, 7) * X(npnw)
                  - A9(np, 6) * X(npe) - A9(np, 9) * X(npne);
            PP(np) = -A9(np, 8) / A9(np, 5);
            QQ(np) = D / A9(np, 5);
            for (j = 2; j <= ny - 1; j++) {
                np = nx * (j - 1) + i; nps = np - nx; npn = np + nx; npw = np - 1; npe = np + 1;
                npsw = nps - 1; npse = nps + 1; npnw = npn - 1; npne = npn + 1;
                if (i == 1)
                    D = BB(np) - A9(np, 3) * X(npse) - A9(np, 6) * X(npe) - A9(np, 9) * X(npne);
                else if (i == nx)
                    D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 4) * X(npw) - A9(np, 7) * X(npnw);
                else
                    D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 4) * X(npw) - A9(np, 7) * X(npnw)
                      - A9(np, 3) * X(npse) - A9(np, 6) * X(npe) - A9(np, 9) * X(npne);
                PP(np) = -A9(np, 8) / (A9(np, 5) + A9(np, 2) * PP(np - nx));
                QQ(np) = (D - A9(np, 2) * QQ(np - nx)) / (A9(np, 5) + A9(np, 2) * PP(np - nx));
            }
            j = ny;
            np = nx * (j - 1) + i; nps = np - nx; npw = np - 1; npe = np + 1;
            npsw = nps - 1; npse = nps + 1;
            if (i == 1)
                D = BB(np) - A9(np, 3) * X(npse) - A9(np, 6) * X(npe);
            else if (i == nx)
                D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 4) * X(npw);
            else
                D = BB(np) - A9(np, 1) * X(npsw) - A9(np, 4) * X(npw)
                  - A9(np, 3) * X(npse) - A9(np, 6) * X(npe);
            PP(np) = -A9(np, 8) / (A9(np, 5) + A9(np, 2) * PP(np - nx));
            QQ(np) = (D - A9(np, 2) * QQ(np - nx)) / (A9(np, 5) + A9(np, 2) * PP(np - nx));
        }
        for (i = 1; i <= nx; i++) {
            j = ny; np = nx * (j - 1) + i;
            X(np) = QQ(np);
            for (j = ny - 1; j >= 1; j--) {
                np = nx * (j - 1) + i;
                X(np) = X(np + nx) * PP(np) + QQ(np);
            }
        }
    }
    free(P); free(Q);
}

#define A5(np, k) a[((size_t)(k) - 1) * N + (size_t)(np) - 1]

/* src/solvers/tdma2d5.f90:38-241 */
void orc_tdma2d5(int nx, int ny, int nitm, const double *a, const double *b, double *x)
{
    size_t N = (size_t)nx * (size_t)ny;
    double *P = (double *)calloc(N, sizeof(double));
    double *Q = (double *)calloc(N, sizeof(double));
    int i, j, np, npn, nps, it;
    double D;
    for (it = 1; it <= nitm; it++) {
        for (j = 1; j <= ny; j++) {
            i = 1;
            np = nx * (j - 1) + i; nps = np - nx; npn = np + nx;
            if (j == 1) D = BB(np) - A5(np, 5) * X(npn);
            else if (j == ny) D = BB(np) - A5(np, 1) * X(nps);
            else D = BB(np) - A5(np, 5) * X(npn) - A5(np, 1) * X(nps);
            PP(np) = -A5(np, 4) / A5(np, 3);
            QQ(np) = D / A5(np, 3);
            for (i = 2; i <= nx; i++) {
                np = nx * (j - 1) + i; nps = np - nx; npn = np + nx;
                if (j == 1) D = BB(np) - A5(np, 5) * X(npn);
                else if (j == ny) D = BB(np) - A5(np, 1) * X(nps);
                else D = BB(np) - A5(np, 5) * X(npn) - A5(np, 1) * X(nps);
                PP(np) = -A5(np, 4) / (A5(np, 3) + A5(np, 2) * PP(np - 1));
                QQ(np) = (D - A5(np, 2) * QQ(np - 1)) / (A5(np, 3) + A5(np, 2) * PP(np - 1));
            }
        }
        for (j = 1; j <= ny; j++) {
            i = nx; np = nx * (j - 1) + i;
            X(np) = QQ(np);
            for (i = nx - 1; i >= 1; i--) {
                np = nx * (j - 1) + i;
                X(np) = PP(np) * X(np + 1) + QQ(np);
            }
        }
        for (i = 1; i <= nx; i++) {
            j = 1; np = nx * (j - 1) + i;
            if (i == 1) D = BB(np) - A5(np, 4) * X(np + 1);
            else if (i == nx) D = BB(np) - A5(np, 2) * X(np - 1);
            else D = BB(np) - A5(np, 2) * X(np - 1) - A5(np, 4) * X(np + 1);
            PP(np) = -A5(np, 5) / A5(np, 3);
            QQ(np) = D / A5(np, 3);
            for (j = 2; j <= ny; j++) {
                np = nx * (j - 1) + i;
                if (i == 1) D = BB(np) - A5(np, 4) * X(np + 1);
                else if (i == nx) D = BB(np) - A5(np, 2) * X(np - 1);
                else D = BB(np) - A5(np, 2) * X(np - 1) - A5(np, 4) * X(np + 1);
                PP(np) = -A5(np, 5) / (A5(np, 3) + A5(np, 1) * PP(np - nx));
                QQ(np) = (D - A5(np, 1) * QQ(np - nx)) / (A5(np, 3) + A5(np, 1) * PP(np - nx));
            }
        }
        for (i = 1; i <= nx; i++) {
            j = ny; np = nx * (j - 1) + i;
            X(np) = QQ(np);
            for (j = ny - 1; j >= 1; j--) {
                np = nx * (j - 1) + i;
                X(np) = X(np + nx) * PP(np) + QQ(np);
            }
        }
    }
    free(P); free(Q);
}

/* Thomas algorithm for one line, in the recurrence form of tdma2d9's
 * x-line sweep: P = -ae/(ap + aw P_w), Q = (d - aw Q_w)/(ap + aw P_w). */
void orc_tdma_line(int n, const double *aw, const double *ap, const double *ae,
                   const double *d, double *x)
{
    double *P = (double *)malloc(sizeof(double) * (size_t)n);
    double *Q = (double *)malloc(sizeof(double) * (size_t)n);
    P[0] = -ae[0] / ap[0];
    Q[0] = d[0] / ap[0];
    for (int i = 1; i < n; i++) {
        P[i] = -ae[i] / (ap[i] + aw[i] * P[i - 1]);
        Q[i] = (d[i] - aw[i] * Q[i - 1]) / (ap[i] + aw[i] * P[i - 1]);
    }
    x[n - 1] = Q[n - 1];
    for (int i = n - 2; i >= 0; i--) x[i] = P[i] * x[i + 1] + Q[i];
    free(P); free(Q);
}

/* ---- norms: src/solvers/mod_solvers.f90:91-277 -------------------------- */
double orc_norm_l1_5d(int nx, int ny, const double *var, const double *b,
                      const double *a, double norm)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i, nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
            norm = norm + fabs(+A5(np, 1) * V(var, nps) + A5(np, 2) * V(var, npw)
                               + A5(np, 3) * V(var, np) + A5(np, 4) * V(var, npe)
                               + A5(np, 5) * V(var, npn) - BB(np));
        }
    return norm;
}

static double res9(int nx, size_t N, const double *a, const double *var,
                   const double *b, int np)
{
    int nps = np - nx, npn = np + nx, npw = np - 1, npe = np + 1;
    int npsw = nps - 1, npse = nps + 1, npnw = npn - 1, npne = npn + 1;
    return +A9(np, 1) * V(var, npsw) + A9(np, 2) * V(var, nps) + A9(np, 3) * V(var, npse)
           + A9(np, 4) * V(var, npw) + A9(np, 5) * V(var, np) + A9(np, 6) * V(var, npe)
           + A9(np, 7) * V(var, npnw) + A9(np, 8) * V(var, npn) + A9(np, 9) * V(var, npne)
           - BB(np);
}

double orc_norm_l1_9d(int nx, int ny, const double *var, const double *b,
                      const double *a, double norm)
{
    size_t N = (size_t)nx * (size_t)ny;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++)
            norm = norm + fabs(res9(nx, N, a, var, b, nx * (j - 1) + i));
    return norm;
}

double orc_norm_l1_9d_relative(int nx, int ny, const double *var, const double *b,
                               const double *a, double norm)
{
    size_t N = (size_t)nx * (size_t)ny;
    const double eps = 10.0 * 2.220446049250313e-16;
    double norma = 0.0, normb = 0.0;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (j - 1) + i;
            norma = norma + fabs(res9(nx, N, a, var, b, np));
            normb = normb + fabs(BB(np));
        }
    if (normb > eps) norm = norm + norma / normb;
    else norm = norm + norma;
    return norm;
}

double orc_norm_l1_b(int nx, int ny, const double *b)
{
    double norm = 0.0;
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx - 1; i++) norm = norm + fabs(BB(nx * (j - 1) + i));
    return norm;
}
