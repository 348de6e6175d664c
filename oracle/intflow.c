/*
 * intflow.c -- oracle restatement of MACH-2D's internal-flow plug-in
 * (src/user/internal_flow/mod_intflow.f90).  TEST INFRASTRUCTURE ONLY (see
 * m2d_oracle.h).  Parity unpinned.
 */
#include <math.h>
#include <stdlib.h>
#include "m2d_oracle.h"

#define F(v, np) (v)[(size_t)(np) - 1]
#define A(np, k) a[((size_t)(k) - 1) * N + (size_t)(np) - 1]
#define V1(v, i) (v)[(size_t)(i) - 1]

/* mod_intflow.f90:142-210 */
void orc_get_u_v_north_slip(int nx, int ny, const double *x, const double *xp,
    const double *xk, const double *yk, const double *u, const double *v,
    double *ubn, double *vbn)
{
    int j = ny - 1, np, npe, npw, npee, npww;
    for (int i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        double Up = sqrt(F(u, np) * F(u, np) + F(v, np) * F(v, np));
        double signal = copysign(1.0, F(xk, np) * F(u, np) + F(yk, np) * F(v, np));
        double t = sqrt(F(xk, np) * F(xk, np) + F(yk, np) * F(yk, np));
        double tx = F(xk, np) / t, ty = F(yk, np) / t;
        V1(ubn, i) = signal * Up * tx;
        V1(vbn, i) = signal * Up * ty;
    }
    np = nx * (j - 1) + 1; npe = np + 1; npee = npe + 1;
    V1(ubn, 1) = V1(ubn, 2) + (V1(ubn, 2) - V1(ubn, 3)) * (F(xp, npe) - F(x, np)) / (F(xp, npee) - F(xp, npe));
    V1(vbn, 1) = V1(vbn, 2) + (V1(vbn, 2) - V1(vbn, 3)) * (F(xp, npe) - F(x, np)) / (F(xp, npee) - F(xp, npe));
    np = nx * (j - 1) + nx; npw = np - 1; npww = npw - 1;
    V1(ubn, nx) = V1(ubn, nx - 1) + (V1(ubn, nx - 1) - V1(ubn, nx - 2)) * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww));
    V1(vbn, nx) = V1(vbn, nx - 1) + (V1(vbn, nx - 1) - V1(vbn, nx - 2)) * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww));
}

static void zero_row(double *a, size_t N, int np, int nd)
{
    for (int k = 1; k <= nd; k++) A(np, k) = 0.0;
}

/* mod_intflow.f90:214-301 */
void orc_intflow_set_bcu(int nx, int ny, int modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u,
    const double *v, double *a, double *b)
{
    size_t N = (size_t)nx * (size_t)ny;
    int i, j, np, npe, npee, npw, npww;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npe = np + 1; npee = npe + 1;
        zero_row(a, N, np, 9); A(np, 6) = -1.0; A(np, 5) = 1.0;
        F(b, np) = (2.0 * F(xp, npe)) / (F(xp, npee) - F(xp, npe)) * (F(u, npe) - F(u, npee));
    }
    i = nx;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npw = np - 1; npww = npw - 1;
        zero_row(a, N, np, 9); A(np, 4) = -1.0; A(np, 5) = 1.0;
        F(b, np) = 2.0 * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww)) * (F(u, npw) - F(u, npww));
    }
    j = 1;
    for (i = 1; i <= nx; i++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 9); A(np, 8) = -1.0; A(np, 5) = 1.0;
        F(b, np) = 0.0;
    }
    j = ny;
    if (modvis == 1) {
        for (i = 1; i <= nx; i++) {
            np = nx * (j - 1) + i;
            zero_row(a, N, np, 9); A(np, 2) = 1.0; A(np, 5) = 1.0;
            F(b, np) = 0.0;
        }
    } else {
        double *ubn = (double *)malloc(sizeof(double) * (size_t)nx);
        double *vbn = (double *)malloc(sizeof(double) * (size_t)nx);
        orc_get_u_v_north_slip(nx, ny, x, xp, xk, yk, u, v, ubn, vbn);
        for (i = 1; i <= nx; i++) {
            np = nx * (j - 1) + i;
            zero_row(a, N, np, 9); A(np, 2) = 1.0; A(np, 5) = 1.0;
            F(b, np) = 2.0 * V1(ubn, i);
        }
        free(ubn); free(vbn);
    }
}

/* mod_intflow.f90:305-392 */
void orc_intflow_set_bcv(int nx, int ny, int modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u,
    const double *v, double *a, double *b)
{
    size_t N = (size_t)nx * (size_t)ny;
    int i, j, np, npw, npww;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 9); A(np, 6) = 1.0; A(np, 5) = 1.0;
        F(b, np) = 0.0;
    }
    i = nx;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npw = np - 1; npww = npw - 1;
        zero_row(a, N, np, 9); A(np, 4) = -1.0; A(np, 5) = 1.0;
        F(b, np) = (F(v, npw) - F(v, npww)) * 2.0 * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww));
    }
    j = 1;
    for (i = 1; i <= nx; i++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 9); A(np, 8) = 1.0; A(np, 5) = 1.0;
        F(b, np) = 0.0;
    }
    j = ny;
    if (modvis == 1) {
        for (i = 1; i <= nx; i++) {
            np = nx * (j - 1) + i;
            zero_row(a, N, np, 9); A(np, 2) = 1.0; A(np, 5) = 1.0;
            F(b, np) = 0.0;
        }
    } else {
        double *ubn = (double *)malloc(sizeof(double) * (size_t)nx);
        double *vbn = (double *)malloc(sizeof(double) * (size_t)nx);
        orc_get_u_v_north_slip(nx, ny, x, xp, xk, yk, u, v, ubn, vbn);
        for (i = 1; i <= nx; i++) {
            np = nx * (j - 1) + i;
            zero_row(a, N, np, 9); A(np, 2) = 1.0; A(np, 5) = 1.0;
            F(b, np) = 2.0 * V1(vbn, i);
        }
        free(ubn); free(vbn);
    }
}

/* mod_intflow.f90:396-459 (corner rows are left untouched) */
void orc_intflow_set_bcpl(int nx, int ny, const double *x, const double *xp,
    const double *pl, const double *plin, double *a, double *bp)
{
    size_t N = (size_t)nx * (size_t)ny;
    int i, j, np, npw, npww;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 5); A(np, 4) = 1.0; A(np, 3) = 1.0;
        F(bp, np) = 2.0 * V1(plin, j);
    }
    i = nx;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npw = np - 1; npww = npw - 1;
        zero_row(a, N, np, 5); A(np, 2) = -1.0; A(np, 3) = 1.0;
        F(bp, np) = 2.0 * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww)) * (F(pl, npw) - F(pl, npww));
    }
    j = 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 5); A(np, 5) = -1.0; A(np, 3) = 1.0;
        F(bp, np) = 0.0;
    }
    j = ny;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 5); A(np, 1) = -1.0; A(np, 3) = 1.0;
        F(bp, np) = 0.0;
    }
}

/* mod_intflow.f90:464-550 */
void orc_intflow_set_bcT(int nx, int ny, const double *x, const double *xp,
    const double *T, double Twall, const double *Tin, double *a, double *bt)
{
    size_t N = (size_t)nx * (size_t)ny;
    int i, j, np, npw, npww, ccTw = 0;
    if (Twall > 0.0) ccTw = 1;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 9); A(np, 6) = 1.0; A(np, 5) = 1.0;
        F(bt, np) = 2.0 * V1(Tin, j);
    }
    i = nx;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npw = np - 1; npww = npw - 1;
        zero_row(a, N, np, 9); A(np, 4) = -1.0; A(np, 5) = 1.0;
        F(bt, np) = 2.0 * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww)) * (F(T, npw) - F(T, npww));
    }
    j = 1;
    for (i = 1; i <= nx; i++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 9); A(np, 8) = -1.0; A(np, 5) = 1.0;
        F(bt, np) = 0.0;
    }
    j = ny;
    for (i = 1; i <= nx; i++) {
        np = nx * (j - 1) + i;
        zero_row(a, N, np, 9);
        if (ccTw == 0) { A(np, 2) = -1.0; A(np, 5) = 1.0; F(bt, np) = 0.0; }
        else { A(np, 2) = 1.0; A(np, 5) = 1.0; F(bt, np) = 2.0 * Twall; }
    }
}

/* mod_intflow.f90:557-688 */
void orc_intflow_boundary_T_from_H_conservation(int nx, int ny, double Cpref,
    double Href, const double *Tin, const double *u, const double *ue,
    const double *un, const double *v, const double *ve, const double *vn,
    double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs)
{
    (void)u; (void)v;
    int i, j, np, npe, npn, nps;
    i = nx - 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        V1(Tbe, j) = (Href - (F(ue, np) * F(ue, np) + F(ve, np) * F(ve, np)) / 2.0) / Cpref;
        npe = np + 1;
        F(T, npe) = 2.0 * V1(Tbe, j) - F(T, np);
    }
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        V1(Tbw, j) = V1(Tin, j);
        npe = np + 1;
        F(T, np) = 2.0 * V1(Tbw, j) - F(T, npe);
    }
    j = ny - 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        V1(Tbn, i) = (Href - (F(un, np) * F(un, np) + F(vn, np) * F(vn, np)) / 2.0) / Cpref;
        npn = np + nx;
        F(T, npn) = 2.0 * V1(Tbn, i) - F(T, np);
    }
    j = 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        V1(Tbs, i) = (Href - (F(un, np) * F(un, np) + F(vn, np) * F(vn, np)) / 2.0) / Cpref;
        npn = np + nx;
        F(T, np) = 2.0 * V1(Tbs, i) - F(T, npn);
    }
    np = 1; npn = np + nx; F(T, np) = F(T, npn);
    np = nx; npn = np + nx; F(T, np) = F(T, npn);
    np = nx * (ny - 1) + 1; nps = np - nx; F(T, np) = F(T, nps);
    np = nx * (ny - 1) + nx; nps = np - nx; F(T, np) = F(T, nps);
}

/* mod_intflow.f90:692-787 */
void orc_intflow_velocities_at_boundary_faces(int nx, int ny, int modvis,
    const double *x, const double *xp, const double *xe, const double *ye,
    const double *xk, const double *yk, const double *u, const double *v,
    double *ue, double *ve, double *un, double *vn, double *Uce, double *Vcn)
{
    int i, j, np, npn, npe;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npe = np + 1;
        F(ue, np) = (F(u, np) + F(u, npe)) / 2.0;
        F(ve, np) = 0.0;
        F(Uce, np) = F(ue, np) * F(ye, np) - F(ve, np) * F(xe, np);
    }
    i = nx - 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npe = np + 1;
        F(ue, np) = (F(u, np) + F(u, npe)) / 2.0;
        F(ve, np) = (F(v, np) + F(v, npe)) / 2.0;
        F(Uce, np) = F(ue, np) * F(ye, np) - F(ve, np) * F(xe, np);
    }
    j = 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i; npn = np + nx;
        F(un, np) = (F(u, np) + F(u, npn)) / 2.0;
        F(vn, np) = 0.0;
        F(Vcn, np) = 0.0;
    }
    double *ubn = (double *)calloc((size_t)nx, sizeof(double));
    double *vbn = (double *)calloc((size_t)nx, sizeof(double));
    if (modvis == 0) orc_get_u_v_north_slip(nx, ny, x, xp, xk, yk, u, v, ubn, vbn);
    j = ny - 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        F(un, np) = V1(ubn, i);
        F(vn, np) = V1(vbn, i);
        F(Vcn, np) = 0.0;
    }
    free(ubn); free(vbn);
}

/* mod_intflow.f90:791-877 */
void orc_intflow_boundary_simplec(int nx, int ny, int modvis, double *due,
    double *dve, double *dun, double *dvn, double *de, double *dn)
{
    (void)modvis;
    int i, j, np;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        F(due, np) = F(due, np + 1); F(dve, np) = 0.0; F(de, np) = F(de, np + 1);
    }
    i = nx - 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        F(due, np) = F(due, np - 1); F(dve, np) = F(dve, np - 1); F(de, np) = F(de, np - 1);
    }
    j = 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        F(dun, np) = F(dun, np + nx); F(dvn, np) = 0.0; F(dn, np) = 0.0;
    }
    j = ny - 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        F(dun, np) = 0.0; F(dvn, np) = 0.0; F(dn, np) = 0.0;
    }
}

/* mod_intflow.f90:881-964 */
void orc_intflow_extrapolate_u_v_to_fictitious(int nx, int ny, int modvis,
    const double *x, const double *xp, const double *xk, const double *yk,
    double *u, double *v)
{
    int i, j, np, npe, npee, npw, npww, nps, npn;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npe = np + 1; npee = np + 2;
        F(u, np) = F(u, npe) + 2.0 * F(xp, npe) / (F(xp, npee) - F(xp, npe)) * (F(u, npe) - F(u, npee));
        F(v, np) = -F(v, npe);
    }
    i = nx;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npw = np - 1; npww = np - 2;
        F(u, np) = F(u, npw) + 2.0 * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww)) * (F(u, npw) - F(u, npww));
        F(v, np) = F(v, npw) + 2.0 * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww)) * (F(v, npw) - F(v, npww));
    }
    j = 1;
    for (i = 1; i <= nx; i++) {
        np = nx * (j - 1) + i; npn = np + nx;
        F(u, np) = F(u, npn);
        F(v, np) = -F(v, npn);
    }
    j = ny;
    if (modvis == 1) {
        for (i = 1; i <= nx; i++) {
            np = nx * (j - 1) + i; nps = np - nx;
            F(u, np) = -F(u, nps);
            F(v, np) = -F(v, nps);
        }
    } else {
        double *ubn = (double *)malloc(sizeof(double) * (size_t)nx);
        double *vbn = (double *)malloc(sizeof(double) * (size_t)nx);
        orc_get_u_v_north_slip(nx, ny, x, xp, xk, yk, u, v, ubn, vbn);
        for (i = 1; i <= nx; i++) {
            np = nx * (j - 1) + i; nps = np - nx;
            F(u, np) = -F(u, nps) + 2.0 * V1(ubn, i);
            F(v, np) = -F(v, nps) + 2.0 * V1(vbn, i);
        }
        free(ubn); free(vbn);
    }
}

/* mod_intflow.f90:968-1006 */
void orc_get_uin_vin_pin_Tin_Mw(int nx, int ny, double gamma, double Rg, double po,
    double T0, const double *u, double *uin, double *vin, double *pin,
    double *Tin, double *Mw)
{
    int i = 1;
    for (int j = 2; j <= ny - 1; j++) {
        int np = nx * (j - 1) + i, npe = np + 1;
        V1(uin, j) = (F(u, np) + F(u, npe)) / 2.0;
        V1(vin, j) = 0.0;
        V1(Tin, j) = T0 - (gamma - 1.0) / (2.0 * gamma * Rg)
                   * (V1(uin, j) * V1(uin, j) + V1(vin, j) * V1(vin, j));
        V1(Mw, j) = sqrt((V1(uin, j) * V1(uin, j) + V1(vin, j) * V1(vin, j)) / (gamma * Rg * V1(Tin, j)));
        V1(pin, j) = po * pow(1.0 + 0.5 * (gamma - 1.0) * (V1(Mw, j) * V1(Mw, j)), -gamma / (gamma - 1.0));
    }
}

/* mod_intflow.f90:1010-1101 */
void orc_get_plin_and_p_fictitious(int nx, int ny, const double *x,
    const double *xp, const double *pina, const double *pin, double *plin,
    double *p)
{
    int i, j, np, npe, npw, npww, npn, nps;
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npe = np + 1;
        F(p, np) = 2.0 * V1(pin, j) - F(p, npe);
        V1(plin, j) = V1(pin, j) - V1(pina, j);
    }
    i = nx;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i; npw = np - 1; npww = npw - 1;
        F(p, np) = F(p, npw) + 2.0 * (F(x, npw) - F(xp, npw)) / (F(xp, npw) - F(xp, npww)) * (F(p, npw) - F(p, npww));
    }
    j = 1;
    for (i = 2; i <= nx - 1; i++) { np = i; npn = np + nx; F(p, np) = F(p, npn); }
    j = ny;
    for (i = 2; i <= nx - 1; i++) { np = nx * (j - 1) + i; nps = np - nx; F(p, np) = F(p, nps); }
    np = 1; F(p, np) = F(p, np + nx);
    np = nx; F(p, np) = F(p, np + nx);
    np = nx * (ny - 1) + 1; F(p, np) = F(p, np - nx);
    np = nx * (ny - 1) + nx; F(p, np) = F(p, np - nx);
}

/* mod_intflow.f90:1591-1643 */
void orc_get_mass_flow_rate_and_thrust(int nx, int ny, const double *re,
    const double *roe, const double *u, const double *Uce, double *fmi,
    double *fme, double *Fd)
{
    const double pi = acos(-1.0);
    double s = 0.0;
    int i = 1;
    for (int j = 2; j <= ny - 1; j++) {
        int np = nx * (j - 1) + i;
        s = s + F(re, np) * F(roe, np) * F(Uce, np);
    }
    *fmi = s * 2.0 * pi;
    double e = 0.0, d = 0.0;
    i = nx - 1;
    for (int j = 2; j <= ny - 1; j++) {
        int np = nx * (j - 1) + i;
        e = e + F(re, np) * F(roe, np) * F(Uce, np);
        d = d + F(re, np) * F(roe, np) * F(Uce, np) * (F(u, np) + F(u, np + 1)) / 2.0;
    }
    *fme = e * 2.0 * pi;
    *Fd = d * 2.0 * pi;
}

/* mod_intflow.f90:1492-1503 */
double orc_get_isentropic_mass_flow(double po, double T0, double gamma, double Rg,
                                    double Sg)
{
    return po * Sg * sqrt(gamma / (Rg * T0)
                          * pow(2.0 / (gamma + 1.0), (gamma + 1.0) / (gamma - 1.0)));
}

/* mod_intflow.f90:1507-1557 */
double orc_get_mach_area(int kf, double ar, double gamma)
{
    double M0, M1, M = 1.0;
#define FMA_(xx) (pow(2.0 * (1.0 + (gamma - 1.0) * ((xx) * (xx)) / 2.0) / (gamma + 1.0), \
                      (gamma + 1.0) / (gamma - 1.0)) - ((xx) * ar) * ((xx) * ar))
    if (fabs(ar - 1.0) < 1.0e-15) return 1.0;
    if (kf == 0) { M0 = 1.0e-4; M1 = 1.0; }
    else { M0 = 1.0; M1 = 100.0; }
    for (int it = 1; it <= 1000; it++) {
        M = 0.5 * (M0 + M1);
        if (FMA_(M) * FMA_(M0) > 0) M0 = M; else M1 = M;
        if (fabs(M1 - M0) < 1.0e-15) break;
    }
#undef FMA_
    return M;
}

/* mod_intflow.f90:1561-1587 */
int orc_get_ig(int nx, int ny, const double *y)
{
    int j = ny - 1;
    for (int i = 2; i <= nx - 1; i++) {
        int np = nx * (j - 1) + i;
        if (F(y, np - 1) < F(y, np)) return i - 1;
    }
    return 1;
}
