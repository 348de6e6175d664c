/*
 * extflow.c -- oracle restatement of MACH-2D's external-flow boundary plug-in:
 * the boundary-row routines of src/user/external_flow/mod_extflow.f90
 * (extflow_set_bcu/bcv/bcpl/bcro/bcT, :166-317), the boundary schemes they
 * call (get_bc_scheme_u/v/pl/ro/T, mod_extflow_procedures.f90:344-701) and
 * the strip helpers of src/boundary_conditions/mach2d_bc9d.f90 and
 * mach2d_bc5d.f90 (Dirichlet, null normal gradient, slip, corners, transfer).
 * The reference keeps UF, ROF, TF and Tsbc as module variables; here they
 * are arguments.  TEST INFRASTRUCTURE ONLY (see m2d_oracle.h).  Parity
 * unpinned.
 *
 * Strips follow the reference: a9bn(nx,9) etc. stored column-major, element
 * (i,k) at [(k-1)*n + i-1] with n = nx for north/south and ny for east/west.
 */
#include <math.h>
#include <string.h>
#include "m2d_oracle.h"

#define F(v, np) (v)[(size_t)(np) - 1]
#define S9(s, n, i, k) (s)[((size_t)(k) - 1) * (size_t)(n) + (size_t)(i) - 1]
#define V1(v, i) (v)[(size_t)(i) - 1]

static void row_zero(double *s, int n, int i, int nk)
{
    for (int k = 1; k <= nk; k++) S9(s, n, i, k) = 0.0;
}

/* mach2d_bc9d.f90:40-62 */
static void bc_dirichlet_south_9d(int nx, const double *Fbs, double *a, double *b)
{
    for (int i = 2; i <= nx - 1; i++) {
        row_zero(a, nx, i, 9);
        S9(a, nx, i, 5) = 1.0; S9(a, nx, i, 8) = 1.0;
        V1(b, i) = 2.0 * V1(Fbs, i);
    }
}
/* :67-89 */
static void bc_dirichlet_west_9d(int ny, const double *Fbw, double *a, double *b)
{
    for (int j = 2; j <= ny - 1; j++) {
        row_zero(a, ny, j, 9);
        S9(a, ny, j, 5) = 1.0; S9(a, ny, j, 6) = 1.0;
        V1(b, j) = 2.0 * V1(Fbw, j);
    }
}
/* :158-179 */
static void ibc_null_normal_grad_east_9d(int ny, double *a, double *b)
{
    for (int j = 2; j <= ny - 1; j++) {
        row_zero(a, ny, j, 9);
        S9(a, ny, j, 4) = -1.0; S9(a, ny, j, 5) = 1.0;
        V1(b, j) = 0.0;
    }
}
/* :184-263 */
static void bc_null_normal_grad_south_9d(int nx, int ny, const double *betan, const double *gamman, double *a,
                                         double *b)
{
    int j = 1, i = 2, np = nx * (j - 1) + i;
    double raux = (F(betan, np) / F(gamman, np)) / 2.0;
    row_zero(a, nx, i, 9);
    S9(a, nx, i, 5) = 1.0 - raux; S9(a, nx, i, 6) = raux; S9(a, nx, i, 8) = -1.0 - raux; S9(a, nx, i, 9) = raux;
    V1(b, i) = 0.0;
    for (i = 3; i <= nx - 2; i++) {
        np = nx * (j - 1) + i;
        raux = (F(betan, np) / F(gamman, np)) / 4.0;
        row_zero(a, nx, i, 9);
        S9(a, nx, i, 4) = -raux; S9(a, nx, i, 5) = 1.0; S9(a, nx, i, 6) = raux;
        S9(a, nx, i, 7) = -raux; S9(a, nx, i, 8) = -1.0; S9(a, nx, i, 9) = raux;
        V1(b, i) = 0.0;
    }
    i = nx - 1; np = nx * (j - 1) + i;
    raux = (F(betan, np) / F(gamman, np)) / 2.0;
    row_zero(a, nx, i, 9);
    S9(a, nx, i, 4) = -raux; S9(a, nx, i, 5) = 1.0 + raux; S9(a, nx, i, 7) = -raux; S9(a, nx, i, 8) = -1.0 + raux;
    V1(b, i) = 0.0;
}
/* :268-346 */
static void bc_null_normal_grad_west_9d(int nx, int ny, const double *alphae, const double *betae, double *a,
                                        double *b)
{
    int i = 1, j = 2, np = nx * (j - 1) + i;
    double raux = 0.5 * F(betae, np) / F(alphae, np);
    row_zero(a, ny, j, 9);
    S9(a, ny, j, 5) = 1.0 - raux; S9(a, ny, j, 6) = -1.0 - raux; S9(a, ny, j, 8) = raux; S9(a, ny, j, 9) = raux;
    V1(b, j) = 0.0;
    for (j = 3; j <= ny - 2; j++) {
        np = nx * (j - 1) + i;
        raux = 0.25 * F(betae, np) / F(alphae, np);
        row_zero(a, ny, j, 9);
        S9(a, ny, j, 2) = -raux; S9(a, ny, j, 3) = -raux; S9(a, ny, j, 5) = 1.0; S9(a, ny, j, 6) = -1.0;
        S9(a, ny, j, 8) = raux; S9(a, ny, j, 9) = raux;
        V1(b, j) = 0.0;
    }
    j = ny - 1; np = nx * (j - 1) + i;
    raux = 0.5 * F(betae, np) / F(alphae, np);
    row_zero(a, ny, j, 9);
    S9(a, ny, j, 2) = -raux; S9(a, ny, j, 3) = -raux; S9(a, ny, j, 5) = 1.0 + raux; S9(a, ny, j, 6) = -1.0 + raux;
    V1(b, j) = 0.0;
}
/* :352-439; comp 0 gives the u row (2 lambda xk), 1 the v row (2 lambda yk) */
static void bc_slip_south_9d(int nx, const double *xk, const double *yk, const double *u, const double *v, int comp,
                             double *a, double *b)
{
    const int j = 1;
    for (int i = 2; i <= nx - 1; i++) {
        row_zero(a, nx, i, 9);
        S9(a, nx, i, 5) = 1.0; S9(a, nx, i, 8) = 1.0;
        const int np = nx * (j - 1) + i, npn = np + nx;
        const double lambda = copysign(1.0, F(xk, np) * F(u, npn) + F(yk, np) * F(v, npn))
                            * sqrt((F(u, npn) * F(u, npn) + F(v, npn) * F(v, npn))
                                   / (F(xk, np) * F(xk, np) + F(yk, np) * F(yk, np)));
        V1(b, i) = 2.0 * lambda * (comp == 0 ? F(xk, np) : F(yk, np));
    }
}
/* :521-615 */
static void bc_corners_9d(int nx, int ny, double *an, double *as, double *ae, double *aw, double *bn, double *bs,
                          double *be, double *bw)
{
    const double third = -1.0 / 3.0;
    row_zero(as, nx, 1, 9);
    S9(as, nx, 1, 5) = 1.0; S9(as, nx, 1, 6) = third; S9(as, nx, 1, 8) = third; S9(as, nx, 1, 9) = third;
    V1(bs, 1) = 0.0;
    for (int k = 1; k <= 9; k++) S9(aw, ny, 1, k) = S9(as, nx, 1, k);
    V1(bw, 1) = V1(bs, 1);
    row_zero(as, nx, nx, 9);
    S9(as, nx, nx, 4) = third; S9(as, nx, nx, 5) = 1.0; S9(as, nx, nx, 7) = third; S9(as, nx, nx, 8) = third;
    V1(bs, nx) = 0.0;
    for (int k = 1; k <= 9; k++) S9(ae, ny, 1, k) = S9(as, nx, nx, k);
    V1(be, 1) = V1(bs, nx);
    row_zero(an, nx, 1, 9);
    S9(an, nx, 1, 2) = third; S9(an, nx, 1, 3) = third; S9(an, nx, 1, 5) = 1.0; S9(an, nx, 1, 6) = third;
    V1(bn, 1) = 0.0;
    for (int k = 1; k <= 9; k++) S9(aw, ny, ny, k) = S9(an, nx, 1, k);
    V1(bw, ny) = V1(bn, 1);
    row_zero(an, nx, nx, 9);
    S9(an, nx, nx, 1) = third; S9(an, nx, nx, 2) = third; S9(an, nx, nx, 4) = third; S9(an, nx, nx, 5) = 1.0;
    V1(bn, nx) = 0.0;
    for (int k = 1; k <= 9; k++) S9(ae, ny, ny, k) = S9(an, nx, nx, k);
    V1(be, ny) = V1(bn, nx);
}
/* :622-706 (nk = 9) and mach2d_bc5d.f90:213-297 (nk = 5) */
static void bc_transfer(int nx, int ny, int nk, const double *an, const double *as, const double *ae,
                        const double *aw, const double *bn, const double *bs, const double *be, const double *bw,
                        double *a, double *b)
{
    const size_t N = (size_t)nx * (size_t)ny;
    int i, j, np;
    j = ny;
    for (i = 1; i <= nx; i++) {
        np = nx * (j - 1) + i;
        for (int k = 1; k <= nk; k++) a[(size_t)(k - 1) * N + np - 1] = S9(an, nx, i, k);
        F(b, np) = V1(bn, i);
    }
    j = 1;
    for (i = 1; i <= nx; i++) {
        np = nx * (j - 1) + i;
        for (int k = 1; k <= nk; k++) a[(size_t)(k - 1) * N + np - 1] = S9(as, nx, i, k);
        F(b, np) = V1(bs, i);
    }
    i = nx;
    for (j = 1; j <= ny; j++) {
        np = nx * (j - 1) + i;
        for (int k = 1; k <= nk; k++) a[(size_t)(k - 1) * N + np - 1] = S9(ae, ny, j, k);
        F(b, np) = V1(be, j);
    }
    i = 1;
    for (j = 1; j <= ny; j++) {
        np = nx * (j - 1) + i;
        for (int k = 1; k <= nk; k++) a[(size_t)(k - 1) * N + np - 1] = S9(aw, ny, j, k);
        F(b, np) = V1(bw, j);
    }
}

/* strip buffers of one call: 9 (or 5) coefficient columns and a source each */
typedef struct {
    double an[9 * ORC_MAX_STRIP], as[9 * ORC_MAX_STRIP], ae[9 * ORC_MAX_STRIP], aw[9 * ORC_MAX_STRIP];
    double bn[ORC_MAX_STRIP], bs[ORC_MAX_STRIP], be[ORC_MAX_STRIP], bw[ORC_MAX_STRIP];
    double F[ORC_MAX_STRIP];
} strips9;

static strips9 g_st;

/* the north strip of every external-flow scheme: a P row with the
 * free-stream value (the "UDS approximation" of get_bc_scheme_*) */
static void north_free_stream(int nx, double value, double *an, double *bn)
{
    for (int i = 1; i <= nx; i++) {
        row_zero(an, nx, i, 9);
        S9(an, nx, i, 5) = 1.0;
        V1(bn, i) = value;
    }
}

/* get_bc_scheme_u (mod_extflow_procedures.f90:403-477) */
void orc_extflow_scheme_u(int nx, int ny, int modvis, double UF, const double *xk, const double *yk,
                          const double *alphae, const double *betae, const double *u, const double *v,
                          double *an, double *as, double *ae, double *aw, double *bn, double *bs, double *be,
                          double *bw)
{
    north_free_stream(nx, UF, an, bn);
    if (modvis == 0) {
        bc_slip_south_9d(nx, xk, yk, u, v, 0, as, bs);
    } else {
        for (int i = 1; i <= nx; i++) V1(g_st.F, i) = 0.0;
        bc_dirichlet_south_9d(nx, g_st.F, as, bs);
    }
    ibc_null_normal_grad_east_9d(ny, ae, be);
    bc_null_normal_grad_west_9d(nx, ny, alphae, betae, aw, bw);
    bc_corners_9d(nx, ny, an, as, ae, aw, bn, bs, be, bw);
}

/* get_bc_scheme_v (:481-556) */
void orc_extflow_scheme_v(int nx, int ny, int modvis, const double *xk, const double *yk, const double *u,
                          const double *v, double *an, double *as, double *ae, double *aw, double *bn, double *bs,
                          double *be, double *bw)
{
    north_free_stream(nx, 0.0, an, bn);
    if (modvis == 0) {
        bc_slip_south_9d(nx, xk, yk, u, v, 1, as, bs);
    } else {
        for (int i = 1; i <= nx; i++) V1(g_st.F, i) = 0.0;
        bc_dirichlet_south_9d(nx, g_st.F, as, bs);
    }
    ibc_null_normal_grad_east_9d(ny, ae, be);
    for (int j = 1; j <= ny; j++) V1(g_st.F, j) = 0.0;
    bc_dirichlet_west_9d(ny, g_st.F, aw, bw);
    bc_corners_9d(nx, ny, an, as, ae, aw, bn, bs, be, bw);
}

/* get_bc_scheme_ro (:560-623) */
void orc_extflow_scheme_ro(int nx, int ny, double ROF, const double *alphae, const double *betae,
                           const double *betan, const double *gamman, double *an, double *as, double *ae,
                           double *aw, double *bn, double *bs, double *be, double *bw)
{
    north_free_stream(nx, ROF, an, bn);
    bc_null_normal_grad_south_9d(nx, ny, betan, gamman, as, bs);
    ibc_null_normal_grad_east_9d(ny, ae, be);
    bc_null_normal_grad_west_9d(nx, ny, alphae, betae, aw, bw);
    bc_corners_9d(nx, ny, an, as, ae, aw, bn, bs, be, bw);
}

/* get_bc_scheme_T (:627-701); Tsbc < 0: adiabatic wall */
void orc_extflow_scheme_T(int nx, int ny, double TF, double Tsbc, const double *alphae, const double *betae,
                          const double *betan, const double *gamman, double *an, double *as, double *ae,
                          double *aw, double *bn, double *bs, double *be, double *bw)
{
    north_free_stream(nx, TF, an, bn);
    if (Tsbc < 0.0) {
        bc_null_normal_grad_south_9d(nx, ny, betan, gamman, as, bs);
    } else {
        for (int i = 1; i <= nx; i++) V1(g_st.F, i) = Tsbc;
        bc_dirichlet_south_9d(nx, g_st.F, as, bs);
    }
    ibc_null_normal_grad_east_9d(ny, ae, be);
    bc_null_normal_grad_west_9d(nx, ny, alphae, betae, aw, bw);
    bc_corners_9d(nx, ny, an, as, ae, aw, bn, bs, be, bw);
}

/* extflow_set_bcu (mod_extflow.f90:166-198) */
void orc_extflow_set_bcu(int nx, int ny, int modvis, double UF, const double *xk, const double *yk,
                         const double *alphae, const double *betae, const double *u, const double *v, double *au,
                         double *bu)
{
    strips9 *s = &g_st;
    orc_extflow_scheme_u(nx, ny, modvis, UF, xk, yk, alphae, betae, u, v, s->an, s->as, s->ae, s->aw, s->bn, s->bs,
                         s->be, s->bw);
    bc_transfer(nx, ny, 9, s->an, s->as, s->ae, s->aw, s->bn, s->bs, s->be, s->bw, au, bu);
}

/* extflow_set_bcv (:202-231) */
void orc_extflow_set_bcv(int nx, int ny, int modvis, const double *xk, const double *yk, const double *u,
                         const double *v, double *av, double *bv)
{
    strips9 *s = &g_st;
    orc_extflow_scheme_v(nx, ny, modvis, xk, yk, u, v, s->an, s->as, s->ae, s->aw, s->bn, s->bs, s->be, s->bw);
    bc_transfer(nx, ny, 9, s->an, s->as, s->ae, s->aw, s->bn, s->bs, s->be, s->bw, av, bv);
}

/* extflow_set_bcpl (:235-259) with get_bc_scheme_pl (mod_extflow_procedures.f90:344-399) and the
 * 5-diagonal helpers of mach2d_bc5d.f90 (:44-206) */
void orc_extflow_set_bcpl(int nx, int ny, double *ap, double *bp)
{
    strips9 *s = &g_st;
    double *an = s->an, *as = s->as, *ae = s->ae, *aw = s->aw;
    for (int i = 1; i <= nx; i++) {          /* north: P row, zero source */
        row_zero(an, nx, i, 5);
        S9(an, nx, i, 3) = 1.0;
        V1(s->bn, i) = 0.0;
    }
    for (int i = 2; i <= nx - 1; i++) {      /* get_ibc_null_normal_grad_south_5d */
        row_zero(as, nx, i, 5);
        S9(as, nx, i, 3) = 1.0; S9(as, nx, i, 5) = -1.0;
        V1(s->bs, i) = 0.0;
    }
    for (int j = 2; j <= ny - 1; j++) {      /* get_ibc_null_normal_grad_east_5d */
        row_zero(ae, ny, j, 5);
        S9(ae, ny, j, 2) = -1.0; S9(ae, ny, j, 3) = 1.0;
        V1(s->be, j) = 0.0;
    }
    for (int j = 2; j <= ny - 1; j++) {      /* get_ibc_null_normal_grad_west_5d */
        row_zero(aw, ny, j, 5);
        S9(aw, ny, j, 3) = 1.0; S9(aw, ny, j, 4) = -1.0;
        V1(s->bw, j) = 0.0;
    }
    /* get_bc_corners_5d: a unit P row at each corner */
    row_zero(as, nx, 1, 5); S9(as, nx, 1, 3) = 1.0; V1(s->bs, 1) = 0.0;
    for (int k = 1; k <= 5; k++) S9(aw, ny, 1, k) = S9(as, nx, 1, k);
    V1(s->bw, 1) = V1(s->bs, 1);
    row_zero(as, nx, nx, 5); S9(as, nx, nx, 3) = 1.0; V1(s->bs, nx) = 0.0;
    for (int k = 1; k <= 5; k++) S9(ae, ny, 1, k) = S9(as, nx, nx, k);
    V1(s->be, 1) = V1(s->bs, nx);
    row_zero(an, nx, 1, 5); S9(an, nx, 1, 3) = 1.0; V1(s->bn, 1) = 0.0;
    for (int k = 1; k <= 5; k++) S9(aw, ny, ny, k) = S9(an, nx, 1, k);
    V1(s->bw, ny) = V1(s->bn, 1);
    row_zero(an, nx, nx, 5); S9(an, nx, nx, 3) = 1.0; V1(s->bn, nx) = 0.0;
    for (int k = 1; k <= 5; k++) S9(ae, ny, ny, k) = S9(an, nx, nx, k);
    V1(s->be, ny) = V1(s->bn, nx);
    bc_transfer(nx, ny, 5, an, as, ae, aw, s->bn, s->bs, s->be, s->bw, ap, bp);
}

/* extflow_set_bcT (:289-317) */
void orc_extflow_set_bcT(int nx, int ny, double TF, double Tsbc, const double *alphae, const double *betae,
                         const double *betan, const double *gamman, double *at, double *bt)
{
    strips9 *s = &g_st;
    orc_extflow_scheme_T(nx, ny, TF, Tsbc, alphae, betae, betan, gamman, s->an, s->as, s->ae, s->aw, s->bn, s->bs,
                         s->be, s->bw);
    bc_transfer(nx, ny, 9, s->an, s->as, s->ae, s->aw, s->bn, s->bs, s->be, s->bw, at, bt);
}

/* tdma of mach2d_bc9d.f90:1292-1329: a(n,3) column-major W, P, E */
static void bc_tdma(int n, const double *a, const double *b, double *x, double *P, double *Q)
{
    P[0] = -a[2 * n] / a[n];
    Q[0] = b[0] / a[n];
    for (int i = 1; i < n; i++) {
        P[i] = -a[2 * n + i] / (a[n + i] + a[i] * P[i - 1]);
        Q[i] = (b[i] - a[i] * Q[i - 1]) / (a[n + i] + a[i] * P[i - 1]);
    }
    x[n - 1] = Q[n - 1];
    for (int i = n - 2; i >= 0; i--) x[i] = x[i + 1] * P[i] + Q[i];
}

static double g_ax[3 * ORC_MAX_STRIP], g_bx[ORC_MAX_STRIP], g_sx[ORC_MAX_STRIP], g_P[ORC_MAX_STRIP],
    g_Q[ORC_MAX_STRIP];

/* get_bc_extrapolation_9d (mach2d_bc9d.f90:711-972): itemax sweeps of the four
 * boundary lines, each a tridiagonal solve along the line with the other
 * couplings of its strip rows on the right-hand side */
void orc_bc_extrapolation_9d(int nx, int ny, int itemax, const double *an, const double *as, const double *ae,
                             const double *aw, const double *bn, const double *bs, const double *be,
                             const double *bw, double *Fv)
{
    double *ax = g_ax, *bx = g_bx, *sx = g_sx;
    int i, j, np;
    for (int it = 1; it <= itemax; it++) {
        /* north line */
        for (i = 1; i <= nx; i++) {
            ax[i - 1] = S9(an, nx, i, 4); ax[nx + i - 1] = S9(an, nx, i, 5); ax[2 * nx + i - 1] = S9(an, nx, i, 6);
        }
        j = ny;
        i = 1; np = nx * (j - 1) + i;
        bx[0] = V1(bn, i) - (S9(an, nx, i, 2) * F(Fv, np - nx) + S9(an, nx, i, 3) * F(Fv, np - nx + 1));
        for (i = 2; i <= nx - 1; i++) {
            np = nx * (j - 1) + i;
            bx[i - 1] = V1(bn, i) - (S9(an, nx, i, 1) * F(Fv, np - nx - 1) + S9(an, nx, i, 2) * F(Fv, np - nx)
                                     + S9(an, nx, i, 3) * F(Fv, np - nx + 1));
        }
        i = nx; np = nx * (j - 1) + i;
        bx[nx - 1] = V1(bn, i) - (S9(an, nx, i, 1) * F(Fv, np - nx - 1) + S9(an, nx, i, 2) * F(Fv, np - nx));
        bc_tdma(nx, ax, bx, sx, g_P, g_Q);
        for (i = 1; i <= nx; i++) F(Fv, nx * (j - 1) + i) = sx[i - 1];
        /* south line */
        for (i = 1; i <= nx; i++) {
            ax[i - 1] = S9(as, nx, i, 4); ax[nx + i - 1] = S9(as, nx, i, 5); ax[2 * nx + i - 1] = S9(as, nx, i, 6);
        }
        j = 1;
        i = 1; np = nx * (j - 1) + i;
        bx[0] = V1(bs, i) - (S9(as, nx, i, 8) * F(Fv, np + nx) + S9(as, nx, i, 9) * F(Fv, np + nx + 1));
        for (i = 2; i <= nx - 1; i++) {
            np = nx * (j - 1) + i;
            bx[i - 1] = V1(bs, i) - (S9(as, nx, i, 7) * F(Fv, np + nx - 1) + S9(as, nx, i, 8) * F(Fv, np + nx)
                                     + S9(as, nx, i, 9) * F(Fv, np + nx + 1));
        }
        i = nx; np = nx * (j - 1) + i;
        bx[nx - 1] = V1(bs, i) - (S9(as, nx, i, 7) * F(Fv, np + nx - 1) + S9(as, nx, i, 8) * F(Fv, np + nx));
        bc_tdma(nx, ax, bx, sx, g_P, g_Q);
        for (i = 1; i <= nx; i++) F(Fv, nx * (j - 1) + i) = sx[i - 1];
        /* east line */
        for (j = 1; j <= ny; j++) {
            ax[j - 1] = S9(ae, ny, j, 2); ax[ny + j - 1] = S9(ae, ny, j, 5); ax[2 * ny + j - 1] = S9(ae, ny, j, 8);
        }
        i = nx;
        j = 1; np = nx * (j - 1) + i;
        bx[0] = V1(be, j) - (S9(ae, ny, j, 4) * F(Fv, np - 1) + S9(ae, ny, j, 7) * F(Fv, np + nx - 1));
        for (j = 2; j <= ny - 1; j++) {
            np = nx * (j - 1) + i;
            bx[j - 1] = V1(be, j) - (S9(ae, ny, j, 1) * F(Fv, np - nx - 1) + S9(ae, ny, j, 4) * F(Fv, np - 1)
                                     + S9(ae, ny, j, 7) * F(Fv, np + nx - 1));
        }
        j = ny; np = nx * (j - 1) + i;
        bx[ny - 1] = V1(be, j) - (S9(ae, ny, j, 1) * F(Fv, np - nx - 1) + S9(ae, ny, j, 4) * F(Fv, np - 1));
        bc_tdma(ny, ax, bx, sx, g_P, g_Q);
        for (j = 1; j <= ny; j++) F(Fv, nx * (j - 1) + i) = sx[j - 1];
        /* west line */
        for (j = 1; j <= ny; j++) {
            ax[j - 1] = S9(aw, ny, j, 2); ax[ny + j - 1] = S9(aw, ny, j, 5); ax[2 * ny + j - 1] = S9(aw, ny, j, 8);
        }
        i = 1;
        j = 1; np = nx * (j - 1) + i;
        bx[0] = V1(bw, j) - (S9(aw, ny, j, 6) * F(Fv, np + 1) + S9(aw, ny, j, 9) * F(Fv, np + nx + 1));
        for (j = 2; j <= ny - 1; j++) {
            np = nx * (j - 1) + i;
            bx[j - 1] = V1(bw, j) - (S9(aw, ny, j, 3) * F(Fv, np - nx + 1) + S9(aw, ny, j, 6) * F(Fv, np + 1)
                                     + S9(aw, ny, j, 9) * F(Fv, np + nx + 1));
        }
        j = ny; np = nx * (j - 1) + i;
        bx[ny - 1] = V1(bw, j) - (S9(aw, ny, j, 3) * F(Fv, np - nx + 1) + S9(aw, ny, j, 6) * F(Fv, np + 1));
        bc_tdma(ny, ax, bx, sx, g_P, g_Q);
        for (j = 1; j <= ny; j++) F(Fv, nx * (j - 1) + i) = sx[j - 1];
    }
}

/* extflow_extrapolate_u_v_to_fictitious (mod_extflow.f90:360-397) */
void orc_extflow_extrapolate_u_v(int nx, int ny, int modvis, int itemax, double UF, const double *xk,
                                 const double *yk, const double *alphae, const double *betae, double *u, double *v)
{
    static double an[9 * ORC_MAX_STRIP], as[9 * ORC_MAX_STRIP], ae[9 * ORC_MAX_STRIP], aw[9 * ORC_MAX_STRIP];
    static double bn[ORC_MAX_STRIP], bs[ORC_MAX_STRIP], be[ORC_MAX_STRIP], bw[ORC_MAX_STRIP];
    orc_extflow_scheme_u(nx, ny, modvis, UF, xk, yk, alphae, betae, u, v, an, as, ae, aw, bn, bs, be, bw);
    orc_bc_extrapolation_9d(nx, ny, itemax, an, as, ae, aw, bn, bs, be, bw, u);
    orc_extflow_scheme_v(nx, ny, modvis, xk, yk, u, v, an, as, ae, aw, bn, bs, be, bw);
    orc_bc_extrapolation_9d(nx, ny, itemax, an, as, ae, aw, bn, bs, be, bw, v);
}

/* extflow_extrapolate_ro_to_fictitious (mod_extflow.f90:401-431) */
void orc_extflow_extrapolate_ro(int nx, int ny, int itemax, double ROF, const double *alphae, const double *betae,
                                const double *betan, const double *gamman, double *ro)
{
    static double an[9 * ORC_MAX_STRIP], as[9 * ORC_MAX_STRIP], ae[9 * ORC_MAX_STRIP], aw[9 * ORC_MAX_STRIP];
    static double bn[ORC_MAX_STRIP], bs[ORC_MAX_STRIP], be[ORC_MAX_STRIP], bw[ORC_MAX_STRIP];
    orc_extflow_scheme_ro(nx, ny, ROF, alphae, betae, betan, gamman, an, as, ae, aw, bn, bs, be, bw);
    orc_bc_extrapolation_9d(nx, ny, itemax, an, as, ae, aw, bn, bs, be, bw, ro);
}

/* get_cdfi (mod_extflow_procedures.f90:994-1041): pressure foredrag over the
 * south boundary, i = iiv..ifv */
double orc_extflow_cdfi(int nx, int iiv, int ifv, double Rg, double PF, double TF, double UF, double rb,
                        const double *yk, const double *rn, const double *p)
{
    const double ROF = PF / (Rg * TF);
    const double QF = ROF * (UF * UF) / 2.0;
    double Cdfi = 0.0;
    for (int i = iiv; i <= ifv; i++) {
        const int np = i, npn = np + nx;
        const double pn = 0.5 * (F(p, np) + F(p, npn));
        Cdfi = Cdfi + (pn - PF) * F(rn, np) * F(yk, np);
    }
    return Cdfi * 2.0 / ((rb * rb) * QF);
}

/* get_cdfv (:1045-1104): viscous foredrag over the south boundary */
double orc_extflow_cdfv(int nx, int iiv, int ifv, double Rg, double PF, double TF, double UF, double rb,
                        const double *xk, const double *yk, const double *rn, const double *Jn, const double *vln,
                        const double *u, const double *v, const double *Vcn)
{
    const double ROF = PF / (Rg * TF);
    const double QF = ROF * (UF * UF) / 2.0;
    double Cdfv = 0.0;
    for (int i = iiv; i <= ifv; i++) {
        const int np = i, npn = np + nx;
        const double Sxx = -2.0 * F(vln, np) * F(Jn, np)
                         * (F(yk, np) * (F(u, npn) - F(u, np)) + F(rn, npn) * F(Vcn, npn) / (3.0 * F(rn, np)));
        const double Sxy = F(vln, np) * F(Jn, np)
                         * (F(xk, np) * (F(u, npn) - F(u, np)) - F(yk, np) * (F(v, npn) - F(v, np)));
        Cdfv = Cdfv - Sxx * F(rn, np) * F(yk, np) + Sxy * F(rn, np) * F(xk, np);
    }
    return Cdfv * 2.0 / (QF * (rb * rb));
}

/* extflow_calc_main_variables (mod_extflow.f90:321-356): Cdfi over i = 2..iocs
 * and, for Navier-Stokes, Cdfv (else 0) */
void orc_extflow_calc_main_variables(int nx, int ny, double Rg, int modvis, double PF, double TF, double UF,
                                     double rb, int iocs, const double *xk, const double *yk, const double *rn,
                                     const double *Jn, const double *vln, const double *p, const double *u,
                                     const double *v, const double *Vcn, double *cd)
{
    (void)ny;
    cd[0] = orc_extflow_cdfi(nx, 2, iocs, Rg, PF, TF, UF, rb, yk, rn, p);
    cd[1] = modvis == 1 ? orc_extflow_cdfv(nx, 2, iocs, Rg, PF, TF, UF, rb, xk, yk, rn, Jn, vln, u, v, Vcn) : 0.0;
}

/* extflow_boundary_T_from_H_conservation (mod_extflow.f90:438-544) */
void orc_extflow_boundary_T_from_H(int nx, int ny, double CPF, double HF, const double *u, const double *ue,
                                   const double *un, const double *v, const double *ve, const double *vn, double *T,
                                   double *Tbe, double *Tbw, double *Tbn, double *Tbs)
{
    const int N = nx * ny;
    int i, j, np;
    for (np = 1; np <= N; np++) F(T, np) = (HF - (F(u, np) * F(u, np) + F(v, np) * F(v, np)) / 2.0) / CPF;
    i = nx - 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        V1(Tbe, j) = (HF - (F(ue, np) * F(ue, np) + F(ve, np) * F(ve, np)) / 2.0) / CPF;
        F(T, np + 1) = 2.0 * V1(Tbe, j) - F(T, np);
    }
    i = 1;
    for (j = 2; j <= ny - 1; j++) {
        np = nx * (j - 1) + i;
        V1(Tbw, j) = (HF - (F(ue, np) * F(ue, np) + F(ve, np) * F(ve, np)) / 2.0) / CPF;
        F(T, np) = 2.0 * V1(Tbw, j) - F(T, np + 1);
    }
    j = ny - 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        V1(Tbn, i) = (HF - (F(un, np) * F(un, np) + F(vn, np) * F(vn, np)) / 2.0) / CPF;
        F(T, np + nx) = 2.0 * V1(Tbn, i) - F(T, np);
    }
    j = 1;
    for (i = 2; i <= nx - 1; i++) {
        np = nx * (j - 1) + i;
        V1(Tbs, i) = (HF - (F(un, np) * F(un, np) + F(vn, np) * F(vn, np)) / 2.0) / CPF;
        F(T, np) = 2.0 * V1(Tbs, i) - F(T, np + nx);
    }
}
