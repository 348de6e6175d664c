/*
 * driver.c -- oracle restatement of MACH-2D's set-up and SIMPLEC outer
 * iteration for internal flow (src/mach2d_main.f90:25-445), constant
 * thermophysical properties (src/thermophysical/
 * mod_class_thermophysical_constant.f90), internal-flow initial guess
 * (src/user/internal_flow/mod_intflow.f90:1137-1488).
 * TEST INFRASTRUCTURE ONLY (see m2d_oracle.h).  Parity unpinned.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "m2d_oracle.h"

#define F(v, np) (v)[(size_t)(np) - 1]
#define V1(v, i) (v)[(size_t)(i) - 1]

#define FIELDS(X) \
    X(x) X(y) X(xp) X(yp) X(xe) X(ye) X(xen) X(yen) X(xk) X(yk) X(xke) X(yke) \
    X(Jp) X(Je) X(Jn) X(alphae) X(gamman) X(betae) X(betan) X(radius) X(re) \
    X(rn) X(rp) X(p) X(pa) X(T) X(Ta) X(ro) X(roa) X(roe) X(ron) X(g) X(u) \
    X(ua) X(v) X(va) X(ue) X(un) X(ve) X(vn) X(Uce) X(Vcn) X(cp) X(vlp) X(vle) \
    X(vln) X(kp) X(ke) X(kn) X(cup) X(sup) X(cvp) X(svp) X(uea) X(vea) X(una) \
    X(vna) X(bu) X(bv) X(bt) X(bp) X(pl) X(due) X(dve) X(dun) X(dvn) X(de) \
    X(dn) X(fbe) X(fbn) X(vtp)

struct orc_state {
    orc_case c;
    int nx, ny, it;
    size_t N;
#define DECL(f) double *f;
    FIELDS(DECL)
#undef DECL
    double *au, *av, *at, *ap;
    double *Tbe, *Tbw, *Tbn, *Tbs;                 /* ny, ny, nx, nx */
    double *uin, *vin, *pin, *Tin, *Mw, *plin, *pina; /* ny */
    double *M1D, *p1D, *T1D, *u1D;                 /* nx */
    double dt, norm, normpl, rmass, p_avg;
    double Rg, gamma, Tref, Cpref, Href, fm1D, Fd1D, Fpv1D, Sg;
    int ktm, it_stop;
    double *blwork;                                /* 9 (ny-2): Baldwin-Lomax line work */
};

int orc_nx(const orc_state *s) { return s->nx; }
int orc_ny(const orc_state *s) { return s->ny; }

static void solve9(orc_state *s, double *a, double *b, double *x)
{
    if (s->c.solver == 0) orc_msi9_solve(s->nx, s->ny, s->c.nitm_u, s->c.tol_u, a, b, x);
    else orc_tdma2d9(s->nx, s->ny, s->c.nitm_u, a, b, x);
}

static void solve5(orc_state *s, double *a, double *b, double *x)
{
    if (s->c.solver == 0) orc_msi5_solve(s->nx, s->ny, s->c.nitm_p, s->c.tol_p, a, b, x);
    else orc_tdma2d5(s->nx, s->ny, s->c.nitm_p, a, b, x);
}

orc_state *orc_create(const orc_case *c)
{
    orc_state *s = (orc_state *)calloc(1, sizeof(orc_state));
    s->c = *c;
    int nx = c->nxr + 2, ny = c->nyr + 2;
    s->nx = nx; s->ny = ny;
    size_t N = (size_t)nx * (size_t)ny;
    s->N = N;
#define ALLOC(f) s->f = (double *)calloc(N, sizeof(double));
    FIELDS(ALLOC)
#undef ALLOC
    s->au = (double *)calloc(9 * N, sizeof(double));
    s->av = (double *)calloc(9 * N, sizeof(double));
    s->at = (double *)calloc(9 * N, sizeof(double));
    s->ap = (double *)calloc(5 * N, sizeof(double));
    for (size_t k = 0; k < N; k++) s->ap[2 * N + k] = 1.0;   /* ap(:,3) = 1 */
    s->Tbe = (double *)calloc((size_t)ny, sizeof(double));
    s->Tbw = (double *)calloc((size_t)ny, sizeof(double));
    s->Tbn = (double *)calloc((size_t)nx, sizeof(double));
    s->Tbs = (double *)calloc((size_t)nx, sizeof(double));
    double **v1[] = {&s->uin, &s->vin, &s->pin, &s->Tin, &s->Mw, &s->plin, &s->pina};
    for (int k = 0; k < 7; k++) *v1[k] = (double *)calloc((size_t)ny, sizeof(double));
    s->blwork = (double *)calloc(9 * (size_t)ny, sizeof(double));
    double **v2[] = {&s->M1D, &s->p1D, &s->T1D, &s->u1D};
    for (int k = 0; k < 4; k++) *v2[k] = (double *)calloc((size_t)nx, sizeof(double));

    /* thermophysical_initialization (mod_thermophysical.f90:20-75) + intflow_init
     * (mod_intflow.f90:72-100); the internal-flow routines take gamma = gm(T0)
     * (:1121, :1186) */
    s->ktm = c->ktm;
    s->Tref = c->T0;
    if (c->ktm == 1) {
        s->Rg = c->mix.Rg;
        s->gamma = orc_mix_gm(&c->mix, c->T0);
        s->Cpref = orc_mix_cp(&c->mix, s->Tref);
    } else {
        s->Rg = c->Rg; s->gamma = c->gamma;
        s->Cpref = c->gamma * c->Rg / (c->gamma - 1.0);
    }
    s->Href = s->Cpref * s->Tref;

    /* grid_create (nmf = nmd: the finest grid is the desired grid) */
    if (c->geom == 0) {
        orc_nozzle_boundary_c01(nx, ny, c->Lc, c->Ld, c->Rin, c->Rout, s->x, s->y);
        s->Sg = acos(-1.0) * 1.0 * 1.0;
    } else {
        orc_nozzle_boundary_n01(nx, ny, c->Rth, c->Rin, c->Rout, c->Rc1, c->Rc2, c->Rc3,
                                c->alf, c->bet, c->Lchamb, s->x, s->y);
        s->Sg = acos(-1.0) * (c->Rth * c->Rth);
    }
    if (c->kg == 1) orc_get_uniform_grid(nx, ny, s->x, s->y);
    else orc_get_pg_grid(1, c->a1, nx, ny, s->x, s->y);
    orc_get_real_centroids_xy(c->kcm, nx, ny, s->x, s->y, s->xp, s->yp);
    orc_get_metrics(nx, ny, s->x, s->y, s->xp, s->yp, s->xe, s->ye, s->xen, s->yen,
                    s->xk, s->yk, s->xke, s->yke, s->Jp, s->Je, s->Jn, s->alphae,
                    s->gamman, s->betae, s->betan);
    orc_get_radius(c->coord, nx, ny, s->y, s->yp, s->radius, s->re, s->rn, s->rp);
    orc_initialize_boundary_faces_flags(nx, ny, s->fbe, s->fbn);

    /* intflow_initial_conditions -> get_initial_guess (mod_intflow.f90:1240-1488) */
    {
        const double pi = acos(-1.0);
        double po = c->p0, T0 = c->T0, gamma = s->gamma, Rg = s->Rg, Sg = s->Sg;
        s->fm1D = orc_get_isentropic_mass_flow(po, T0, gamma, Rg, Sg);
        int ig = orc_get_ig(nx, ny, s->y);
        for (int i = 2; i <= nx - 1; i++) {
            int np = nx * (ny - 2) + i;
            double Si = pi * (F(s->rn, np) * F(s->rn, np));
            int kf = (i > ig) ? 1 : 0;
            V1(s->M1D, i) = orc_get_mach_area(kf, Si / Sg, gamma);
            double aux = 1.0 + 0.5 * (gamma - 1.0) * (V1(s->M1D, i) * V1(s->M1D, i));
            V1(s->p1D, i) = po * pow(aux, -gamma / (gamma - 1.0));
            V1(s->T1D, i) = T0 / aux;
            V1(s->u1D, i) = V1(s->M1D, i) * sqrt(gamma * Rg * V1(s->T1D, i));
            for (int j = 1; j <= ny; j++) {
                np = nx * (j - 1) + i;
                F(s->p, np) = V1(s->p1D, i);
                F(s->T, np) = V1(s->T1D, i);
                F(s->u, np) = V1(s->u1D, i);
                if (j > 1 && j < ny - 1) {
                    F(s->un, np) = V1(s->u1D, i);
                    F(s->Vcn, np) = -F(s->un, np) * F(s->yk, np);
                }
            }
        }
        orc_intflow_extrapolate_u_v_to_fictitious(nx, ny, c->modvis, s->x, s->xp, s->xk, s->yk, s->u, s->v);
        orc_get_uin_vin_pin_Tin_Mw(nx, ny, gamma, Rg, po, T0, s->u, s->uin, s->vin, s->pin, s->Tin, s->Mw);
        for (int j = 2; j <= ny - 1; j++) {
            int np = nx * (j - 1) + 1, npe = np + 1;
            F(s->p, np) = 2.0 * V1(s->pin, j) - F(s->p, npe);
            F(s->T, np) = 2.0 * V1(s->Tin, j) - F(s->T, npe);
        }
        for (int j = 2; j <= ny - 1; j++) {
            int np = nx * (j - 1) + nx, npw = np - 1, npww = np - 2;
            double f = 2.0 * (F(s->x, npw) - F(s->xp, npw)) / (F(s->xp, npw) - F(s->xp, npww));
            F(s->p, np) = F(s->p, npw) + f * (F(s->p, npw) - F(s->p, npww));
            F(s->T, np) = F(s->T, npw) + f * (F(s->T, npw) - F(s->T, npww));
        }
        int corners[4][2] = {{1, 1 + nx}, {nx, nx + nx}, {nx * (ny - 1) + 1, nx * (ny - 2) + 1},
                             {nx * ny, nx * (ny - 1)}};
        for (int k = 0; k < 4; k++) {
            F(s->p, corners[k][0]) = F(s->p, corners[k][1]);
            F(s->T, corners[k][0]) = F(s->T, corners[k][1]);
        }
        for (int i = 1; i <= nx - 1; i++) {
            int np = nx * (ny - 2) + i;
            double Si = pi * (F(s->radius, np) * F(s->radius, np));
            int kf = (i > ig) ? 1 : 0;
            double Me1D = orc_get_mach_area(kf, Si / Sg, gamma);
            double aux = 1.0 + 0.5 * (gamma - 1.0) * (Me1D * Me1D);
            double pe1D = po * pow(aux, -gamma / (gamma - 1.0));
            double Te1D = T0 / aux;
            double ue1D = Me1D * sqrt(gamma * Rg * Te1D);
            for (int j = 2; j <= ny - 1; j++) {
                np = nx * (j - 1) + i;
                F(s->ue, np) = ue1D;
                F(s->Uce, np) = ue1D * F(s->ye, np);
            }
            if (i == 1) {
                V1(s->u1D, 1) = ue1D; V1(s->p1D, 1) = pe1D; V1(s->T1D, 1) = Te1D; V1(s->M1D, 1) = Me1D;
            }
            if (i == nx - 1) {
                V1(s->u1D, nx) = ue1D; V1(s->p1D, nx) = pe1D; V1(s->T1D, nx) = Te1D; V1(s->M1D, nx) = Me1D;
                s->Fd1D = s->fm1D * ue1D;
                s->Fpv1D = pe1D * Si;
            }
        }
        orc_intflow_velocities_at_boundary_faces(nx, ny, c->modvis, s->x, s->xp, s->xe, s->ye,
            s->xk, s->yk, s->u, s->v, s->ue, s->ve, s->un, s->vn, s->Uce, s->Vcn);
        orc_get_density_at_nodes(nx, ny, Rg, s->p, s->T, s->ro);
        orc_get_density_at_faces(nx, ny, c->beta, s->ro, s->Uce, s->Vcn, s->roe, s->ron);
        memcpy(s->Tbw, s->Tin, (size_t)ny * sizeof(double));
        memcpy(s->Tbs, s->T1D, (size_t)nx * sizeof(double));
        memcpy(s->Tbn, s->T1D, (size_t)nx * sizeof(double));
        for (int j = 0; j < ny; j++) s->Tbe[j] = V1(s->T1D, nx - 1);
    }
    /* get_cp_mu_kappa_initialization (mod_thermophysical.f90:514-591) */
    if (c->ktm == 1) {
        orc_set_cp(&c->mix, nx, ny, s->Tbn, s->Tbs, s->Tbe, s->Tbw, s->T, s->cp);
        if (c->modvis == 1) {
            orc_transport_nodes(&c->mix, nx, ny, 1, s->T, s->vlp);
            orc_transport_nodes(&c->mix, nx, ny, 0, s->T, s->kp);
            orc_transport_faces(&c->mix, nx, ny, 1, s->Tbn, s->Tbs, s->Tbe, s->Tbw, s->vlp, s->vle, s->vln);
            orc_transport_faces(&c->mix, nx, ny, 0, s->Tbn, s->Tbs, s->Tbe, s->Tbw, s->kp, s->ke, s->kn);
        }
    } else {
        for (size_t k = 0; k < N; k++) s->cp[k] = s->Cpref;
        if (c->modvis == 1)
            for (size_t k = 0; k < N; k++) {
                s->vlp[k] = c->mu; s->vle[k] = c->mu; s->vln[k] = c->mu;
                s->kp[k] = c->kappa; s->ke[k] = c->kappa; s->kn[k] = c->kappa;
            }
    }
    /* first time step */
    if (c->dtmodel == 1) s->dt = orc_tstepper_dt0_scarborough(nx, ny, s->Jp, s->u, s->v);
    else s->dt = orc_tstepper_dt_ramp(0, c->dt1, c->dt2, c->it1, c->it2);
    s->it = 0;
    s->it_stop = -1;
    return s;
}

void orc_destroy(orc_state *s)
{
    if (!s) return;
#define FREE(f) free(s->f);
    FIELDS(FREE)
#undef FREE
    free(s->au); free(s->av); free(s->at); free(s->ap);
    free(s->Tbe); free(s->Tbw); free(s->Tbn); free(s->Tbs);
    free(s->uin); free(s->vin); free(s->pin); free(s->Tin); free(s->Mw); free(s->plin); free(s->pina);
    free(s->M1D); free(s->p1D); free(s->T1D); free(s->u1D);
    free(s->blwork);
    free(s);
}

/* src/mach2d_main.f90:94-445, one pass of the `it` loop body */
int orc_iterate(orc_state *s, orc_report *rep)
{
    const orc_case *c = &s->c;
    int nx = s->nx, ny = s->ny, modvis = c->modvis;
    size_t N = s->N, nb = N * sizeof(double);
    int it = ++s->it;
    memcpy(s->roa, s->ro, nb); memcpy(s->Ta, s->T, nb); memcpy(s->pa, s->p, nb);
    memcpy(s->ua, s->u, nb); memcpy(s->va, s->v, nb); memcpy(s->uea, s->ue, nb);
    memcpy(s->vea, s->ve, nb); memcpy(s->una, s->un, nb); memcpy(s->vna, s->vn, nb);
    /* intflow_time_cycle_update */
    memcpy(s->pina, s->pin, (size_t)ny * sizeof(double));
    orc_get_uin_vin_pin_Tin_Mw(nx, ny, s->gamma, s->Rg, c->p0, c->T0, s->u, s->uin, s->vin,
                               s->pin, s->Tin, s->Mw);
    orc_get_plin_and_p_fictitious(nx, ny, s->x, s->xp, s->pina, s->pin, s->plin, s->p);
    /* temperature-dependent properties, src/mach2d_main.f90:112-149 */
    if (s->ktm == 1) {
        orc_get_boundary_fields(nx, ny, s->T, s->Tbn, s->Tbs, s->Tbe, s->Tbw);
        orc_set_cp(&c->mix, nx, ny, s->Tbn, s->Tbs, s->Tbe, s->Tbw, s->T, s->cp);
        if (modvis == 1) {
            orc_transport_nodes(&c->mix, nx, ny, 1, s->T, s->vlp);
            orc_transport_nodes(&c->mix, nx, ny, 0, s->T, s->kp);
            orc_transport_faces(&c->mix, nx, ny, 1, s->Tbn, s->Tbs, s->Tbe, s->Tbw, s->vlp, s->vle, s->vln);
            orc_transport_faces(&c->mix, nx, ny, 0, s->Tbn, s->Tbs, s->Tbe, s->Tbw, s->kp, s->ke, s->kn);
        }
    }
    /* Baldwin-Lomax eddy viscosity from the previous iteration's flow
     * (blomax.f90:285-490), added to the laminar transport coefficients */
    if (modvis == 1 && c->modtur == 1) {
        orc_get_eddy_viscosity_blomax(nx, ny, s->x, s->y, s->xp, s->yp, s->xk, s->yk, s->Jp, s->Jn, s->vln,
                                      s->ro, s->ron, s->u, s->v, s->vtp, s->blwork);
        orc_get_eddy_viscosity_fictitious(nx, ny, s->vtp);
        orc_add_eddy_viscosity(nx, ny, s->ktm, c->mu, c->kappa, c->prt, s->vtp, s->cp, s->vlp, s->vle, s->vln,
                               s->kp, s->ke, s->kn);
    }
    /* get_average(p) */
    {
        double a = 0.0;
        for (int j = 2; j <= ny - 1; j++)
            for (int i = 2; i <= nx - 1; i++) a = a + F(s->p, nx * (j - 1) + i);
        s->p_avg = a / ((double)(nx - 2) * (double)(ny - 2));
    }
    for (size_t k = 0; k < N; k++) s->g[k] = 1.0 / (s->Rg * s->T[k]);
    int itp_used = 0;
    for (int itm = 1; itm <= c->itmmax; itm++) {
        s->norm = 0.0;
        orc_get_u_coefficients(nx, ny, modvis, s->dt, s->rp, s->re, s->rn, s->Jp, s->Je, s->Jn,
            s->ye, s->yk, s->alphae, s->betae, s->betan, s->gamman, s->vle, s->vln, s->roe,
            s->ron, s->roa, s->Uce, s->Vcn, s->au);
        orc_get_u_source(nx, ny, modvis, c->beta, s->dt, s->rp, s->re, s->rn, s->xe, s->ye,
            s->xk, s->yk, s->xke, s->yke, s->xen, s->yen, s->Jp, s->Je, s->Jn, s->roe, s->ron,
            s->roa, s->p, s->vle, s->vln, s->Uce, s->Vcn, s->ua, s->u, s->v, s->cup, s->sup, s->bu);
        orc_intflow_set_bcu(nx, ny, modvis, s->x, s->xp, s->xk, s->yk, s->u, s->v, s->au, s->bu);
        orc_get_v_coefficients(nx, ny, c->coord, modvis, s->dt, s->rp, s->re, s->rn, s->Jp,
            s->Je, s->Jn, s->xe, s->xk, s->alphae, s->betae, s->betan, s->gamman, s->vle,
            s->vln, s->vlp, s->roe, s->ron, s->roa, s->Uce, s->Vcn, s->av);
        orc_get_v_source(nx, ny, c->coord, modvis, c->beta, s->dt, s->rp, s->re, s->rn, s->xe,
            s->ye, s->xk, s->yk, s->xke, s->yke, s->xen, s->yen, s->Jp, s->Je, s->Jn, s->roe,
            s->ron, s->roa, s->p, s->vle, s->vln, s->Uce, s->Vcn, s->va, s->u, s->v, s->cvp,
            s->svp, s->bv);
        orc_intflow_set_bcv(nx, ny, modvis, s->x, s->xp, s->xk, s->yk, s->u, s->v, s->av, s->bv);
        orc_get_internal_simplec_coefficients(nx, ny, s->re, s->rn, s->xe, s->ye, s->xk, s->yk,
            s->au, s->av, s->due, s->dve, s->dun, s->dvn, s->de, s->dn);
        orc_intflow_boundary_simplec(nx, ny, modvis, s->due, s->dve, s->dun, s->dvn, s->de, s->dn);
        solve9(s, s->au, s->bu, s->u);
        s->norm = orc_norm_l1_9d_relative(nx, ny, s->u, s->bu, s->au, s->norm);
        solve9(s, s->av, s->bv, s->v);
        s->norm = orc_norm_l1_9d_relative(nx, ny, s->v, s->bv, s->av, s->norm);
        orc_get_velocities_at_internal_faces(nx, ny, s->dt, s->rp, s->re, s->rn, s->xe, s->ye,
            s->xk, s->yk, s->xen, s->yen, s->xke, s->yke, s->Jp, s->cup, s->cvp, s->sup, s->svp,
            s->au, s->av, s->roa, s->p, s->u, s->v, s->uea, s->vea, s->una, s->vna, s->ue,
            s->ve, s->un, s->vn, s->Uce, s->Vcn);
        orc_intflow_velocities_at_boundary_faces(nx, ny, modvis, s->x, s->xp, s->xe, s->ye,
            s->xk, s->yk, s->u, s->v, s->ue, s->ve, s->un, s->vn, s->Uce, s->Vcn);
        memset(s->pl, 0, nb);
        for (int itp = 1; itp <= c->itpmax; itp++) {
            itp_used = itp;
            orc_get_p_coefficients(nx, ny, s->dt, s->rp, s->re, s->rn, s->Jp, s->Uce, s->Vcn,
                                   s->roe, s->ron, s->g, s->de, s->dn, s->ap);
            orc_intflow_set_bcpl(nx, ny, s->x, s->xp, s->pl, s->plin, s->ap, s->bp);
            orc_get_p_source(nx, ny, s->dt, s->rp, s->re, s->rn, s->Jp, s->roe, s->ron, s->ro,
                             s->roa, s->Uce, s->Vcn, s->de, s->dn, s->g, s->pl, s->bp);
            solve5(s, s->ap, s->bp, s->pl);
            orc_get_velocity_correction_at_faces_with_pl(nx, ny, s->xe, s->ye, s->xk, s->yk,
                s->due, s->dve, s->dun, s->dvn, s->de, s->dn, s->pl, s->ue, s->ve, s->un,
                s->vn, s->Uce, s->Vcn);
            orc_intflow_velocities_at_boundary_faces(nx, ny, modvis, s->x, s->xp, s->xe, s->ye,
                s->xk, s->yk, s->u, s->v, s->ue, s->ve, s->un, s->vn, s->Uce, s->Vcn);
            orc_get_pressure_correction_with_pl(nx, ny, s->pl, s->p);
            orc_get_density_correction_with_pl(nx, ny, s->pl, s->g, s->ro);
            orc_get_density_at_faces(nx, ny, c->beta, s->ro, s->Uce, s->Vcn, s->roe, s->ron);
            double mx = 0.0;
            for (size_t k = 0; k < N; k++) if (fabs(s->pl[k]) > mx) mx = fabs(s->pl[k]);
            s->normpl = mx / s->p_avg;
            if (s->normpl < c->tolm) break;
        }
        s->norm = orc_norm_l1_5d(nx, ny, s->pl, s->bp, s->ap, s->norm);
        orc_get_u_v_at_real_nodes_with_pl(nx, ny, s->xe, s->ye, s->xk, s->yk, s->rp, s->pl,
                                          s->au, s->av, s->u, s->v);
        orc_intflow_extrapolate_u_v_to_fictitious(nx, ny, modvis, s->x, s->xp, s->xk, s->yk,
                                                  s->u, s->v);
    }
    s->rmass = orc_check_mass_conservation(nx, ny, s->dt, s->rp, s->re, s->rn, s->Jp, s->ro,
                                           s->roa, s->ron, s->roe, s->Uce, s->Vcn);
    if (modvis == 0 && s->ktm == 0) {
        for (size_t k = 0; k < N; k++)
            s->T[k] = (s->Href - (s->u[k] * s->u[k] + s->v[k] * s->v[k]) / 2.0) / s->Cpref;
        orc_intflow_boundary_T_from_H_conservation(nx, ny, s->Cpref, s->Href, s->Tin, s->u,
            s->ue, s->un, s->v, s->ve, s->vn, s->T, s->Tbe, s->Tbw, s->Tbn, s->Tbs);
    } else {
        orc_get_T_coefficients_and_source(nx, ny, modvis, c->beta, s->dt, s->rp, s->re, s->rn,
            s->xe, s->ye, s->xk, s->yk, s->xke, s->yke, s->xen, s->yen, s->alphae, s->betae,
            s->betan, s->gamman, s->Jp, s->Je, s->Jn, s->roe, s->ron, s->ro, s->roa, s->p,
            s->pa, s->cp, s->vle, s->vln, s->ke, s->kn, s->Uce, s->Vcn, s->u, s->v, s->ue,
            s->ve, s->un, s->vn, s->ua, s->va, s->T, s->Ta, s->fbe, s->fbn, s->at, s->bt);
        orc_intflow_set_bcT(nx, ny, s->x, s->xp, s->T, c->Twall, s->Tin, s->at, s->bt);
        solve9(s, s->at, s->bt, s->T);
        s->norm = orc_norm_l1_9d_relative(nx, ny, s->T, s->bt, s->at, s->norm);
    }
    orc_get_density_at_nodes(nx, ny, s->Rg, s->p, s->T, s->ro);
    orc_get_density_at_faces(nx, ny, c->beta, s->ro, s->Uce, s->Vcn, s->roe, s->ron);
    if (c->dtmodel == 1)
        s->dt = orc_tstepper_dt_scarborough(nx, ny, s->dt, s->au, s->av, s->at, s->ap, c->h0,
                                            c->mincc, c->maxcc, c->nan_policy);
    else
        s->dt = orc_tstepper_dt_ramp(it, c->dt1, c->dt2, c->it1, c->it2);
    if (rep) {
        rep->it = it; rep->dt = s->dt; rep->norm = s->norm; rep->normpl = s->normpl;
        rep->rmass = s->rmass; rep->itp_used = itp_used;
        orc_get_mass_flow_rate_and_thrust(nx, ny, s->re, s->roe, s->u, s->Uce, &rep->fmi,
                                          &rep->fme, &rep->Fd);
    }
    if (isnan(s->norm)) return 3;
    if (s->normpl < c->tolt && s->it_stop < 0) s->it_stop = it * 2;
    return 0;
}

long orc_field(orc_state *s, const char *name, double **ptr)
{
#define MATCH(f) if (strcmp(name, #f) == 0) { *ptr = s->f; return (long)s->N; }
    FIELDS(MATCH)
#undef MATCH
    if (!strcmp(name, "au")) { *ptr = s->au; return (long)(9 * s->N); }
    if (!strcmp(name, "av")) { *ptr = s->av; return (long)(9 * s->N); }
    if (!strcmp(name, "at")) { *ptr = s->at; return (long)(9 * s->N); }
    if (!strcmp(name, "ap")) { *ptr = s->ap; return (long)(5 * s->N); }
    if (!strcmp(name, "Tbe")) { *ptr = s->Tbe; return s->ny; }
    if (!strcmp(name, "Tbw")) { *ptr = s->Tbw; return s->ny; }
    if (!strcmp(name, "Tbn")) { *ptr = s->Tbn; return s->nx; }
    if (!strcmp(name, "Tbs")) { *ptr = s->Tbs; return s->nx; }
    if (!strcmp(name, "pin")) { *ptr = s->pin; return s->ny; }
    if (!strcmp(name, "plin")) { *ptr = s->plin; return s->ny; }
    if (!strcmp(name, "Tin")) { *ptr = s->Tin; return s->ny; }
    if (!strcmp(name, "uin")) { *ptr = s->uin; return s->ny; }
    if (!strcmp(name, "Mw")) { *ptr = s->Mw; return s->ny; }
    if (!strcmp(name, "vin")) { *ptr = s->vin; return s->ny; }
    if (!strcmp(name, "pina")) { *ptr = s->pina; return s->ny; }
    if (!strcmp(name, "p1D")) { *ptr = s->p1D; return s->nx; }
    if (!strcmp(name, "M1D")) { *ptr = s->M1D; return s->nx; }
    return -1;
}

double orc_scalar(const orc_state *s, const char *name)
{
    if (!strcmp(name, "dt")) return s->dt;
    if (!strcmp(name, "norm")) return s->norm;
    if (!strcmp(name, "normpl")) return s->normpl;
    if (!strcmp(name, "rmass")) return s->rmass;
    if (!strcmp(name, "p_avg")) return s->p_avg;
    if (!strcmp(name, "Href")) return s->Href;
    if (!strcmp(name, "Cpref")) return s->Cpref;
    if (!strcmp(name, "fm1D")) return s->fm1D;
    if (!strcmp(name, "Fd1D")) return s->Fd1D;
    if (!strcmp(name, "Fpv1D")) return s->Fpv1D;
    if (!strcmp(name, "Sg")) return s->Sg;
    if (!strcmp(name, "it")) return (double)s->it;
    if (!strcmp(name, "it_stop")) return (double)s->it_stop;
    return NAN;
}
