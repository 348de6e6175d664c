/*
 * m2d_oracle.h -- CPU FP64 restatement of MACH-2D's SIMPLEC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (mach2d_b200/) may link,
 * load or call this code; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py use it, as the checker.
 *
 * PARITY UNPINNED.  The reference (gbertoldo/MACH-2D v5.10.2) is Fortran 2003
 * and no Fortran compiler exists in this image, so the reference cannot be
 * built or run here; the reference ships no tests and no golden vectors.
 * This restatement follows the reference routine by routine, in the same
 * evaluation order, compiled with -O2 -ffp-contract=off (no FMA contraction,
 * SSE2 double arithmetic, i.e. what gfortran -O2 does on x86-64), and is
 * checked against analytic known answers (dense solves, isentropic flow).
 *
 * Conventions (same as the reference):
 *   nx, ny  volumes per direction INCLUDING the ghost ring;  N = nx*ny.
 *   1-based cell index np = nx*(j-1)+i, stored at offset np-1.
 *   Coefficient arrays are Fortran column-major a(N,k): diagonal k occupies
 *   [(k-1)N, kN).  9-diagonal order SW,S,SE,W,P,E,NW,N,NE; 5-diagonal order
 *   S,W,P,E,N.
 */
#ifndef M2D_ORACLE_H
#define M2D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- linear solvers: src/solvers/msi2d9-v03.f90, msi2d5-v03.f90,
 *      tdma2d9.f90, tdma2d5.f90, mod_solvers.f90 ------------------------- */
void orc_lu2d9(const double *b, double *dl, double *du, int nij, int ni, int nj);
int  orc_fb2d9(const double *b, const double *dl, const double *du, int nj, int ni,
               int nij, double *var, double gamma, int nitm, const double *rhs);
void orc_lu2d5(const double *b, double *dl, double *du, int nij, int ni, int nj);
int  orc_fb2d5(const double *b, const double *dl, const double *du, int nj, int ni,
               int nij, double *var, double gamma, int nitm, const double *rhs);
/* solve9d/solve5d of class_solver_msi: lu then fb; returns iterations used */
int  orc_msi9_solve(int nx, int ny, int nitm, double tol, const double *a,
                    const double *b, double *x);
int  orc_msi5_solve(int nx, int ny, int nitm, double tol, const double *a,
                    const double *b, double *x);
void orc_tdma2d9(int nx, int ny, int nitm, const double *a, const double *b, double *x);
void orc_tdma2d5(int nx, int ny, int nitm, const double *a, const double *b, double *x);
double orc_norm_l1_5d(int nx, int ny, const double *var, const double *b,
                      const double *a, double norm);
double orc_norm_l1_9d(int nx, int ny, const double *var, const double *b,
                      const double *a, double norm);
double orc_norm_l1_9d_relative(int nx, int ny, const double *var, const double *b,
                               const double *a, double norm);
double orc_norm_l1_b(int nx, int ny, const double *b);
/* single tridiagonal line (Thomas), used by the line-batch checks */
void orc_tdma_line(int n, const double *aw, const double *ap, const double *ae,
                   const double *d, double *x);

/* ---- coefficient assembly: src/equations/mach2d_coef.f90 --------------- */
void orc_get_density_at_nodes(int nx, int ny, double Rg, const double *p,
                              const double *T, double *ro);
void orc_get_density_at_faces(int nx, int ny, double beta, const double *ro,
                              const double *Uce, const double *Vcn, double *roe,
                              double *ron);
void orc_get_u_coefficients(int nx, int ny, int modvis, double dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *Je,
    const double *Jn, const double *ye, const double *yk, const double *alphae,
    const double *betae, const double *betan, const double *gamman,
    const double *vle, const double *vln, const double *roe, const double *ron,
    const double *roa, const double *Uce, const double *Vcn, double *a);
void orc_get_u_source(int nx, int ny, int modvis, double beta, double dt,
    const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *Jp,
    const double *Je, const double *Jn, const double *roe, const double *ron,
    const double *roa, const double *p, const double *vle, const double *vln,
    const double *Uce, const double *Vcn, const double *ua, const double *u,
    const double *v, double *cup, double *sup, double *b);
void orc_get_v_coefficients(int nx, int ny, int coord, int modvis, double dt,
    const double *rp, const double *re, const double *rn, const double *Jp,
    const double *Je, const double *Jn, const double *xe, const double *xk,
    const double *alphae, const double *betae, const double *betan,
    const double *gamman, const double *vle, const double *vln, const double *vlp,
    const double *roe, const double *ron, const double *roa, const double *Uce,
    const double *Vcn, double *a);
void orc_get_v_source(int nx, int ny, int coord, int modvis, double beta, double dt,
    const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *Jp,
    const double *Je, const double *Jn, const double *roe, const double *ron,
    const double *roa, const double *p, const double *vle, const double *vln,
    const double *Uce, const double *Vcn, const double *va, const double *u,
    const double *v, double *cvp, double *svp, double *b);
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
    const double *fbn, double *a, double *b);
void orc_get_p_coefficients(int nx, int ny, double dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *Uce,
    const double *Vcn, const double *roe, const double *ron, const double *g,
    const double *de, const double *dn, double *a);
void orc_get_p_source(int nx, int ny, double dt, const double *rp, const double *re,
    const double *rn, const double *Jp, const double *roe, const double *ron,
    const double *ro, const double *roa, const double *Uce, const double *Vcn,
    const double *de, const double *dn, const double *g, const double *pl,
    double *b);
void orc_get_velocities_at_internal_faces(int nx, int ny, double dt,
    const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xen,
    const double *yen, const double *xke, const double *yke, const double *Jp,
    const double *cup, const double *cvp, const double *sup, const double *svp,
    const double *au, const double *av, const double *roa, const double *p,
    const double *u, const double *v, const double *uea, const double *vea,
    const double *una, const double *vna, double *ue, double *ve, double *un,
    double *vn, double *Uce, double *Vcn);
void orc_get_internal_simplec_coefficients(int nx, int ny, const double *re,
    const double *rn, const double *xe, const double *ye, const double *xk,
    const double *yk, const double *au, const double *av, double *due,
    double *dve, double *dun, double *dvn, double *de, double *dn);
void orc_get_pressure_correction_with_pl(int nx, int ny, const double *pl, double *p);
void orc_get_density_correction_with_pl(int nx, int ny, const double *pl,
                                        const double *g, double *ro);
void orc_get_u_v_at_real_nodes_with_pl(int nx, int ny, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *rp,
    const double *pl, const double *au, const double *av, double *u, double *v);
void orc_get_velocity_correction_at_faces_with_pl(int nx, int ny, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *due,
    const double *dve, const double *dun, const double *dvn, const double *de,
    const double *dn, const double *pl, double *ue, double *ve, double *un,
    double *vn, double *Uce, double *Vcn);
void orc_initialize_boundary_faces_flags(int nx, int ny, double *fbe, double *fbn);
double orc_check_mass_conservation(int nx, int ny, double dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *ro,
    const double *roa, const double *ron, const double *roe, const double *Uce,
    const double *Vcn);

/* ---- internal flow plug-in: src/user/internal_flow/mod_intflow.f90 ------ */
void orc_get_u_v_north_slip(int nx, int ny, const double *x, const double *xp,
    const double *xk, const double *yk, const double *u, const double *v,
    double *ubn, double *vbn);
void orc_intflow_set_bcu(int nx, int ny, int modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u,
    const double *v, double *au, double *b);
void orc_intflow_set_bcv(int nx, int ny, int modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u,
    const double *v, double *av, double *b);
void orc_intflow_set_bcpl(int nx, int ny, const double *x, const double *xp,
    const double *pl, const double *plin, double *ap, double *bp);
void orc_intflow_set_bcT(int nx, int ny, const double *x, const double *xp,
    const double *T, double Twall, const double *Tin, double *at, double *bt);
void orc_intflow_boundary_T_from_H_conservation(int nx, int ny, double Cpref,
    double Href, const double *Tin, const double *u, const double *ue,
    const double *un, const double *v, const double *ve, const double *vn,
    double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs);
void orc_intflow_velocities_at_boundary_faces(int nx, int ny, int modvis,
    const double *x, const double *xp, const double *xe, const double *ye,
    const double *xk, const double *yk, const double *u, const double *v,
    double *ue, double *ve, double *un, double *vn, double *Uce, double *Vcn);
void orc_intflow_boundary_simplec(int nx, int ny, int modvis, double *due,
    double *dve, double *dun, double *dvn, double *de, double *dn);
void orc_intflow_extrapolate_u_v_to_fictitious(int nx, int ny, int modvis,
    const double *x, const double *xp, const double *xk, const double *yk,
    double *u, double *v);
void orc_get_uin_vin_pin_Tin_Mw(int nx, int ny, double gamma, double Rg, double po,
    double T0, const double *u, double *uin, double *vin, double *pin,
    double *Tin, double *Mw);
void orc_get_plin_and_p_fictitious(int nx, int ny, const double *x,
    const double *xp, const double *pina, const double *pin, double *plin,
    double *p);
void orc_get_mass_flow_rate_and_thrust(int nx, int ny, const double *re,
    const double *roe, const double *u, const double *Uce, double *fmi,
    double *fme, double *Fd);
double orc_get_isentropic_mass_flow(double po, double T0, double gamma, double Rg,
                                    double Sg);
double orc_get_mach_area(int kf, double ar, double gamma);
int    orc_get_ig(int nx, int ny, const double *y);

/* ---- grid: src/grid/mod_grid.f90, mod_grid_procedures.f90 and the nozzle
 *      contours (N01: src/user/internal_flow/mod_intflow_geometry.f90;
 *      C01 cosine nozzle: new geometry, no counterpart in the reference) --- */
void orc_nozzle_boundary_c01(int nx, int ny, double Lc, double Ld, double Rin,
                             double Rout, double *x, double *y);
void orc_nozzle_boundary_n01(int nx, int ny, double Rth, double Rin, double Rout,
    double Rc1, double Rc2, double Rc3, double alf_deg, double bet_deg,
    double Lchamb, double *x, double *y);
void orc_get_uniform_grid(int nx, int ny, double *x, double *y);
void orc_get_pg_grid(int isReversed, double a1, int nx, int ny, double *x, double *y);
double orc_get_gp_ratio(int n, double r);
void orc_get_real_centroids_xy(int opt, int nx, int ny, const double *x,
                               const double *y, double *xp, double *yp);
void orc_get_metrics(int nx, int ny, const double *x, const double *y,
    const double *xp, const double *yp, double *xe, double *ye, double *xen,
    double *yen, double *xk, double *yk, double *xke, double *yke, double *Jp,
    double *Je, double *Jn, double *alphae, double *gamman, double *betae,
    double *betan);
void orc_get_radius(int coord, int nx, int ny, const double *y, const double *yp,
                    double *radius, double *re, double *rn, double *rp);

/* ---- time stepper: src/tstepper/mod_tstepper*.f90 ----------------------------------- */
double orc_tstepper_dt0_scarborough(int nx, int ny, const double *Jp,
                                    const double *u, const double *v);
double orc_get_mean_cc_9d(int nx, int ny, const double *a);
double orc_get_mean_cc_5d(int nx, int ny, const double *a);
/* nan_policy 0: NaN operands of max() are dropped (IEEE fmax);
 * nan_policy 1: a NaN operand makes c NaN, so h = 0 and dt is unchanged. */
double orc_tstepper_dt_scarborough(int nx, int ny, double dt, const double *au,
    const double *av, const double *at, const double *ap, double h0, double mincc,
    double maxcc, int nan_policy);
double orc_tstepper_dt_ramp(int it, double dt1, double dt2, int it1, int it2);

/* gas mixture (thermo.c); the layout of the library's m2d_mixture */
#define ORC_MAX_SPECIES 8
typedef struct orc_mixture {
    int ngs;
    double Rg;
    double Xi[ORC_MAX_SPECIES], Yi[ORC_MAX_SPECIES], Mi[ORC_MAX_SPECIES], Ri[ORC_MAX_SPECIES];
    double cpi[ORC_MAX_SPECIES][10], mui[ORC_MAX_SPECIES][8], kpi[ORC_MAX_SPECIES][8];
} orc_mixture;

/* ---- driver: src/mach2d_main.f90:25-445 --------------------------------- */
typedef struct orc_case {
    /* geometry: 0 = C01 cosine nozzle, 1 = N01 */
    int geom;
    double Lc, Ld, Rin, Rout;                      /* C01 */
    double Rth, Rc1, Rc2, Rc3, alf, bet, Lchamb;   /* N01 (Rin, Rout shared) */
    int nxr, nyr;          /* real volumes per direction */
    int kg, kcm;           /* grid kind (1 uniform, 2 geometric), centroid mean */
    double a1;             /* first-cell width for kg=2 */
    int coord, modvis;
    double beta;
    double p0, T0, Twall;  /* Twall <= 0: adiabatic */
    double Rg, gamma;      /* constant thermophysical model */
    double mu, kappa;
    int itmmax, itpmax;
    double tolm, tolt;
    int solver;            /* 0 = MSI, 1 = TDMA */
    int nitm_u, nitm_p;
    double tol_u, tol_p;
    int dtmodel;           /* 0 = RAMP, 1 = SCARBOROUGH */
    double dt1, dt2; int it1, it2;
    double h0, mincc, maxcc;
    int nan_policy;
    int ktm;               /* 0 = CONSTANT, 1 = MIXTURE */
    orc_mixture mix;       /* ktm = 1 */
    int modtur;            /* 1: Baldwin-Lomax eddy viscosity in the transport coefficients (modvis = 1) */
    double prt;            /* turbulent Prandtl number (modtur = 1) */
    int msi_lag;           /* device solver option (factor reuse); the oracle factorises every solve */
} orc_case;

typedef struct orc_report {
    int it;
    double dt, norm, normpl, rmass, fmi, fme, Fd;
    int itp_used;
} orc_report;

typedef struct orc_state orc_state;

orc_state *orc_create(const orc_case *c);
void orc_destroy(orc_state *s);
int  orc_nx(const orc_state *s);
int  orc_ny(const orc_state *s);
/* Runs one SIMPLEC outer iteration it (1-based); returns 0, or 3 on NaN. */
int  orc_iterate(orc_state *s, orc_report *rep);
/* Field access by name ("u", "p", "au", ...); returns element count or -1. */
long orc_field(orc_state *s, const char *name, double **ptr);
double orc_scalar(const orc_state *s, const char *name);

/* ---- external-flow boundary plug-in (extflow.c):
 *      src/user/external_flow/mod_extflow.f90:166-317,
 *      mod_extflow_procedures.f90:344-701, src/boundary_conditions/ */
#define ORC_MAX_STRIP 16384
void orc_extflow_scheme_u(int nx, int ny, int modvis, double UF, const double *xk, const double *yk,
                          const double *alphae, const double *betae, const double *u, const double *v,
                          double *an, double *as, double *ae, double *aw, double *bn, double *bs, double *be,
                          double *bw);
void orc_extflow_scheme_v(int nx, int ny, int modvis, const double *xk, const double *yk, const double *u,
                          const double *v, double *an, double *as, double *ae, double *aw, double *bn, double *bs,
                          double *be, double *bw);
void orc_extflow_scheme_ro(int nx, int ny, double ROF, const double *alphae, const double *betae,
                           const double *betan, const double *gamman, double *an, double *as, double *ae,
                           double *aw, double *bn, double *bs, double *be, double *bw);
void orc_extflow_scheme_T(int nx, int ny, double TF, double Tsbc, const double *alphae, const double *betae,
                          const double *betan, const double *gamman, double *an, double *as, double *ae,
                          double *aw, double *bn, double *bs, double *be, double *bw);
void orc_extflow_set_bcu(int nx, int ny, int modvis, double UF, const double *xk, const double *yk,
                         const double *alphae, const double *betae, const double *u, const double *v, double *au,
                         double *bu);
void orc_extflow_set_bcv(int nx, int ny, int modvis, const double *xk, const double *yk, const double *u,
                         const double *v, double *av, double *bv);
void orc_extflow_set_bcpl(int nx, int ny, double *ap, double *bp);
void orc_extflow_set_bcT(int nx, int ny, double TF, double Tsbc, const double *alphae, const double *betae,
                         const double *betan, const double *gamman, double *at, double *bt);
void orc_bc_extrapolation_9d(int nx, int ny, int itemax, const double *an, const double *as, const double *ae,
                             const double *aw, const double *bn, const double *bs, const double *be,
                             const double *bw, double *F);
void orc_extflow_extrapolate_u_v(int nx, int ny, int modvis, int itemax, double UF, const double *xk,
                                 const double *yk, const double *alphae, const double *betae, double *u, double *v);
void orc_extflow_extrapolate_ro(int nx, int ny, int itemax, double ROF, const double *alphae, const double *betae,
                                const double *betan, const double *gamman, double *ro);
double orc_extflow_cdfi(int nx, int iiv, int ifv, double Rg, double PF, double TF, double UF, double rb,
                        const double *yk, const double *rn, const double *p);
double orc_extflow_cdfv(int nx, int iiv, int ifv, double Rg, double PF, double TF, double UF, double rb,
                        const double *xk, const double *yk, const double *rn, const double *Jn, const double *vln,
                        const double *u, const double *v, const double *Vcn);
void orc_extflow_calc_main_variables(int nx, int ny, double Rg, int modvis, double PF, double TF, double UF,
                                     double rb, int iocs, const double *xk, const double *yk, const double *rn,
                                     const double *Jn, const double *vln, const double *p, const double *u,
                                     const double *v, const double *Vcn, double *cd);
void orc_extflow_boundary_T_from_H(int nx, int ny, double CPF, double HF, const double *u, const double *ue,
                                   const double *un, const double *v, const double *ve, const double *vn, double *T,
                                   double *Tbe, double *Tbw, double *Tbn, double *Tbs);

/* ---- Baldwin-Lomax: src/equations/blomax.f90 (blomax.c) ---------------- */
void orc_set_blomax_coefficients(double kappa, double Aop, double alpha, double Ccp, double Ckleb,
                                 double Cwk);
/* work: 9 (ny-2) doubles */
void orc_get_eddy_viscosity_blomax(int nx, int ny, const double *x, const double *y, const double *xp,
                                   const double *yp, const double *xk, const double *yk, const double *Jp,
                                   const double *Jn, const double *vln, const double *ro, const double *ron,
                                   const double *u, const double *v, double *vtp, double *work);
void orc_get_eddy_viscosity_fictitious(int nx, int ny, double *phi);
/* the eddy viscosity into the transport coefficients (no reference call
 * site: blomax.f90 is compiled but never used); ktm = 0 takes the laminar
 * values from the constants mu, kappa, ktm = 1 from the arrays themselves */
void orc_add_eddy_viscosity(int nx, int ny, int ktm, double mu, double kappa, double prt, const double *vtp,
                            const double *cp, double *vlp, double *vle, double *vln, double *kp, double *ke,
                            double *kn);

/* ---- thermophysical model (thermo.c): mod_class_thermophysical_mixture.f90,
 *      mod_thermophysical.f90, mod_field_operations.f90.  orc_mixture has
 *      the layout of the library's m2d_mixture. */
int orc_mixture_init(int base, int ngs, const double *fractions, const double *Mi, const double *cpi,
                     const double *mui, const double *kpi, orc_mixture *out);
double orc_mix_cp(const orc_mixture *m, double T);
double orc_mix_mu(const orc_mixture *m, double T);
double orc_mix_kp(const orc_mixture *m, double T);
double orc_mix_gm(const orc_mixture *m, double T);
void orc_get_boundary_fields(int nx, int ny, const double *F, double *Fbn, double *Fbs, double *Fbe,
                             double *Fbw);
void orc_set_cp(const orc_mixture *m, int nx, int ny, const double *Tbn, const double *Tbs, const double *Tbe,
                const double *Tbw, const double *T, double *cp);
void orc_set_gamma(int nx, int ny, double Rg, const double *cp, double *gcp);
/* visc = 1: laminar viscosity; 0: thermal conductivity */
void orc_transport_nodes(const orc_mixture *m, int nx, int ny, int visc, const double *T, double *phip);
void orc_transport_faces(const orc_mixture *m, int nx, int ny, int visc, const double *Tbn, const double *Tbs,
                         const double *Tbe, const double *Tbw, const double *p, double *pe, double *pn);

#ifdef __cplusplus
}
#endif
#endif
