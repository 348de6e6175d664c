/*
 * mach2d_b200.h -- C ABI of the B200 (sm_100a) implementation of MACH-2D's
 * SIMPLEC outer iteration.
 *
 * Two layers:
 *
 *  1. Drop-ins for the reference's routines.  Each entry point takes the
 *     reference routine's argument list in the reference's order, with HOST
 *     pointers and every argument by reference, exactly what a Fortran
 *     `bind(C)` interface passes.  Arrays use the
 *     reference layout: nx, ny count the ghost ring, cell (i,j) 1-based sits
 *     at offset nx*(j-1)+i-1, a coefficient matrix a(nx*ny,k) is stored
 *     diagonal after diagonal (9-diagonal order SW,S,SE,W,P,E,NW,N,NE;
 *     5-diagonal order S,W,P,E,N).  Each call copies its inputs to the GPU,
 *     runs the kernel and copies its outputs back; it is meant for swapping
 *     one routine at a time.
 *
 *  2. A device-resident context (m2d_ctx) that holds every field of one
 *     nozzle instance in HBM and runs whole outer iterations; host copies are
 *     made only on request.  This is the fast path.
 *
 * Every function returns 0 on success or an M2D_ERR_* code; m2d_last_error()
 * describes the last failure of the calling thread.  Nothing in the library
 * calls exit() or stop.  Errors of the solver kernels (non-finite pivots, an
 * unbounded MSI iteration that reached its cap) are reported through the
 * status code, never by trapping the GPU.
 */
#ifndef MACH2D_B200_H
#define MACH2D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define M2D_OK 0
#define M2D_ERR_CUDA 1         /* a CUDA call failed (m2d_last_error has it) */
#define M2D_ERR_ARG 2          /* invalid argument (sizes, null pointer, ...) */
#define M2D_ERR_NAN 3          /* NaN in the iteration norm (src/mach2d_main.f90:424-436) */
#define M2D_ERR_TIMEOUT 4      /* bounded iteration / wait reached its limit */
#define M2D_ERR_NOMEM 5        /* device allocation failed */
#define M2D_ERR_TOO_LARGE 6    /* grid larger than the kernel supports */
#define M2D_ERR_PIVOT 7        /* zero or non-finite pivot in the MSI factorisation */

const char *m2d_last_error(void);
int m2d_version(void);

/* ===================== 1. drop-ins for reference routines ================ */

/* ---- linear solvers ------------------------------------------------------
 * m2d_msi9_solve / m2d_msi5_solve replace class_solver_msi9d%solve and
 * class_solver_msi5d%solve (src/solvers/mod_solver_msi.f90:79-93,119-133):
 * incomplete LU (lu2d9 src/solvers/msi2d9-v03.f90:277-432, lu2d5
 * src/solvers/msi2d5-v03.f90:247-330) recomputed on every call, then the
 * fb2d9 / fb2d5 iteration (msi2d9-v03.f90:42-262, msi2d5-v03.f90:42-233) to
 * |r| < tol |r0| or nitm iterations (nitm <= 0: until converged, capped at
 * 10000 iterations with M2D_ERR_TIMEOUT).  x is the initial guess on entry.
 * Precondition of the reference (msi2d9-v03.f90:16-17): no coefficient couples
 * a cell to a neighbour outside the nx x ny grid.  ny <= m2d_msi_max_ny(). */
int m2d_msi9_solve(const int *nx, const int *ny, const int *nitm, const double *tol,
                   const double *a, const double *b, double *x);
int m2d_msi5_solve(const int *nx, const int *ny, const int *nitm, const double *tol,
                   const double *a, const double *b, double *x);
int m2d_msi_max_ny(void);
/* same, also returning the iterations performed */
int m2d_msi9_solve_it(const int *nx, const int *ny, const int *nitm, const double *tol,
                      const double *a, const double *b, double *x, int *nit);
int m2d_msi5_solve_it(const int *nx, const int *ny, const int *nitm, const double *tol,
                      const double *a, const double *b, double *x, int *nit);

/* Device-resident variant of the same solve for callers whose arrays already
 * live in GPU memory (CUDA Fortran / OpenACC data, or another library):
 * nd = 9 or 5; d_a, d_b, d_x device pointers in the layout above; d_work a
 * caller-allocated device buffer of m2d_msi_workspace_doubles(nd,nx,ny)
 * doubles (16-byte aligned, as cudaMalloc returns it, for the cluster kernel;
 * otherwise the slower one-CTA kernel runs); `stream` a cudaStream_t (NULL:
 * the default stream).  The call is
 * asynchronous: the iteration count is written to the device int *d_nit
 * (may be NULL) when the solve completes on `stream`. */
long m2d_msi_workspace_doubles(int nd, int nx, int ny);
int m2d_msi_solve_device(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                         const double *d_b, double *d_x, double *d_work, void *stream,
                         int *d_nit);
/* Diagnostics: the same solve, also writing seven %globaltimer stamps (ns)
 * to the device array d_times[7]: start, after the factorisation, after the
 * initial residual, after the first forward sweep, the first backward sweep
 * and the first residual, and at the end (ny <= 1024 only; otherwise the
 * stamps are left untouched). */
int m2d_msi_solve_device_timed(int nd, int nx, int ny, int nitm, double tol,
                               const double *d_a, const double *d_b, double *d_x,
                               double *d_work, void *stream, int *d_nit,
                               unsigned long long *d_times);
/* The device solve with its options spelled out: prec 0 (FP64, the
 * reference's arithmetic) or 1 (FP32 factors and sweeps in the FP64
 * iteration); reuse_factors = 1 when d_work already holds the factors of
 * this same d_a from an earlier solve with the same prec and sizes, d_work
 * untouched since (the cluster kernel then skips the transpose of A and the
 * factorisation; the one-CTA kernel factorises anyway; the iterates are the
 * same); d_times (may be null) as for m2d_msi_solve_device_timed, the
 * factorisation phase empty when reused. */
int m2d_msi_solve_device_ex(int nd, int nx, int ny, int nitm, double tol, const double *d_a, const double *d_b,
                            double *d_x, double *d_work, void *stream, int *d_nit, int prec, int reuse_factors,
                            unsigned long long *d_times);
/* Diagnostics: the FP64 solves factorise with reciprocal-based (Markstein)
 * quotients and check every factor against IEEE division while the first
 * sweeps run; when one differs (operands near the subnormal or overflow
 * range), the factorisation is repeated with IEEE division before x changes.
 * Returns how many factorisations were repeated on the current device since
 * the library was loaded (-1 on a CUDA error).  No counterpart in the
 * reference. */
long long m2d_msi_lu_redo_count(void);

/* Test hook for failure detection, no counterpart in the reference (whose
 * only failure check is the NaN test of src/mach2d_main.f90:424-436).  Every
 * device-side wait of the MSI cluster kernel (warp-to-warp hand-offs, staged
 * copies) and of the tcgen05 convolution is bounded by 4 s of %globaltimer
 * time; when one runs out the kernel records it, stops waiting, runs to its
 * end and the call returns M2D_ERR_TIMEOUT -- no trap, the context stays
 * usable.  kernel = 1 (MSI cluster kernel) or 2 (tcgen05 convolution) makes
 * the next launches of that kernel wait once more, on an mbarrier that
 * nothing completes, bounded by limit_s seconds (<= 10), so that this wait
 * runs out: the MSI solve then returns M2D_ERR_TIMEOUT from the host
 * drop-ins and m2d_iterate, the convolution through m2d_unet_status.
 * kernel = 0 (or limit_s = 0) switches the hook off. */
int m2d_test_wait_hook(int kernel, double limit_s);

/* No counterpart in the reference ("MSI_MIXED" in solvers_init).  The same
 * MSI iteration with the factorisation and both sweeps in FP32: the residual
 * r = A x - b, x, the norm and the stopping test |r| < tol |r0| stay FP64, so
 * the iteration is FP64 iterative refinement preconditioned by the FP32
 * incomplete LU and converges to the FP64 solution; it is not bitwise equal
 * to m2d_msi9_solve.  Same arguments as m2d_msi9_solve_it / the device
 * variant above; ny <= 1024 runs the FP32 cluster kernel, larger ny the FP64
 * one-CTA kernel. */
int m2d_msi9_solve_mixed(const int *nx, const int *ny, const int *nitm, const double *tol,
                         const double *a, const double *b, double *x, int *nit);
int m2d_msi5_solve_mixed(const int *nx, const int *ny, const int *nitm, const double *tol,
                         const double *a, const double *b, double *x, int *nit);
int m2d_msi_solve_device_mixed(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                               const double *d_b, double *d_x, double *d_work, void *stream,
                               int *d_nit);

/* No counterpart in the reference.  The same device-resident solve for
 * callers that cannot allocate device memory when they solve: a host program
 * whose device memory is all owned by its own pool (an OpenACC or CUDA
 * Fortran runtime, a framework's caching allocator), or a time-critical loop
 * that must not call cudaMalloc/cudaFree because they synchronise the device.
 * Allocates nothing: the workspace is a 12 MiB array in the library's own
 * device memory, held on every GPU that loads the library until exit.  Limit:
 * nx*ny <= m2d_msi_noalloc_max_cells(nd) (157286 cells for nd = 9, 196607 for
 * nd = 5); larger grids return M2D_ERR_TOO_LARGE.  Every call looks up the
 * array's device address on the current device (cudaGetSymbolAddress), so a
 * device reset between calls leaves no stale address; the first call on a
 * device also loads the device code there, so make it before any stream
 * capture.  The fast cluster kernel runs only while its wavefront-major
 * layout fits in the array (32*ceil(ny/32) * (nx + 62) <= 74849 for nd = 9,
 * <= 104789 for nd = 5); other grids under the cell limit, 514 x 258 with
 * nd = 9 among them, run the bitwise-equal but slower one-CTA kernel.  All
 * calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
long m2d_msi_noalloc_max_cells(int nd);
int m2d_msi_solve_device_noalloc(int nd, int nx, int ny, int nitm, double tol,
                                 const double *d_a, const double *d_b, double *d_x,
                                 void *stream, int *d_nit);

/* class_solver_tdma9d%solve / class_solver_tdma5d%solve
 * (src/solvers/mod_solver_tdma.f90:63-100): tdma2d9 src/solvers/tdma2d9.f90:38-322,
 * tdma2d5 src/solvers/tdma2d5.f90:38-241 */
int m2d_tdma9_solve(const int *nx, const int *ny, const int *nitm, const double *a,
                    const double *b, double *x);
int m2d_tdma5_solve(const int *nx, const int *ny, const int *nitm, const double *a,
                    const double *b, double *x);

/* A batch of independent tridiagonal lines (the x-line kernel of tdma2d9,
 * src/solvers/tdma2d9.f90:80-192, on caller-supplied lines): line l element
 * i at offset l*n + i; aw, ap, ae the W, P, E coefficients, d the rhs. */
int m2d_tdma_lines(const int *n, const int *nlines, const double *aw, const double *ap,
                   const double *ae, const double *d, double *x);
/* The same batch on device arrays (layout as above), asynchronous on
 * `stream`.  method 0: the sequential recurrence of the reference's line
 * sweep, one line per thread, bitwise m2d_tdma_lines; d_work holds 2 n
 * nlines doubles.  method 1 (no counterpart in the reference): parallel
 * cyclic reduction, one thread block per line in shared memory, n <= 2048
 * (else M2D_ERR_TOO_LARGE), d_work unused; its rounding differs from the
 * recurrence's (about 1e-15 relative on diagonally dominant lines). */
int m2d_tdma_lines_device(int n, int nlines, const double *d_aw, const double *d_ap, const double *d_ae,
                          const double *d_d, double *d_x, double *d_work, int method, void *stream);

/* norms: src/solvers/mod_solvers.f90:91-277.  `norm` is in/out (the routines
 * add to it); the sums run in a fixed tree order on the GPU. */
int m2d_norm_l1_5d(const int *nx, const int *ny, const double *var, const double *b,
                   const double *a, double *norm);
int m2d_norm_l1_9d(const int *nx, const int *ny, const double *var, const double *b,
                   const double *a, double *norm);
int m2d_norm_l1_9d_relative(const int *nx, const int *ny, const double *var,
                            const double *b, const double *a, double *norm);

/* ---- grid metrics: src/grid/mod_grid.f90 --------------------------------
 * Same arguments as the reference subroutines (Fortran by-reference scalars,
 * arrays of nx*ny doubles in host memory).  Every element of every output is
 * written, as the reference zero- (or one-) fills its outputs first; the
 * results are bitwise those of the reference's loops.  nx, ny >= 4. */
int m2d_get_real_centroids_xy(const int *opt, const int *nx, const int *ny, const double *x,
    const double *y, double *xp, double *yp);                                     /* :237-300 */
int m2d_get_metrics(const int *nx, const int *ny, const double *x, const double *y,
    const double *xp, const double *yp, double *xe, double *ye, double *xen, double *yen,
    double *xk, double *yk, double *xke, double *yke, double *Jp, double *Je, double *Jn,
    double *alphae, double *gamman, double *betae, double *betan);               /* :304-558 */
int m2d_get_radius(const int *coord, const int *nx, const int *ny, const double *y,
    const double *yp, double *radius, double *re, double *rn, double *rp);        /* :562-723 */

/* ---- coefficient assembly and corrections: src/equations/mach2d_coef.f90 */
int m2d_get_density_at_nodes(const int *nx, const int *ny, const double *Rg, const double *p,
                             const double *T, double *ro);                          /* :6-17 */
int m2d_get_density_at_faces(const int *nx, const int *ny, const double *beta,
                             const double *ro, const double *Uce, const double *Vcn,
                             double *roe, double *ron);                             /* :20-60 */
int m2d_get_u_coefficients(const int *nx, const int *ny, const int *modvis, const double *dt,
    const double *rp, const double *re, const double *rn, const double *Jp, const double *Je,
    const double *Jn, const double *ye, const double *yk, const double *alphae,
    const double *betae, const double *betan, const double *gamman, const double *vle,
    const double *vln, const double *roe, const double *ron, const double *roa,
    const double *Uce, const double *Vcn, double *a);                              /* :63-218 */
int m2d_get_u_source(const int *nx, const int *ny, const int *modvis, const double *beta,
    const double *dt, const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xke, const double *yke,
    const double *xen, const double *yen, const double *Jp, const double *Je, const double *Jn,
    const double *roe, const double *ron, const double *roa, const double *p, const double *vle,
    const double *vln, const double *Uce, const double *Vcn, const double *ua, const double *u,
    const double *v, double *cup, double *sup, double *b);                         /* :221-451 */
int m2d_get_v_coefficients(const int *nx, const int *ny, const int *coord, const int *modvis,
    const double *dt, const double *rp, const double *re, const double *rn, const double *Jp,
    const double *Je, const double *Jn, const double *xe, const double *xk,
    const double *alphae, const double *betae, const double *betan, const double *gamman,
    const double *vle, const double *vln, const double *vlp, const double *roe,
    const double *ron, const double *roa, const double *Uce, const double *Vcn,
    double *a);                                                                    /* :454-613 */
int m2d_get_v_source(const int *nx, const int *ny, const int *coord, const int *modvis,
    const double *beta, const double *dt, const double *rp, const double *re, const double *rn,
    const double *xe, const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *Jp, const double *Je,
    const double *Jn, const double *roe, const double *ron, const double *roa, const double *p,
    const double *vle, const double *vln, const double *Uce, const double *Vcn,
    const double *va, const double *u, const double *v, double *cvp, double *svp,
    double *b);                                                                    /* :616-783 */
int m2d_get_T_coefficients_and_source(const int *nx, const int *ny, const int *modvis,
    const double *beta, const double *dt, const double *rp, const double *re, const double *rn,
    const double *xe, const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *alphae,
    const double *betae, const double *betan, const double *gamman, const double *Jp,
    const double *Je, const double *Jn, const double *roe, const double *ron, const double *ro,
    const double *roa, const double *p, const double *pa, const double *cp, const double *vle,
    const double *vln, const double *ke, const double *kn, const double *Uce, const double *Vcn,
    const double *u, const double *v, const double *ue, const double *ve, const double *un,
    const double *vn, const double *ua, const double *va, const double *T, const double *Ta,
    const double *fbe, const double *fbn, double *a, double *b);                   /* :787-1203 */
int m2d_get_p_coefficients(const int *nx, const int *ny, const double *dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *Uce, const double *Vcn,
    const double *roe, const double *ron, const double *g, const double *de, const double *dn,
    double *a);                                                                    /* :1207-1278 */
int m2d_get_p_source(const int *nx, const int *ny, const double *dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *roe, const double *ron,
    const double *ro, const double *roa, const double *Uce, const double *Vcn, const double *de,
    const double *dn, const double *g, const double *pl, double *b);               /* :1281-1348 */
int m2d_get_velocities_at_internal_faces(const int *nx, const int *ny, const double *dt,
    const double *rp, const double *re, const double *rn, const double *xe, const double *ye,
    const double *xk, const double *yk, const double *xen, const double *yen, const double *xke,
    const double *yke, const double *Jp, const double *cup, const double *cvp, const double *sup,
    const double *svp, const double *au, const double *av, const double *roa, const double *p,
    const double *u, const double *v, const double *uea, const double *vea, const double *una,
    const double *vna, double *ue, double *ve, double *un, double *vn, double *Uce,
    double *Vcn);                                                                  /* :1350-1501 */
int m2d_get_internal_simplec_coefficients(const int *nx, const int *ny, const double *re,
    const double *rn, const double *xe, const double *ye, const double *xk, const double *yk,
    const double *au, const double *av, double *due, double *dve, double *dun, double *dvn,
    double *de, double *dn);                                                       /* :1504-1600 */
int m2d_get_pressure_correction_with_pl(const int *nx, const int *ny, const double *pl,
                                        double *p);                               /* :1602-1611 */
int m2d_get_density_correction_with_pl(const int *nx, const int *ny, const double *pl,
                                       const double *g, double *ro);              /* :1614-1624 */
int m2d_get_u_v_at_real_nodes_with_pl(const int *nx, const int *ny, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *rp, const double *pl,
    const double *au, const double *av, double *u, double *v);                     /* :1626-1675 */
int m2d_get_velocity_correction_at_faces_with_pl(const int *nx, const int *ny,
    const double *xe, const double *ye, const double *xk, const double *yk, const double *due,
    const double *dve, const double *dun, const double *dvn, const double *de, const double *dn,
    const double *pl, double *ue, double *ve, double *un, double *vn, double *Uce,
    double *Vcn);                                                                  /* :1679-1758 */
int m2d_initialize_boundary_faces_flags(const int *nx, const int *ny, double *fbe,
                                        double *fbn);                             /* :1764-1828 */
int m2d_check_mass_conservation(const int *nx, const int *ny, const double *dt,
    const double *rp, const double *re, const double *rn, const double *Jp, const double *ro,
    const double *roa, const double *ron, const double *roe, const double *Uce,
    const double *Vcn, double *res);                                               /* :1833-1880 */

/* ---- Baldwin-Lomax eddy viscosity: src/equations/blomax.f90 -------------
 * set/get_blomax_coefficients (:25-62), initialize_blomax (:67-80; the
 * vorticity metrics of :83-115 are evaluated inside the kernel, so this only
 * checks its arguments), get_eddy_viscosity_blomax (:285-395: vtp at the real
 * volumes, ghost entries left as passed), get_eddy_viscosity_fictitious
 * (:397-490).  The reference never calls the model from its main loop. */
int m2d_set_blomax_coefficients(const double *kappa, const double *Aop, const double *alpha,
                                const double *Ccp, const double *Ckleb, const double *Cwk);
int m2d_get_blomax_coefficients(double *kappa, double *Aop, double *alpha, double *Ccp,
                                double *Ckleb, double *Cwk);
int m2d_initialize_blomax(const int *nx, const int *ny, const double *x, const double *y);
int m2d_get_eddy_viscosity_blomax(const int *nx, const int *ny, const double *x, const double *y,
    const double *xp, const double *yp, const double *xk, const double *yk, const double *Jp,
    const double *Jn, const double *vln, const double *ro, const double *ron, const double *u,
    const double *v, double *vtp);
int m2d_get_eddy_viscosity_fictitious(const int *nx, const int *ny, double *phi);

/* ---- internal-flow plug-in: src/user/internal_flow/mod_intflow.f90 ------- */
int m2d_intflow_set_bcu(const int *nx, const int *ny, const int *modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u, const double *v,
    double *au, double *b);                                                        /* :214-301 */
int m2d_intflow_set_bcv(const int *nx, const int *ny, const int *modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u, const double *v,
    double *av, double *b);                                                        /* :305-392 */
/* plin(ny) stands for iflow%plin of the derived-type argument */
int m2d_intflow_set_bcpl(const int *nx, const int *ny, const double *x, const double *xp,
    const double *pl, const double *plin, double *ap, double *bp);                 /* :396-459 */
/* Twall and Tin(ny) stand for iflow%Twall and iflow%Tin */
int m2d_intflow_set_bcT(const int *nx, const int *ny, const double *x, const double *xp,
    const double *T, const double *Twall, const double *Tin, double *at, double *bt); /* :464-550 */
int m2d_intflow_boundary_T_from_H_conservation(const int *nx, const int *ny,
    const double *Cpref, const double *Href, const double *Tin, const double *u,
    const double *ue, const double *un, const double *v, const double *ve, const double *vn,
    double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs);               /* :557-688 */
int m2d_intflow_velocities_at_boundary_faces(const int *nx, const int *ny, const int *modvis,
    const double *x, const double *xp, const double *xe, const double *ye, const double *xk,
    const double *yk, const double *u, const double *v, double *ue, double *ve, double *un,
    double *vn, double *Uce, double *Vcn);                                         /* :692-787 */
int m2d_intflow_boundary_simplec(const int *nx, const int *ny, const int *modvis, double *due,
    double *dve, double *dun, double *dvn, double *de, double *dn);                /* :791-877 */
int m2d_intflow_extrapolate_u_v_to_fictitious(const int *nx, const int *ny, const int *modvis,
    const double *x, const double *xp, const double *xk, const double *yk, double *u,
    double *v);                                                                    /* :881-964 */
/* intflow_time_cycle_update (:1106-1134): gamma, Rg, P0, T0 and the inlet
 * arrays (ny each) stand for the thermophysical model and iflow members */
int m2d_intflow_time_cycle_update(const int *nx, const int *ny, const double *x,
    const double *xp, const double *u, const double *gamma, const double *Rg,
    const double *P0, const double *T0, double *uin, double *vin, double *pin, double *Tin,
    double *Mw, double *plin, double *pina, double *p);

/* ---- external-flow plug-in: src/user/external_flow/mod_extflow.f90 ------
 * The boundary rows of the external-flow problem (far field north, body
 * wall south, outflow east, symmetry axis west), from the schemes of
 * get_bc_scheme_u/v/pl/ro/T (mod_extflow_procedures.f90:344-701) and the
 * strip helpers of src/boundary_conditions/mach2d_bc9d.f90 and
 * mach2d_bc5d.f90, corners and transfer included; bitwise the reference's.
 * UF, ROF, TF and Tsbc stand for the module's free-stream speed, density
 * and temperature and the wall temperature (Tsbc < 0: adiabatic).  Only the
 * boundary rows of a and b are written.  The reference's external-flow
 * geometry library, grid generator and driver set-up are not part of this
 * library. */
int m2d_extflow_set_bcu(const int *nx, const int *ny, const int *modvis, const double *UF, const double *xk,
    const double *yk, const double *alphae, const double *betae, const double *u, const double *v, double *au,
    double *bu);                                                                   /* :166-198 */
int m2d_extflow_set_bcv(const int *nx, const int *ny, const int *modvis, const double *xk, const double *yk,
    const double *u, const double *v, double *av, double *bv);                     /* :202-231 */
int m2d_extflow_set_bcpl(const int *nx, const int *ny, double *ap, double *bp);  /* :235-259 */
/* returns the four strips (a9bn(nx,9), a9bs(nx,9), a9be(ny,9), a9bw(ny,9),
 * column-major, and b9bn(nx), b9bs(nx), b9be(ny), b9bw(ny)), as the
 * reference's routine does */
int m2d_extflow_set_bcro(const int *nx, const int *ny, const double *ROF, const double *alphae,
    const double *betae, const double *betan, const double *gamman, double *a9bn, double *a9bs, double *a9be,
    double *a9bw, double *b9bn, double *b9bs, double *b9be, double *b9bw);        /* :263-285 */
int m2d_extflow_set_bcT(const int *nx, const int *ny, const double *TF, const double *Tsbc,
    const double *alphae, const double *betae, const double *betan, const double *gamman, double *at,
    double *bt);                                                                   /* :289-317 */
/* extflow_extrapolate_u_v_to_fictitious (:360-397) and
 * extflow_extrapolate_ro_to_fictitious (:401-431): the ring cells of u and v
 * (or ro) from the strips of get_bc_scheme_u/v (or extflow_set_bcro) by
 * itemax sweeps of get_bc_extrapolation_9d (mach2d_bc9d.f90:711-972), one
 * tridiagonal solve per boundary line in the reference's order and
 * arithmetic; bitwise the reference's.  nx, ny >= 4 and max(nx, ny) <=
 * 14336 (one line's recurrences in shared memory), else M2D_ERR_ARG. */
int m2d_extflow_extrapolate_u_v_to_fictitious(const int *nx, const int *ny, const int *modvis, const int *itemax,
    const double *UF, const double *xk, const double *yk, const double *alphae, const double *betae, double *u,
    double *v);
int m2d_extflow_extrapolate_ro_to_fictitious(const int *nx, const int *ny, const int *itemax, const double *ROF,
    const double *alphae, const double *betae, const double *betan, const double *gamman, double *ro);
/* extflow_calc_main_variables (:321-356): the pressure foredrag Cdfi
 * (get_cdfi, mod_extflow_procedures.f90:994-1041) and, for modvis = 1, the
 * viscous foredrag Cdfv (get_cdfv, :1045-1104; else 0) over the south
 * boundary cells i = 2..iocs, summed in the reference's order.  PF, TF, UF,
 * rb and iocs stand for the module's far-field pressure, temperature and
 * speed, base radius and the index of the ogive-cylinder junction; the two
 * coefficients are returned instead of the reference's message lines. */
int m2d_extflow_calc_main_variables(const int *nx, const int *ny, const double *Rg, const int *modvis,
    const double *PF, const double *TF, const double *UF, const double *rb, const int *iocs, const double *xk,
    const double *yk, const double *rn, const double *Jn, const double *vln, const double *p, const double *u,
    const double *v, const double *Vcn, double *Cdfi, double *Cdfv);
/* extflow_boundary_T_from_H_conservation (:438-544): T = (HF - |V|^2 / 2) /
 * CPF at every node, the boundary temperatures Tbe, Tbw (j = 2..ny-1) and
 * Tbn, Tbs (i = 2..nx-1) from the face velocities, and the ring cells by
 * linear extrapolation through them; the end entries of Tb* keep the
 * caller's values. */
int m2d_extflow_boundary_T_from_H_conservation(const int *nx, const int *ny, const double *CPF, const double *HF,
    const double *u, const double *ue, const double *un, const double *v, const double *ve, const double *vn,
    double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs);

/* ---- thermophysical properties: src/thermophysical/ ----------------------
 * The gas-mixture model (class_thermophysical_mixture,
 * mod_class_thermophysical_mixture.f90): cp(T) from 5-coefficient
 * polynomials per species (below / above 1000 K), mu(T) and k(T) from
 * exp(a ln T + b/T + c/T^2 + d) per species combined by Wilke's rule.
 * m2d_mixture_init (init, :56-224) takes the species of the mixture
 * (fractions <= 1e-8 are skipped, as the reference does): base 0 = molar,
 * 1 = mass fractions; Mi in kg/mol; cpi ngs x 10, mui and kpi ngs x 8,
 * species-major, in the database's coefficient order.  It fills Xi, Yi, Ri
 * and Rg = Ru / Mg, and returns M2D_ERR_ARG if the fractions do not sum to 1
 * within 10 epsilon.  The field routines below take the mixture in place of
 * the reference's thermomodel pointer. */
#define M2D_MAX_SPECIES 8
typedef struct m2d_mixture {
    int ngs;                                         /* gaseous species */
    double Rg;                                       /* J/(kg K) */
    double Xi[M2D_MAX_SPECIES], Yi[M2D_MAX_SPECIES]; /* molar and mass fractions */
    double Mi[M2D_MAX_SPECIES], Ri[M2D_MAX_SPECIES]; /* kg/mol, Ru/Mi */
    double cpi[M2D_MAX_SPECIES][10];
    double mui[M2D_MAX_SPECIES][8];
    double kpi[M2D_MAX_SPECIES][8];
} m2d_mixture;
int m2d_mixture_init(int base, int ngs, const double *fractions, const double *Mi,
                     const double *cpi, const double *mui, const double *kpi, m2d_mixture *out);
/* point values: cp, mu, kp, gm (mixture functions :227-272); NULL outputs skipped */
int m2d_mixture_eval(const m2d_mixture *mix, double T, double *cp, double *mu, double *kp,
                     double *gm);
/* mod_thermophysical.f90 field routines (:79-509) and the boundary averages
 * of src/util/mod_field_operations.f90:1-110 (get_north/south/east/west_
 * boundary_field in one call) */
int m2d_set_cp(const m2d_mixture *mix, const int *nx, const int *ny, const double *Tbn,
    const double *Tbs, const double *Tbe, const double *Tbw, const double *T, double *cp);
int m2d_set_gamma(const int *nx, const int *ny, const double *Rg, const double *cp, double *gcp);
int m2d_set_laminar_viscosity_at_nodes(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *T, double *vlp);
int m2d_set_thermal_conductivity_at_nodes(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *T, double *kp);
int m2d_get_laminar_viscosity_at_faces(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *Tbn, const double *Tbs, const double *Tbe, const double *Tbw,
    const double *vlp, double *vle, double *vln);
int m2d_get_thermal_conductivity_at_faces(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *Tbn, const double *Tbs, const double *Tbe, const double *Tbw,
    const double *kp, double *ke, double *kn);
int m2d_get_boundary_fields(const int *nx, const int *ny, const double *F, double *Fbn,
    double *Fbs, double *Fbe, double *Fbw);

/* ===================== 2. device-resident SIMPLEC context =================
 * Mirrors the set-up and the `it` loop body of src/mach2d_main.f90:25-445 for
 * internal flow, with the CONSTANT (ktm = 0) or MIXTURE (ktm = 1)
 * thermophysical model. */

typedef struct m2d_case {
    int geom;                               /* 0: C01 cosine nozzle, 1: N01 nozzle */
    double Lc, Ld, Rin, Rout;               /* C01 (Rin, Rout also N01) */
    double Rth, Rc1, Rc2, Rc3, alf, bet, Lchamb;  /* N01, geometry_n01.txt */
    int nxr, nyr;                           /* real volumes (nxi-2, nyi-2 at nmd = nmf) */
    int kg, kcm;                            /* grid kind 1 uniform / 2 geometric; centroid mean */
    double a1;                              /* first wall-cell width for kg = 2 */
    int coord, modvis;
    double beta;
    double p0, T0, Twall;                   /* Tnbc: Twall <= 0 means adiabatic */
    double Rg, gamma, mu, kappa;            /* CONSTANT thermophysical model (ktm = 0) */
    int itmmax, itpmax;
    double tolm, tolt;
    int solver;                             /* 0 MSI, 1 TDMA, 2 MSI with FP32 factors and sweeps,
                                               3 as 2 with the learned p' correction first
                                               (m2d_ctx_set_unet), 4 as 3 with a kept correction
                                               that already meets MSI's stopping test standing
                                               alone (no MSI iteration for that p' solve) */
    int nitm_u, nitm_p;
    double tol_u, tol_p;
    int dtmodel;                            /* 0 RAMP, 1 SCARBOROUGH */
    double dt1, dt2; int it1, it2;
    double h0, mincc, maxcc;
    int nan_policy;                         /* max() with the NaN of at = 0: 0 drop, 1 propagate */
    int ktm;                                /* 0 CONSTANT, 1 MIXTURE (thermophysical_initialization) */
    m2d_mixture mix;                        /* ktm = 1: the gas mixture (m2d_mixture_init) */
    int modtur;                             /* 1 (with modvis = 1): Baldwin-Lomax eddy viscosity
                                               (src/equations/blomax.f90:285-490), which the
                                               reference compiles but never calls, evaluated at the
                                               start of each outer iteration from the previous
                                               flow and added to the transport coefficients:
                                               mu + mu_t and k + cp mu_t / prt at the nodes, the
                                               arithmetic face means of mu_t and cp mu_t at the
                                               east and north faces, the wall faces laminar */
    double prt;                             /* turbulent Prandtl number (modtur = 1) */
    int msi_lag;                            /* solvers 2-4, cluster MSI kernel: 0 factorises every
                                               solve, as the reference; n > 0 lets a solve reuse
                                               the FP32 factors its workspace holds for the same
                                               equation from fewer than n solves ago while one
                                               iteration still meets the tolerance (the FP64
                                               residual and stopping test are unchanged; a stale
                                               solve that needs a second iteration renews the
                                               factors at the next one).  Not the reference's
                                               algorithm: only the preconditioner ages. */
} m2d_case;

typedef struct m2d_report {
    int it;
    double dt, norm, normpl, rmass, fmi, fme, Fd;
    int itp_used;
} m2d_report;

typedef struct m2d_ctx m2d_ctx;

int m2d_create(const m2d_case *c, int device, m2d_ctx **out);
int m2d_destroy(m2d_ctx *ctx);
int m2d_dims(const m2d_ctx *ctx, int *nx, int *ny);
/* one pass of the `it` loop body, src/mach2d_main.f90:94-445 */
int m2d_iterate(m2d_ctx *ctx, m2d_report *rep);
/* up to itmax iterations with the reference's stopping rule
 * (normpl < tolt first at it, then stop at it_stop = 2 it; :441-443) */
int m2d_run(m2d_ctx *ctx, int itmax, m2d_report *last);
/* copy a named field (reference variable name: "u", "p", "au", "Tbn", ...) */
int m2d_get_field(m2d_ctx *ctx, const char *name, double *host, long n);
int m2d_set_field(m2d_ctx *ctx, const char *name, const double *host, long n);
/* several fields per call (one copy each, one synchronisation; pinned host
 * buffers make the copies asynchronous DMA) */
int m2d_set_fields(m2d_ctx *ctx, int count, const char *const *names, const double *const *host,
                   const long *n);
int m2d_get_fields(m2d_ctx *ctx, int count, const char *const *names, double *const *host,
                   const long *n);
/* named scalars: dt, norm, normpl, rmass, p_avg, Href, Cpref, fm1D, Fd1D,
 * Fpv1D, Sg, it, it_stop; and of the last iteration itp_used and the MSI
 * iterations nit_u, nit_v, nit_p (last p' cycle), nit_T; launches (kernels
 * started so far), learned_calls, learned_accepted, learned_alone (p' solves
 * the correction alone settled, solver 4), solver, msi_schedule */
int m2d_get_scalar(const m2d_ctx *ctx, const char *name, double *out);
/* post-processing integrals (src/user/internal_flow/mod_intflow.f90:1591-1643,
 * mod_intflow_postp.f90:1211 Cd = fme/fm1D, :430-445,1454-1465 wall pressure
 * p(i,ny-1) for i = 1..nx into pwall, may be null) */
int m2d_integrals(m2d_ctx *ctx, double *fmi, double *fme, double *Fd, double *Cd,
                  double *pwall);
/* the cudaStream_t the context launches on, and the device address of a
 * named field (for callers that time or chain their own kernels) */
int m2d_ctx_stream(const m2d_ctx *ctx, void **stream);
/* the network of solver 3 (not owned; its images must hold the real cells);
 * NULL detaches.  Scalars learned_calls / learned_accepted count the p'
 * solves and the corrections kept. */
struct m2d_unet;
int m2d_ctx_set_unet(m2d_ctx *ctx, struct m2d_unet *net);
/* 1: run each outer iteration as one captured CUDA graph (built on the next
 * m2d_iterate): the p' loop is a conditional WHILE node whose exit
 * (normpl < tolm or itpmax cycles) and the next time step are computed on
 * the device, so an iteration costs one graph launch and one read-back
 * instead of about 60 launches and a host synchronisation per p' cycle.
 * Results are bitwise those of the default mode (0).  Not with solver 3. */
int m2d_ctx_set_graph(m2d_ctx *ctx, int on);
int m2d_ctx_field_device(m2d_ctx *ctx, const char *name, double **dptr, long *n);
/* The wavefront schedule of the context's MSI solves, no counterpart in the
 * reference: 0 automatic (one wavefront warp per SM when the thread-block
 * cluster fits, else two), 1 one warp per SM with 4 staging stages, 2 two
 * warps per SM with 2 stages (half the SMs per solve), 3 the one-CTA kernel
 * (FP64 solvers only; with FP32 sweeps it means 0).  A schedule that cannot
 * run falls back to the one-CTA kernel.  All schedules give the same
 * iterates; a captured iteration is captured again on its next call. */
int m2d_ctx_set_msi_schedule(m2d_ctx *ctx, int variant);

/* ---- batches of instances (no counterpart in the reference) ------------
 * n independent nozzle instances on one GPU, each a full context with its
 * own stream.  m2d_batch_create sets the instances up with `workers` host
 * threads (<= 0: min(n, 16)); if one fails, none is kept and the call
 * returns that failure.  m2d_batch_iterate runs `iters` outer iterations of
 * every instance with the same threads, so that several
 * instances have kernels in flight at once; reps[k] (may be NULL) receives
 * instance k's last report.  An instance whose iteration fails stops there
 * (m2d_batch_status); the call returns the first failure.  Each instance's
 * results equal those of running it alone.  m2d_batch_ctx gives an
 * instance's context for fields and integrals. */
typedef struct m2d_batch m2d_batch;
int m2d_batch_create(const m2d_case *cases, int n, int device, int workers, m2d_batch **out);
int m2d_batch_size(const m2d_batch *b, int *n);
int m2d_batch_ctx(m2d_batch *b, int k, m2d_ctx **ctx);
int m2d_batch_iterate(m2d_batch *b, int iters, m2d_report *reps);
int m2d_batch_status(const m2d_batch *b, int k, int *status);
/* Instances whose iterations run as captured graphs (m2d_ctx_set_graph on
 * m2d_batch_ctx) are advanced with every graph in flight at once: each
 * iteration launches all of them, then waits for each.  Each instance has its
 * own stream; for more than a few instances set the environment variable
 * CUDA_DEVICE_MAX_CONNECTIONS=32 before the process's first CUDA call, so
 * that the streams do not share the default 8 hardware queues (256 uneven
 * nozzles: 131 M cell-updates/s with 8, 310 M with 32 on one B200).
 * m2d_batch_set_msi_schedule: m2d_ctx_set_msi_schedule on every instance.
 * m2d_batch_autotune: the schedule autotuner -- runs the batch's next
 * 1 + iters iterations with each candidate schedule (1, 2, and 3 when every
 * instance solves in FP64), times the last iters of each on the host clock,
 * keeps the fastest (*chosen, may be NULL) and writes each candidate's
 * milliseconds per iteration to ms_per_iter[variant] (4 doubles, may be
 * NULL; -1 for schedules not tried).  Schedules give the same iterates, so
 * the tuned run's results equal an untuned one's. */
int m2d_batch_set_msi_schedule(m2d_batch *b, int variant);
int m2d_batch_autotune(m2d_batch *b, int iters, int *chosen, double *ms_per_iter);

/* ===================== 3. learned p' preconditioner ======================
 * No counterpart in the reference.  A 4-level U-Net (3x3 convolutions with
 * 16/32/64/128 channels, GELU, 2x2 mean pooling, nearest upsampling with
 * skip concatenation, 1x1 head; BF16 weights and activations, FP32
 * accumulation) maps 11 planes of a p' system to a p' correction.
 * Images are H x W (multiples of 8), pixel (y, x) = real cell (x+2, y+2).
 * Parameters (FP32 master copy, m2d_unet_param_count() floats): per
 * convolution in network order -- enc0 (16->16, 16->16), enc1 (16->32,
 * 32->32), enc2 (32->64, 64->64), bottleneck (64->128, 128->128), dec2
 * (192->64, 64->64), dec1 (96->32, 32->32), dec0 (48->16, 16->16) --
 * W[cout][9][cin] (tap = 3 dy + dx) then b[cout]; last the head's 16
 * weights and bias.  The input layer's channels 11..15 see zeros.
 * All data pointers are device pointers; calls are asynchronous on `stream`
 * unless they return host values. */
typedef struct m2d_unet m2d_unet;
long m2d_unet_param_count(void);
/* bmax images per call at most; allocates activations, gradients and Adam state */
int m2d_unet_create(int bmax, int H, int W, int device, m2d_unet **out);
int m2d_unet_destroy(m2d_unet *net);
int m2d_unet_shape(const m2d_unet *net, int *bmax, int *H, int *W);
/* host FP32 parameters in and out (set also resets the Adam state) */
int m2d_unet_set_params(m2d_unet *net, const float *host, long n);
int m2d_unet_get_params(m2d_unet *net, float *host, long n);
int m2d_unet_get_grads(m2d_unet *net, float *host, long n);
/* d_in: [nimg][11][H][W] FP32 planes; d_out: [nimg][H][W] FP32 */
int m2d_unet_forward(m2d_unet *net, int nimg, const float *d_in, float *d_out, void *stream);
/* forward, loss = scale * sum mask (out - target)^2 (mask may be NULL), and
 * backward into the gradients (zeroed first); *loss (host, may be NULL)
 * receives the loss after a stream synchronisation */
int m2d_unet_loss_grad(m2d_unet *net, int nimg, const float *d_in, const float *d_target,
                       const float *d_mask, float scale, float *loss, void *stream);
/* one Adam step on the master parameters, then their BF16 copies */
int m2d_unet_adam(m2d_unet *net, float lr, float beta1, float beta2, float eps, void *stream);
/* which convolutions run on the tcgen05 kernel: 0 none (all on the mma.sync
 * kernel); 1 (default) or 2 every one whose image has an even height and a
 * width that is a multiple of 128 (the others use the mma.sync kernel) */
int m2d_unet_set_tensor_path(int mode);
/* synchronises; *flags = device error word (8: a tensor-core kernel's
 * bounded wait ran out, returned as M2D_ERR_TIMEOUT); the word is cleared
 * after it is read */
int m2d_unet_status(m2d_unet *net, int *flags);

/* p' system <-> images.  d_a: 5 planes (S, W, P, E, N), d_stats: 16 doubles.
 * Features: r/(aP sigma) with sigma the RMS of r/aP, the nine coefficient
 * planes over aP (SW, S, SE, W, P, E, NW, N, NE; corners zero), and the
 * standardised log Jp.  apply: x_out = x + sigma y on the real cells and,
 * on the ghost ring, the value that satisfies the cell's own row given its
 * corrected neighbours (x_out must not alias x).  target: t = delta /
 * sigma and mask = 1 on real cells.  residual5: r = b - A x on every cell
 * (the norm of the MSI stopping test), *d_rr = |r|^2 (may be NULL). */
int m2d_residual5(int nx, int ny, const double *d_a, const double *d_b, const double *d_x,
                  double *d_r, double *d_rr, void *stream);
int m2d_pprime_features(int nx, int ny, int H, int W, const double *d_a, const double *d_r,
                        const double *d_Jp, float *d_feat, double *d_stats, void *stream);
int m2d_pprime_apply(int nx, int ny, int H, int W, const double *d_a, const double *d_b,
                     const float *d_y, const double *d_stats, const double *d_x, double *d_xout,
                     void *stream);
int m2d_pprime_target(int nx, int ny, int H, int W, const double *d_delta, const double *d_stats,
                      float *d_t, float *d_mask, void *stream);
/* Flexible pressure-correction solve of the 5-diagonal p' system: the
 * network's correction is kept only when it lowers |b - A x|; the MSI
 * iteration (prec bit 0: 0 FP64, 1 FP32 sweeps) then runs with its stopping
 * test relative to the residual before the correction; like plain MSI it
 * runs at least one iteration, unless prec bit 1 is set and the corrected
 * residual (FP64, every cell) already meets |r| < tol |r0|: then the
 * correction is the solution and rep->nit = 0.
 * d_work: m2d_msi_workspace_doubles(5, nx, ny). */
typedef struct m2d_learned_report {
    int accepted;          /* 1: the network's correction was kept */
    double r0, r1;         /* |r| before and after the correction */
    int nit;               /* MSI iterations that followed */
} m2d_learned_report;
int m2d_pprime_solve_learned(m2d_unet *net, int nx, int ny, int nitm, double tol,
                             const double *d_a, const double *d_b, double *d_x, const double *d_Jp,
                             double *d_work, int prec, void *stream, m2d_learned_report *rep);
/* Two-level cycles: the network's correction (kept only when it lowers |r|)
 * alternating with m MSI iterations (the last step of a cycle is always MSI)
 * until |r| <= tol |r0| or max_cycles;
 * rep->nit counts every MSI iteration, rep->accepted the kept corrections,
 * rep->r1 is the final |r|. */
int m2d_pprime_solve_cycles(m2d_unet *net, int nx, int ny, int m, int max_cycles, double tol,
                            const double *d_a, const double *d_b, double *d_x, const double *d_Jp,
                            double *d_work, int prec, void *stream, m2d_learned_report *rep);
int m2d_batch_destroy(m2d_batch *b);

/* ===================== 4. flexible GMRES (no counterpart in the reference) =====
 * The reference iterates MSI as a stationary method (x += (LU)^-1 (b - A x),
 * fb2d9 / fb2d5).  m2d_fgmres_solve keeps MSI's incomplete factorisation
 * (computed once per call) as the right preconditioner of flexible GMRES
 * (Saad 1993) with restart length `restart` (1..32), to |b - A x| <= tol |b|
 * or maxit preconditioner applications (then M2D_ERR_TIMEOUT).  prec 0: MSI
 * with FP64 factors; 1: FP32 factors and sweeps; 2 (nd = 5): the learned
 * correction of `net` (images covering the real cells; Jp for its features)
 * followed by one FP32 MSI step from it, z = N(v) + (LU)^-1 (v - A N(v)).
 * All device pointers; x is the initial guess on entry; d_work holds
 * m2d_fgmres_workspace_doubles(nd, nx, ny, restart) doubles, 16-byte
 * aligned.  Synchronises `stream` once per Krylov step (the Hessenberg
 * least-squares problem is solved on the host); dot products are FP64 in a
 * fixed order, so a solve is reproducible bit for bit. */
typedef struct m2d_fgmres_report {
    int iterations;              /* Krylov steps = preconditioner applications */
    int msi_applications;        /* MSI forward/backward sweep pairs */
    int learned_applications;    /* network corrections (prec 2) */
    int cycles;                  /* restart cycles */
    int converged;
    double rel_residual;         /* |b - A x| / |b| of the returned x, recomputed */
} m2d_fgmres_report;
long m2d_fgmres_workspace_doubles(int nd, int nx, int ny, int restart);
int m2d_fgmres_solve(int nd, int nx, int ny, int restart, int maxit, double tol, const double *d_a,
                     const double *d_b, double *d_x, int prec, m2d_unet *net, const double *d_Jp,
                     double *d_work, void *stream, m2d_fgmres_report *rep);

#ifdef __cplusplus
}
#endif
#endif
