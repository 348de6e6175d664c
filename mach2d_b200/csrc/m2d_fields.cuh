// m2d_fields.cuh -- the device-resident field set of one nozzle instance and
// the launchers of the stencil kernels (src/equations/mach2d_coef.f90 and the
// internal-flow plug-in src/user/internal_flow/mod_intflow.f90).
#pragma once
#include "m2d_common.cuh"

namespace m2d {

// Every array is a device pointer of N doubles unless noted.  Names follow
// the reference's module variables (src/mod_mach2d_data.f90:30-173).
struct Fields {
    int nx, ny;
    // grid and metrics (src/grid/mod_grid.f90:304-723)
    double *x, *y, *xp, *yp, *xe, *ye, *xen, *yen, *xk, *yk, *xke, *yke;
    double *Jp, *Je, *Jn, *alphae, *gamman, *betae, *betan, *radius, *re, *rn, *rp;
    double *fbe, *fbn;
    // state
    double *p, *pa, *T, *Ta, *ro, *roa, *roe, *ron, *g, *u, *ua, *v, *va;
    double *ue, *un, *ve, *vn, *Uce, *Vcn, *uea, *vea, *una, *vna;
    double *cp, *vlp, *vle, *vln, *kp, *ke, *kn;
    double *cup, *sup, *cvp, *svp, *bu, *bv, *bt, *bp, *pl;
    double *due, *dve, *dun, *dvn, *de, *dn;
    double *vtp;            // Baldwin-Lomax eddy viscosity at the nodes (modtur = 1)
    double *au, *av, *at;   // 9N each
    double *ap;             // 5N
    // boundary strips
    double *uin, *vin, *pin, *Tin, *Mw, *plin, *pina;   // ny each
    double *Tbe, *Tbw;                                  // ny each
    double *Tbn, *Tbs;                                  // nx each
};

struct Params {
    int modvis, coord;
    double beta, dt, Rg, gamma, p0, T0, Cpref, Href, Twall;
    const double *dtp;     // when set, dt is read from this device word (captured iterations)
    double *maxpl;         // when set, the p' coefficient pass zeroes it for k_p_cycle_update's max|p'|
};

// what = bit 1: coefficients, bit 2: source (lets one kernel serve both the
// fused assembly and the separate drop-ins of get_*_coefficients/get_*_source)
enum { ASM_COEF = 1, ASM_SRC = 2 };

// ---- launchers (m2d_stencil.cu); all run on `st` and return cudaError_t ----
cudaError_t launch_density_at_nodes(const Fields &f, double Rg, cudaStream_t st);
cudaError_t launch_density_at_faces(const Fields &f, double beta, cudaStream_t st);
cudaError_t launch_u_assembly(const Fields &f, const Params &q, int what, cudaStream_t st);
// fused launches of the iteration (bitwise the separate kernels): u and v
// assembly with their boundary rows; internal and boundary face
// velocities; the p' coefficients, source and boundary rows of one cycle
cudaError_t launch_uv_assembly_bc(const Fields &f, const Params &q, int modvis, cudaStream_t st);
cudaError_t launch_faces_all(const Fields &f, double dt, int modvis, cudaStream_t st, const double *dtp);
cudaError_t launch_p_assembly_bc(const Fields &f, const Params &q, cudaStream_t st);
cudaError_t launch_v_assembly(const Fields &f, const Params &q, int what, cudaStream_t st);
cudaError_t launch_T_assembly(const Fields &f, const Params &q, cudaStream_t st);
cudaError_t launch_p_assembly(const Fields &f, const Params &q, int what, cudaStream_t st);
cudaError_t launch_velocities_at_internal_faces(const Fields &f, double dt, cudaStream_t st,
                                                const double *dtp = nullptr);
cudaError_t launch_internal_simplec(const Fields &f, cudaStream_t st);
cudaError_t launch_p_ro_correction(const Fields &f, int do_p, int do_ro, cudaStream_t st);
cudaError_t launch_uv_nodes_correction(const Fields &f, cudaStream_t st);
cudaError_t launch_velocity_correction_at_faces(const Fields &f, cudaStream_t st);
// the p' cycle's update after the solve, in one pass: the face velocities
// corrected with p' (mach2d_coef.f90:1679-1758) or, on the boundary faces,
// set by the internal-flow strips (mod_intflow.f90:692-787), p += p' and
// rho += g p' (mach2d_coef.f90:1602-1624), and max|p'| over every cell into
// *maxpl (zeroed earlier in the cycle; NaN counts as 0, as fmax drops it)
cudaError_t launch_p_cycle_update(const Fields &f, int modvis, double *maxpl, cudaStream_t st);
cudaError_t launch_boundary_faces_flags(const Fields &f, cudaStream_t st);
cudaError_t launch_set_bcu(const Fields &f, int modvis, cudaStream_t st);
cudaError_t launch_set_bcv(const Fields &f, int modvis, cudaStream_t st);
cudaError_t launch_set_bcpl(const Fields &f, cudaStream_t st);
cudaError_t launch_set_bcT(const Fields &f, double Twall, cudaStream_t st);
cudaError_t launch_velocities_at_boundary_faces(const Fields &f, int modvis, cudaStream_t st);
cudaError_t launch_boundary_simplec(const Fields &f, cudaStream_t st);
cudaError_t launch_extrapolate_uv(const Fields &f, int modvis, cudaStream_t st);
cudaError_t launch_T_from_H(const Fields &f, double Href, double Cpref, cudaStream_t st);
cudaError_t launch_T_boundary_H(const Fields &f, double Href, double Cpref, cudaStream_t st);
cudaError_t launch_inlet_update(const Fields &f, const Params &q, cudaStream_t st);
cudaError_t launch_g(const Fields &f, double Rg, cudaStream_t st);
cudaError_t launch_backup(const Fields &f, cudaStream_t st);

// ---- reductions (m2d_reduce.cu): deterministic two-pass FP64 trees.  The
// result is written to a device double so graphs and later kernels can use it
// without a host round trip.  `part` is scratch of at least red_parts() doubles.
int red_parts();
enum RedKind {
    RED_SUM_REAL = 0,     // sum of v over real cells                 (get_average)
    RED_MAXABS_ALL,       // max |v| over all N cells                 (normpl numerator)
    RED_NORM_L1_9D,       // sum |A x - b| over real cells, A 9-diag  (norm_l1_9d)
    RED_NORM_L1_5D,       // same, 5-diag in the order of norm_l1_5d
    RED_SUM_ABS_B,        // sum |b| over real cells                  (norm_l1_b)
    RED_MASS,             // sum |mass imbalance|                     (check_mass_conservation)
    RED_MEAN_CC_9D,       // sum of sum|a_nb|/|a_P| over real cells   (get_mean_cc_9d)
    RED_MEAN_CC_5D,
    RED_DT0,              // min 1/sqrt(Jp (u^2+v^2))                 (tstepper_dt0_scarborough)
};
struct RedArgs {
    int kind, nx, ny;
    const double *a, *x, *b;                 // matrix / vector / rhs or generic field
    // mass-conservation inputs
    const double *rp, *re, *rn, *Jp, *ro, *roa, *ron, *roe, *Uce, *Vcn, *u, *v;
    double dt;
    const double *dtp;     // when set, dt is read from this device word
};
cudaError_t launch_reduce(const RedArgs &r, double *part, double *out, cudaStream_t st);
// n (<= kMaxMultiReduce) reductions in one launch, each bitwise what
// launch_reduce gives; part holds n x red_parts() doubles
constexpr int kMaxMultiReduce = 4;
cudaError_t launch_reduce_multi(const RedArgs *r, double *const *out, int n, double *part, cudaStream_t st);

// inlet/outlet strip integrals of get_mass_flow_rate_and_thrust: out[0..2] = fmi, fme, Fd
cudaError_t launch_mass_flow_thrust(const Fields &f, double *out, cudaStream_t st);

}  // namespace m2d
