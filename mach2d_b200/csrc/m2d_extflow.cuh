// m2d_extflow.cuh -- launchers of the external-flow boundary plug-in
// (m2d_extflow.cu; src/user/external_flow/mod_extflow.f90:166-317).
#pragma once
#include "m2d_common.cuh"

namespace m2d {

enum ExtScheme { EXT_U = 0, EXT_V = 1, EXT_RO = 2, EXT_T = 3, EXT_PL = 4 };

struct ExtArgs {
    int nx, ny, scheme, modvis;
    double value;               // free-stream value of the north strip: UF, 0, ROF, TF
    double Tsbc;                // wall temperature (< 0: adiabatic), scheme T
    const double *xk, *yk, *alphae, *betae, *betan, *gamman, *u, *v;
};

// the boundary rows of the 9-diagonal (schemes u, v, ro, T) or 5-diagonal
// (pl) matrix a and its source b; interior rows untouched
cudaError_t launch_extflow_rows(const ExtArgs &A, double *a, double *b, cudaStream_t st);
// the four boundary strips (north and south nx entries, east and west ny),
// column-major (entry, coefficient), 9 coefficients
cudaError_t launch_extflow_strips9(const ExtArgs &A, double *an, double *as, double *ae, double *aw, double *bn,
                                   double *bs, double *be, double *bw, cudaStream_t st);

// the strips of one scheme packed in one buffer of 20 (nx + ny) doubles:
// an, as (9 nx each), ae, aw (9 ny each), bn, bs (nx), be, bw (ny)
inline size_t extflow_strips_doubles(int nx, int ny) { return 20 * ((size_t)nx + (size_t)ny); }
cudaError_t launch_extflow_strips9_packed(const ExtArgs &A, double *strips, cudaStream_t st);
// longest boundary line the extrapolation takes: P and Q of one line in
// shared memory
constexpr int kExtExtrapolateMaxLine = 14336;
bool extflow_extrapolate_supported(int nx, int ny);
// get_bc_extrapolation_9d on the field F (nx*ny) from packed strips
cudaError_t launch_extflow_extrapolate(int nx, int ny, int itemax, const double *strips, double *F, cudaStream_t st);

// get_cdfi / get_cdfv over i = iiv..ifv of the south boundary; cd[0] =
// Cdfi, cd[1] = Cdfv (0 unless viscous)
struct DragArgs {
    int nx, iiv, ifv, viscous;
    double Rg, PF, TF, UF, rb;
    const double *xk, *yk, *rn, *Jn, *vln, *p, *u, *v, *Vcn;
};
cudaError_t launch_extflow_drag(const DragArgs &D, double *cd, cudaStream_t st);

// extflow_boundary_T_from_H_conservation
struct THArgs {
    int nx, ny;
    double CPF, HF;
    const double *u, *ue, *un, *v, *ve, *vn;
};
cudaError_t launch_extflow_T_from_H(const THArgs &H, double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs,
                                    cudaStream_t st);

}  // namespace m2d
