// m2d_blomax.cuh -- Baldwin-Lomax eddy viscosity (src/equations/blomax.f90).
#pragma once
#include <cuda_runtime.h>

namespace m2d {

// model constants, blomax.f90:5-10 (set_blomax_coefficients, :25-43)
struct BlConst {
    double kappa = 0.40, Aop = 26.0, alpha = 0.0168, Ccp = 1.6, Ckleb = 0.3, Cwk = 1.0;
};

// get_eddy_viscosity_blomax (blomax.f90:285-395): vtp at the real volumes,
// one warp per eta line
cudaError_t launch_blomax(int nx, int ny, const BlConst &c, const double *x, const double *y, const double *xp,
                          const double *yp, const double *xk, const double *yk, const double *Jp,
                          const double *Jn, const double *vln, const double *ro, const double *ron,
                          const double *u, const double *v, double *vtp, cudaStream_t st);
// get_eddy_viscosity_fictitious (blomax.f90:397-490)
cudaError_t launch_blomax_fictitious(int nx, int ny, double *phi, cudaStream_t st);
// the eddy viscosity into the transport coefficients (no reference call site:
// blomax.f90 is never called): mu + mu_t and k + cp mu_t / prt at the nodes,
// arithmetic face means of mu_t and cp mu_t at the east and north faces, the
// wall faces (north of the last real row) and the outermost faces laminar;
// ktm = 0 takes the laminar values from mu and kappa, ktm = 1 from the arrays
cudaError_t launch_add_eddy(int nx, int ny, int ktm, double mu, double kappa, double prt, const double *vtp,
                            const double *cp, double *vlp, double *vle, double *vln, double *kp, double *ke,
                            double *kn, cudaStream_t st);

}  // namespace m2d
