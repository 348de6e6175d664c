// m2d_thermo.cu -- thermophysical field kernels: set_cp, set_gamma,
// viscosity and conductivity at nodes and faces
// (src/thermophysical/mod_thermophysical.f90:79-509) and the boundary
// averages of src/util/mod_field_operations.f90:1-110.  One thread per cell
// or boundary element; every value uses the reference's expression order.
#include "m2d_thermo.cuh"

namespace m2d {

namespace {
constexpr int kBlock = 256;
inline unsigned blocks(long long n) { return (unsigned)((n + kBlock - 1) / kBlock); }
}

#define IDX(i, j) ((long long)nx * ((j) - 1) + (i) - 1)

// Fbn, Fbs (i = 2..nx-1) and Fbe, Fbw (j = 2..ny-1): mean of the last real
// volume and its ghost neighbour
__global__ void k_boundary_fields(int nx, int ny, const double *F, double *Fbn, double *Fbs, double *Fbe,
                                  double *Fbw)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nx - 2) {
        const int i = t + 2;
        Fbn[i - 1] = 0.5 * (F[IDX(i, ny - 1)] + F[IDX(i, ny)]);
        Fbs[i - 1] = 0.5 * (F[IDX(i, 2)] + F[IDX(i, 1)]);
    } else if (t < nx - 2 + ny - 2) {
        const int j = t - (nx - 2) + 2;
        Fbe[j - 1] = 0.5 * (F[IDX(nx - 1, j)] + F[IDX(nx, j)]);
        Fbw[j - 1] = 0.5 * (F[IDX(2, j)] + F[IDX(1, j)]);
    }
}

// cp at the real volumes and, stored in the ghost volumes, over the
// boundaries (corners by k_set_cp_corners)
__global__ void k_set_cp(int nx, int ny, const m2d_mixture *__restrict__ mix, const double *Tbn, const double *Tbs,
                         const double *Tbe, const double *Tbw, const double *T, double *cp)
{
    const long long np = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (np >= (long long)nx * ny) return;
    const int j = (int)(np / nx) + 1, i = (int)(np - (long long)(j - 1) * nx) + 1;
    const bool ci = i > 1 && i < nx, cj = j > 1 && j < ny;
    double Tv;
    if (ci && cj) Tv = T[np];
    else if (ci && j == ny) Tv = Tbn[i - 1];
    else if (ci && j == 1) Tv = Tbs[i - 1];
    else if (cj && i == nx) Tv = Tbe[j - 1];
    else if (cj && i == 1) Tv = Tbw[j - 1];
    else return;                                   // corner
    cp[np] = mix_cp(*mix, Tv);
}
// corners: mean of the three neighbours (end of set_cp, :79-218)
__global__ void k_set_cp_corners(int nx, int ny, double *cp)
{
    long long np = IDX(1, 1);
    cp[np] = (cp[np + nx] + cp[np + 1] + cp[np + nx + 1]) / 3.0;
    np = IDX(nx, 1);
    cp[np] = (cp[np + nx] + cp[np - 1] + cp[np + nx - 1]) / 3.0;
    np = IDX(1, ny);
    cp[np] = (cp[np - nx] + cp[np + 1] + cp[np - nx + 1]) / 3.0;
    np = IDX(nx, ny);
    cp[np] = (cp[np - nx] + cp[np - 1] + cp[np - nx - 1]) / 3.0;
}

__global__ void k_set_gamma(long long n, double Rg, const double *cp, double *gcp)
{
    const long long np = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (np < n) gcp[np] = cp[np] / (cp[np] - Rg);
}

__global__ void k_transport_nodes(int nx, int ny, const m2d_mixture *__restrict__ mix, bool viscosity,
                                  const double *T, double *phip)
{
    const long long np = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (np >= (long long)nx * ny) return;
    const int j = (int)(np / nx) + 1, i = (int)(np - (long long)(j - 1) * nx) + 1;
    if (i > 1 && i < nx && j > 1 && j < ny) phip[np] = viscosity ? mix_mu(*mix, T[np]) : mix_kp(*mix, T[np]);
}

// east faces (i = 1..nx-1, j = 2..ny-1) and north faces (i = 2..nx-1, j = 1..ny-1)
__global__ void k_transport_faces(int nx, int ny, const m2d_mixture *__restrict__ mix, bool viscosity,
                                  const double *Tbn, const double *Tbs, const double *Tbe, const double *Tbw,
                                  const double *phip, double *phie, double *phin)
{
    const long long np = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (np >= (long long)nx * ny) return;
    const int j = (int)(np / nx) + 1, i = (int)(np - (long long)(j - 1) * nx) + 1;
    auto model = [&](double Tv) { return viscosity ? mix_mu(*mix, Tv) : mix_kp(*mix, Tv); };
    if (j >= 2 && j <= ny - 1) {
        if (i >= 2 && i <= nx - 2) phie[np] = 2.0 * phip[np] * phip[np + 1] / (phip[np] + phip[np + 1]);
        else if (i == 1) phie[np] = model(Tbw[j - 1]);
        else if (i == nx - 1) phie[np] = model(Tbe[j - 1]);
    }
    if (i >= 2 && i <= nx - 1) {
        if (j >= 2 && j <= ny - 2) phin[np] = 2.0 * phip[np] * phip[np + nx] / (phip[np] + phip[np + nx]);
        else if (j == 1) phin[np] = model(Tbs[i - 1]);
        else if (j == ny - 1) phin[np] = model(Tbn[i - 1]);
    }
}

cudaError_t launch_boundary_fields(int nx, int ny, const double *F, double *Fbn, double *Fbs, double *Fbe,
                                   double *Fbw, cudaStream_t st)
{
    k_boundary_fields<<<blocks(nx + ny), kBlock, 0, st>>>(nx, ny, F, Fbn, Fbs, Fbe, Fbw);
    return cudaGetLastError();
}

cudaError_t launch_set_cp(int nx, int ny, const m2d_mixture *mix, const double *Tbn, const double *Tbs,
                          const double *Tbe, const double *Tbw, const double *T, double *cp, cudaStream_t st)
{
    k_set_cp<<<blocks((long long)nx * ny), kBlock, 0, st>>>(nx, ny, mix, Tbn, Tbs, Tbe, Tbw, T, cp);
    k_set_cp_corners<<<1, 1, 0, st>>>(nx, ny, cp);
    return cudaGetLastError();
}

cudaError_t launch_set_gamma(int nx, int ny, double Rg, const double *cp, double *gcp, cudaStream_t st)
{
    const long long n = (long long)nx * ny;
    k_set_gamma<<<blocks(n), kBlock, 0, st>>>(n, Rg, cp, gcp);
    return cudaGetLastError();
}

cudaError_t launch_transport_nodes(int nx, int ny, const m2d_mixture *mix, bool viscosity, const double *T,
                                   double *phip, cudaStream_t st)
{
    k_transport_nodes<<<blocks((long long)nx * ny), kBlock, 0, st>>>(nx, ny, mix, viscosity, T, phip);
    return cudaGetLastError();
}

cudaError_t launch_transport_faces(int nx, int ny, const m2d_mixture *mix, bool viscosity, const double *Tbn,
                                   const double *Tbs, const double *Tbe, const double *Tbw, const double *phip,
                                   double *phie, double *phin, cudaStream_t st)
{
    k_transport_faces<<<blocks((long long)nx * ny), kBlock, 0, st>>>(nx, ny, mix, viscosity, Tbn, Tbs, Tbe, Tbw,
                                                                    phip, phie, phin);
    return cudaGetLastError();
}

}  // namespace m2d
