// m2d_thermo.cuh -- gas-mixture thermophysical model
// (src/thermophysical/mod_class_thermophysical_mixture.f90) and the field
// routines of src/thermophysical/mod_thermophysical.f90.
#pragma once
#include <cmath>
#include <cuda_runtime.h>
#include "../../include/mach2d_b200.h"

namespace m2d {

// species cp (J/kg.K): 5-coefficient polynomial in T below / above 1000 K,
// times R_i (cp_i, :563-581); powers as gfortran expands T**2, T**3, T**4
__host__ __device__ __forceinline__ double mix_cp_i(double T, double Ri, const double *a)
{
    const double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
    const double *c = (T <= 1000.0) ? a : a + 5;
    const double v = c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4;
    return v * Ri;
}
// exp(a ln T + b/T + c/T^2 + d) for the species viscosity (scale 1e-7, mu_i
// :639-654) and conductivity (scale 1e-4, kp_i :712-727)
__host__ __device__ __forceinline__ double mix_transport_i(double T, const double *a, double scale)
{
    const double *c = (T <= 1000.0) ? a : a + 4;
    return exp(c[0] * log(T) + c[1] / T + c[2] / (T * T) + c[3]) * scale;
}
// cp_mix (:539-559)
__host__ __device__ __forceinline__ double mix_cp(const m2d_mixture &m, double T)
{
    double s = 0.0;
    for (int i = 0; i < m.ngs; i++) s = s + m.Yi[i] * mix_cp_i(T, m.Ri[i], m.cpi[i]);
    return s;
}
// Wilke's rule of mu_mix (:585-635) and kp_mix (:658-708)
__host__ __device__ __forceinline__ double mix_wilke(const m2d_mixture &m, double T, bool viscosity)
{
    double r[M2D_MAX_SPECIES];
    for (int i = 0; i < m.ngs; i++)
        r[i] = viscosity ? mix_transport_i(T, m.mui[i], 1.0e-7) : mix_transport_i(T, m.kpi[i], 1.0e-4);
    double s = 0.0;
    for (int i = 0; i < m.ngs; i++) {
        double d = 0.0;
        for (int j = 0; j < m.ngs; j++) {
            const double t = 1.0 + sqrt(r[i] / r[j] * sqrt(m.Mi[j] / m.Mi[i]));
            d = d + m.Xi[j] * (t * t) / sqrt(8.0 * (1.0 + m.Mi[i] / m.Mi[j]));
        }
        s = s + m.Xi[i] * r[i] / d;
    }
    return s;
}
__host__ __device__ __forceinline__ double mix_mu(const m2d_mixture &m, double T) { return mix_wilke(m, T, true); }
__host__ __device__ __forceinline__ double mix_kp(const m2d_mixture &m, double T) { return mix_wilke(m, T, false); }
// gm (:261-272)
__host__ __device__ __forceinline__ double mix_gm(const m2d_mixture &m, double T)
{
    const double c = mix_cp(m, T);
    return c / (c - m.Rg);
}

// field launchers (m2d_thermo.cu); `mix` points to device memory
cudaError_t launch_boundary_fields(int nx, int ny, const double *F, double *Fbn, double *Fbs, double *Fbe,
                                   double *Fbw, cudaStream_t st);
cudaError_t launch_set_cp(int nx, int ny, const m2d_mixture *mix, const double *Tbn, const double *Tbs,
                          const double *Tbe, const double *Tbw, const double *T, double *cp, cudaStream_t st);
cudaError_t launch_set_gamma(int nx, int ny, double Rg, const double *cp, double *gcp, cudaStream_t st);
// vlp (viscosity = true) or kp at the real nodes
cudaError_t launch_transport_nodes(int nx, int ny, const m2d_mixture *mix, bool viscosity, const double *T,
                                   double *phip, cudaStream_t st);
// vle/vln or ke/kn: harmonic means inside, the model at the boundary faces
cudaError_t launch_transport_faces(int nx, int ny, const m2d_mixture *mix, bool viscosity, const double *Tbn,
                                   const double *Tbs, const double *Tbe, const double *Tbw, const double *phip,
                                   double *phie, double *phin, cudaStream_t st);

}  // namespace m2d
