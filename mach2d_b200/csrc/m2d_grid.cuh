// m2d_grid.cuh -- grid metrics (src/grid/mod_grid.f90:237-723) and the
// per-cell parts of the internal-flow initial guess
// (src/user/internal_flow/mod_intflow.f90:1240-1488) on the device.
//
// The face radii are written once here, as expressions of one cell, and used
// both by the radius kernel and by the host set-up (which needs them on the
// north row for the quasi-1D isentropic strips), so the two agree bitwise.
#pragma once
#include "m2d_fields.cuh"

namespace m2d {

// radius at the centre of the north face of (i, j), get_radius
// (mod_grid.f90:606-614): the mean of the two north corners for i = 2..nx-1,
// j = 1..ny-1 of a cylindrical grid, 1 elsewhere
__host__ __device__ __forceinline__ double rn_value(int coord, int nx, int ny, const double *y, int i, int j)
{
    if (coord != 1 || i < 2 || i > nx - 1 || j < 1 || j > ny - 1) return 1.0;
    const long long np = cell(nx, i, j);
    return (y[np] + y[np - 1]) / 2.0;
}

// radius at the centre of the east face of (i, j) (mod_grid.f90:593-601):
// i = 1..nx-1, j = 2..ny-1
__host__ __device__ __forceinline__ double re_value(int coord, int nx, int ny, const double *y, int i, int j)
{
    if (coord != 1 || i < 1 || i > nx - 1 || j < 2 || j > ny - 1) return 1.0;
    const long long np = cell(nx, i, j);
    return (y[np] + y[np - nx]) / 2.0;
}

// radius of the north-east corner of (i, j) (mod_grid.f90:589)
__host__ __device__ __forceinline__ double radius_value(int coord, int nx, const double *y, int i, int j)
{
    return coord == 1 ? y[cell(nx, i, j)] : 1.0;
}

// the output planes of get_metrics, in its argument order
struct Metrics {
    double *xe, *ye, *xen, *yen, *xk, *yk, *xke, *yke, *Jp, *Je, *Jn, *alphae, *gamman, *betae, *betan;
};

// get_real_centroids_xy (mod_grid.f90:237-300): xp, yp of every cell
// (0 on the ghost ring); opt 1 = mean of the corners, else area-weighted
cudaError_t launch_centroids(int opt, int nx, int ny, const double *x, const double *y, double *xp, double *yp,
                             cudaStream_t st);
// get_metrics (mod_grid.f90:304-558): all 15 planes, every cell
cudaError_t launch_metrics(int nx, int ny, const double *x, const double *y, const double *xp, const double *yp,
                           const Metrics &m, cudaStream_t st);
// get_radius (mod_grid.f90:562-723): radius, re, rn, rp of every cell
cudaError_t launch_radius(int coord, int nx, int ny, const double *y, const double *yp, double *radius, double *re,
                          double *rn, double *rp, cudaStream_t st);

// initial guess, per-cell parts.  col holds 4 x nx doubles (0-based column
// index i-1): p1D, T1D, u1D of columns 2..nx-1 and the isentropic east-face
// velocity ue1D of columns 1..nx-1.  Writes p, T, u of columns 2..nx-1,
// un and Vcn of rows 2..ny-2, ue and Uce of the east faces; the rest of those
// planes keeps its value (zero in a fresh instance).
cudaError_t launch_initial_columns(const Fields &f, const double *col, cudaStream_t st);
// uin(j) = (u(1,j) + u(2,j)) / 2, j = 2..ny-1 (get_uin_vin_pin_Tin_Mw,
// mod_intflow.f90:988-994: the part that reads the extrapolated field)
cudaError_t launch_initial_inlet_u(const Fields &f, cudaStream_t st);
// p and T of the west ghosts from pin and Tin, of the east ghosts by
// extrapolation, and of the four corners (mod_intflow.f90:1363-1420)
cudaError_t launch_initial_pT_ghosts(const Fields &f, cudaStream_t st);
// p[k] = v for k < n
cudaError_t launch_fill(double *p, long long n, double v, cudaStream_t st);

}  // namespace m2d
