// m2d_grid.cu -- grid metrics and the per-cell parts of the initial guess.
//
// One thread per cell, 32x8 blocks: each kernel reads the corner coordinates
// (and centroids) of a cell and its west/south neighbours and writes every
// output plane at that cell, including the zeros (or ones) the reference
// writes before its loops, so no output needs clearing first.  Where the
// reference fills a boundary strip in a separate loop after the interior
// (the one-sided xke/xen of the first and last faces, the ghost radii rp),
// the thread of that cell evaluates the strip's expression itself: every
// cell is written by exactly one of the reference's loops (or by a later one
// that only reads values of other loops), so the result does not depend on
// the order of the threads.  FP64 with -fmad=false: bitwise equal to the
// reference's sequential loops.
#include "m2d_grid.cuh"

namespace m2d {

#define IDX(i, j) ((long long)((j) - 1) * nx + ((i) - 1))

static inline dim3 grid2d(int nx, int ny)
{
    return dim3((unsigned)((nx + 31) / 32), (unsigned)((ny + 7) / 8));
}
static const dim3 kBlock2d(32, 8);
#define CELL_IJ                                      \
    const int i = blockIdx.x * 32 + threadIdx.x + 1; \
    const int j = blockIdx.y * 8 + threadIdx.y + 1;  \
    if (i > nx || j > ny) return;                    \
    const long long np = IDX(i, j);

// get_real_centroids_xy  mod_grid.f90:237-300
__global__ void k_centroids(int opt, int nx, int ny, const double *__restrict__ x, const double *__restrict__ y,
                            double *__restrict__ xp, double *__restrict__ yp)
{
    CELL_IJ
    double xo = 0.0, yo = 0.0;
    if (i >= 2 && i <= nx - 1 && j >= 2 && j <= ny - 1) {
        const long long nps = np - nx, npw = np - 1, npsw = nps - 1;
        if (opt == 1) {
            xo = (x[np] + x[npw] + x[npsw] + x[nps]) / 4.0;
            yo = (y[np] + y[npw] + y[npsw] + y[nps]) / 4.0;
        } else {
            // two triangles of areas A1, A2; the centroid is the area-weighted
            // mean of their corner means
            const double A1 = 0.5 * (x[npsw] * (y[nps] - y[np]) + x[nps] * (y[np] - y[npsw])
                                     + x[np] * (y[npsw] - y[nps]));
            const double A2 = 0.5 * (x[npsw] * (y[np] - y[npw]) + x[np] * (y[npw] - y[npsw])
                                     + x[npw] * (y[npsw] - y[np]));
            xo = ((x[npsw] + x[nps] + x[np]) * A1 + (x[npsw] + x[np] + x[npw]) * A2) / (3.0 * (A1 + A2));
            yo = ((y[npsw] + y[nps] + y[np]) * A1 + (y[npsw] + y[np] + y[npw]) * A2) / (3.0 * (A1 + A2));
        }
    }
    xp[np] = xo;
    yp[np] = yo;
}

// get_metrics  mod_grid.f90:304-558
__global__ void k_metrics(int nx, int ny, const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ xp, const double *__restrict__ yp, Metrics m)
{
    CELL_IJ
    double xe = 0.0, ye = 0.0, alphae = 0.0, xke = 0.0, yke = 0.0, betae = 0.0, Je = 0.0;
    double xk = 0.0, yk = 0.0, gamman = 0.0, xen = 0.0, yen = 0.0, betan = 0.0, Jn = 0.0, Jp = 0.0;
    // east face of (i, j): i = 1..nx-1, j = 2..ny-1
    if (i <= nx - 1 && j >= 2 && j <= ny - 1) {
        const long long nps = np - nx;
        xe = x[np] - x[nps];
        ye = y[np] - y[nps];
        alphae = xe * xe + ye * ye;
        if (i == 1) {
            // one-sided x_csi at the west boundary face, written by the
            // reference's i = 2 loop at npw (:394-411)
            const long long q = np + 1, qs = q - nx, qw = q - 1, qsw = qs - 1;
            double fw = (x[qw] + x[qsw]) / 2.0, fe = (x[q] + x[qs]) / 2.0;
            xke = -3.0 * fw + 4.0 * xp[q] - fe;
            fw = (y[qw] + y[qsw]) / 2.0;
            fe = (y[q] + y[qs]) / 2.0;
            yke = -3.0 * fw + 4.0 * yp[q] - fe;
        } else if (i == nx - 1) {
            // east boundary face (:416-432)
            const long long npw = np - 1, npsw = nps - 1;
            double fw = (x[npw] + x[npsw]) / 2.0, fe = (x[np] + x[nps]) / 2.0;
            xke = fw - 4.0 * xp[np] + 3.0 * fe;
            fw = (y[npw] + y[npsw]) / 2.0;
            fe = (y[np] + y[nps]) / 2.0;
            yke = fw - 4.0 * yp[np] + 3.0 * fe;
        } else {
            xke = xp[np + 1] - xp[np];
            yke = yp[np + 1] - yp[np];
        }
        betae = xke * xe + yke * ye;
        Je = fabs(1.0 / (xke * ye - xe * yke));
    }
    // north face of (i, j): i = 2..nx-1, j = 1..ny-1
    if (i >= 2 && i <= nx - 1 && j <= ny - 1) {
        const long long npw = np - 1;
        xk = x[np] - x[npw];
        yk = y[np] - y[npw];
        gamman = xk * xk + yk * yk;
        if (j == 1) {
            // south boundary face, written by the reference's j = 2 loop at nps
            // (:452-470); the north one below by the j = ny-1 loop (:474-492)
            const long long q = np + nx, qw = q - 1;
            double fs = (x[np] + x[npw]) / 2.0, fn = (x[q] + x[qw]) / 2.0;
            xen = -3.0 * fs + 4.0 * xp[q] - fn;
            fs = (y[np] + y[npw]) / 2.0;
            fn = (y[q] + y[qw]) / 2.0;
            yen = -3.0 * fs + 4.0 * yp[q] - fn;
        } else if (j == ny - 1) {
            const long long nps = np - nx, npsw = nps - 1;
            double fs = (x[nps] + x[npsw]) / 2.0, fn = (x[np] + x[npw]) / 2.0;
            xen = fs - 4.0 * xp[np] + 3.0 * fn;
            fs = (y[nps] + y[npsw]) / 2.0;
            fn = (y[np] + y[npw]) / 2.0;
            yen = fs - 4.0 * yp[np] + 3.0 * fn;
        } else {
            xen = xp[np + nx] - xp[np];
            yen = yp[np + nx] - yp[np];
        }
        betan = xk * xen + yk * yen;
        Jn = fabs(1.0 / (xk * yen - xen * yk));
    }
    // Jacobian at the centre of a real volume, from the face-centre means of
    // its corners
    if (i >= 2 && i <= nx - 1 && j >= 2 && j <= ny - 1) {
        const long long nps = np - nx, npw = np - 1, npsw = nps - 1;
        double fw = (x[npw] + x[npsw]) / 2.0, fe = (x[np] + x[nps]) / 2.0;
        double fs = (x[nps] + x[npsw]) / 2.0, fn = (x[np] + x[npw]) / 2.0;
        const double xkp = fe - fw, xep = fn - fs;
        fw = (y[npw] + y[npsw]) / 2.0;
        fe = (y[np] + y[nps]) / 2.0;
        fs = (y[nps] + y[npsw]) / 2.0;
        fn = (y[np] + y[npw]) / 2.0;
        const double ykp = fe - fw, yep = fn - fs;
        Jp = fabs(1.0 / (xkp * yep - xep * ykp));
    }
    m.xe[np] = xe; m.ye[np] = ye; m.alphae[np] = alphae; m.xke[np] = xke; m.yke[np] = yke;
    m.betae[np] = betae; m.Je[np] = Je;
    m.xk[np] = xk; m.yk[np] = yk; m.gamman[np] = gamman; m.xen[np] = xen; m.yen[np] = yen;
    m.betan[np] = betan; m.Jn[np] = Jn; m.Jp[np] = Jp;
}

// rp of a ghost cell that is not a corner (mod_grid.f90:621-670): the face
// radius reflected about the boundary face, r - rp(inner) + r
__device__ __forceinline__ double rp_edge(int nx, int ny, const double *y, const double *yp, int i, int j)
{
    double r;
    if (j == 1) { r = rn_value(1, nx, ny, y, i, 1); return r - yp[IDX(i, 2)] + r; }
    if (j == ny) { r = rn_value(1, nx, ny, y, i, ny - 1); return r - yp[IDX(i, ny - 1)] + r; }
    if (i == 1) { r = re_value(1, nx, ny, y, 1, j); return r - yp[IDX(2, j)] + r; }
    r = re_value(1, nx, ny, y, nx - 1, j);
    return r - yp[IDX(nx - 1, j)] + r;
}

// get_radius  mod_grid.f90:562-723
__global__ void k_radius(int coord, int nx, int ny, const double *__restrict__ y, const double *__restrict__ yp,
                         double *__restrict__ radius, double *__restrict__ re, double *__restrict__ rn,
                         double *__restrict__ rp)
{
    CELL_IJ
    if (coord != 1) {
        radius[np] = 1.0; re[np] = 1.0; rn[np] = 1.0; rp[np] = 1.0;
        return;
    }
    radius[np] = y[np];
    re[np] = re_value(1, nx, ny, y, i, j);
    rn[np] = rn_value(1, nx, ny, y, i, j);
    const bool wi = i == 1, ei = i == nx, sj = j == 1, nj = j == ny;
    double r;
    if ((wi || ei) && (sj || nj)) {
        // corners (:673-720): 4 y of the nearest interior corner minus the
        // three neighbouring rp
        const int ii = wi ? 1 : nx - 1, jj = sj ? 1 : ny - 1;       // corner node y(ii, jj)
        const int ia = wi ? 2 : nx - 1, jb = sj ? 2 : ny - 1;       // the neighbours' indices
        const int ic = wi ? 1 : nx, jc = sj ? 1 : ny;
        r = 4.0 * y[IDX(ii, jj)] - rp_edge(nx, ny, y, yp, ia, jc) - rp_edge(nx, ny, y, yp, ic, jb)
            - yp[IDX(ia, jb)];
    } else if (wi || ei || sj || nj) {
        r = rp_edge(nx, ny, y, yp, i, j);
    } else {
        r = yp[np];
    }
    rp[np] = r;
}

// ---------------------------------------------------------------------------
// get_initial_guess  mod_intflow.f90:1240-1488, per-cell parts

// p, T, u of columns 2..nx-1 (:1310-1350), un and Vcn of rows 2..ny-2, and
// the isentropic ue, Uce of the east faces (:1423-1453)
__global__ void k_initial_columns(Fields f, const double *__restrict__ col)
{
    const int nx = f.nx, ny = f.ny;
    CELL_IJ
    if (i >= 2 && i <= nx - 1) {
        const double p1 = col[i - 1], T1 = col[nx + i - 1], u1 = col[2 * nx + i - 1];
        f.p[np] = p1;
        f.T[np] = T1;
        f.u[np] = u1;
        if (j > 1 && j < ny - 1) {
            f.un[np] = u1;
            f.Vcn[np] = -u1 * f.yk[np];
        }
    }
    if (i <= nx - 1 && j >= 2 && j <= ny - 1) {
        const double ue1 = col[3 * nx + i - 1];
        f.ue[np] = ue1;
        f.Uce[np] = ue1 * f.ye[np];
    }
}

__global__ void k_initial_inlet_u(Fields f)
{
    const int nx = f.nx, ny = f.ny;
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    if (j > ny - 1) return;
    const long long np = IDX(1, j);
    f.uin[j - 1] = (f.u[np] + f.u[np + 1]) / 2.0;
}

__device__ __forceinline__ void west_ghost_pT(const Fields &f, int j, double &p, double &T)
{
    const int nx = f.nx;
    const long long npe = IDX(1, j) + 1;
    p = 2.0 * f.pin[j - 1] - f.p[npe];
    T = 2.0 * f.Tin[j - 1] - f.T[npe];
}
__device__ __forceinline__ void east_ghost_pT(const Fields &f, int j, double &p, double &T)
{
    const int nx = f.nx;
    const long long npw = IDX(nx, j) - 1, npww = npw - 1;
    p = f.p[npw] + 2.0 * (f.x[npw] - f.xp[npw]) / (f.xp[npw] - f.xp[npww]) * (f.p[npw] - f.p[npww]);
    T = f.T[npw] + 2.0 * (f.x[npw] - f.xp[npw]) / (f.xp[npw] - f.xp[npww]) * (f.T[npw] - f.T[npww]);
}

// one thread per row j = 1..ny, writing (1, j) and (nx, j); the corners copy
// the ghost of their neighbouring row, computed here again
__global__ void k_initial_pT_ghosts(Fields f)
{
    const int nx = f.nx, ny = f.ny;
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > ny) return;
    const int jr = j == 1 ? 2 : (j == ny ? ny - 1 : j);
    double p, T;
    west_ghost_pT(f, jr, p, T);
    f.p[IDX(1, j)] = p; f.T[IDX(1, j)] = T;
    east_ghost_pT(f, jr, p, T);
    f.p[IDX(nx, j)] = p; f.T[IDX(nx, j)] = T;
}

__global__ void k_fill(double *p, long long n, double v)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        p[k] = v;
}

// ---------------------------------------------------------------------------
cudaError_t launch_centroids(int opt, int nx, int ny, const double *x, const double *y, double *xp, double *yp,
                             cudaStream_t st)
{ k_centroids<<<grid2d(nx, ny), kBlock2d, 0, st>>>(opt, nx, ny, x, y, xp, yp); return cudaGetLastError(); }

cudaError_t launch_metrics(int nx, int ny, const double *x, const double *y, const double *xp, const double *yp,
                           const Metrics &m, cudaStream_t st)
{ k_metrics<<<grid2d(nx, ny), kBlock2d, 0, st>>>(nx, ny, x, y, xp, yp, m); return cudaGetLastError(); }

cudaError_t launch_radius(int coord, int nx, int ny, const double *y, const double *yp, double *radius, double *re,
                          double *rn, double *rp, cudaStream_t st)
{
    k_radius<<<grid2d(nx, ny), kBlock2d, 0, st>>>(coord, nx, ny, y, yp, radius, re, rn, rp);
    return cudaGetLastError();
}

cudaError_t launch_initial_columns(const Fields &f, const double *col, cudaStream_t st)
{ k_initial_columns<<<grid2d(f.nx, f.ny), kBlock2d, 0, st>>>(f, col); return cudaGetLastError(); }

cudaError_t launch_initial_inlet_u(const Fields &f, cudaStream_t st)
{ k_initial_inlet_u<<<(f.ny + 127) / 128, 128, 0, st>>>(f); return cudaGetLastError(); }

cudaError_t launch_initial_pT_ghosts(const Fields &f, cudaStream_t st)
{ k_initial_pT_ghosts<<<(f.ny + 127) / 128, 128, 0, st>>>(f); return cudaGetLastError(); }

cudaError_t launch_fill(double *p, long long n, double v, cudaStream_t st)
{
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    k_fill<<<(unsigned)b, 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

}  // namespace m2d
