// m2d_extflow.cu -- the external-flow boundary plug-in on the device: the
// boundary rows that extflow_set_bcu / bcv / bcpl / bcro / bcT write
// (src/user/external_flow/mod_extflow.f90:166-317), from the schemes of
// get_bc_scheme_u / v / pl / ro / T (mod_extflow_procedures.f90:344-701) and
// the strip helpers of src/boundary_conditions/mach2d_bc9d.f90 and
// mach2d_bc5d.f90.
//
// The reference builds four boundary strips (north, south, east, west; each
// a row of coefficients and a source per boundary cell), overwrites their
// corner entries (get_bc_corners_9d / _5d) and copies them into the matrix
// north, south, east, then west (get_bc_transfer_9d / _5d), so a corner cell
// ends with its west or east strip entry.  Here one thread computes the
// final row of one ring cell directly: the strip entry that the transfer
// leaves there, with the same expressions, so the results are bitwise the
// reference's.  Every strip entry is O(1) work; the kernels touch only the
// 2 nx + 2 ny - 4 ring cells.
#include "m2d_extflow.cuh"

namespace m2d {

enum Side { SIDE_N = 0, SIDE_S = 1, SIDE_E = 2, SIDE_W = 3 };

// F(v, np) with the reference's 1-based np
#define E1(p, np) (p)[(long long)(np) - 1]

// the final entry `idx` (1-based) of boundary strip `side`, 9 coefficients
// in the order SW, S, SE, W, P, E, NW, N, NE, and the source
__device__ void strip_row9(const ExtArgs &A, int side, int idx, double *c, double &b)
{
    const int nx = A.nx, ny = A.ny;
    for (int k = 0; k < 9; k++) c[k] = 0.0;
    b = 0.0;
    const double third = -1.0 / 3.0;
    // the corners (get_bc_corners_9d, mach2d_bc9d.f90:521-615)
    const bool sw = (side == SIDE_S && idx == 1) || (side == SIDE_W && idx == 1);
    const bool se = (side == SIDE_S && idx == nx) || (side == SIDE_E && idx == 1);
    const bool nw = (side == SIDE_N && idx == 1) || (side == SIDE_W && idx == ny);
    const bool ne = (side == SIDE_N && idx == nx) || (side == SIDE_E && idx == ny);
    if (sw) { c[4] = 1.0; c[5] = third; c[7] = third; c[8] = third; return; }
    if (se) { c[3] = third; c[4] = 1.0; c[6] = third; c[7] = third; return; }
    if (nw) { c[1] = third; c[2] = third; c[4] = 1.0; c[5] = third; return; }
    if (ne) { c[0] = third; c[1] = third; c[3] = third; c[4] = 1.0; return; }
    if (side == SIDE_N) {                 // the free-stream value (UDS approximation)
        c[4] = 1.0;
        b = A.value;
        return;
    }
    if (side == SIDE_E) {                 // get_ibc_null_normal_grad_east_9d (:158-179)
        c[3] = -1.0; c[4] = 1.0;
        return;
    }
    if (side == SIDE_S) {
        const int i = idx, np = i;        // j = 1
        const bool slip = (A.scheme == EXT_U || A.scheme == EXT_V) && A.modvis == 0;
        const bool dirichlet = ((A.scheme == EXT_U || A.scheme == EXT_V) && A.modvis != 0) ||
                               (A.scheme == EXT_T && !(A.Tsbc < 0.0));
        if (slip) {                       // get_bc_u_slip_south_9d / get_bc_v_slip_south_9d (:352-439)
            const int npn = np + nx;
            const double xk = E1(A.xk, np), yk = E1(A.yk, np), u = E1(A.u, npn), v = E1(A.v, npn);
            const double lambda = copysign(1.0, xk * u + yk * v) * sqrt((u * u + v * v) / (xk * xk + yk * yk));
            c[4] = 1.0; c[7] = 1.0;
            b = 2.0 * lambda * (A.scheme == EXT_U ? xk : yk);
        } else if (dirichlet) {           // get_bc_dirichlet_south_9d (:40-62)
            c[4] = 1.0; c[7] = 1.0;
            b = 2.0 * (A.scheme == EXT_T ? A.Tsbc : 0.0);
        } else {                          // get_bc_null_normal_grad_south_9d (:184-263)
            const double bg = E1(A.betan, np) / E1(A.gamman, np);
            if (i == nx - 1) {
                const double raux = bg / 2.0;
                c[3] = -raux; c[4] = 1.0 + raux; c[6] = -raux; c[7] = -1.0 + raux;
            } else if (i == 2) {
                const double raux = bg / 2.0;
                c[4] = 1.0 - raux; c[5] = raux; c[7] = -1.0 - raux; c[8] = raux;
            } else {
                const double raux = bg / 4.0;
                c[3] = -raux; c[4] = 1.0; c[5] = raux; c[6] = -raux; c[7] = -1.0; c[8] = raux;
            }
        }
        return;
    }
    // west
    const int j = idx, np = nx * (j - 1) + 1;
    if (A.scheme == EXT_V) {              // get_bc_dirichlet_west_9d (:67-89), zero value
        c[4] = 1.0; c[5] = 1.0;
        b = 2.0 * 0.0;
        return;
    }
    // get_bc_null_normal_grad_west_9d (:268-346)
    if (j == ny - 1) {
        const double raux = 0.5 * E1(A.betae, np) / E1(A.alphae, np);
        c[1] = -raux; c[2] = -raux; c[4] = 1.0 + raux; c[5] = -1.0 + raux;
    } else if (j == 2) {
        const double raux = 0.5 * E1(A.betae, np) / E1(A.alphae, np);
        c[4] = 1.0 - raux; c[5] = -1.0 - raux; c[7] = raux; c[8] = raux;
    } else {
        const double raux = 0.25 * E1(A.betae, np) / E1(A.alphae, np);
        c[1] = -raux; c[2] = -raux; c[4] = 1.0; c[5] = -1.0; c[7] = raux; c[8] = raux;
    }
}

// the p' strips (get_bc_scheme_pl, mod_extflow_procedures.f90:344-399, and
// mach2d_bc5d.f90:44-206): S, W, P, E, N; every source zero
__device__ void strip_row5(const ExtArgs &A, int side, int idx, double *c)
{
    const int nx = A.nx, ny = A.ny;
    for (int k = 0; k < 5; k++) c[k] = 0.0;
    c[2] = 1.0;
    const int n = (side == SIDE_N || side == SIDE_S) ? nx : ny;
    if (idx == 1 || idx == n || side == SIDE_N) return;     // corners and the north strip: P only
    if (side == SIDE_S) c[4] = -1.0;
    else if (side == SIDE_E) c[1] = -1.0;
    else c[3] = -1.0;
}

// ring cell q -> (i, j) and the strip entry the transfer leaves there
__device__ __forceinline__ bool ring_cell(int q, int nx, int ny, int &i, int &j, int &side, int &idx)
{
    if (q < nx) { i = q + 1; j = 1; }
    else if (q < 2 * nx) { i = q - nx + 1; j = ny; }
    else if (q < 2 * nx + ny - 2) { i = 1; j = q - 2 * nx + 2; }
    else if (q < 2 * nx + 2 * (ny - 2)) { i = nx; j = q - 2 * nx - (ny - 2) + 2; }
    else return false;
    if (i == 1) { side = SIDE_W; idx = j; }
    else if (i == nx) { side = SIDE_E; idx = j; }
    else if (j == 1) { side = SIDE_S; idx = i; }
    else { side = SIDE_N; idx = i; }
    return true;
}

// boundary rows into the matrix (nd = 9 or 5) and its source
__global__ void k_extflow_rows(ExtArgs A, double *a, double *b)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, side, idx;
    if (!ring_cell(q, A.nx, A.ny, i, j, side, idx)) return;
    const long long N = (long long)A.nx * A.ny, np = (long long)A.nx * (j - 1) + (i - 1);
    if (A.scheme == EXT_PL) {
        double c[5];
        strip_row5(A, side, idx, c);
        for (int k = 0; k < 5; k++) a[k * N + np] = c[k];
        b[np] = 0.0;
    } else {
        double c[9], s;
        strip_row9(A, side, idx, c, s);
        for (int k = 0; k < 9; k++) a[k * N + np] = c[k];
        b[np] = s;
    }
}

// the four strips themselves (extflow_set_bcro returns them): entry e of the
// concatenation north (nx), south (nx), east (ny), west (ny); strip arrays
// column-major (entry, coefficient)
__global__ void k_extflow_strips9(ExtArgs A, double *an, double *as, double *ae, double *aw, double *bn, double *bs,
                                  double *be, double *bw)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = A.nx, ny = A.ny;
    int side, idx, n;
    double *a, *b;
    if (e < nx) { side = SIDE_N; idx = e + 1; a = an; b = bn; n = nx; }
    else if (e < 2 * nx) { side = SIDE_S; idx = e - nx + 1; a = as; b = bs; n = nx; }
    else if (e < 2 * nx + ny) { side = SIDE_E; idx = e - 2 * nx + 1; a = ae; b = be; n = ny; }
    else if (e < 2 * nx + 2 * ny) { side = SIDE_W; idx = e - 2 * nx - ny + 1; a = aw; b = bw; n = ny; }
    else return;
    double c[9], s;
    strip_row9(A, side, idx, c, s);
    for (int k = 0; k < 9; k++) a[(long long)k * n + idx - 1] = c[k];
    b[idx - 1] = s;
}

// get_bc_extrapolation_9d (mach2d_bc9d.f90:711-972): itemax sweeps of the
// north, south, east and west lines, in that order; each line is a
// tridiagonal system along the line (the strip's W, P, E or S, P, N
// coefficients) whose source is the strip source less the strip row's
// couplings to the real cells next to the line.  The lines depend on one
// another through the corner cells, so the sweeps stay in order inside one
// CTA: the block forms the line's right-hand side in parallel, then one
// thread runs the Thomas recurrences of the reference's tdma
// (mach2d_bc9d.f90:1292-1329) in the same operation order, P and the
// right-hand side / Q in shared memory, and writes the solution into F.
//
// Line L's three off-line couplings are strip columns c[L][0..2] at cell
// offsets o[L][0..2]; the first entry of a line drops the first coupling and
// the last entry the third, as the reference's end rows do.
struct ExtLines {
    const double *a[4], *b[4];  // strips north, south, east, west
};

__global__ void __launch_bounds__(256) k_extflow_extrapolate(ExtLines S, int nx, int ny, int itemax, double *F)
{
    extern __shared__ double sm[];
    const int nmax = nx > ny ? nx : ny;
    double *P = sm, *Q = sm + nmax;
    const int tid = threadIdx.x;
    // strip columns (0-based) of the couplings and of the line's own W/S, P, E/N
    const int cc[4][3] = {{0, 1, 2}, {6, 7, 8}, {0, 3, 6}, {2, 5, 8}};
    const int cl[4][3] = {{3, 4, 5}, {3, 4, 5}, {1, 4, 7}, {1, 4, 7}};
    const long long o[4][3] = {{-nx - 1, -nx, -nx + 1}, {nx - 1, nx, nx + 1}, {-nx - 1, -1, nx - 1},
                               {-nx + 1, 1, nx + 1}};
    for (int it = 0; it < itemax; it++) {
        for (int L = 0; L < 4; L++) {
            const int n = L < 2 ? nx : ny;
            const double *a = S.a[L], *b = S.b[L];
            // cell (0-based) of line entry e
            auto cell = [&](int e) -> long long {
                if (L == 0) return (long long)nx * (ny - 1) + e;
                if (L == 1) return e;
                if (L == 2) return (long long)nx * e + (nx - 1);
                return (long long)nx * e;
            };
            for (int e = tid; e < n; e += blockDim.x) {
                const long long np = cell(e);
                // coupling k of entry e; the end entries leave out the
                // coupling whose cell lies beyond the line (outside F for
                // the east and west lines)
                auto t = [&](int k) { return a[(long long)cc[L][k] * n + e] * F[np + o[L][k]]; };
                double r;
                if (e == 0) r = b[e] - (t(1) + t(2));
                else if (e == n - 1) r = b[e] - (t(0) + t(1));
                else r = b[e] - ((t(0) + t(1)) + t(2));
                Q[e] = r;
            }
            __syncthreads();
            if (tid == 0) {
                const double *aw = a + (long long)cl[L][0] * n, *ap = a + (long long)cl[L][1] * n,
                             *ae = a + (long long)cl[L][2] * n;
                P[0] = -ae[0] / ap[0];
                Q[0] = Q[0] / ap[0];
                for (int i = 1; i < n; i++) {
                    const double den = ap[i] + aw[i] * P[i - 1];
                    P[i] = -ae[i] / den;
                    Q[i] = (Q[i] - aw[i] * Q[i - 1]) / den;
                }
                double x = Q[n - 1];
                F[cell(n - 1)] = x;
                for (int i = n - 2; i >= 0; i--) {
                    x = x * P[i] + Q[i];
                    F[cell(i)] = x;
                }
            }
            __syncthreads();
        }
    }
}

bool extflow_extrapolate_supported(int nx, int ny)
{
    const int nmax = nx > ny ? nx : ny;
    return nx >= 4 && ny >= 4 && nmax <= kExtExtrapolateMaxLine;
}

cudaError_t launch_extflow_extrapolate(int nx, int ny, int itemax, const double *strips, double *F, cudaStream_t st)
{
    if (!extflow_extrapolate_supported(nx, ny) || itemax < 0) return cudaErrorInvalidValue;
    if (itemax == 0) return cudaSuccess;
    ExtLines S;
    const long long X = nx, Y = ny;
    S.a[0] = strips;
    S.a[1] = S.a[0] + 9 * X;
    S.a[2] = S.a[1] + 9 * X;
    S.a[3] = S.a[2] + 9 * Y;
    S.b[0] = S.a[3] + 9 * Y;
    S.b[1] = S.b[0] + X;
    S.b[2] = S.b[1] + X;
    S.b[3] = S.b[2] + Y;
    const size_t smem = 2 * sizeof(double) * (size_t)(nx > ny ? nx : ny);
    cudaError_t e = cudaFuncSetAttribute(k_extflow_extrapolate, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k_extflow_extrapolate<<<1, 256, smem, st>>>(S, nx, ny, itemax, F);
    return cudaGetLastError();
}

cudaError_t launch_extflow_strips9_packed(const ExtArgs &A, double *strips, cudaStream_t st)
{
    const long long X = A.nx, Y = A.ny;
    double *an = strips, *as = an + 9 * X, *ae = as + 9 * X, *aw = ae + 9 * Y;
    double *bn = aw + 9 * Y, *bs = bn + X, *be = bs + X, *bw = be + Y;
    return launch_extflow_strips9(A, an, as, ae, aw, bn, bs, be, bw, st);
}

// get_cdfi and get_cdfv (mod_extflow_procedures.f90:994-1104): the pressure
// and viscous foredrag sums over the south boundary, i = iiv..ifv, in the
// reference's order.  The block forms a chunk of the summands in shared
// memory, then one thread adds them in order: the sums are bitwise the
// reference's sequential loops.
constexpr int kDragChunk = 2048;

__global__ void __launch_bounds__(256) k_extflow_drag(DragArgs D, double *cd)
{
    __shared__ double ti[kDragChunk], tsx[kDragChunk], tsy[kDragChunk];
    const int nx = D.nx;
    const double ROF = D.PF / (D.Rg * D.TF);
    const double QF = ROF * (D.UF * D.UF) / 2.0;
    double cdfi = 0.0, cdfv = 0.0;
    for (int c0 = D.iiv; c0 <= D.ifv; c0 += kDragChunk) {
        const int n = min(kDragChunk, D.ifv - c0 + 1);
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const long long np = c0 + e, npn = np + nx;   // 1-based, j = 1
            const double pn = 0.5 * (E1(D.p, np) + E1(D.p, npn));
            ti[e] = (pn - D.PF) * E1(D.rn, np) * E1(D.yk, np);
            if (D.viscous) {
                const double du = E1(D.u, npn) - E1(D.u, np), dv = E1(D.v, npn) - E1(D.v, np);
                const double Sxx = -2.0 * E1(D.vln, np) * E1(D.Jn, np)
                                 * (E1(D.yk, np) * du + E1(D.rn, npn) * E1(D.Vcn, npn) / (3.0 * E1(D.rn, np)));
                const double Sxy = E1(D.vln, np) * E1(D.Jn, np) * (E1(D.xk, np) * du - E1(D.yk, np) * dv);
                tsx[e] = Sxx * E1(D.rn, np) * E1(D.yk, np);
                tsy[e] = Sxy * E1(D.rn, np) * E1(D.xk, np);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int e = 0; e < n; e++) cdfi = cdfi + ti[e];
            if (D.viscous)
                for (int e = 0; e < n; e++) cdfv = cdfv - tsx[e] + tsy[e];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        cd[0] = cdfi * 2.0 / ((D.rb * D.rb) * QF);
        cd[1] = D.viscous ? cdfv * 2.0 / (QF * (D.rb * D.rb)) : 0.0;
    }
}

cudaError_t launch_extflow_drag(const DragArgs &D, double *cd, cudaStream_t st)
{
    k_extflow_drag<<<1, 256, 0, st>>>(D, cd);
    return cudaGetLastError();
}

// extflow_boundary_T_from_H_conservation (mod_extflow.f90:438-544): T from
// the total enthalpy at every node, then the boundary temperatures of the
// four sides (faces of the first real or last real cells) and the ring cells
// by linear extrapolation through them.  Each ring write reads one real
// cell, which this thread recomputes with the same expression.
__global__ void k_extflow_T_from_H(THArgs H, double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = H.nx, ny = H.ny;
    if (c >= (long long)nx * ny) return;
    const int i = (int)(c % nx) + 1, j = (int)(c / nx) + 1;
    auto tnode = [&](long long q) {           // q 0-based
        return (H.HF - (H.u[q] * H.u[q] + H.v[q] * H.v[q]) / 2.0) / H.CPF;
    };
    auto tface = [&](const double *a, const double *b, long long q) {
        return (H.HF - (a[q] * a[q] + b[q] * b[q]) / 2.0) / H.CPF;
    };
    double t = tnode(c);
    const bool jin = j >= 2 && j <= ny - 1, iin = i >= 2 && i <= nx - 1;
    // the reference's order: east, west, north, south; no ring cell is
    // written twice (corners are not written at all)
    if (i == nx && jin) {
        const double tb = tface(H.ue, H.ve, c - 1);
        Tbe[j - 1] = tb;
        t = 2.0 * tb - tnode(c - 1);
    } else if (i == 1 && jin) {
        const double tb = tface(H.ue, H.ve, c);
        Tbw[j - 1] = tb;
        t = 2.0 * tb - tnode(c + 1);
    } else if (j == ny && iin) {
        const double tb = tface(H.un, H.vn, c - nx);
        Tbn[i - 1] = tb;
        t = 2.0 * tb - tnode(c - nx);
    } else if (j == 1 && iin) {
        const double tb = tface(H.un, H.vn, c);
        Tbs[i - 1] = tb;
        t = 2.0 * tb - tnode(c + nx);
    }
    T[c] = t;
}

cudaError_t launch_extflow_T_from_H(const THArgs &H, double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs,
                                    cudaStream_t st)
{
    const long long n = (long long)H.nx * H.ny;
    k_extflow_T_from_H<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(H, T, Tbe, Tbw, Tbn, Tbs);
    return cudaGetLastError();
}

cudaError_t launch_extflow_rows(const ExtArgs &A, double *a, double *b, cudaStream_t st)
{
    const int n = 2 * A.nx + 2 * (A.ny - 2);
    k_extflow_rows<<<(n + 127) / 128, 128, 0, st>>>(A, a, b);
    return cudaGetLastError();
}

cudaError_t launch_extflow_strips9(const ExtArgs &A, double *an, double *as, double *ae, double *aw, double *bn,
                                   double *bs, double *be, double *bw, cudaStream_t st)
{
    const int n = 2 * A.nx + 2 * A.ny;
    k_extflow_strips9<<<(n + 127) / 128, 128, 0, st>>>(A, an, as, ae, aw, bn, bs, be, bw);
    return cudaGetLastError();
}

}  // namespace m2d
