// m2d_msi.cu -- MSI wavefront kernels (lu2d9/fb2d9, lu2d5/fb2d5) and line TDMA.
//
// Dependency structure.  The incomplete factorisation and the forward sweep
// of cell (i,j) read (i-1,j), (i-1,j-1), (i,j-1) and (i+1,j-1)
// (src/solvers/msi2d9-v03.f90:155,357-366); the backward sweep reads the
// mirror image.  Cells on the hyperplane t = i + 2j are therefore mutually
// independent and the whole grid is swept in nx + 2(ny-1) steps.
//
// Execution.  One CTA per linear system.  Thread t owns rows j = t, t+T, ...
// and at step s processes column i = s - 2j of each owned row, so a row lags
// the one below it by two columns.  The factor values a row produces are
// published in a 4-step shared-memory ring [slot][value][row] (conflict-free:
// consecutive threads read consecutive rows); one __syncthreads per step.
// Residuals and the L2 norm of the stopping test run over all cells with
// coalesced accesses and a fixed-order block tree.
//
// Parity.  The reference's special cases for the first/last rows and columns
// are the general formula with out-of-grid neighbours taken as zero and the
// relaxation alpha = 0 there; under the reference's own precondition (no
// coupling to neighbours outside the grid, msi2d9-v03.f90:16-17) the zero
// terms add exact zeros, so with -fmad=false every factor and every sweep
// value is bitwise equal to the lexicographic reference loop.  Only the
// stopping test's sum of squares is ordered differently.
#include "m2d_solvers.cuh"

namespace m2d {

static const int kMaxThreads = 1024;
static const int kRingSlots = 4;
static const int kMaxIterUnbounded = 10000;   // nitm <= 0: loop until converged, bounded

int msi_block_threads(int ny)
{
    int t = ((ny + 31) / 32) * 32;
    return t > kMaxThreads ? kMaxThreads : t;
}
size_t msi_smem_bytes(int nd, int ny)
{
    int nu = (nd == 9) ? 4 : 3;
    return (size_t)kRingSlots * nu * ny * sizeof(double) + (size_t)msi_block_threads(ny) * sizeof(double);
}
size_t msi_skew_plane(int nx, int ny)
{
    return (size_t)((ny + 31) / 32) * (size_t)(nx + 62) * 32;
}
size_t msi_generic_work_doubles(int nd, int nx, int ny)
{
    return (size_t)(nd == 9 ? 10 : 8) * (size_t)nx * ny;                 // dl, du, residual
}
size_t msi_cluster_work_doubles(int nd, int nx, int ny)
{
    // dl, du, 1/dl1, residual, correction and A, wavefront-major, then the
    // scratch of the whole-GPU residual passes
    return (size_t)(nd == 9 ? 21 : 15) * msi_skew_plane(nx, ny) + kMsiExtScratch;
}
size_t msi_work_doubles(int nd, int nx, int ny)
{
    const size_t g = msi_generic_work_doubles(nd, nx, ny), c = msi_cluster_work_doubles(nd, nx, ny);
    return g > c ? g : c;
}
int msi_max_ny()
{
    // 227 KB of opt-in shared memory per CTA on sm_100
    int ny = 16;
    while (msi_smem_bytes(9, ny + 16) <= 227 * 1024) ny += 16;
    return ny;
}

#define RING(slot, k, row) ring[((size_t)(slot) * NU + (k)) * ny + (row)]
#define PL(p, k, np) (p)[(long long)((k) - 1) * N + (np)]

// fixed-order block sum for any blockDim.x (a multiple of 32): fold the
// tail onto the largest power of two, then a binary tree
template <int ND>
__device__ double block_sum(double v, double *red)
{
    const int T = blockDim.x;
    int P = 1;
    while (P * 2 <= T) P *= 2;
    red[threadIdx.x] = v;
    __syncthreads();
    if (threadIdx.x < T - P) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + P];
    __syncthreads();
    for (int s = P / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    double r = red[0];
    __syncthreads();
    return r;
}

// r = A x - b over all cells, in-range neighbours only, in ascending diagonal
// order (msi2d9-v03.f90:61-131 / msi2d5-v03.f90:61-119); returns this
// thread's partial sum of r^2.
template <int ND>
__device__ double residual(const double *__restrict__ a, const double *__restrict__ b,
                           const double *x, double *r, int nx, int ny)
{
    const long long N = (long long)nx * ny;
    double acc = 0.0;
    for (long long np = threadIdx.x; np < N; np += blockDim.x) {
        const int i = (int)(np % nx), j = (int)(np / nx);
        const bool w = i > 0, e = i < nx - 1, s = j > 0, n = j < ny - 1;
        double v = -b[np];
        if (ND == 9) {
            if (s && w) v = v + PL(a, 1, np) * x[np - nx - 1];
            if (s) v = v + PL(a, 2, np) * x[np - nx];
            if (s && e) v = v + PL(a, 3, np) * x[np - nx + 1];
            if (w) v = v + PL(a, 4, np) * x[np - 1];
            v = v + PL(a, 5, np) * x[np];
            if (e) v = v + PL(a, 6, np) * x[np + 1];
            if (n && w) v = v + PL(a, 7, np) * x[np + nx - 1];
            if (n) v = v + PL(a, 8, np) * x[np + nx];
            if (n && e) v = v + PL(a, 9, np) * x[np + nx + 1];
        } else {
            if (s) v = v + PL(a, 1, np) * x[np - nx];
            if (w) v = v + PL(a, 2, np) * x[np - 1];
            v = v + PL(a, 3, np) * x[np];
            if (e) v = v + PL(a, 4, np) * x[np + 1];
            if (n) v = v + PL(a, 5, np) * x[np + nx];
        }
        r[np] = v;
        acc = acc + v * v;
    }
    return acc;
}

template <int ND>
__global__ void __launch_bounds__(kMaxThreads) k_msi(MsiLaunch L)
{
    constexpr int NU = (ND == 9) ? 4 : 3;
    extern __shared__ double smem[];
    const MsiSys S = L.dev ? L.dev[blockIdx.x] : L.s[blockIdx.x];
    const int nx = L.nx, ny = L.ny;
    const long long N = (long long)nx * ny;
    const int T = blockDim.x;
    const int nsteps = nx + 2 * (ny - 1);
    double *ring = smem;
    double *red = smem + (size_t)kRingSlots * NU * ny;
    const double *__restrict__ a = S.a;
    // plain plane-major scratch: dl planes, du planes, one residual plane
    double *__restrict__ dl = S.ws;
    double *__restrict__ du = S.ws + (ND == 9 ? 5 : 4) * N;
    double *wk = du + NU * N;
    double *x = S.x;
    bool bad_pivot = false;

    // ---- incomplete LU (lu2d9 msi2d9-v03.f90:277-432, lu2d5 msi2d5-v03.f90:247-330)
    for (int s = 0; s < nsteps; s++) {
        const int c0 = s & 3, c1 = (s + 3) & 3, c2 = (s + 2) & 3, c3 = (s + 1) & 3;
        for (int j = threadIdx.x; j < ny; j += T) {
            const int i = s - 2 * j;
            if (i < 0 || i >= nx) continue;
            const long long np = (long long)j * nx + i;
            const bool hw = i > 0, hs = j > 0, hsw = hs && i > 0, hse = hs && i < nx - 1;
            const double alpha = (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) ? 0.5 : 0.0;
            if (ND == 9) {
                double w1 = hw ? RING(c1, 0, j) : 0.0, w2 = hw ? RING(c1, 1, j) : 0.0;
                double w3 = hw ? RING(c1, 2, j) : 0.0, w4 = hw ? RING(c1, 3, j) : 0.0;
                double s1 = hs ? RING(c2, 0, j - 1) : 0.0, s2 = hs ? RING(c2, 1, j - 1) : 0.0;
                double s3 = hs ? RING(c2, 2, j - 1) : 0.0, s4 = hs ? RING(c2, 3, j - 1) : 0.0;
                double sw1 = hsw ? RING(c3, 0, j - 1) : 0.0, sw2 = hsw ? RING(c3, 1, j - 1) : 0.0;
                double sw3 = hsw ? RING(c3, 2, j - 1) : 0.0, sw4 = hsw ? RING(c3, 3, j - 1) : 0.0;
                double se1 = hse ? RING(c1, 0, j - 1) : 0.0, se2 = hse ? RING(c1, 1, j - 1) : 0.0;
                double se3 = hse ? RING(c1, 2, j - 1) : 0.0, se4 = hse ? RING(c1, 3, j - 1) : 0.0;
                const double b1 = PL(a, 1, np), b2 = PL(a, 2, np), b3 = PL(a, 3, np);
                const double b4 = PL(a, 4, np), b5 = PL(a, 5, np), b6 = PL(a, 6, np);
                const double b7 = PL(a, 7, np), b8 = PL(a, 8, np), b9 = PL(a, 9, np);
                double l5 = b1;
                double l4 = (b2 - l5 * sw1 - alpha * b3 * se1) / (1.0 - alpha * s1 * se1);
                double l3 = b3 - l4 * s1;
                double l2 = (b4 - l4 * s2 - l5 * sw3 - 2.0 * alpha * l5 * sw2) / (1 + 2.0 * alpha * w2);
                double phi1 = l3 * se1, phi2 = l5 * sw2, phi3 = l3 * se4, phi4 = l2 * w2;
                double l1 = b5 - l2 * w1 - l3 * se2 - l4 * s3 - l5 * sw4
                          + alpha * (2.0 * phi1 + phi2 + phi3 + 2.0 * phi4);
                double u1 = (b6 - l3 * se3 - l4 * s4 - 2.0 * alpha * (phi1 + phi3)) / l1;
                double u2 = (b7 - l2 * w3) / l1;
                double u3 = (b8 - l2 * w4 - alpha * phi4) / l1;
                double u4 = b9 / l1;
                if (!(fabs(l1) > 0.0) || !isfinite(l1)) bad_pivot = true;
                PL(dl, 1, np) = l1; PL(dl, 2, np) = l2; PL(dl, 3, np) = l3; PL(dl, 4, np) = l4; PL(dl, 5, np) = l5;
                PL(du, 1, np) = u1; PL(du, 2, np) = u2; PL(du, 3, np) = u3; PL(du, 4, np) = u4;
                RING(c0, 0, j) = u1; RING(c0, 1, j) = u2; RING(c0, 2, j) = u3; RING(c0, 3, j) = u4;
            } else {
                double w1 = hw ? RING(c1, 0, j) : 0.0, w2 = hw ? RING(c1, 1, j) : 0.0;
                double w3 = hw ? RING(c1, 2, j) : 0.0;
                double s1 = hs ? RING(c2, 0, j - 1) : 0.0, s2 = hs ? RING(c2, 1, j - 1) : 0.0;
                double s3 = hs ? RING(c2, 2, j - 1) : 0.0;
                double se1 = hse ? RING(c1, 0, j - 1) : 0.0, se2 = hse ? RING(c1, 1, j - 1) : 0.0;
                double se3 = hse ? RING(c1, 2, j - 1) : 0.0;
                (void)hsw;
                const double b1 = PL(a, 1, np), b2 = PL(a, 2, np), b3 = PL(a, 3, np);
                const double b4 = PL(a, 4, np), b5 = PL(a, 5, np);
                double l4 = b1 / (1.0 - alpha * s1 * se1);
                double l3 = -l4 * s1;
                double l2 = (b2 - l4 * s2) / (1.0 + 2.0 * alpha * w2);
                double phi1 = l3 * se1, phi4 = l2 * w2;
                double l1 = b3 - l2 * w1 - l3 * se2 - l4 * s3 + 2.0 * alpha * (phi1 + phi4);
                double u1 = (b4 - l3 * se3 - 2.0 * alpha * phi1) / l1;
                double u2 = -l2 * w3 / l1;
                double u3 = (b5 - alpha * phi4) / l1;
                if (!(fabs(l1) > 0.0) || !isfinite(l1)) bad_pivot = true;
                PL(dl, 1, np) = l1; PL(dl, 2, np) = l2; PL(dl, 3, np) = l3; PL(dl, 4, np) = l4;
                PL(du, 1, np) = u1; PL(du, 2, np) = u2; PL(du, 3, np) = u3;
                RING(c0, 0, j) = u1; RING(c0, 1, j) = u2; RING(c0, 2, j) = u3;
            }
        }
        __syncthreads();
    }
    if (bad_pivot && L.err) atomicOr(L.err, ERR_NONFINITE_PIVOT);

    // ---- fb2d9 / fb2d5 (msi2d9-v03.f90:42-262, msi2d5-v03.f90:42-233)
    double rr0 = block_sum<ND>(residual<ND>(a, S.b, x, wk, nx, ny), red);
    const double gammarp = L.tol * sqrt(rr0);
    const int cap = (L.nitm > 0) ? L.nitm : kMaxIterUnbounded;
    int nit = 0;
    double rr = rr0;
    for (;;) {
        nit = nit + 1;
        // forward: L w = -r, w overwrites r in wk
        for (int s = 0; s < nsteps; s++) {
            const int c0 = s & 3, c1 = (s + 3) & 3, c2 = (s + 2) & 3, c3 = (s + 1) & 3;
            for (int j = threadIdx.x; j < ny; j += T) {
                const int i = s - 2 * j;
                if (i < 0 || i >= nx) continue;
                const long long np = (long long)j * nx + i;
                const bool hw = i > 0, hs = j > 0;
                const double ww = hw ? RING(c1, 0, j) : 0.0;
                const double wse = (hs && i < nx - 1) ? RING(c1, 0, j - 1) : 0.0;
                const double ws = hs ? RING(c2, 0, j - 1) : 0.0;
                double w;
                if (ND == 9) {
                    const double wsw = (hs && hw) ? RING(c3, 0, j - 1) : 0.0;
                    w = -(wk[np] + PL(dl, 2, np) * ww + PL(dl, 3, np) * wse + PL(dl, 4, np) * ws
                          + PL(dl, 5, np) * wsw) / PL(dl, 1, np);
                } else {
                    w = -(wk[np] + PL(dl, 2, np) * ww + PL(dl, 3, np) * wse + PL(dl, 4, np) * ws)
                        / PL(dl, 1, np);
                }
                wk[np] = w;
                RING(c0, 0, j) = w;
            }
            __syncthreads();
        }
        // backward: U z = w, var = z + var
        for (int s = 0; s < nsteps; s++) {
            const int c0 = s & 3, c1 = (s + 3) & 3, c2 = (s + 2) & 3, c3 = (s + 1) & 3;
            for (int j = threadIdx.x; j < ny; j += T) {
                const int i = nx - 1 - (s - 2 * (ny - 1 - j));
                if (i < 0 || i >= nx) continue;
                const long long np = (long long)j * nx + i;
                const bool he = i < nx - 1, hn = j < ny - 1;
                const double ze = he ? RING(c1, 0, j) : 0.0;
                const double znw = (hn && i > 0) ? RING(c1, 0, j + 1) : 0.0;
                const double zn = hn ? RING(c2, 0, j + 1) : 0.0;
                double z;
                if (ND == 9) {
                    const double zne = (hn && he) ? RING(c3, 0, j + 1) : 0.0;
                    z = wk[np] - PL(du, 1, np) * ze - PL(du, 2, np) * znw - PL(du, 3, np) * zn
                        - PL(du, 4, np) * zne;
                } else {
                    z = wk[np] - PL(du, 1, np) * ze - PL(du, 2, np) * znw - PL(du, 3, np) * zn;
                }
                x[np] = z + x[np];
                RING(c0, 0, j) = z;
            }
            __syncthreads();
        }
        rr = block_sum<ND>(residual<ND>(a, S.b, x, wk, nx, ny), red);
        if (sqrt(rr) < gammarp) break;
        if (nit == cap) {
            if (L.nitm <= 0 && L.err && threadIdx.x == 0) atomicOr(L.err, ERR_WAIT_TIMEOUT);
            break;
        }
    }
    if (threadIdx.x == 0) {
        if (S.nit) *S.nit = nit;
        if (S.rr) { S.rr[0] = rr0; S.rr[1] = rr; }
    }
}

static thread_local int g_msi_launches = 0;
void msi_note_launches(int n) { g_msi_launches = n; }
int msi_last_launch_count() { return g_msi_launches; }

cudaError_t launch_msi(int nd, const MsiLaunch &L, int nsys, cudaStream_t st)
{
    if (L.ny > msi_max_ny() || L.nx < 3 || L.ny < 3) return cudaErrorInvalidValue;
    if (L.variant == 3 && L.prec == 0) return launch_msi_generic(nd, L, nsys, st);
    if (msi_warp_supported(L.ny)) return launch_msi_warp(nd, L, nsys, st);
    return launch_msi_generic(nd, L, nsys, st);
}

cudaError_t launch_msi_generic(int nd, const MsiLaunch &L, int nsys, cudaStream_t st)
{
    if (L.ny > msi_max_ny() || L.nx < 3 || L.ny < 3) return cudaErrorInvalidValue;
    const int T = msi_block_threads(L.ny);
    const size_t sm = msi_smem_bytes(nd, L.ny);
    if (nd == 9) {
        cudaError_t e = cudaFuncSetAttribute(k_msi<9>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_msi<9><<<nsys, T, sm, st>>>(L);
    } else {
        cudaError_t e = cudaFuncSetAttribute(k_msi<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_msi<5><<<nsys, T, sm, st>>>(L);
    }
    msi_note_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// line TDMA (src/solvers/tdma2d9.f90:38-322, tdma2d5.f90:38-241).  Each phase
// is two launches: the recurrence for every line first, then every
// back-substitution, because the right-hand sides of a line read the old
// values of the neighbouring lines (the reference's separate loops).

// x lines: one thread per row j; P, Q over the row
template <int ND>
__global__ void k_tdma_xfwd(int nx, int ny, const double *__restrict__ a, const double *__restrict__ b,
                            const double *__restrict__ x, double *P, double *Q)
{
    const long long N = (long long)nx * ny;
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > ny) return;
    for (int i = 1; i <= nx; i++) {
        const long long np = (long long)(j - 1) * nx + (i - 1), nps = np - nx, npn = np + nx;
        double D;
        if (ND == 9) {
            if (j == 1) {
                D = b[np];
                if (i > 1) D = D - PL(a, 7, np) * x[npn - 1];
                D = D - PL(a, 8, np) * x[npn];
                if (i < nx) D = D - PL(a, 9, np) * x[npn + 1];
            } else if (j == ny) {
                D = b[np];
                if (i > 1) D = D - PL(a, 1, np) * x[nps - 1];
                D = D - PL(a, 2, np) * x[nps];
                if (i < nx) D = D - PL(a, 3, np) * x[nps + 1];
            } else {
                D = b[np];
                if (i > 1) D = D - PL(a, 1, np) * x[nps - 1];
                D = D - PL(a, 2, np) * x[nps];
                if (i < nx) D = D - PL(a, 3, np) * x[nps + 1];
                if (i > 1) D = D - PL(a, 7, np) * x[npn - 1];
                D = D - PL(a, 8, np) * x[npn];
                if (i < nx) D = D - PL(a, 9, np) * x[npn + 1];
            }
            if (i == 1) {
                P[np] = -PL(a, 6, np) / PL(a, 5, np);
                Q[np] = D / PL(a, 5, np);
            } else {
                P[np] = -PL(a, 6, np) / (PL(a, 5, np) + PL(a, 4, np) * P[np - 1]);
                Q[np] = (D - PL(a, 4, np) * Q[np - 1]) / (PL(a, 5, np) + PL(a, 4, np) * P[np - 1]);
            }
        } else {
            if (j == 1) D = b[np] - PL(a, 5, np) * x[npn];
            else if (j == ny) D = b[np] - PL(a, 1, np) * x[nps];
            else D = b[np] - PL(a, 5, np) * x[npn] - PL(a, 1, np) * x[nps];
            if (i == 1) {
                P[np] = -PL(a, 4, np) / PL(a, 3, np);
                Q[np] = D / PL(a, 3, np);
            } else {
                P[np] = -PL(a, 4, np) / (PL(a, 3, np) + PL(a, 2, np) * P[np - 1]);
                Q[np] = (D - PL(a, 2, np) * Q[np - 1]) / (PL(a, 3, np) + PL(a, 2, np) * P[np - 1]);
            }
        }
    }
}

__global__ void k_tdma_xback(int nx, int ny, const double *P, const double *Q, double *x)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > ny) return;
    long long np = (long long)(j - 1) * nx + (nx - 1);
    x[np] = Q[np];
    for (int i = nx - 1; i >= 1; i--) {
        np = (long long)(j - 1) * nx + (i - 1);
        x[np] = P[np] * x[np + 1] + Q[np];
    }
}

// y lines: one thread per column i, consecutive threads on consecutive columns
template <int ND>
__global__ void k_tdma_yfwd(int nx, int ny, const double *__restrict__ a, const double *__restrict__ b,
                            const double *__restrict__ x, double *P, double *Q)
{
    const long long N = (long long)nx * ny;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > nx) return;
    for (int j = 1; j <= ny; j++) {
        const long long np = (long long)(j - 1) * nx + (i - 1), nps = np - nx, npn = np + nx;
        double D;
        if (ND == 9) {
            const bool hs = j > 1, hn = j < ny;
            if (i == 1) {
                D = b[np];
                if (hs) D = D - PL(a, 3, np) * x[nps + 1];
                D = D - PL(a, 6, np) * x[np + 1];
                if (hn) D = D - PL(a, 9, np) * x[npn + 1];
            } else if (i == nx) {
                D = b[np];
                if (hs) D = D - PL(a, 1, np) * x[nps - 1];
                D = D - PL(a, 4, np) * x[np - 1];
                if (hn) D = D - PL(a, 7, np) * x[npn - 1];
            } else {
                D = b[np];
                if (hs) D = D - PL(a, 1, np) * x[nps - 1];
                D = D - PL(a, 4, np) * x[np - 1];
                if (hn) D = D - PL(a, 7, np) * x[npn - 1];
                if (hs) D = D - PL(a, 3, np) * x[nps + 1];
                D = D - PL(a, 6, np) * x[np + 1];
                if (hn) D = D - PL(a, 9, np) * x[npn + 1];
            }
            if (j == 1) {
                P[np] = -PL(a, 8, np) / PL(a, 5, np);
                Q[np] = D / PL(a, 5, np);
            } else {
                P[np] = -PL(a, 8, np) / (PL(a, 5, np) + PL(a, 2, np) * P[nps]);
                Q[np] = (D - PL(a, 2, np) * Q[nps]) / (PL(a, 5, np) + PL(a, 2, np) * P[nps]);
            }
        } else {
            if (i == 1) D = b[np] - PL(a, 4, np) * x[np + 1];
            else if (i == nx) D = b[np] - PL(a, 2, np) * x[np - 1];
            else D = b[np] - PL(a, 2, np) * x[np - 1] - PL(a, 4, np) * x[np + 1];
            if (j == 1) {
                P[np] = -PL(a, 5, np) / PL(a, 3, np);
                Q[np] = D / PL(a, 3, np);
            } else {
                P[np] = -PL(a, 5, np) / (PL(a, 3, np) + PL(a, 1, np) * P[nps]);
                Q[np] = (D - PL(a, 1, np) * Q[nps]) / (PL(a, 3, np) + PL(a, 1, np) * P[nps]);
            }
        }
    }
}

__global__ void k_tdma_yback(int nx, int ny, const double *P, const double *Q, double *x)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > nx) return;
    long long np = (long long)(ny - 1) * nx + (i - 1);
    x[np] = Q[np];
    for (int j = ny - 1; j >= 1; j--) {
        np = (long long)(j - 1) * nx + (i - 1);
        x[np] = x[np + nx] * P[np] + Q[np];
    }
}

cudaError_t launch_tdma(int nd, int nx, int ny, int nitm, const double *a, const double *b,
                        double *x, double *P, double *Q, cudaStream_t st)
{
    const int tb = 64;
    for (int it = 0; it < nitm; it++) {
        if (nd == 9) k_tdma_xfwd<9><<<(ny + tb - 1) / tb, tb, 0, st>>>(nx, ny, a, b, x, P, Q);
        else k_tdma_xfwd<5><<<(ny + tb - 1) / tb, tb, 0, st>>>(nx, ny, a, b, x, P, Q);
        k_tdma_xback<<<(ny + tb - 1) / tb, tb, 0, st>>>(nx, ny, P, Q, x);
        if (nd == 9) k_tdma_yfwd<9><<<(nx + tb - 1) / tb, tb, 0, st>>>(nx, ny, a, b, x, P, Q);
        else k_tdma_yfwd<5><<<(nx + tb - 1) / tb, tb, 0, st>>>(nx, ny, a, b, x, P, Q);
        k_tdma_yback<<<(nx + tb - 1) / tb, tb, 0, st>>>(nx, ny, P, Q, x);
    }
    return cudaGetLastError();
}

// independent lines: P = -ae/(ap + aw P_w), Q = (d - aw Q_w)/(ap + aw P_w)
__global__ void k_tdma_lines(int n, int nlines, const double *__restrict__ aw, const double *__restrict__ ap,
                             const double *__restrict__ ae, const double *__restrict__ d, double *x,
                             double *P, double *Q)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const long long o = (long long)l * n;
    double p = -ae[o] / ap[o], q = d[o] / ap[o];
    P[o] = p; Q[o] = q;
    for (int i = 1; i < n; i++) {
        const long long k = o + i;
        const double den = ap[k] + aw[k] * p;
        const double pn = -ae[k] / den;
        q = (d[k] - aw[k] * q) / den;
        p = pn;
        P[k] = p; Q[k] = q;
    }
    double xv = Q[o + n - 1];
    x[o + n - 1] = xv;
    for (int i = n - 2; i >= 0; i--) {
        xv = P[o + i] * xv + Q[o + i];
        x[o + i] = xv;
    }
}

cudaError_t launch_tdma_lines(int n, int nlines, const double *aw, const double *ap,
                              const double *ae, const double *d, double *x, double *P,
                              double *Q, cudaStream_t st)
{
    k_tdma_lines<<<(nlines + 63) / 64, 64, 0, st>>>(n, nlines, aw, ap, ae, d, x, P, Q);
    return cudaGetLastError();
}

// Parallel cyclic reduction, one CTA per line, the line's four coefficient
// arrays in shared memory (ping-pong between two copies).  With the line
// written aw_i x_{i-1} + ap_i x_i + ae_i x_{i+1} = d_i, a step of stride s
// eliminates x_{i-s} and x_{i+s} from row i with rows i-s and i+s:
//   k1 = aw_i / ap_{i-s},  k2 = ae_i / ap_{i+s}   (0 past the line's ends)
//   aw'_i = -aw_{i-s} k1,  ae'_i = -ae_{i+s} k2
//   ap'_i = ap_i - ae_{i-s} k1 - aw_{i+s} k2
//   d'_i  = d_i - d_{i-s} k1 - d_{i+s} k2
// so after ceil(log2 n) steps every row holds one unknown: x_i = d_i / ap_i
// (Hockney's cyclic reduction in its parallel form).  Global loads and
// stores are whole coalesced lines.  The rounding differs from the
// sequential Thomas algorithm (k_tdma_lines); for diagonally dominant lines
// the two agree to about 1e-15 relative.
constexpr int kPcrThreads = 256;
constexpr int kPcrMaxN = 2048;

__global__ void __launch_bounds__(kPcrThreads) k_tdma_lines_pcr(int n, int nlines, const double *__restrict__ aw,
                                                                const double *__restrict__ ap,
                                                                const double *__restrict__ ae,
                                                                const double *__restrict__ d, double *x)
{
    extern __shared__ double pcr[];   // 2 copies x {aw, ap, ae, d} x n
    const int l = blockIdx.x;
    if (l >= nlines) return;
    const long long o = (long long)l * n;
    double *A0 = pcr, *B0 = A0 + n, *C0 = B0 + n, *D0 = C0 + n;
    double *A1 = D0 + n, *B1 = A1 + n, *C1 = B1 + n, *D1 = C1 + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        A0[i] = aw[o + i]; B0[i] = ap[o + i]; C0[i] = ae[o + i]; D0[i] = d[o + i];
    }
    __syncthreads();
    for (int sft = 1; sft < n; sft <<= 1) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int im = i - sft, ip = i + sft;
            const double k1 = im >= 0 ? A0[i] / B0[im] : 0.0;
            const double k2 = ip < n ? C0[i] / B0[ip] : 0.0;
            const double am = im >= 0 ? A0[im] : 0.0, cm = im >= 0 ? C0[im] : 0.0, dm = im >= 0 ? D0[im] : 0.0;
            const double ap_ = ip < n ? A0[ip] : 0.0, cp = ip < n ? C0[ip] : 0.0, dp = ip < n ? D0[ip] : 0.0;
            A1[i] = -am * k1;
            C1[i] = -cp * k2;
            B1[i] = B0[i] - cm * k1 - ap_ * k2;
            D1[i] = D0[i] - dm * k1 - dp * k2;
        }
        __syncthreads();
        double *t;
        t = A0; A0 = A1; A1 = t;
        t = B0; B0 = B1; B1 = t;
        t = C0; C0 = C1; C1 = t;
        t = D0; D0 = D1; D1 = t;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[o + i] = D0[i] / B0[i];
}

bool tdma_lines_pcr_supported(int n) { return n >= 1 && n <= kPcrMaxN; }

cudaError_t launch_tdma_lines_pcr(int n, int nlines, const double *aw, const double *ap, const double *ae,
                                  const double *d, double *x, cudaStream_t st)
{
    if (!tdma_lines_pcr_supported(n) || nlines < 1) return cudaErrorInvalidValue;
    const size_t smem = (size_t)8 * n * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_tdma_lines_pcr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_tdma_lines_pcr<<<nlines, kPcrThreads, smem, st>>>(n, nlines, aw, ap, ae, d, x);
    return cudaGetLastError();
}

}  // namespace m2d
