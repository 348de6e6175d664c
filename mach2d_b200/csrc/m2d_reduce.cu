// m2d_reduce.cu -- FP64 reductions of the SIMPLEC iteration.
//
// Two passes with a fixed schedule (kParts blocks x 256 threads, fixed
// per-thread stride, fixed shared-memory tree), so every result is bitwise
// reproducible from run to run.  The reference sums sequentially; a tree sum
// differs from it only in rounding (relative 1e-15 level).  Sums, max and min
// all stay in FP64 on the GPU: the linear-system residual norms, the mass
// imbalance and the outer convergence norm.
#include "m2d_fields.cuh"

namespace m2d {

static const int kParts = 296;     // 2 x 148 SMs
static const int kThreads = 256;
// per-block partials, then one word for the count of finished blocks
int red_parts() { return kParts + 1; }

#define A9(a, np, k) (a)[(long long)((k) - 1) * N + (np)]

enum Combine { C_SUM, C_MAX, C_MIN };

__device__ __forceinline__ int combine_of(int kind)
{
    if (kind == RED_MAXABS_ALL) return C_MAX;
    if (kind == RED_DT0) return C_MIN;
    return C_SUM;
}

__device__ __forceinline__ double comb(int c, double a, double b)
{
    if (c == C_SUM) return a + b;
    if (c == C_MAX) return fmax(a, b);
    return (a > b) ? b : a;   // tstepper_dt0_scarborough: if (dt > aux) dt = aux
}

__device__ __forceinline__ double ident(int c)
{
    if (c == C_SUM) return 0.0;
    if (c == C_MAX) return 0.0;
    return 1.0e10;
}

// value of one real cell (i,j) for the cell-wise kinds
__device__ __forceinline__ double cell_value(const RedArgs &r, int i, int j)
{
    const int nx = r.nx;
    const long long N = (long long)r.nx * r.ny;
    const long long np = (long long)(j - 1) * nx + (i - 1);
    switch (r.kind) {
    case RED_SUM_REAL: return r.x[np];
    case RED_NORM_L1_9D: {
        const double *a = r.a, *x = r.x;
        const long long nps = np - nx, npn = np + nx;
        return fabs(+A9(a, np, 1) * x[nps - 1] + A9(a, np, 2) * x[nps] + A9(a, np, 3) * x[nps + 1]
                    + A9(a, np, 4) * x[np - 1] + A9(a, np, 5) * x[np] + A9(a, np, 6) * x[np + 1]
                    + A9(a, np, 7) * x[npn - 1] + A9(a, np, 8) * x[npn] + A9(a, np, 9) * x[npn + 1]
                    - r.b[np]);
    }
    case RED_NORM_L1_5D: {
        const double *a = r.a, *x = r.x;
        return fabs(+A9(a, np, 1) * x[np - nx] + A9(a, np, 2) * x[np - 1] + A9(a, np, 3) * x[np]
                    + A9(a, np, 4) * x[np + 1] + A9(a, np, 5) * x[np + nx] - r.b[np]);
    }
    case RED_SUM_ABS_B: return fabs(r.b[np]);
    case RED_MASS: {
        const long long nps = np - nx, npw = np - 1;
        double fme = r.roe[np] * r.re[np] * r.Uce[np];
        double fmw = r.roe[npw] * r.re[npw] * r.Uce[npw];
        double fmn = r.ron[np] * r.rn[np] * r.Vcn[np];
        double fms = r.ron[nps] * r.rn[nps] * r.Vcn[nps];
        return fabs((r.ro[np] - r.roa[np]) * r.rp[np] / (r.Jp[np] * (r.dtp ? *r.dtp : r.dt)) + fme - fmw + fmn - fms);
    }
    case RED_MEAN_CC_9D: {
        const double *a = r.a;
        double s1 = 0.0, s2 = 0.0;
        for (int k = 1; k <= 4; k++) s1 = s1 + fabs(A9(a, np, k));
        for (int k = 6; k <= 9; k++) s2 = s2 + fabs(A9(a, np, k));
        return (s1 + s2) / fabs(A9(a, np, 5));
    }
    case RED_MEAN_CC_5D: {
        const double *a = r.a;
        double s1 = fabs(A9(a, np, 1)) + fabs(A9(a, np, 2));
        double s2 = fabs(A9(a, np, 4)) + fabs(A9(a, np, 5));
        return (s1 + s2) / fabs(A9(a, np, 3));
    }
    case RED_DT0: {
        double uu = r.u[np], vv = r.v[np];
        return 1.0 / sqrt(r.Jp[np] * (uu * uu + vv * vv));
    }
    }
    return 0.0;
}

__device__ __forceinline__ double block_reduce(double v, int c)
{
    __shared__ double sh[kThreads];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = comb(c, sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    return sh[0];
}

// One launch: every block reduces its share into part[block]; the last
// block to finish (a counter in part[kParts], back to zero afterwards)
// combines the kParts partials in index order with the same tree, so the
// result does not depend on which block finishes last.
__device__ __forceinline__ void reduce_one(const RedArgs &r, double *part, double *out)
{
    const int c = combine_of(r.kind);
    double acc = ident(c);
    if (r.kind == RED_MAXABS_ALL) {
        const long long N = (long long)r.nx * r.ny;
        for (long long k = blockIdx.x * (long long)kThreads + threadIdx.x; k < N; k += (long long)kParts * kThreads)
            acc = fmax(acc, fabs(r.x[k]));
    } else {
        const int ni = r.nx - 2;
        const long long nr = (long long)(r.nx - 2) * (r.ny - 2);
        for (long long k = blockIdx.x * (long long)kThreads + threadIdx.x; k < nr; k += (long long)kParts * kThreads) {
            int i = (int)(k % ni) + 2, j = (int)(k / ni) + 2;
            acc = comb(c, acc, cell_value(r, i, j));
        }
    }
    double s = block_reduce(acc, c);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(reinterpret_cast<unsigned *>(part + kParts), 1u) == (unsigned)(kParts - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    acc = ident(c);
    for (int k = threadIdx.x; k < kParts; k += kThreads) acc = comb(c, acc, __ldcg(part + k));
    s = block_reduce(acc, c);
    if (threadIdx.x == 0) {
        if (r.kind == RED_MEAN_CC_9D || r.kind == RED_MEAN_CC_5D) s = s / (double)((r.nx - 2) * (r.ny - 2));
        if (r.kind == RED_DT0) s = s * 0.25;
        *out = s;
        *reinterpret_cast<unsigned *>(part + kParts) = 0u;
    }
}

__global__ void __launch_bounds__(kThreads) k_reduce(RedArgs r, double *part, double *out)
{
    reduce_one(r, part, out);
}

cudaError_t launch_reduce(const RedArgs &r, double *part, double *out, cudaStream_t st)
{
    k_reduce<<<kParts, kThreads, 0, st>>>(r, part, out);
    return cudaGetLastError();
}

// up to kMaxMultiReduce independent reductions in one launch: blockIdx.y
// picks one, which runs exactly as k_reduce would (same shares, trees and
// final combine, its own partials), so each result is bitwise that of its
// own launch
struct RedMulti {
    RedArgs r[kMaxMultiReduce];
    double *out[kMaxMultiReduce];
};
__global__ void __launch_bounds__(kThreads) k_reduce_multi(RedMulti m, double *part)
{
    const int y = blockIdx.y;
    reduce_one(m.r[y], part + (long long)y * (kParts + 1), m.out[y]);
}

cudaError_t launch_reduce_multi(const RedArgs *r, double *const *out, int n, double *part, cudaStream_t st)
{
    if (n < 1 || n > kMaxMultiReduce) return cudaErrorInvalidValue;
    RedMulti m;
    for (int k = 0; k < n; k++) {
        m.r[k] = r[k];
        m.out[k] = out[k];
    }
    k_reduce_multi<<<dim3(kParts, (unsigned)n), kThreads, 0, st>>>(m, part);
    return cudaGetLastError();
}

// get_mass_flow_rate_and_thrust  src/user/internal_flow/mod_intflow.f90:1591-1643
__global__ void k_mass_flow_thrust(Fields f, double *out)
{
    const int nx = f.nx, ny = f.ny;
    double fi = 0.0, fe = 0.0, fd = 0.0;
    for (int j = 2 + threadIdx.x; j <= ny - 1; j += blockDim.x) {
        long long np = (long long)(j - 1) * nx;                   // i = 1
        fi = fi + f.re[np] * f.roe[np] * f.Uce[np];
        long long ne = (long long)(j - 1) * nx + (nx - 2);        // i = nx-1
        double m = f.re[ne] * f.roe[ne] * f.Uce[ne];
        fe = fe + m;
        fd = fd + f.re[ne] * f.roe[ne] * f.Uce[ne] * (f.u[ne] + f.u[ne + 1]) / 2.0;
    }
    __shared__ double sh[3][kThreads];
    sh[0][threadIdx.x] = fi; sh[1][threadIdx.x] = fe; sh[2][threadIdx.x] = fd;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 3; q++) sh[q][threadIdx.x] = sh[q][threadIdx.x] + sh[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double pi = 3.141592653589793;
        out[0] = sh[0][0] * 2.0 * pi;
        out[1] = sh[1][0] * 2.0 * pi;
        out[2] = sh[2][0] * 2.0 * pi;
    }
}

cudaError_t launch_mass_flow_thrust(const Fields &f, double *out, cudaStream_t st)
{
    k_mass_flow_thrust<<<1, kThreads, 0, st>>>(f, out);
    return cudaGetLastError();
}

}  // namespace m2d
