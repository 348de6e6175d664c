// m2d_krylov.cu -- flexible GMRES around the MSI preconditioner and the
// learned p' correction.  No counterpart in the reference: MACH-2D iterates
// MSI as a stationary method (fb2d9 / fb2d5, src/solvers/msi2d9-v03.f90:
// 42-262).  This solver keeps MSI's incomplete factorisation (lu2d9 /
// lu2d5, computed once per solve, as the reference computes it once per
// call) and uses it as the right preconditioner of Saad's flexible GMRES
// (SIAM J. Sci. Comput. 14, 1993), so the Krylov space replaces the fixed
// point iteration x += (LU)^-1 (b - A x).  The preconditioner may change
// from one Krylov step to the next, which lets the learned correction (a
// nonlinear map) act as a preconditioner too: z = N(v), then one MSI step
// from it, z += (LU)^-1 (v - A z).
//
// Device work per step: one MSI application (the cluster kernel with
// reused factors: forward and backward sweeps only), one product A z, two
// passes of classical Gram-Schmidt (h = V^T w in one launch, w -= V h in
// another, done twice for orthogonality), a norm.  The FP64 dot products use
// a fixed per-block order and a fixed final order, so a solve is bitwise
// reproducible.  The small Hessenberg least-squares problem (Givens
// rotations) lives on the host.
#include <cmath>
#include <cstring>
#include <vector>
#include "m2d_solvers.cuh"
#include "../../include/mach2d_b200.h"

void m2d_set_last_error_msg(const char *);

namespace m2d {
// the learned correction x_out = x + N(b - A x) (m2d_unet.cu), no acceptance test
cudaError_t unet_correct(m2d_unet *n, int nx, int ny, const double *d_a, const double *d_b, const double *d_x,
                         double *d_xout, const double *d_Jp, cudaStream_t st);
}

using namespace m2d;

namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 296;          // 2 per SM
constexpr int kMaxRestart = 32;       // accumulators per thread in the multi-dot

#define PLK(a, k, np) (a)[(long long)(k) * N + (np)]

// r = b - A x (sign 1) or w = A x (sign 0, b unused), every cell; couplings
// to cells outside the grid are dropped, as in the MSI residual
template <int ND>
__global__ void k_apply_a(int nx, int ny, const double *__restrict__ a, const double *__restrict__ b,
                          const double *__restrict__ x, double *y, int residual)
{
    const long long N = (long long)nx * ny;
    for (long long np = blockIdx.x * (long long)blockDim.x + threadIdx.x; np < N;
         np += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(np / nx), i = (int)(np - (long long)j * nx);
        const bool w = i > 0, e = i < nx - 1, s = j > 0, n = j < ny - 1;
        double v = 0.0;
        if (ND == 9) {
            if (s && w) v = v + PLK(a, 0, np) * x[np - nx - 1];
            if (s) v = v + PLK(a, 1, np) * x[np - nx];
            if (s && e) v = v + PLK(a, 2, np) * x[np - nx + 1];
            if (w) v = v + PLK(a, 3, np) * x[np - 1];
            v = v + PLK(a, 4, np) * x[np];
            if (e) v = v + PLK(a, 5, np) * x[np + 1];
            if (n && w) v = v + PLK(a, 6, np) * x[np + nx - 1];
            if (n) v = v + PLK(a, 7, np) * x[np + nx];
            if (n && e) v = v + PLK(a, 8, np) * x[np + nx + 1];
        } else {
            if (s) v = v + PLK(a, 0, np) * x[np - nx];
            if (w) v = v + PLK(a, 1, np) * x[np - 1];
            v = v + PLK(a, 2, np) * x[np];
            if (e) v = v + PLK(a, 3, np) * x[np + 1];
            if (n) v = v + PLK(a, 4, np) * x[np + nx];
        }
        y[np] = residual ? b[np] - v : v;
    }
}

// part[i * kBlocks + block] = this block's share of sum_c V_i[c] w[c] over
// c < N, i < k (k <= kMaxRestart, rows of V ld doubles apart); each block
// takes a contiguous slice of cells
__global__ void __launch_bounds__(kThreads) k_multidot(int k, long long N, long long ld, const double *__restrict__ V,
                                                       const double *__restrict__ w, double *part)
{
    double acc[kMaxRestart];
#pragma unroll
    for (int i = 0; i < kMaxRestart; i++) acc[i] = 0.0;
    const long long per = (N + gridDim.x - 1) / gridDim.x;
    const long long lo = per * blockIdx.x, hi = lo + per < N ? lo + per : N;
    for (long long c = lo + threadIdx.x; c < hi; c += kThreads) {
        const double wc = w[c];
#pragma unroll
        for (int i = 0; i < kMaxRestart; i++)
            if (i < k) acc[i] = acc[i] + V[(long long)i * ld + c] * wc;
    }
    __shared__ double red[kThreads / 32][kMaxRestart];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < kMaxRestart; i++) {
        if (i >= k) break;
        double v = acc[i];
        for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[wp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double v = 0.0;
        for (int q = 0; q < kThreads / 32; q++) v = v + red[q][threadIdx.x];
        part[(long long)threadIdx.x * kBlocks + blockIdx.x] = v;
    }
}

// out[i] = sum over blocks of part[i][*] in block order
__global__ void k_multidot_finish(int k, const double *part, double *out)
{
    const int i = threadIdx.x;
    if (i >= k) return;
    double v = 0.0;
    for (int b = 0; b < kBlocks; b++) v = v + part[(long long)i * kBlocks + b];
    out[i] = v;
}

// y += sign * sum_{i < k} h[i] X_i over c < N (rows of X ld apart, h in
// device memory)
__global__ void k_multi_axpy(int k, long long N, long long ld, const double *__restrict__ X,
                             const double *__restrict__ h, double sign, double *y)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x) {
        double v = y[c];
        for (int i = 0; i < k; i++) v = v + sign * h[i] * X[(long long)i * ld + c];
        y[c] = v;
    }
}

__global__ void k_scale_copy(long long N, const double *__restrict__ x, const double *s, double *y)
{
    const double f = 1.0 / *s;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x)
        y[c] = x[c] * f;
}

int fail(int code, const char *msg)
{
    m2d_set_last_error_msg(msg);
    return code;
}

struct Layout {
    long long N;
    double *V, *Z, *w, *t, *ws, *part, *h;
    size_t ws_doubles;
};

size_t align32(size_t n) { return (n + 31) / 32 * 32; }

Layout layout(int nd, int nx, int ny, int m, double *base)
{
    Layout L;
    L.N = (long long)nx * ny;
    const size_t Na = align32((size_t)L.N);
    double *p = base;
    L.V = p; p += (size_t)(m + 1) * Na;
    L.Z = p; p += (size_t)m * Na;
    L.w = p; p += Na;
    L.t = p; p += Na;
    L.ws_doubles = align32(msi_work_doubles(nd, nx, ny) + 4);
    L.ws = p; p += L.ws_doubles;
    L.part = p; p += align32((size_t)kMaxRestart * kBlocks);
    L.h = p; p += align32(2 * kMaxRestart + 8);
    return L;
}

size_t workspace_doubles(int nd, int nx, int ny, int m)
{
    const size_t Na = align32((size_t)nx * ny);
    return (size_t)(2 * m + 3) * Na + align32(msi_work_doubles(nd, nx, ny) + 4) + align32((size_t)kMaxRestart * kBlocks)
           + align32(2 * kMaxRestart + 8);
}

}  // namespace

extern "C" long m2d_fgmres_workspace_doubles(int nd, int nx, int ny, int restart)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4 || restart < 1 || restart > kMaxRestart) return -1;
    return (long)workspace_doubles(nd, nx, ny, restart);
}

extern "C" int m2d_fgmres_solve(int nd, int nx, int ny, int restart, int maxit, double tol, const double *d_a,
                                const double *d_b, double *d_x, int prec, m2d_unet *net, const double *d_Jp,
                                double *d_work, void *stream, m2d_fgmres_report *rep)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4 || restart < 1 || restart > kMaxRestart || maxit < 1 ||
        !(tol > 0.0) || !d_a || !d_b || !d_x || !d_work || prec < 0 || prec > 2)
        return fail(M2D_ERR_ARG, "m2d_fgmres_solve: bad arguments");
    if (prec == 2 && (nd != 5 || !net || !d_Jp))
        return fail(M2D_ERR_ARG, "m2d_fgmres_solve: the learned preconditioner needs nd = 5, a network and Jp");
    if (ny > msi_max_ny()) return fail(M2D_ERR_TOO_LARGE, "m2d_fgmres_solve: ny exceeds m2d_msi_max_ny()");
    if (((uintptr_t)d_work) % 16) return fail(M2D_ERR_ARG, "m2d_fgmres_solve: d_work must be 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    const int m = restart;
    Layout W = layout(nd, nx, ny, m, d_work);
    const long long N = W.N;
    const size_t Na = align32((size_t)N);
    const unsigned g = (unsigned)((N + kThreads - 1) / kThreads < 1184 ? (N + kThreads - 1) / kThreads : 1184);
    cudaError_t e = cudaSuccess;
    int msi_apps = 0, net_apps = 0, total = 0, restarts = 0;
    bool factored = false, converged = false;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gv(m + 1), hcol(m + 2);
    double bnorm = 0.0, resid = 0.0;

    auto apply_a = [&](const double *x, double *y, const double *b, int residual) {
        if (nd == 9) k_apply_a<9><<<g, kThreads, 0, st>>>(nx, ny, d_a, b, x, y, residual);
        else k_apply_a<5><<<g, kThreads, 0, st>>>(nx, ny, d_a, b, x, y, residual);
    };
    // dots of the first k rows of X with y into W.h[0..k), copied to host
    auto dots = [&](int k, const double *X, const double *y, double *host) -> cudaError_t {
        k_multidot<<<kBlocks, kThreads, 0, st>>>(k, N, (long long)Na, X, y, W.part);
        k_multidot_finish<<<1, kMaxRestart, 0, st>>>(k, W.part, W.h);
        cudaError_t ee = cudaMemcpyAsync(host, W.h, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (ee == cudaSuccess) ee = cudaStreamSynchronize(st);
        return ee;
    };
    // one application of the factors: y = (LU)^-1 rhs, y zeroed here; the
    // first call of a solve also factorises (and runs the full iteration
    // step, which from y = 0 gives the same y)
    auto apply_factors = [&](const double *rhs, double *y) -> cudaError_t {
        cudaError_t ee = cudaMemsetAsync(y, 0, (size_t)N * sizeof(double), st);
        if (ee != cudaSuccess) return ee;
        MsiLaunch L;
        memset(&L, 0, sizeof L);
        L.nx = nx; L.ny = ny; L.nitm = 1; L.tol = 0.0;
        L.prec = (prec >= 1) ? 1 : 0;
        L.reuse_lu = factored ? 1 : 0;
        L.apply_only = factored ? 1 : 0;
        L.s[0].a = d_a; L.s[0].b = rhs; L.s[0].x = y;
        L.s[0].ws = W.ws;
        L.s[0].rr = W.ws + (W.ws_doubles - 4);
        L.ws_cap = W.ws_doubles - 4;
        ee = launch_msi(nd, L, 1, st);
        factored = true;
        msi_apps++;
        return ee;
    };
    // the preconditioner: z = P(v)
    auto precondition = [&](const double *v, double *z) -> cudaError_t {
        if (prec != 2) return apply_factors(v, z);
        // z = N(v) from the zero guess, then z += (LU)^-1 (v - A z)
        cudaError_t ee = cudaMemsetAsync(W.w, 0, (size_t)N * sizeof(double), st);
        if (ee == cudaSuccess) ee = unet_correct(net, nx, ny, d_a, v, W.w, z, d_Jp, st);
        if (ee != cudaSuccess) return ee;
        net_apps++;
        apply_a(z, W.t, v, 1);
        ee = apply_factors(W.t, W.w);
        if (ee != cudaSuccess) return ee;
        const double one = 1.0;
        ee = cudaMemcpyAsync(W.h + 2 * kMaxRestart, &one, sizeof(double), cudaMemcpyHostToDevice, st);
        if (ee != cudaSuccess) return ee;
        k_multi_axpy<<<g, kThreads, 0, st>>>(1, N, (long long)Na, W.w, W.h + 2 * kMaxRestart, 1.0, z);
        return cudaGetLastError();
    };

    e = cudaSuccess;
    {
        // |b|
        double hb = 0.0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(W.w, d_b, (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = dots(1, W.w, W.w, &hb);
        bnorm = std::sqrt(hb);
    }
    while (e == cudaSuccess && !converged && total < maxit) {
        // r = b - A x into V_0, beta = |r|
        apply_a(d_x, W.V, d_b, 1);
        double hb = 0.0;
        e = dots(1, W.V, W.V, &hb);
        if (e != cudaSuccess) break;
        const double beta = std::sqrt(hb);
        resid = beta;
        if (!(beta > tol * bnorm)) { converged = std::isfinite(beta); break; }
        e = cudaMemcpyAsync(W.h, &beta, sizeof(double), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) break;
        k_scale_copy<<<g, kThreads, 0, st>>>(N, W.V, W.h, W.V);
        std::fill(gv.begin(), gv.end(), 0.0);
        gv[0] = beta;
        int jdone = 0;
        for (int j = 0; j < m && total < maxit; j++) {
            double *Vj = W.V + (size_t)j * Na, *Zj = W.Z + (size_t)j * Na, *Vn = W.V + (size_t)(j + 1) * Na;
            e = precondition(Vj, Zj);
            if (e != cudaSuccess) break;
            apply_a(Zj, W.w, nullptr, 0);
            // classical Gram-Schmidt, twice
            std::fill(hcol.begin(), hcol.end(), 0.0);
            for (int pass = 0; pass < 2 && e == cudaSuccess; pass++) {
                std::vector<double> hp(j + 1);
                e = dots(j + 1, W.V, W.w, hp.data());
                if (e != cudaSuccess) break;
                e = cudaMemcpyAsync(W.h, hp.data(), (size_t)(j + 1) * sizeof(double), cudaMemcpyHostToDevice, st);
                if (e != cudaSuccess) break;
                k_multi_axpy<<<g, kThreads, 0, st>>>(j + 1, N, (long long)Na, W.V, W.h, -1.0, W.w);
                for (int i = 0; i <= j; i++) hcol[i] += hp[i];
            }
            if (e != cudaSuccess) break;
            double hw = 0.0;
            e = dots(1, W.w, W.w, &hw);
            if (e != cudaSuccess) break;
            hcol[j + 1] = std::sqrt(hw);
            e = cudaMemcpyAsync(W.h, &hcol[j + 1], sizeof(double), cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) break;
            k_scale_copy<<<g, kThreads, 0, st>>>(N, W.w, W.h, Vn);
            // Givens rotations on the new column
            for (int i = 0; i < j; i++) {
                const double t = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
                hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
                hcol[i] = t;
            }
            const double den = std::hypot(hcol[j], hcol[j + 1]);
            cs[j] = den > 0.0 ? hcol[j] / den : 1.0;
            sn[j] = den > 0.0 ? hcol[j + 1] / den : 0.0;
            hcol[j] = den;
            hcol[j + 1] = 0.0;
            gv[j + 1] = -sn[j] * gv[j];
            gv[j] = cs[j] * gv[j];
            for (int i = 0; i <= j; i++) H[(size_t)i * m + j] = hcol[i];
            total++;
            jdone = j + 1;
            resid = std::fabs(gv[j + 1]);
            if (!std::isfinite(resid)) { e = cudaErrorUnknown; break; }
            if (resid <= tol * bnorm) break;
        }
        if (e != cudaSuccess || jdone == 0) break;
        // y = H^-1 g, x += Z y
        std::vector<double> y(jdone);
        for (int i = jdone - 1; i >= 0; i--) {
            double s = gv[i];
            for (int k = i + 1; k < jdone; k++) s -= H[(size_t)i * m + k] * y[k];
            y[i] = s / H[(size_t)i * m + i];
        }
        e = cudaMemcpyAsync(W.h, y.data(), (size_t)jdone * sizeof(double), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) break;
        k_multi_axpy<<<g, kThreads, 0, st>>>(jdone, N, (long long)Na, W.Z, W.h, 1.0, d_x);
        restarts++;
        if (resid <= tol * bnorm) converged = true;
    }
    if (e == cudaErrorUnknown) return fail(M2D_ERR_NAN, "m2d_fgmres_solve: non-finite residual");
    if (e != cudaSuccess) {
        m2d_set_last_error(e, "m2d_fgmres_solve", __FILE__, __LINE__);
        return M2D_ERR_CUDA;
    }
    // the true residual of the result
    double rr = 0.0;
    apply_a(d_x, W.w, d_b, 1);
    e = dots(1, W.w, W.w, &rr);
    if (e != cudaSuccess) {
        m2d_set_last_error(e, "m2d_fgmres_solve", __FILE__, __LINE__);
        return M2D_ERR_CUDA;
    }
    if (rep) {
        rep->iterations = total;
        rep->msi_applications = msi_apps;
        rep->learned_applications = net_apps;
        rep->cycles = restarts;
        rep->converged = converged ? 1 : 0;
        rep->rel_residual = bnorm > 0.0 ? std::sqrt(rr) / bnorm : std::sqrt(rr);
    }
    return converged ? M2D_OK : M2D_ERR_TIMEOUT;
}
