// m2d_blomax.cu -- Baldwin-Lomax eddy viscosity (src/equations/blomax.f90).
//
// One warp per eta line (column i).  The reference walks each line from the
// north wall (j = ny-1) down to j = 2 with per-line arrays; here every lane
// evaluates the same per-cell expressions for its cells, and the line-wide
// operations become warp reductions: maxval (order-free), maxloc (first
// index of the maximum), and the first sign change of nu_outer - nu_inner
// (smallest index whose predicate holds).  Each per-cell value is computed
// with the reference's expression and operand order, so the result equals
// the sequential loop except where exp() differs from the host's libm.
#include "m2d_common.cuh"
#include "m2d_blomax.cuh"

namespace m2d {

namespace {
constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;
}

#define IDX(i, j) ((long long)nx * ((j) - 1) + (i) - 1)

struct BlCell {           // per-cell quantities of one eta line, m = 0 at the wall
    double yplus, omgplus, lmp;
};

__device__ __forceinline__ double bl_omega(int nx, const double *x, const double *y, const double *Jp,
                                           const double *u, const double *v, int i, int j)
{   // blomax.f90:83-148
    const long long np = IDX(i, j), nps = np - nx, npw = np - 1, npsw = nps - 1, npn = np + nx, npe = np + 1;
    const double xkp = 0.5 * (x[np] + x[nps] - x[npw] - x[npsw]);
    const double ykp = 0.5 * (y[np] + y[nps] - y[npw] - y[npsw]);
    const double xep = 0.5 * (x[np] + x[npw] - x[nps] - x[npsw]);
    const double yep = 0.5 * (y[np] + y[npw] - y[nps] - y[npsw]);
    return 0.5 * Jp[np] * fabs((v[npe] - v[npw]) * yep - (v[npn] - v[nps]) * ykp
                               + (u[npe] - u[npw]) * xep - (u[npn] - u[nps]) * xkp);
}

// warp argmax, ties to the smaller index (Fortran maxloc)
__device__ __forceinline__ void warp_argmax(double &val, int &idx)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(kFull, val, o);
        const int oi = __shfl_xor_sync(kFull, idx, o);
        if (ov > val || (ov == val && oi < idx) || (idx < 0 && oi >= 0)) { val = ov; idx = oi; }
    }
}
__device__ __forceinline__ double warp_max(double v, bool &have)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(kFull, v, o);
        const bool oh = __shfl_xor_sync(kFull, (int)have, o);
        if (oh && (!have || ov > v)) v = ov;
        have = have || oh;
    }
    return v;
}

__global__ void k_blomax(int nx, int ny, BlConst c, const double *__restrict__ x, const double *__restrict__ y,
                         const double *__restrict__ xp, const double *__restrict__ yp,
                         const double *__restrict__ xk, const double *__restrict__ yk,
                         const double *__restrict__ Jp, const double *__restrict__ Jn,
                         const double *__restrict__ vln, const double *__restrict__ ro,
                         const double *__restrict__ ron, const double *__restrict__ u,
                         const double *__restrict__ v, double *__restrict__ vtp)
{
    const int lane = threadIdx.x & 31;
    const int i = 2 + (int)blockIdx.x * kWarpsPerBlock + (int)(threadIdx.x >> 5);
    if (i > nx - 1) return;                       // whole warp leaves together
    const int n = ny - 2;
    // wall quantities at the north face of (i, ny-1), blomax.f90:336-349
    const long long np = IDX(i, ny - 1), npw = np - 1;
    const double tauw = fabs(vln[np] * Jn[np] * 2.0 * (u[np] * xk[np] + v[np] * yk[np]));
    const double row = ron[np], vlw = vln[np];
    const double nuw = vlw / row;
    const double utau = sqrt(fabs(tauw / row));
    const double xw = 0.5 * (x[np] + x[npw]);
    const double yw = 0.5 * (y[np] + y[npw]);
    auto cell = [&](int m) -> BlCell {            // m-th node from the wall: j = ny-1-m
        const int k = ny - 1 - m;
        const long long npl = IDX(i, k);
        const double dx = xp[npl] - xw, dy = yp[npl] - yw;
        const double dw = sqrt(dx * dx + dy * dy);
        BlCell r;
        r.yplus = dw * utau / nuw;
        r.omgplus = bl_omega(nx, x, y, Jp, u, v, i, k) * nuw / (utau * utau);
        r.lmp = c.kappa * r.yplus * (1.0 - exp(-r.yplus / c.Aop));
        return r;
    };
    // maxval(sqrt(u^2+v^2)), maxval(|omg+|) and maxloc(F) along the line
    double udif = 0.0, amax = 0.0, fmax = 0.0;
    int kmax = -1;
    bool hu = false, ha = false;
    for (int m = lane; m < n; m += 32) {
        const long long npl = IDX(i, ny - 1 - m);
        const double s = sqrt(u[npl] * u[npl] + v[npl] * v[npl]);
        if (!hu || s > udif) udif = s;
        hu = true;
        const BlCell q = cell(m);
        const double ao = fabs(q.omgplus);
        if (!ha || ao > amax) amax = ao;
        ha = true;
        const double f = q.lmp * fabs(q.omgplus) / c.kappa;
        if (kmax < 0 || f > fmax) { fmax = f; kmax = m; }
    }
    udif = warp_max(udif, hu);
    amax = warp_max(amax, ha);
    warp_argmax(fmax, kmax);
    if (amax < 1.0e-15) {                         // no vorticity: nu_t = 0 on the line
        for (int m = lane; m < n; m += 32) {
            const long long npl = IDX(i, ny - 1 - m);
            vtp[npl] = ro[npl] * 0.0 * nuw;
        }
        return;
    }
    // three-point parabola around the maximum, blomax.f90:244-283
    const int k0 = (kmax == 0) ? 0 : (kmax == n - 1 ? n - 3 : kmax - 1);
    double px[3], py[3];
    for (int t = 0; t < 3; t++) {
        const BlCell q = cell(k0 + t);
        px[t] = q.yplus;
        py[t] = q.lmp * fabs(q.omgplus) / c.kappa;
    }
    double ymaxp, Fmaxp;
    {
        const double a1 = (py[1] - py[0]) / (px[1] - px[0]);
        const double a2 = ((py[2] - py[1]) / (px[2] - px[1]) - a1) / (px[2] - px[0]);
        int kk = 0;
        for (int m = 1; m < 3; m++) if (py[m] > py[kk]) kk = m;
        ymaxp = px[kk]; Fmaxp = py[kk];
        if (a2 < 0.0) {
            const double xm = 0.5 * (px[0] + px[1] - a1 / a2);
            if (px[0] <= xm && xm <= px[2]) {
                ymaxp = xm;
                Fmaxp = py[0] + a1 * (xm - px[0]) + a2 * (xm - px[0]) * (xm - px[1]);
            }
        }
    }
    const double Udp = udif / utau;
    const double w1 = ymaxp * Fmaxp, w2 = c.Cwk * ymaxp * (Udp * Udp) / Fmaxp;
    const double Fwakep = (w2 < w1) ? w2 : w1;
    auto split = [&](const BlCell &q, double &nutip, double &nutop) {
        nutip = q.lmp * q.lmp * fabs(q.omgplus);
        const double cc = c.Ckleb * q.yplus / ymaxp;
        const double c3 = cc * cc * cc;
        nutop = c.alpha * c.Ccp * Fwakep / (1.0 + 5.5 * (c3 * c3));
    };
    // first k >= 1 with f(k-1) f(k) <= 0, f = nu_outer - nu_inner
    int kswitch = n;
    for (int base = 0; base < n; base += 32) {
        const int m = base + lane;
        bool hit = false;
        if (m >= 1 && m < n) {
            double i0, o0, i1, o1;
            split(cell(m - 1), i0, o0);
            split(cell(m), i1, o1);
            hit = (o0 - i0) * (o1 - i1) <= 0.0;
        }
        const unsigned bal = __ballot_sync(kFull, hit);
        if (bal) { kswitch = base + __ffs(bal) - 1; break; }
    }
    for (int m = lane; m < n; m += 32) {
        double nutip, nutop;
        split(cell(m), nutip, nutop);
        const long long npl = IDX(i, ny - 1 - m);
        vtp[npl] = ro[npl] * (m < kswitch ? nutip : nutop) * nuw;
    }
}

// blomax.f90:397-490: ghost values copy the adjacent real value, corners diagonally
__global__ void k_blomax_fictitious(int nx, int ny, double *phi)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nx - 2) {
        const int i = t + 2;
        phi[IDX(i, 1)] = phi[IDX(i, 2)];
        phi[IDX(i, ny)] = phi[IDX(i, ny - 1)];
    } else if (t < nx - 2 + ny - 2) {
        const int j = t - (nx - 2) + 2;
        phi[IDX(1, j)] = phi[IDX(2, j)];
        phi[IDX(nx, j)] = phi[IDX(nx - 1, j)];
    } else if (t == nx - 2 + ny - 2) {
        phi[IDX(1, 1)] = phi[IDX(2, 2)];
        phi[IDX(nx, 1)] = phi[IDX(nx - 1, 2)];
        phi[IDX(1, ny)] = phi[IDX(2, ny - 1)];
        phi[IDX(nx, ny)] = phi[IDX(nx - 1, ny - 1)];
    }
}

cudaError_t launch_blomax(int nx, int ny, const BlConst &c, const double *x, const double *y, const double *xp,
                          const double *yp, const double *xk, const double *yk, const double *Jp,
                          const double *Jn, const double *vln, const double *ro, const double *ron,
                          const double *u, const double *v, double *vtp, cudaStream_t st)
{
    if (nx < 3 || ny < 5) return cudaErrorInvalidValue;
    const int cols = nx - 2;
    k_blomax<<<(cols + kWarpsPerBlock - 1) / kWarpsPerBlock, 32 * kWarpsPerBlock, 0, st>>>(
        nx, ny, c, x, y, xp, yp, xk, yk, Jp, Jn, vln, ro, ron, u, v, vtp);
    return cudaGetLastError();
}

cudaError_t launch_blomax_fictitious(int nx, int ny, double *phi, cudaStream_t st)
{
    const int n = (nx - 2) + (ny - 2) + 1;
    k_blomax_fictitious<<<(n + 127) / 128, 128, 0, st>>>(nx, ny, phi);
    return cudaGetLastError();
}

// One thread per cell; the arithmetic and its order are those of the
// oracle's restatement, so the results are bitwise equal.
__global__ void k_add_eddy(int nx, int ny, int ktm, double mu, double kappa, double prt,
                           const double *__restrict__ vtp, const double *__restrict__ cp, double *vlp,
                           double *vle, double *vln, double *kp, double *ke, double *kn)
{
    const long long np = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (np >= (long long)nx * ny) return;
    const int j = (int)(np / nx) + 1, i = (int)(np - (long long)(j - 1) * nx) + 1;
    const double mp = ktm ? vlp[np] : mu, me = ktm ? vle[np] : mu, mn = ktm ? vln[np] : mu;
    const double kpl = ktm ? kp[np] : kappa, kel = ktm ? ke[np] : kappa, knl = ktm ? kn[np] : kappa;
    const double tp = cp[np] * vtp[np];
    vlp[np] = mp + vtp[np];
    kp[np] = kpl + tp / prt;
    if (i < nx) {
        const double te = cp[np + 1] * vtp[np + 1];
        vle[np] = me + 0.5 * (vtp[np] + vtp[np + 1]);
        ke[np] = kel + 0.5 * (tp + te) / prt;
    } else {
        vle[np] = me;
        ke[np] = kel;
    }
    if (j < ny - 1) {
        const double tn = cp[np + nx] * vtp[np + nx];
        vln[np] = mn + 0.5 * (vtp[np] + vtp[np + nx]);
        kn[np] = knl + 0.5 * (tp + tn) / prt;
    } else {
        vln[np] = mn;
        kn[np] = knl;
    }
}

cudaError_t launch_add_eddy(int nx, int ny, int ktm, double mu, double kappa, double prt, const double *vtp,
                            const double *cp, double *vlp, double *vle, double *vln, double *kp, double *ke,
                            double *kn, cudaStream_t st)
{
    const long long N = (long long)nx * ny;
    k_add_eddy<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(nx, ny, ktm, mu, kappa, prt, vtp, cp, vlp, vle, vln, kp,
                                                           ke, kn);
    return cudaGetLastError();
}

}  // namespace m2d
