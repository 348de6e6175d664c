// m2d_capi.cu -- the per-routine drop-ins of include/mach2d_b200.h.
//
// Each entry point stages the caller's host arrays into device memory, runs
// the same kernel the device-resident iteration uses, and copies the
// routine's outputs back.  Output arrays are copied in as well, because the
// reference routines write only part of them (interior rows, boundary
// strips) and the rest must keep the caller's values.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "m2d_fields.cuh"
#include "m2d_grid.cuh"
#include "m2d_solvers.cuh"
#include "m2d_extflow.cuh"
#include "m2d_blomax.cuh"
#include "m2d_thermo.cuh"
#include <cmath>
#include "../../include/mach2d_b200.h"

static thread_local std::string g_last_error;

void m2d_set_last_error(cudaError_t e, const char *what, const char *file, int line)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_last_error = buf;
}
void m2d_set_last_error_msg(const char *msg) { g_last_error = msg; }

static int fail(int code, const char *msg)
{
    g_last_error = msg;
    return code;
}

extern "C" const char *m2d_last_error(void) { return g_last_error.c_str(); }
extern "C" int m2d_version(void) { return 100; }

namespace {

using namespace m2d;

// device staging of host arrays for one drop-in call
struct Stage {
    struct Out { double *d; double *h; size_t n; };
    std::vector<void *> allocs;
    std::vector<Out> outs;
    int status = ST_OK;

    double *alloc(size_t n)
    {
        void *p = nullptr;
        if (status) return nullptr;
        cudaError_t e = cudaMalloc(&p, (n ? n : 1) * sizeof(double));
        if (e != cudaSuccess) { m2d_set_last_error(e, "cudaMalloc", __FILE__, __LINE__); status = ST_NOMEM; return nullptr; }
        allocs.push_back(p);
        return (double *)p;
    }
    double *in(const double *h, size_t n)
    {
        if (!h) { status = status ? status : ST_ARG; g_last_error = "null array argument"; return nullptr; }
        double *d = alloc(n);
        if (!d) return nullptr;
        cudaError_t e = cudaMemcpy(d, h, n * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { m2d_set_last_error(e, "cudaMemcpy H2D", __FILE__, __LINE__); status = ST_CUDA; }
        return d;
    }
    double *inout(double *h, size_t n)
    {
        double *d = in(h, n);
        if (d) outs.push_back({d, h, n});
        return d;
    }
    // an output the routine writes in full: no copy in
    double *out(double *h, size_t n)
    {
        if (!h) { status = status ? status : ST_ARG; g_last_error = "null array argument"; return nullptr; }
        double *d = alloc(n);
        if (d) outs.push_back({d, h, n});
        return d;
    }
    double *scratch(size_t n)
    {
        double *d = alloc(n);
        if (d && cudaMemset(d, 0, n * sizeof(double)) != cudaSuccess) status = ST_CUDA;
        return d;
    }
    int finish(cudaError_t launch)
    {
        if (!status && launch != cudaSuccess) { m2d_set_last_error(launch, "kernel launch", __FILE__, __LINE__); status = ST_CUDA; }
        if (!status) {
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) { m2d_set_last_error(e, "kernel", __FILE__, __LINE__); status = ST_CUDA; }
        }
        if (!status)
            for (auto &o : outs) {
                cudaError_t e = cudaMemcpy(o.h, o.d, o.n * sizeof(double), cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) { m2d_set_last_error(e, "cudaMemcpy D2H", __FILE__, __LINE__); status = ST_CUDA; break; }
            }
        return status;
    }
    ~Stage()
    {
        for (void *p : allocs) cudaFree(p);
    }
};

bool dims_ok(const int *nx, const int *ny)
{
    return nx && ny && *nx >= 4 && *ny >= 4 && (long long)*nx * *ny < (1LL << 31);
}

Fields empty_fields(int nx, int ny)
{
    Fields f;
    memset(&f, 0, sizeof f);
    f.nx = nx; f.ny = ny;
    return f;
}

int msi_solve_host(int nd, const int *nx, const int *ny, const int *nitm, const double *tol,
                   const double *a, const double *b, double *x, int *nit_out, int prec = 0)
{
    if (!dims_ok(nx, ny) || !nitm || !tol) return fail(ST_ARG, "msi: bad arguments");
    if (*ny > msi_max_ny()) return fail(ST_TOO_LARGE, "msi: ny exceeds m2d_msi_max_ny()");
    const size_t N = (size_t)*nx * *ny;
    Stage s;
    MsiLaunch L;
    memset(&L, 0, sizeof L);
    L.nx = *nx; L.ny = *ny; L.nitm = *nitm; L.tol = *tol;
    L.prec = prec;
    MsiSys &S = L.s[0];
    S.a = s.in(a, (size_t)nd * N);
    S.b = s.in(b, N);
    S.x = s.inout(x, N);
    S.ws = s.scratch(msi_work_doubles(nd, *nx, *ny));
    double *misc = s.scratch(4);
    if (s.status) return s.status;
    S.nit = (int *)misc;
    S.rr = misc + 1;
    L.err = (int *)(misc + 3);
    int rc = s.finish(launch_msi(nd, L, 1, 0));
    if (rc) return rc;
    int hv[2] = {0, 0};
    cudaMemcpy(&hv[0], misc, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(&hv[1], misc + 3, sizeof(int), cudaMemcpyDeviceToHost);
    if (nit_out) *nit_out = hv[0];
    if (hv[1] & ERR_SPIN_TIMEOUT) return fail(ST_TIMEOUT, "msi: a bounded device-side wait ran out");
    if (hv[1] & ERR_WAIT_TIMEOUT) return fail(ST_TIMEOUT, "msi: unbounded iteration reached its cap");
    if (hv[1] & ERR_NONFINITE_PIVOT) return fail(7, "msi: zero or non-finite pivot in the factorisation");
    return ST_OK;
}

int reduce_host(RedArgs r, double *out)
{
    Stage s;
    double *part = s.scratch((size_t)red_parts() + 1);
    if (s.status) return s.status;
    int rc = s.finish(launch_reduce(r, part, part + red_parts(), 0));
    if (rc) return rc;
    if (cudaMemcpy(out, part + red_parts(), sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(ST_CUDA, "reduce: D2H copy failed");
    return ST_OK;
}

}  // namespace

extern "C" {

int m2d_msi_max_ny(void) { return m2d::msi_max_ny(); }

int m2d_test_wait_hook(int kernel, double limit_s)
{
    if (kernel < 0 || kernel > 2 || !(limit_s >= 0.0) || limit_s > 10.0)
        return fail(ST_ARG, "m2d_test_wait_hook: kernel 0..2, limit 0..10 s");
    const unsigned long long ns = (unsigned long long)(limit_s * 1e9);
    m2d::set_msi_wait_hook(kernel == 1 ? ns : 0ull);
    m2d::set_conv_wait_hook(kernel == 2 ? ns : 0ull);
    return ST_OK;
}

int m2d_msi9_solve(const int *nx, const int *ny, const int *nitm, const double *tol,
                   const double *a, const double *b, double *x)
{ return msi_solve_host(9, nx, ny, nitm, tol, a, b, x, nullptr); }
int m2d_msi5_solve(const int *nx, const int *ny, const int *nitm, const double *tol,
                   const double *a, const double *b, double *x)
{ return msi_solve_host(5, nx, ny, nitm, tol, a, b, x, nullptr); }
int m2d_msi9_solve_mixed(const int *nx, const int *ny, const int *nitm, const double *tol,
                         const double *a, const double *b, double *x, int *nit)
{ return msi_solve_host(9, nx, ny, nitm, tol, a, b, x, nit, 1); }
int m2d_msi5_solve_mixed(const int *nx, const int *ny, const int *nitm, const double *tol,
                         const double *a, const double *b, double *x, int *nit)
{ return msi_solve_host(5, nx, ny, nitm, tol, a, b, x, nit, 1); }
int m2d_msi9_solve_it(const int *nx, const int *ny, const int *nitm, const double *tol,
                      const double *a, const double *b, double *x, int *nit)
{ return msi_solve_host(9, nx, ny, nitm, tol, a, b, x, nit); }
int m2d_msi5_solve_it(const int *nx, const int *ny, const int *nitm, const double *tol,
                      const double *a, const double *b, double *x, int *nit)
{ return msi_solve_host(5, nx, ny, nitm, tol, a, b, x, nit); }

long m2d_msi_workspace_doubles(int nd, int nx, int ny)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4) return -1;
    // factor and residual planes, then 4 doubles for rr and the error word
    return (long)msi_work_doubles(nd, nx, ny) + 4;
}

// one device-resident solve on caller scratch of work_doubles doubles (the
// factor planes, then rr in the last 4 doubles); the caller has checked that
// work_doubles covers at least the plain-layout kernel
int m2d_msi_solve_device_ws(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                            const double *d_b, double *d_x, double *d_work, long work_doubles,
                            void *stream, int *d_nit, unsigned long long *d_times, int prec)
{
    MsiLaunch L;
    memset(&L, 0, sizeof L);
    L.nx = nx; L.ny = ny; L.nitm = nitm; L.tol = tol;
    L.prec = prec;
    MsiSys &S = L.s[0];
    S.a = d_a; S.b = d_b; S.x = d_x;
    S.ws = d_work;
    S.rr = d_work + (work_doubles - 4);
    S.nit = d_nit;
    L.ws_cap = (size_t)(work_doubles - 4);
    L.prof = d_times;
    cudaError_t e = launch_msi(nd, L, 1, (cudaStream_t)stream);
    if (e != cudaSuccess) { m2d_set_last_error(e, "msi_solve_device launch", __FILE__, __LINE__); return ST_CUDA; }
    return ST_OK;
}

int m2d_msi_solve_device(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                         const double *d_b, double *d_x, double *d_work, void *stream, int *d_nit)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4 || !d_a || !d_b || !d_x || !d_work)
        return fail(ST_ARG, "msi_solve_device: bad arguments");
    if (ny > msi_max_ny()) return fail(ST_TOO_LARGE, "msi_solve_device: ny exceeds m2d_msi_max_ny()");
    return m2d_msi_solve_device_ws(nd, nx, ny, nitm, tol, d_a, d_b, d_x, d_work,
                                   m2d_msi_workspace_doubles(nd, nx, ny), stream, d_nit, nullptr, 0);
}

int m2d_msi_solve_device_mixed(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                               const double *d_b, double *d_x, double *d_work, void *stream, int *d_nit)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4 || !d_a || !d_b || !d_x || !d_work)
        return fail(ST_ARG, "msi_solve_device_mixed: bad arguments");
    if (ny > msi_max_ny()) return fail(ST_TOO_LARGE, "msi_solve_device_mixed: ny exceeds m2d_msi_max_ny()");
    return m2d_msi_solve_device_ws(nd, nx, ny, nitm, tol, d_a, d_b, d_x, d_work,
                                   m2d_msi_workspace_doubles(nd, nx, ny), stream, d_nit, nullptr, 1);
}

int m2d_msi_solve_device_ex(int nd, int nx, int ny, int nitm, double tol, const double *d_a, const double *d_b,
                            double *d_x, double *d_work, void *stream, int *d_nit, int prec, int reuse_factors,
                            unsigned long long *d_times)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4 || !d_a || !d_b || !d_x || !d_work || (prec != 0 && prec != 1) ||
        (reuse_factors != 0 && reuse_factors != 1))
        return fail(ST_ARG, "msi_solve_device_ex: bad arguments");
    if (ny > msi_max_ny()) return fail(ST_TOO_LARGE, "msi_solve_device_ex: ny exceeds m2d_msi_max_ny()");
    const long wd = m2d_msi_workspace_doubles(nd, nx, ny);
    MsiLaunch L;
    memset(&L, 0, sizeof L);
    L.nx = nx; L.ny = ny; L.nitm = nitm; L.tol = tol;
    L.prec = prec;
    L.reuse_lu = reuse_factors;
    MsiSys &S = L.s[0];
    S.a = d_a; S.b = d_b; S.x = d_x;
    S.ws = d_work;
    S.rr = d_work + (wd - 4);
    S.nit = d_nit;
    L.ws_cap = (size_t)(wd - 4);
    L.prof = d_times;
    cudaError_t e = launch_msi(nd, L, 1, (cudaStream_t)stream);
    if (e != cudaSuccess) { m2d_set_last_error(e, "msi_solve_device_ex launch", __FILE__, __LINE__); return ST_CUDA; }
    return ST_OK;
}

int m2d_msi_solve_device_timed(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                               const double *d_b, double *d_x, double *d_work, void *stream,
                               int *d_nit, unsigned long long *d_times)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4 || !d_a || !d_b || !d_x || !d_work || !d_times)
        return fail(ST_ARG, "msi_solve_device_timed: bad arguments");
    if (ny > msi_max_ny()) return fail(ST_TOO_LARGE, "msi_solve_device_timed: ny exceeds m2d_msi_max_ny()");
    return m2d_msi_solve_device_ws(nd, nx, ny, nitm, tol, d_a, d_b, d_x, d_work,
                                   m2d_msi_workspace_doubles(nd, nx, ny), stream, d_nit, d_times, 0);
}

long long m2d_msi_lu_redo_count(void) { return msi_lu_redo_count(); }

static int tdma_host(int nd, const int *nx, const int *ny, const int *nitm, const double *a,
                     const double *b, double *x)
{
    if (!dims_ok(nx, ny) || !nitm) return fail(ST_ARG, "tdma: bad arguments");
    const size_t N = (size_t)*nx * *ny;
    Stage s;
    const double *da = s.in(a, (size_t)nd * N);
    const double *db = s.in(b, N);
    double *dx = s.inout(x, N);
    double *P = s.scratch(N), *Q = s.scratch(N);
    if (s.status) return s.status;
    return s.finish(launch_tdma(nd, *nx, *ny, *nitm, da, db, dx, P, Q, 0));
}
int m2d_tdma9_solve(const int *nx, const int *ny, const int *nitm, const double *a,
                    const double *b, double *x)
{ return tdma_host(9, nx, ny, nitm, a, b, x); }
int m2d_tdma5_solve(const int *nx, const int *ny, const int *nitm, const double *a,
                    const double *b, double *x)
{ return tdma_host(5, nx, ny, nitm, a, b, x); }

int m2d_tdma_lines(const int *n, const int *nlines, const double *aw, const double *ap,
                   const double *ae, const double *d, double *x)
{
    if (!n || !nlines || *n < 1 || *nlines < 1) return fail(ST_ARG, "tdma_lines: bad arguments");
    const size_t M = (size_t)*n * *nlines;
    Stage s;
    const double *daw = s.in(aw, M), *dap = s.in(ap, M), *dae = s.in(ae, M), *dd = s.in(d, M);
    double *dx = s.inout(x, M);
    double *P = s.scratch(M), *Q = s.scratch(M);
    if (s.status) return s.status;
    return s.finish(launch_tdma_lines(*n, *nlines, daw, dap, dae, dd, dx, P, Q, 0));
}

int m2d_tdma_lines_device(int n, int nlines, const double *d_aw, const double *d_ap, const double *d_ae,
                          const double *d_d, double *d_x, double *d_work, int method, void *stream)
{
    if (n < 1 || nlines < 1 || !d_aw || !d_ap || !d_ae || !d_d || !d_x || (method != 0 && method != 1))
        return fail(ST_ARG, "tdma_lines_device: bad arguments");
    cudaError_t e;
    if (method == 0) {
        if (!d_work) return fail(ST_ARG, "tdma_lines_device: method 0 needs d_work (2 n nlines doubles)");
        const size_t M = (size_t)n * nlines;
        e = launch_tdma_lines(n, nlines, d_aw, d_ap, d_ae, d_d, d_x, d_work, d_work + M, (cudaStream_t)stream);
    } else {
        if (!tdma_lines_pcr_supported(n)) return fail(ST_TOO_LARGE, "tdma_lines_device: cyclic reduction needs n <= 2048");
        e = launch_tdma_lines_pcr(n, nlines, d_aw, d_ap, d_ae, d_d, d_x, (cudaStream_t)stream);
    }
    if (e != cudaSuccess) { m2d_set_last_error(e, "tdma_lines_device launch", __FILE__, __LINE__); return ST_CUDA; }
    return ST_OK;
}

int m2d_norm_l1_5d(const int *nx, const int *ny, const double *var, const double *b,
                   const double *a, double *norm)
{
    if (!dims_ok(nx, ny) || !norm) return fail(ST_ARG, "norm_l1_5d: bad arguments");
    size_t N = (size_t)*nx * *ny;
    Stage s;
    RedArgs r; memset(&r, 0, sizeof r);
    r.kind = RED_NORM_L1_5D; r.nx = *nx; r.ny = *ny;
    r.x = s.in(var, N); r.b = s.in(b, N); r.a = s.in(a, 5 * N);
    if (s.status) return s.status;
    double v;
    int rc = reduce_host(r, &v);
    if (!rc) *norm = *norm + v;
    return rc;
}

int m2d_norm_l1_9d(const int *nx, const int *ny, const double *var, const double *b,
                   const double *a, double *norm)
{
    if (!dims_ok(nx, ny) || !norm) return fail(ST_ARG, "norm_l1_9d: bad arguments");
    size_t N = (size_t)*nx * *ny;
    Stage s;
    RedArgs r; memset(&r, 0, sizeof r);
    r.kind = RED_NORM_L1_9D; r.nx = *nx; r.ny = *ny;
    r.x = s.in(var, N); r.b = s.in(b, N); r.a = s.in(a, 9 * N);
    if (s.status) return s.status;
    double v;
    int rc = reduce_host(r, &v);
    if (!rc) *norm = *norm + v;
    return rc;
}

int m2d_norm_l1_9d_relative(const int *nx, const int *ny, const double *var, const double *b,
                            const double *a, double *norm)
{
    if (!dims_ok(nx, ny) || !norm) return fail(ST_ARG, "norm_l1_9d_relative: bad arguments");
    size_t N = (size_t)*nx * *ny;
    Stage s;
    RedArgs r; memset(&r, 0, sizeof r);
    r.kind = RED_NORM_L1_9D; r.nx = *nx; r.ny = *ny;
    r.x = s.in(var, N); r.b = s.in(b, N); r.a = s.in(a, 9 * N);
    if (s.status) return s.status;
    double na, nb;
    int rc = reduce_host(r, &na);
    if (rc) return rc;
    r.kind = RED_SUM_ABS_B;
    rc = reduce_host(r, &nb);
    if (rc) return rc;
    const double eps = 10.0 * 2.220446049250313e-16;
    if (nb > eps) *norm = *norm + na / nb;
    else *norm = *norm + na;
    return ST_OK;
}

#define ND_ (size_t)(*nx) * (size_t)(*ny)
#define CHK if (!dims_ok(nx, ny)) return fail(ST_ARG, "bad grid dimensions")

int m2d_get_density_at_nodes(const int *nx, const int *ny, const double *Rg, const double *p,
                             const double *T, double *ro)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.p = s.in(p, N); f.T = s.in(T, N); f.ro = s.inout(ro, N);
    if (s.status) return s.status;
    return s.finish(launch_density_at_nodes(f, *Rg, 0));
}

int m2d_get_density_at_faces(const int *nx, const int *ny, const double *beta,
                             const double *ro, const double *Uce, const double *Vcn,
                             double *roe, double *ron)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.ro = s.in(ro, N); f.Uce = s.in(Uce, N); f.Vcn = s.in(Vcn, N);
    f.roe = s.inout(roe, N); f.ron = s.inout(ron, N);
    if (s.status) return s.status;
    return s.finish(launch_density_at_faces(f, *beta, 0));
}

int m2d_get_u_coefficients(const int *nx, const int *ny, const int *modvis, const double *dt,
    const double *rp, const double *re, const double *rn, const double *Jp, const double *Je,
    const double *Jn, const double *ye, const double *yk, const double *alphae,
    const double *betae, const double *betan, const double *gamman, const double *vle,
    const double *vln, const double *roe, const double *ron, const double *roa,
    const double *Uce, const double *Vcn, double *a)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.Jp = s.in(Jp, N);
    f.Je = s.in(Je, N); f.Jn = s.in(Jn, N); f.ye = s.in(ye, N); f.yk = s.in(yk, N);
    f.alphae = s.in(alphae, N); f.betae = s.in(betae, N); f.betan = s.in(betan, N);
    f.gamman = s.in(gamman, N); f.vle = s.in(vle, N); f.vln = s.in(vln, N);
    f.roe = s.in(roe, N); f.ron = s.in(ron, N); f.roa = s.in(roa, N);
    f.Uce = s.in(Uce, N); f.Vcn = s.in(Vcn, N); f.au = s.inout(a, 9 * N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q); q.modvis = *modvis; q.dt = *dt;
    return s.finish(launch_u_assembly(f, q, ASM_COEF, 0));
}

int m2d_get_u_source(const int *nx, const int *ny, const int *modvis, const double *beta,
    const double *dt, const double *rp, const double *re, const double *rn, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *xke, const double *yke,
    const double *xen, const double *yen, const double *Jp, const double *Je, const double *Jn,
    const double *roe, const double *ron, const double *roa, const double *p, const double *vle,
    const double *vln, const double *Uce, const double *Vcn, const double *ua, const double *u,
    const double *v, double *cup, double *sup, double *b)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.xe = s.in(xe, N);
    f.ye = s.in(ye, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N); f.xke = s.in(xke, N);
    f.yke = s.in(yke, N); f.xen = s.in(xen, N); f.yen = s.in(yen, N); f.Jp = s.in(Jp, N);
    f.Je = s.in(Je, N); f.Jn = s.in(Jn, N); f.roe = s.in(roe, N); f.ron = s.in(ron, N);
    f.roa = s.in(roa, N); f.p = s.in(p, N); f.vle = s.in(vle, N); f.vln = s.in(vln, N);
    f.Uce = s.in(Uce, N); f.Vcn = s.in(Vcn, N); f.ua = s.in(ua, N); f.u = s.in(u, N);
    f.v = s.in(v, N); f.cup = s.inout(cup, N); f.sup = s.inout(sup, N); f.bu = s.inout(b, N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q); q.modvis = *modvis; q.dt = *dt; q.beta = *beta;
    return s.finish(launch_u_assembly(f, q, ASM_SRC, 0));
}

int m2d_get_v_coefficients(const int *nx, const int *ny, const int *coord, const int *modvis,
    const double *dt, const double *rp, const double *re, const double *rn, const double *Jp,
    const double *Je, const double *Jn, const double *xe, const double *xk,
    const double *alphae, const double *betae, const double *betan, const double *gamman,
    const double *vle, const double *vln, const double *vlp, const double *roe,
    const double *ron, const double *roa, const double *Uce, const double *Vcn, double *a)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.Jp = s.in(Jp, N);
    f.Je = s.in(Je, N); f.Jn = s.in(Jn, N); f.xe = s.in(xe, N); f.xk = s.in(xk, N);
    f.alphae = s.in(alphae, N); f.betae = s.in(betae, N); f.betan = s.in(betan, N);
    f.gamman = s.in(gamman, N); f.vle = s.in(vle, N); f.vln = s.in(vln, N); f.vlp = s.in(vlp, N);
    f.roe = s.in(roe, N); f.ron = s.in(ron, N); f.roa = s.in(roa, N);
    f.Uce = s.in(Uce, N); f.Vcn = s.in(Vcn, N); f.av = s.inout(a, 9 * N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q); q.modvis = *modvis; q.coord = *coord; q.dt = *dt;
    return s.finish(launch_v_assembly(f, q, ASM_COEF, 0));
}

int m2d_get_v_source(const int *nx, const int *ny, const int *coord, const int *modvis,
    const double *beta, const double *dt, const double *rp, const double *re, const double *rn,
    const double *xe, const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *Jp, const double *Je,
    const double *Jn, const double *roe, const double *ron, const double *roa, const double *p,
    const double *vle, const double *vln, const double *Uce, const double *Vcn,
    const double *va, const double *u, const double *v, double *cvp, double *svp, double *b)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.xe = s.in(xe, N);
    f.ye = s.in(ye, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N); f.xke = s.in(xke, N);
    f.yke = s.in(yke, N); f.xen = s.in(xen, N); f.yen = s.in(yen, N); f.Jp = s.in(Jp, N);
    f.Je = s.in(Je, N); f.Jn = s.in(Jn, N); f.roe = s.in(roe, N); f.ron = s.in(ron, N);
    f.roa = s.in(roa, N); f.p = s.in(p, N); f.vle = s.in(vle, N); f.vln = s.in(vln, N);
    f.Uce = s.in(Uce, N); f.Vcn = s.in(Vcn, N); f.va = s.in(va, N); f.u = s.in(u, N);
    f.v = s.in(v, N); f.cvp = s.inout(cvp, N); f.svp = s.inout(svp, N); f.bv = s.inout(b, N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q); q.modvis = *modvis; q.coord = *coord; q.dt = *dt; q.beta = *beta;
    return s.finish(launch_v_assembly(f, q, ASM_SRC, 0));
}

int m2d_get_T_coefficients_and_source(const int *nx, const int *ny, const int *modvis,
    const double *beta, const double *dt, const double *rp, const double *re, const double *rn,
    const double *xe, const double *ye, const double *xk, const double *yk, const double *xke,
    const double *yke, const double *xen, const double *yen, const double *alphae,
    const double *betae, const double *betan, const double *gamman, const double *Jp,
    const double *Je, const double *Jn, const double *roe, const double *ron, const double *ro,
    const double *roa, const double *p, const double *pa, const double *cp, const double *vle,
    const double *vln, const double *ke, const double *kn, const double *Uce, const double *Vcn,
    const double *u, const double *v, const double *ue, const double *ve, const double *un,
    const double *vn, const double *ua, const double *va, const double *T, const double *Ta,
    const double *fbe, const double *fbn, double *a, double *b)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.xe = s.in(xe, N);
    f.ye = s.in(ye, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N); f.xke = s.in(xke, N);
    f.yke = s.in(yke, N); f.xen = s.in(xen, N); f.yen = s.in(yen, N);
    f.alphae = s.in(alphae, N); f.betae = s.in(betae, N); f.betan = s.in(betan, N);
    f.gamman = s.in(gamman, N); f.Jp = s.in(Jp, N); f.Je = s.in(Je, N); f.Jn = s.in(Jn, N);
    f.roe = s.in(roe, N); f.ron = s.in(ron, N); f.ro = s.in(ro, N); f.roa = s.in(roa, N);
    f.p = s.in(p, N); f.pa = s.in(pa, N); f.cp = s.in(cp, N); f.vle = s.in(vle, N);
    f.vln = s.in(vln, N); f.ke = s.in(ke, N); f.kn = s.in(kn, N); f.Uce = s.in(Uce, N);
    f.Vcn = s.in(Vcn, N); f.u = s.in(u, N); f.v = s.in(v, N); f.ue = s.in(ue, N);
    f.ve = s.in(ve, N); f.un = s.in(un, N); f.vn = s.in(vn, N); f.ua = s.in(ua, N);
    f.va = s.in(va, N); f.T = s.in(T, N); f.Ta = s.in(Ta, N); f.fbe = s.in(fbe, N);
    f.fbn = s.in(fbn, N); f.at = s.inout(a, 9 * N); f.bt = s.inout(b, N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q); q.modvis = *modvis; q.dt = *dt; q.beta = *beta;
    return s.finish(launch_T_assembly(f, q, 0));
}

int m2d_get_p_coefficients(const int *nx, const int *ny, const double *dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *Uce, const double *Vcn,
    const double *roe, const double *ron, const double *g, const double *de, const double *dn,
    double *a)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.Jp = s.in(Jp, N);
    f.Uce = s.in(Uce, N); f.Vcn = s.in(Vcn, N); f.roe = s.in(roe, N); f.ron = s.in(ron, N);
    f.g = s.in(g, N); f.de = s.in(de, N); f.dn = s.in(dn, N); f.ap = s.inout(a, 5 * N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q); q.dt = *dt;
    return s.finish(launch_p_assembly(f, q, ASM_COEF, 0));
}

int m2d_get_p_source(const int *nx, const int *ny, const double *dt, const double *rp,
    const double *re, const double *rn, const double *Jp, const double *roe, const double *ron,
    const double *ro, const double *roa, const double *Uce, const double *Vcn, const double *de,
    const double *dn, const double *g, const double *pl, double *b)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.Jp = s.in(Jp, N);
    f.roe = s.in(roe, N); f.ron = s.in(ron, N); f.ro = s.in(ro, N); f.roa = s.in(roa, N);
    f.Uce = s.in(Uce, N); f.Vcn = s.in(Vcn, N); f.de = s.in(de, N); f.dn = s.in(dn, N);
    f.g = s.in(g, N); f.pl = s.in(pl, N); f.bp = s.inout(b, N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q); q.dt = *dt;
    return s.finish(launch_p_assembly(f, q, ASM_SRC, 0));
}

int m2d_get_velocities_at_internal_faces(const int *nx, const int *ny, const double *dt,
    const double *rp, const double *re, const double *rn, const double *xe, const double *ye,
    const double *xk, const double *yk, const double *xen, const double *yen, const double *xke,
    const double *yke, const double *Jp, const double *cup, const double *cvp, const double *sup,
    const double *svp, const double *au, const double *av, const double *roa, const double *p,
    const double *u, const double *v, const double *uea, const double *vea, const double *una,
    const double *vna, double *ue, double *ve, double *un, double *vn, double *Uce, double *Vcn)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.rp = s.in(rp, N); f.re = s.in(re, N); f.rn = s.in(rn, N); f.xe = s.in(xe, N);
    f.ye = s.in(ye, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N); f.xen = s.in(xen, N);
    f.yen = s.in(yen, N); f.xke = s.in(xke, N); f.yke = s.in(yke, N); f.Jp = s.in(Jp, N);
    f.cup = s.in(cup, N); f.cvp = s.in(cvp, N); f.sup = s.in(sup, N); f.svp = s.in(svp, N);
    f.au = s.in(au, 9 * N); f.av = s.in(av, 9 * N); f.roa = s.in(roa, N); f.p = s.in(p, N);
    f.u = s.in(u, N); f.v = s.in(v, N); f.uea = s.in(uea, N); f.vea = s.in(vea, N);
    f.una = s.in(una, N); f.vna = s.in(vna, N); f.ue = s.inout(ue, N); f.ve = s.inout(ve, N);
    f.un = s.inout(un, N); f.vn = s.inout(vn, N); f.Uce = s.inout(Uce, N); f.Vcn = s.inout(Vcn, N);
    if (s.status) return s.status;
    return s.finish(launch_velocities_at_internal_faces(f, *dt, 0));
}

int m2d_get_internal_simplec_coefficients(const int *nx, const int *ny, const double *re,
    const double *rn, const double *xe, const double *ye, const double *xk, const double *yk,
    const double *au, const double *av, double *due, double *dve, double *dun, double *dvn,
    double *de, double *dn)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.re = s.in(re, N); f.rn = s.in(rn, N); f.xe = s.in(xe, N); f.ye = s.in(ye, N);
    f.xk = s.in(xk, N); f.yk = s.in(yk, N); f.au = s.in(au, 9 * N); f.av = s.in(av, 9 * N);
    f.due = s.inout(due, N); f.dve = s.inout(dve, N); f.dun = s.inout(dun, N);
    f.dvn = s.inout(dvn, N); f.de = s.inout(de, N); f.dn = s.inout(dn, N);
    if (s.status) return s.status;
    return s.finish(launch_internal_simplec(f, 0));
}

int m2d_get_pressure_correction_with_pl(const int *nx, const int *ny, const double *pl, double *p)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.pl = s.in(pl, N); f.p = s.inout(p, N);
    if (s.status) return s.status;
    return s.finish(launch_p_ro_correction(f, 1, 0, 0));
}

int m2d_get_density_correction_with_pl(const int *nx, const int *ny, const double *pl,
                                       const double *g, double *ro)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.pl = s.in(pl, N); f.g = s.in(g, N); f.ro = s.inout(ro, N);
    if (s.status) return s.status;
    return s.finish(launch_p_ro_correction(f, 0, 1, 0));
}

int m2d_get_u_v_at_real_nodes_with_pl(const int *nx, const int *ny, const double *xe,
    const double *ye, const double *xk, const double *yk, const double *rp, const double *pl,
    const double *au, const double *av, double *u, double *v)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.xe = s.in(xe, N); f.ye = s.in(ye, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N);
    f.rp = s.in(rp, N); f.pl = s.in(pl, N); f.au = s.in(au, 9 * N); f.av = s.in(av, 9 * N);
    f.u = s.inout(u, N); f.v = s.inout(v, N);
    if (s.status) return s.status;
    return s.finish(launch_uv_nodes_correction(f, 0));
}

int m2d_get_velocity_correction_at_faces_with_pl(const int *nx, const int *ny,
    const double *xe, const double *ye, const double *xk, const double *yk, const double *due,
    const double *dve, const double *dun, const double *dvn, const double *de, const double *dn,
    const double *pl, double *ue, double *ve, double *un, double *vn, double *Uce, double *Vcn)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.xe = s.in(xe, N); f.ye = s.in(ye, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N);
    f.due = s.in(due, N); f.dve = s.in(dve, N); f.dun = s.in(dun, N); f.dvn = s.in(dvn, N);
    f.de = s.in(de, N); f.dn = s.in(dn, N); f.pl = s.in(pl, N);
    f.ue = s.inout(ue, N); f.ve = s.inout(ve, N); f.un = s.inout(un, N); f.vn = s.inout(vn, N);
    f.Uce = s.inout(Uce, N); f.Vcn = s.inout(Vcn, N);
    if (s.status) return s.status;
    return s.finish(launch_velocity_correction_at_faces(f, 0));
}

int m2d_initialize_boundary_faces_flags(const int *nx, const int *ny, double *fbe, double *fbn)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.fbe = s.inout(fbe, N); f.fbn = s.inout(fbn, N);
    if (s.status) return s.status;
    return s.finish(launch_boundary_faces_flags(f, 0));
}

int m2d_check_mass_conservation(const int *nx, const int *ny, const double *dt,
    const double *rp, const double *re, const double *rn, const double *Jp, const double *ro,
    const double *roa, const double *ron, const double *roe, const double *Uce,
    const double *Vcn, double *res)
{
    CHK; if (!res) return fail(ST_ARG, "check_mass_conservation: null res");
    Stage s; size_t N = ND_;
    RedArgs r; memset(&r, 0, sizeof r);
    r.kind = RED_MASS; r.nx = *nx; r.ny = *ny; r.dt = *dt;
    r.rp = s.in(rp, N); r.re = s.in(re, N); r.rn = s.in(rn, N); r.Jp = s.in(Jp, N);
    r.ro = s.in(ro, N); r.roa = s.in(roa, N); r.ron = s.in(ron, N); r.roe = s.in(roe, N);
    r.Uce = s.in(Uce, N); r.Vcn = s.in(Vcn, N);
    if (s.status) return s.status;
    return reduce_host(r, res);
}

int m2d_intflow_set_bcu(const int *nx, const int *ny, const int *modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u, const double *v,
    double *au, double *b)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.x = s.in(x, N); f.xp = s.in(xp, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N);
    f.u = s.in(u, N); f.v = s.in(v, N); f.au = s.inout(au, 9 * N); f.bu = s.inout(b, N);
    if (s.status) return s.status;
    return s.finish(launch_set_bcu(f, *modvis, 0));
}

int m2d_intflow_set_bcv(const int *nx, const int *ny, const int *modvis, const double *x,
    const double *xp, const double *xk, const double *yk, const double *u, const double *v,
    double *av, double *b)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.x = s.in(x, N); f.xp = s.in(xp, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N);
    f.u = s.in(u, N); f.v = s.in(v, N); f.av = s.inout(av, 9 * N); f.bv = s.inout(b, N);
    if (s.status) return s.status;
    return s.finish(launch_set_bcv(f, *modvis, 0));
}

int m2d_intflow_set_bcpl(const int *nx, const int *ny, const double *x, const double *xp,
    const double *pl, const double *plin, double *ap, double *bp)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.x = s.in(x, N); f.xp = s.in(xp, N); f.pl = s.in(pl, N); f.plin = s.in(plin, (size_t)*ny);
    f.ap = s.inout(ap, 5 * N); f.bp = s.inout(bp, N);
    if (s.status) return s.status;
    return s.finish(launch_set_bcpl(f, 0));
}

int m2d_intflow_set_bcT(const int *nx, const int *ny, const double *x, const double *xp,
    const double *T, const double *Twall, const double *Tin, double *at, double *bt)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.x = s.in(x, N); f.xp = s.in(xp, N); f.T = s.in(T, N); f.Tin = s.in(Tin, (size_t)*ny);
    f.at = s.inout(at, 9 * N); f.bt = s.inout(bt, N);
    if (s.status) return s.status;
    return s.finish(launch_set_bcT(f, *Twall, 0));
}

int m2d_intflow_boundary_T_from_H_conservation(const int *nx, const int *ny,
    const double *Cpref, const double *Href, const double *Tin, const double *u,
    const double *ue, const double *un, const double *v, const double *ve, const double *vn,
    double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    (void)u; (void)v;
    f.Tin = s.in(Tin, (size_t)*ny); f.ue = s.in(ue, N); f.un = s.in(un, N);
    f.ve = s.in(ve, N); f.vn = s.in(vn, N); f.T = s.inout(T, N);
    f.Tbe = s.inout(Tbe, (size_t)*ny); f.Tbw = s.inout(Tbw, (size_t)*ny);
    f.Tbn = s.inout(Tbn, (size_t)*nx); f.Tbs = s.inout(Tbs, (size_t)*nx);
    if (s.status) return s.status;
    // boundary part only: the nodal T is the caller's (src/mach2d_main.f90:362)
    return s.finish(launch_T_boundary_H(f, *Href, *Cpref, 0));
}

int m2d_intflow_velocities_at_boundary_faces(const int *nx, const int *ny, const int *modvis,
    const double *x, const double *xp, const double *xe, const double *ye, const double *xk,
    const double *yk, const double *u, const double *v, double *ue, double *ve, double *un,
    double *vn, double *Uce, double *Vcn)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.x = s.in(x, N); f.xp = s.in(xp, N); f.xe = s.in(xe, N); f.ye = s.in(ye, N);
    f.xk = s.in(xk, N); f.yk = s.in(yk, N); f.u = s.in(u, N); f.v = s.in(v, N);
    f.ue = s.inout(ue, N); f.ve = s.inout(ve, N); f.un = s.inout(un, N); f.vn = s.inout(vn, N);
    f.Uce = s.inout(Uce, N); f.Vcn = s.inout(Vcn, N);
    if (s.status) return s.status;
    return s.finish(launch_velocities_at_boundary_faces(f, *modvis, 0));
}

int m2d_intflow_boundary_simplec(const int *nx, const int *ny, const int *modvis, double *due,
    double *dve, double *dun, double *dvn, double *de, double *dn)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    (void)modvis;
    f.due = s.inout(due, N); f.dve = s.inout(dve, N); f.dun = s.inout(dun, N);
    f.dvn = s.inout(dvn, N); f.de = s.inout(de, N); f.dn = s.inout(dn, N);
    if (s.status) return s.status;
    return s.finish(launch_boundary_simplec(f, 0));
}

int m2d_intflow_extrapolate_u_v_to_fictitious(const int *nx, const int *ny, const int *modvis,
    const double *x, const double *xp, const double *xk, const double *yk, double *u, double *v)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_;
    f.x = s.in(x, N); f.xp = s.in(xp, N); f.xk = s.in(xk, N); f.yk = s.in(yk, N);
    f.u = s.inout(u, N); f.v = s.inout(v, N);
    if (s.status) return s.status;
    return s.finish(launch_extrapolate_uv(f, *modvis, 0));
}

int m2d_intflow_time_cycle_update(const int *nx, const int *ny, const double *x,
    const double *xp, const double *u, const double *gamma, const double *Rg,
    const double *P0, const double *T0, double *uin, double *vin, double *pin, double *Tin,
    double *Mw, double *plin, double *pina, double *p)
{
    CHK; Stage s; Fields f = empty_fields(*nx, *ny); size_t N = ND_, M = (size_t)*ny;
    f.x = s.in(x, N); f.xp = s.in(xp, N); f.u = s.in(u, N);
    f.uin = s.inout(uin, M); f.vin = s.inout(vin, M); f.pin = s.inout(pin, M);
    f.Tin = s.inout(Tin, M); f.Mw = s.inout(Mw, M); f.plin = s.inout(plin, M);
    f.pina = s.inout(pina, M); f.p = s.inout(p, N);
    if (s.status) return s.status;
    Params q; memset(&q, 0, sizeof q);
    q.gamma = *gamma; q.Rg = *Rg; q.p0 = *P0; q.T0 = *T0;
    return s.finish(launch_inlet_update(f, q, 0));
}

/* ---- Baldwin-Lomax eddy viscosity: src/equations/blomax.f90 ------------- */
static m2d::BlConst g_blomax;   // the module's coefficients (blomax.f90:5-10)

int m2d_set_blomax_coefficients(const double *kappa, const double *Aop, const double *alpha,
                                const double *Ccp, const double *Ckleb, const double *Cwk)
{
    if (!kappa || !Aop || !alpha || !Ccp || !Ckleb || !Cwk) return fail(ST_ARG, "set_blomax_coefficients: null argument");
    g_blomax.kappa = *kappa; g_blomax.Aop = *Aop; g_blomax.alpha = *alpha;
    g_blomax.Ccp = *Ccp; g_blomax.Ckleb = *Ckleb; g_blomax.Cwk = *Cwk;
    return ST_OK;
}

int m2d_get_blomax_coefficients(double *kappa, double *Aop, double *alpha, double *Ccp, double *Ckleb,
                                double *Cwk)
{
    if (!kappa || !Aop || !alpha || !Ccp || !Ckleb || !Cwk) return fail(ST_ARG, "get_blomax_coefficients: null argument");
    *kappa = g_blomax.kappa; *Aop = g_blomax.Aop; *alpha = g_blomax.alpha;
    *Ccp = g_blomax.Ccp; *Ckleb = g_blomax.Ckleb; *Cwk = g_blomax.Cwk;
    return ST_OK;
}

int m2d_initialize_blomax(const int *nx, const int *ny, const double *x, const double *y)
{
    CHK;
    if (!x || !y) return fail(ST_ARG, "initialize_blomax: null argument");
    return ST_OK;   // the vorticity metrics are evaluated inside the kernel
}

int m2d_get_eddy_viscosity_blomax(const int *nx, const int *ny, const double *x, const double *y,
    const double *xp, const double *yp, const double *xk, const double *yk, const double *Jp,
    const double *Jn, const double *vln, const double *ro, const double *ron, const double *u,
    const double *v, double *vtp)
{
    CHK;
    if (*ny < 5) return fail(ST_ARG, "get_eddy_viscosity_blomax: ny < 5");
    Stage s; size_t N = ND_;
    const double *dx = s.in(x, N), *dy = s.in(y, N), *dxp = s.in(xp, N), *dyp = s.in(yp, N);
    const double *dxk = s.in(xk, N), *dyk = s.in(yk, N), *dJp = s.in(Jp, N), *dJn = s.in(Jn, N);
    const double *dvln = s.in(vln, N), *dro = s.in(ro, N), *dron = s.in(ron, N);
    const double *du = s.in(u, N), *dv = s.in(v, N);
    double *dvtp = s.inout(vtp, N);
    if (s.status) return s.status;
    return s.finish(launch_blomax(*nx, *ny, g_blomax, dx, dy, dxp, dyp, dxk, dyk, dJp, dJn, dvln, dro, dron,
                                  du, dv, dvtp, 0));
}

int m2d_get_eddy_viscosity_fictitious(const int *nx, const int *ny, double *phi)
{
    CHK; Stage s; size_t N = ND_;
    double *d = s.inout(phi, N);
    if (s.status) return s.status;
    return s.finish(launch_blomax_fictitious(*nx, *ny, d, 0));
}

/* ---- thermophysical model: src/thermophysical/ ------------------------- */
static const m2d_mixture *mixture_in(Stage &s, const m2d_mixture *h)
{
    if (!h) { s.status = s.status ? s.status : ST_ARG; m2d_set_last_error_msg("null mixture"); return nullptr; }
    double *d = s.alloc(sizeof(m2d_mixture) / sizeof(double) + 1);
    if (d && cudaMemcpy(d, h, sizeof(m2d_mixture), cudaMemcpyHostToDevice) != cudaSuccess) s.status = ST_CUDA;
    return (const m2d_mixture *)d;
}

int m2d_mixture_init(int base, int ngs, const double *fractions, const double *Mi, const double *cpi,
                     const double *mui, const double *kpi, m2d_mixture *out)
{
    // class_thermophysical_mixture%init, mod_class_thermophysical_mixture.f90:56-224
    if (!fractions || !Mi || !cpi || !mui || !kpi || !out || ngs < 1 || (base != 0 && base != 1))
        return fail(ST_ARG, "mixture_init: bad arguments");
    m2d_mixture m;
    memset(&m, 0, sizeof m);
    const double Ru = 8.31451000e+00;
    for (int k = 0; k < ngs; k++) {
        if (!(fractions[k] > 1.0e-8)) continue;          // species below 1e-8 are left out
        if (m.ngs == M2D_MAX_SPECIES) return fail(ST_ARG, "mixture_init: more than 8 species");
        const int q = m.ngs++;
        (base == 0 ? m.Xi : m.Yi)[q] = fractions[k];
        m.Mi[q] = Mi[k];
        for (int c = 0; c < 10; c++) m.cpi[q][c] = cpi[k * 10 + c];
        for (int c = 0; c < 8; c++) { m.mui[q][c] = mui[k * 8 + c]; m.kpi[q][c] = kpi[k * 8 + c]; }
    }
    if (m.ngs == 0) return fail(ST_ARG, "mixture_init: no species");
    double sum = 0.0;
    for (int q = 0; q < m.ngs; q++) sum = sum + (base == 0 ? m.Xi[q] : m.Yi[q]);
    if (std::fabs(1.0 - sum) > 2.220446049250313e-16 * 10.0)
        return fail(ST_ARG, "mixture_init: the fractions do not sum to one");
    double Mg = 0.0;
    if (base == 0) {
        for (int q = 0; q < m.ngs; q++) Mg = Mg + m.Xi[q] * m.Mi[q];
        for (int q = 0; q < m.ngs; q++) m.Yi[q] = m.Xi[q] * m.Mi[q] / Mg;
    } else {
        double t = 0.0;
        for (int q = 0; q < m.ngs; q++) t = t + m.Yi[q] / m.Mi[q];
        for (int q = 0; q < m.ngs; q++) m.Xi[q] = (m.Yi[q] / m.Mi[q]) / t;
        for (int q = 0; q < m.ngs; q++) Mg = Mg + m.Xi[q] * m.Mi[q];
    }
    for (int q = 0; q < m.ngs; q++) m.Ri[q] = Ru / m.Mi[q];
    m.Rg = Ru / Mg;
    *out = m;
    return ST_OK;
}

int m2d_mixture_eval(const m2d_mixture *mix, double T, double *cp, double *mu, double *kp, double *gm)
{
    if (!mix) return fail(ST_ARG, "mixture_eval: null mixture");
    if (cp) *cp = m2d::mix_cp(*mix, T);
    if (mu) *mu = m2d::mix_mu(*mix, T);
    if (kp) *kp = m2d::mix_kp(*mix, T);
    if (gm) *gm = m2d::mix_gm(*mix, T);
    return ST_OK;
}

// ---- grid metrics (src/grid/mod_grid.f90:237-723) ----
int m2d_get_real_centroids_xy(const int *opt, const int *nx, const int *ny, const double *x,
    const double *y, double *xp, double *yp)
{
    CHK;
    if (!opt) return fail(ST_ARG, "get_real_centroids_xy: null opt");
    Stage s; size_t N = ND_;
    const double *dx = s.in(x, N), *dy = s.in(y, N);
    double *dxp = s.out(xp, N), *dyp = s.out(yp, N);
    if (s.status) return s.status;
    return s.finish(launch_centroids(*opt, *nx, *ny, dx, dy, dxp, dyp, 0));
}

int m2d_get_metrics(const int *nx, const int *ny, const double *x, const double *y,
    const double *xp, const double *yp, double *xe, double *ye, double *xen, double *yen,
    double *xk, double *yk, double *xke, double *yke, double *Jp, double *Je, double *Jn,
    double *alphae, double *gamman, double *betae, double *betan)
{
    CHK; Stage s; size_t N = ND_;
    const double *dx = s.in(x, N), *dy = s.in(y, N), *dxp = s.in(xp, N), *dyp = s.in(yp, N);
    Metrics m;
    double **dm[] = {&m.xe, &m.ye, &m.xen, &m.yen, &m.xk, &m.yk, &m.xke, &m.yke, &m.Jp, &m.Je, &m.Jn,
                     &m.alphae, &m.gamman, &m.betae, &m.betan};
    double *hm[] = {xe, ye, xen, yen, xk, yk, xke, yke, Jp, Je, Jn, alphae, gamman, betae, betan};
    for (int k = 0; k < 15; k++) *dm[k] = s.out(hm[k], N);
    if (s.status) return s.status;
    return s.finish(launch_metrics(*nx, *ny, dx, dy, dxp, dyp, m, 0));
}

int m2d_get_radius(const int *coord, const int *nx, const int *ny, const double *y,
    const double *yp, double *radius, double *re, double *rn, double *rp)
{
    CHK;
    if (!coord) return fail(ST_ARG, "get_radius: null coord");
    Stage s; size_t N = ND_;
    const double *dy = s.in(y, N), *dyp = s.in(yp, N);
    double *dr = s.out(radius, N), *de = s.out(re, N), *dn = s.out(rn, N), *dp = s.out(rp, N);
    if (s.status) return s.status;
    return s.finish(launch_radius(*coord, *nx, *ny, dy, dyp, dr, de, dn, dp, 0));
}

int m2d_get_boundary_fields(const int *nx, const int *ny, const double *F, double *Fbn, double *Fbs,
                            double *Fbe, double *Fbw)
{
    CHK; Stage s; size_t N = ND_, X = (size_t)*nx, Y = (size_t)*ny;
    const double *dF = s.in(F, N);
    double *dn = s.inout(Fbn, X), *ds = s.inout(Fbs, X), *de = s.inout(Fbe, Y), *dw = s.inout(Fbw, Y);
    if (s.status) return s.status;
    return s.finish(launch_boundary_fields(*nx, *ny, dF, dn, ds, de, dw, 0));
}

int m2d_set_cp(const m2d_mixture *mix, const int *nx, const int *ny, const double *Tbn,
    const double *Tbs, const double *Tbe, const double *Tbw, const double *T, double *cp)
{
    CHK; Stage s; size_t N = ND_, X = (size_t)*nx, Y = (size_t)*ny;
    const m2d_mixture *dm = mixture_in(s, mix);
    const double *dn = s.in(Tbn, X), *ds = s.in(Tbs, X), *de = s.in(Tbe, Y), *dw = s.in(Tbw, Y), *dT = s.in(T, N);
    double *dcp = s.inout(cp, N);
    if (s.status) return s.status;
    return s.finish(launch_set_cp(*nx, *ny, dm, dn, ds, de, dw, dT, dcp, 0));
}

int m2d_set_gamma(const int *nx, const int *ny, const double *Rg, const double *cp, double *gcp)
{
    CHK;
    if (!Rg) return fail(ST_ARG, "set_gamma: null Rg");
    Stage s; size_t N = ND_;
    const double *dcp = s.in(cp, N);
    double *dg = s.inout(gcp, N);
    if (s.status) return s.status;
    return s.finish(launch_set_gamma(*nx, *ny, *Rg, dcp, dg, 0));
}

static int transport_nodes(const m2d_mixture *mix, const int *nx, const int *ny, bool visc, const double *T,
                           double *phip)
{
    CHK; Stage s; size_t N = ND_;
    const m2d_mixture *dm = mixture_in(s, mix);
    const double *dT = s.in(T, N);
    double *dp = s.inout(phip, N);
    if (s.status) return s.status;
    return s.finish(launch_transport_nodes(*nx, *ny, dm, visc, dT, dp, 0));
}
int m2d_set_laminar_viscosity_at_nodes(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *T, double *vlp)
{ return transport_nodes(mix, nx, ny, true, T, vlp); }
int m2d_set_thermal_conductivity_at_nodes(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *T, double *kp)
{ return transport_nodes(mix, nx, ny, false, T, kp); }

static int transport_faces(const m2d_mixture *mix, const int *nx, const int *ny, bool visc, const double *Tbn,
                           const double *Tbs, const double *Tbe, const double *Tbw, const double *phip,
                           double *phie, double *phin)
{
    CHK; Stage s; size_t N = ND_, X = (size_t)*nx, Y = (size_t)*ny;
    const m2d_mixture *dm = mixture_in(s, mix);
    const double *dn = s.in(Tbn, X), *ds = s.in(Tbs, X), *de = s.in(Tbe, Y), *dw = s.in(Tbw, Y);
    const double *dp = s.in(phip, N);
    double *dpe = s.inout(phie, N), *dpn = s.inout(phin, N);
    if (s.status) return s.status;
    return s.finish(launch_transport_faces(*nx, *ny, dm, visc, dn, ds, de, dw, dp, dpe, dpn, 0));
}
int m2d_get_laminar_viscosity_at_faces(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *Tbn, const double *Tbs, const double *Tbe, const double *Tbw,
    const double *vlp, double *vle, double *vln)
{ return transport_faces(mix, nx, ny, true, Tbn, Tbs, Tbe, Tbw, vlp, vle, vln); }
int m2d_get_thermal_conductivity_at_faces(const m2d_mixture *mix, const int *nx, const int *ny,
    const double *Tbn, const double *Tbs, const double *Tbe, const double *Tbw,
    const double *kp, double *ke, double *kn)
{ return transport_faces(mix, nx, ny, false, Tbn, Tbs, Tbe, Tbw, kp, ke, kn); }

// ---- external-flow boundary plug-in (m2d_extflow.cu) --------------------
int m2d_extflow_set_bcu(const int *nx, const int *ny, const int *modvis, const double *UF, const double *xk,
    const double *yk, const double *alphae, const double *betae, const double *u, const double *v, double *au,
    double *bu)
{
    CHK; if (!modvis || !UF) return fail(ST_ARG, "extflow_set_bcu: null argument");
    Stage s; size_t N = ND_;
    ExtArgs A; memset(&A, 0, sizeof A);
    A.nx = *nx; A.ny = *ny; A.scheme = EXT_U; A.modvis = *modvis; A.value = *UF;
    A.xk = s.in(xk, N); A.yk = s.in(yk, N); A.alphae = s.in(alphae, N); A.betae = s.in(betae, N);
    A.u = s.in(u, N); A.v = s.in(v, N);
    double *da = s.inout(au, 9 * N), *db = s.inout(bu, N);
    if (s.status) return s.status;
    return s.finish(launch_extflow_rows(A, da, db, 0));
}

int m2d_extflow_set_bcv(const int *nx, const int *ny, const int *modvis, const double *xk, const double *yk,
    const double *u, const double *v, double *av, double *bv)
{
    CHK; if (!modvis) return fail(ST_ARG, "extflow_set_bcv: null argument");
    Stage s; size_t N = ND_;
    ExtArgs A; memset(&A, 0, sizeof A);
    A.nx = *nx; A.ny = *ny; A.scheme = EXT_V; A.modvis = *modvis; A.value = 0.0;
    A.xk = s.in(xk, N); A.yk = s.in(yk, N); A.u = s.in(u, N); A.v = s.in(v, N);
    double *da = s.inout(av, 9 * N), *db = s.inout(bv, N);
    if (s.status) return s.status;
    return s.finish(launch_extflow_rows(A, da, db, 0));
}

int m2d_extflow_set_bcpl(const int *nx, const int *ny, double *ap, double *bp)
{
    CHK;
    Stage s; size_t N = ND_;
    ExtArgs A; memset(&A, 0, sizeof A);
    A.nx = *nx; A.ny = *ny; A.scheme = EXT_PL;
    double *da = s.inout(ap, 5 * N), *db = s.inout(bp, N);
    if (s.status) return s.status;
    return s.finish(launch_extflow_rows(A, da, db, 0));
}

int m2d_extflow_set_bcro(const int *nx, const int *ny, const double *ROF, const double *alphae,
    const double *betae, const double *betan, const double *gamman, double *a9bn, double *a9bs, double *a9be,
    double *a9bw, double *b9bn, double *b9bs, double *b9be, double *b9bw)
{
    CHK; if (!ROF) return fail(ST_ARG, "extflow_set_bcro: null argument");
    Stage s; size_t N = ND_, X = (size_t)*nx, Y = (size_t)*ny;
    ExtArgs A; memset(&A, 0, sizeof A);
    A.nx = *nx; A.ny = *ny; A.scheme = EXT_RO; A.value = *ROF;
    A.alphae = s.in(alphae, N); A.betae = s.in(betae, N); A.betan = s.in(betan, N); A.gamman = s.in(gamman, N);
    double *an = s.out(a9bn, 9 * X), *as = s.out(a9bs, 9 * X), *ae = s.out(a9be, 9 * Y), *aw = s.out(a9bw, 9 * Y);
    double *bn = s.out(b9bn, X), *bs = s.out(b9bs, X), *be = s.out(b9be, Y), *bw = s.out(b9bw, Y);
    if (s.status) return s.status;
    return s.finish(launch_extflow_strips9(A, an, as, ae, aw, bn, bs, be, bw, 0));
}

static int extrapolate_args(const int *nx, const int *ny, const int *itemax, const char *who)
{
    if (!nx || !ny || !itemax) return fail(ST_ARG, who);
    if (!extflow_extrapolate_supported(*nx, *ny) || *itemax < 0) return fail(ST_ARG, who);
    return ST_OK;
}

int m2d_extflow_extrapolate_u_v_to_fictitious(const int *nx, const int *ny, const int *modvis, const int *itemax,
    const double *UF, const double *xk, const double *yk, const double *alphae, const double *betae, double *u,
    double *v)
{
    CHK; if (!modvis || !UF) return fail(ST_ARG, "extflow_extrapolate_u_v_to_fictitious: null argument");
    if (int st = extrapolate_args(nx, ny, itemax, "extflow_extrapolate_u_v_to_fictitious: nx, ny >= 4, "
                                  "max(nx, ny) <= 14336, itemax >= 0")) return st;
    Stage s; size_t N = ND_;
    ExtArgs A; memset(&A, 0, sizeof A);
    A.nx = *nx; A.ny = *ny; A.scheme = EXT_U; A.modvis = *modvis; A.value = *UF;
    A.xk = s.in(xk, N); A.yk = s.in(yk, N); A.alphae = s.in(alphae, N); A.betae = s.in(betae, N);
    double *du = s.inout(u, N), *dv = s.inout(v, N);
    double *strips = s.scratch(extflow_strips_doubles(*nx, *ny));
    if (s.status) return s.status;
    A.u = du; A.v = dv;
    cudaError_t e = launch_extflow_strips9_packed(A, strips, 0);
    if (e == cudaSuccess) e = launch_extflow_extrapolate(*nx, *ny, *itemax, strips, du, 0);
    A.scheme = EXT_V; A.value = 0.0;
    if (e == cudaSuccess) e = launch_extflow_strips9_packed(A, strips, 0);
    if (e == cudaSuccess) e = launch_extflow_extrapolate(*nx, *ny, *itemax, strips, dv, 0);
    return s.finish(e);
}

int m2d_extflow_extrapolate_ro_to_fictitious(const int *nx, const int *ny, const int *itemax, const double *ROF,
    const double *alphae, const double *betae, const double *betan, const double *gamman, double *ro)
{
    CHK; if (!ROF) return fail(ST_ARG, "extflow_extrapolate_ro_to_fictitious: null argument");
    if (int st = extrapolate_args(nx, ny, itemax, "extflow_extrapolate_ro_to_fictitious: nx, ny >= 4, "
                                  "max(nx, ny) <= 14336, itemax >= 0")) return st;
    Stage s; size_t N = ND_;
    ExtArgs A; memset(&A, 0, sizeof A);
    A.nx = *nx; A.ny = *ny; A.scheme = EXT_RO; A.value = *ROF;
    A.alphae = s.in(alphae, N); A.betae = s.in(betae, N); A.betan = s.in(betan, N); A.gamman = s.in(gamman, N);
    double *dro = s.inout(ro, N);
    double *strips = s.scratch(extflow_strips_doubles(*nx, *ny));
    if (s.status) return s.status;
    cudaError_t e = launch_extflow_strips9_packed(A, strips, 0);
    if (e == cudaSuccess) e = launch_extflow_extrapolate(*nx, *ny, *itemax, strips, dro, 0);
    return s.finish(e);
}

int m2d_extflow_calc_main_variables(const int *nx, const int *ny, const double *Rg, const int *modvis,
    const double *PF, const double *TF, const double *UF, const double *rb, const int *iocs, const double *xk,
    const double *yk, const double *rn, const double *Jn, const double *vln, const double *p, const double *u,
    const double *v, const double *Vcn, double *Cdfi, double *Cdfv)
{
    CHK;
    if (!Rg || !modvis || !PF || !TF || !UF || !rb || !iocs || !Cdfi || !Cdfv)
        return fail(ST_ARG, "extflow_calc_main_variables: null argument");
    if (*iocs < 1 || *iocs > *nx) return fail(ST_ARG, "extflow_calc_main_variables: iocs outside 1..nx");
    Stage s; size_t N = ND_;
    DragArgs D; memset(&D, 0, sizeof D);
    D.nx = *nx; D.iiv = 2; D.ifv = *iocs; D.viscous = *modvis == 1;
    D.Rg = *Rg; D.PF = *PF; D.TF = *TF; D.UF = *UF; D.rb = *rb;
    D.xk = s.in(xk, N); D.yk = s.in(yk, N); D.rn = s.in(rn, N); D.Jn = s.in(Jn, N); D.vln = s.in(vln, N);
    D.p = s.in(p, N); D.u = s.in(u, N); D.v = s.in(v, N); D.Vcn = s.in(Vcn, N);
    double cd[2] = {0.0, 0.0};
    double *dcd = s.out(cd, 2);
    if (s.status) return s.status;
    int st = s.finish(launch_extflow_drag(D, dcd, 0));
    if (st == ST_OK) { *Cdfi = cd[0]; *Cdfv = cd[1]; }
    return st;
}

int m2d_extflow_boundary_T_from_H_conservation(const int *nx, const int *ny, const double *CPF, const double *HF,
    const double *u, const double *ue, const double *un, const double *v, const double *ve, const double *vn,
    double *T, double *Tbe, double *Tbw, double *Tbn, double *Tbs)
{
    CHK; if (!CPF || !HF) return fail(ST_ARG, "extflow_boundary_T_from_H_conservation: null argument");
    Stage s; size_t N = ND_, X = (size_t)*nx, Y = (size_t)*ny;
    THArgs H; memset(&H, 0, sizeof H);
    H.nx = *nx; H.ny = *ny; H.CPF = *CPF; H.HF = *HF;
    H.u = s.in(u, N); H.ue = s.in(ue, N); H.un = s.in(un, N); H.v = s.in(v, N); H.ve = s.in(ve, N);
    H.vn = s.in(vn, N);
    double *dT = s.out(T, N);
    double *de = s.inout(Tbe, Y), *dw = s.inout(Tbw, Y), *dn = s.inout(Tbn, X), *ds = s.inout(Tbs, X);
    if (s.status) return s.status;
    return s.finish(launch_extflow_T_from_H(H, dT, de, dw, dn, ds, 0));
}

int m2d_extflow_set_bcT(const int *nx, const int *ny, const double *TF, const double *Tsbc,
    const double *alphae, const double *betae, const double *betan, const double *gamman, double *at, double *bt)
{
    CHK; if (!TF || !Tsbc) return fail(ST_ARG, "extflow_set_bcT: null argument");
    Stage s; size_t N = ND_;
    ExtArgs A; memset(&A, 0, sizeof A);
    A.nx = *nx; A.ny = *ny; A.scheme = EXT_T; A.value = *TF; A.Tsbc = *Tsbc;
    A.alphae = s.in(alphae, N); A.betae = s.in(betae, N); A.betan = s.in(betan, N); A.gamman = s.in(gamman, N);
    double *da = s.inout(at, 9 * N), *db = s.inout(bt, N);
    if (s.status) return s.status;
    return s.finish(launch_extflow_rows(A, da, db, 0));
}

}  // extern "C"
