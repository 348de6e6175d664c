// m2d_ctx.cu -- device-resident SIMPLEC context: one nozzle instance whose
// every field lives in HBM for the whole run.  m2d_iterate is the `it` loop
// body of src/mach2d_main.f90:94-445, launched on one stream; the only host
// round trips are the ones where the reference takes a control decision
// (the p' loop exit, :307-309) and one copy of the iteration's scalars at the
// end (norms, mass residual, convergence coefficients for dt).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include "m2d_blomax.cuh"
#include "m2d_fields.cuh"
#include "m2d_grid.cuh"
#include "m2d_setup.h"
#include "m2d_solvers.cuh"
#include "m2d_thermo.cuh"

using namespace m2d;

namespace {
enum Slot {
    S_PSUM = 0, S_MAXPL, S_NU_A, S_NU_B, S_NV_A, S_NV_B, S_NP, S_NT_A, S_NT_B, S_RMASS,
    S_CC_U, S_CC_V, S_CC_T, S_CC_P, S_FMI, S_FME, S_FD, S_RR = 20,
    // device-resident control of a captured iteration
    S_DT = 30, S_PAVG, S_NORMPL, S_NORM, S_IT, S_COUNT = 40
};
enum ISlot { I_NIT_U = 0, I_NIT_V, I_NIT_P, I_NIT_T, I_ERR, I_ITP, I_ITP_TOTAL, I_COUNT = 8 };

// what the end of an iteration needs to pick the next time step
struct StepCtl {
    int dtmodel, nan_policy, it1, it2, energy_eq, itpmax;
    double dt1, dt2, h0, mincc, maxcc, tolm;
};
}

struct m2d_ctx {
    m2d_case c;
    int device = 0;
    cudaStream_t st = nullptr;
    int nx = 0, ny = 0;
    size_t N = 0;
    Fields f;
    Params q;
    double *arena = nullptr;
    double *ws9[3], *ws5, *P, *Q, *part;   // ws9: u, v and (energy equation) T
    double *dsc = nullptr;
    int *dint = nullptr;
    int *dlag = nullptr;           // MSI factor records (MsiSys::lag), two ints per workspace
    m2d_mixture *dmix = nullptr;   // device copy of c.mix (ktm = 1)
    m2d_unet *net = nullptr;       // learned p' correction (solver 3), not owned
    long long learned_calls = 0, learned_accepted = 0, learned_alone = 0;
    // captured iteration (m2d_ctx_set_graph): the whole `it` body as one CUDA
    // graph, the p' loop a conditional WHILE node, dt and the loop exit on the
    // device
    bool graph_on = false;
    cudaStream_t st2 = nullptr;    // captures the p' loop body
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long launches_fixed = 0, launches_body = 0;
    double *hsc = nullptr;   // pinned mirror of dsc
    int *hint = nullptr;     // pinned mirror of dint
    double *hsc_b = nullptr; // second mirrors and their events: m2d_run keeps two
    int *hint_b = nullptr;   // captured iterations in flight
    cudaEvent_t ev[2] = {nullptr, nullptr};
    double dt = 0, norm = 0, normpl = 0, rmass = 0, p_avg = 0;
    double Href = 0, Cpref = 0, fm1D = 0, Fd1D = 0, Fpv1D = 0, Sg = 0;
    int it = 0, it_stop = -1, itp_used = 0;
    long long launches = 0;   // kernels launched by m2d_iterate so far
    int msi_variant = 0;      // MSI wavefront schedule (MsiLaunch::variant)
};

static int ctx_fail(int code, const char *msg)
{
    extern void m2d_set_last_error_msg(const char *);
    m2d_set_last_error_msg(msg);
    return code;
}

#define TRY(expr)                                                                 \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess) { m2d_set_last_error(_e, #expr, __FILE__, __LINE__); return M2D_ERR_CUDA; } \
    } while (0)

// launch through the context `x`, counting the kernels it starts
#define KL(expr, n)              \
    do {                         \
        TRY(expr);               \
        x->launches += (n);      \
    } while (0)

static double *plane_ptr(m2d_ctx *x, const char *name, long *n)
{
    Fields &f = x->f;
    const long N = (long)x->N;
#define M2D_MATCH(nm) if (!strcmp(name, #nm)) { *n = N; return f.nm; }
    M2D_PLANES(M2D_MATCH)
#undef M2D_MATCH
    if (!strcmp(name, "au")) { *n = 9 * N; return f.au; }
    if (!strcmp(name, "av")) { *n = 9 * N; return f.av; }
    if (!strcmp(name, "at")) { *n = 9 * N; return f.at; }
    if (!strcmp(name, "ap")) { *n = 5 * N; return f.ap; }
    const struct { const char *nm; double *p; long len; } strips[] = {
        {"uin", f.uin, x->ny}, {"vin", f.vin, x->ny}, {"pin", f.pin, x->ny}, {"Tin", f.Tin, x->ny},
        {"Mw", f.Mw, x->ny}, {"plin", f.plin, x->ny}, {"pina", f.pina, x->ny}, {"Tbe", f.Tbe, x->ny},
        {"Tbw", f.Tbw, x->ny}, {"Tbn", f.Tbn, x->nx}, {"Tbs", f.Tbs, x->nx}};
    for (auto &s : strips)
        if (!strcmp(name, s.nm)) { *n = s.len; return s.p; }
    return nullptr;
}

// cp, and for Navier-Stokes vlp, kp and their face values, from T and the
// boundary temperatures (src/mach2d_main.f90:112-149); with `boundary` the
// boundary temperatures are first taken as face averages of T
static cudaError_t mixture_properties(m2d_ctx *x, bool boundary)
{
    Fields &f = x->f;
    const int nx = x->nx, ny = x->ny;
    cudaStream_t st = x->st;
    cudaError_t e = cudaSuccess;
    if (boundary) e = launch_boundary_fields(nx, ny, f.T, f.Tbn, f.Tbs, f.Tbe, f.Tbw, st);
    if (e == cudaSuccess) e = launch_set_cp(nx, ny, x->dmix, f.Tbn, f.Tbs, f.Tbe, f.Tbw, f.T, f.cp, st);
    if (e == cudaSuccess && x->c.modvis == 1) {
        e = launch_transport_nodes(nx, ny, x->dmix, true, f.T, f.vlp, st);
        if (e == cudaSuccess) e = launch_transport_nodes(nx, ny, x->dmix, false, f.T, f.kp, st);
        if (e == cudaSuccess)
            e = launch_transport_faces(nx, ny, x->dmix, true, f.Tbn, f.Tbs, f.Tbe, f.Tbw, f.vlp, f.vle, f.vln, st);
        if (e == cudaSuccess)
            e = launch_transport_faces(nx, ny, x->dmix, false, f.Tbn, f.Tbs, f.Tbe, f.Tbw, f.kp, f.ke, f.kn, st);
    }
    if (boundary) x->launches += 3 + (x->c.modvis == 1 ? 4 : 0);   // counted inside m2d_iterate only
    return e;
}

// The instance set-up on the device (src/mach2d_main.f90:25-84): from the
// grid nodes and the strips the host computed (m2d_setup.cpp), the centroids,
// metrics and radii (mod_grid.f90:237-723), ap(:,3) = 1
// (src/mod_mach2d_data.f90:403), the boundary-face flags and the internal-flow
// initial guess (mod_intflow.f90:1240-1488) in the reference's order; the
// inlet strips, which call pow, come back to the host once.  Then the
// constant or MIXTURE properties and, with dtmodel = 1, the first time step
// (tstepper_dt0_scarborough).  Only the nodes (2 N doubles) and O(nx + ny)
// strips cross PCIe.
static cudaError_t device_setup(m2d_ctx *x, const m2d_case &c, HostInstance &h)
{
    Fields &f = x->f;
    const int nx = x->nx, ny = x->ny;
    const size_t N = x->N;
    cudaStream_t st = x->st;
    cudaError_t e = cudaSuccess;
    auto up = [&](double *d, const std::vector<double> &v) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    };
    auto run = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    up(f.x, h.x);
    up(f.y, h.y);
    up(x->P, h.col);                  // 4 nx <= N doubles of TDMA scratch, cleared below
    run(launch_fill(f.ap + 2 * N, (long long)N, 1.0, st));
    run(launch_centroids(c.kcm, nx, ny, f.x, f.y, f.xp, f.yp, st));
    const Metrics m = {f.xe, f.ye, f.xen, f.yen, f.xk, f.yk, f.xke, f.yke, f.Jp, f.Je, f.Jn,
                       f.alphae, f.gamman, f.betae, f.betan};
    run(launch_metrics(nx, ny, f.x, f.y, f.xp, f.yp, m, st));
    run(launch_radius(c.coord, nx, ny, f.y, f.yp, f.radius, f.re, f.rn, f.rp, st));
    run(launch_boundary_faces_flags(f, st));
    run(launch_initial_columns(f, x->P, st));
    run(launch_extrapolate_uv(f, c.modvis, st));
    run(launch_initial_inlet_u(f, st));
    std::vector<double> uin((size_t)ny, 0.0);
    run(cudaMemcpyAsync(uin.data(), f.uin, (size_t)ny * sizeof(double), cudaMemcpyDeviceToHost, st));
    run(cudaStreamSynchronize(st));
    if (e != cudaSuccess) return e;
    inlet_strips(c, h, uin);
    up(f.vin, h.vin); up(f.pin, h.pin); up(f.Tin, h.Tin); up(f.Mw, h.Mw);
    up(f.Tbe, h.Tbe); up(f.Tbw, h.Tbw); up(f.Tbn, h.Tbn); up(f.Tbs, h.Tbs);
    run(launch_initial_pT_ghosts(f, st));
    run(launch_velocities_at_boundary_faces(f, c.modvis, st));
    run(launch_density_at_nodes(f, h.Rg, st));
    run(launch_density_at_faces(f, c.beta, st));
    // get_cp_mu_kappa_initialization (mod_thermophysical.f90:560-589): constant
    // properties, or the MIXTURE model from the initial T and Tbn..Tbw
    run(cudaMemcpyAsync(x->dmix, &c.mix, sizeof(m2d_mixture), cudaMemcpyHostToDevice, st));
    if (c.ktm != 1) {
        run(launch_fill(f.cp, (long long)N, h.Cpref, st));
        if (c.modvis == 1) {
            for (double *d : {f.vlp, f.vle, f.vln}) run(launch_fill(d, (long long)N, c.mu, st));
            for (double *d : {f.kp, f.ke, f.kn}) run(launch_fill(d, (long long)N, c.kappa, st));
        }
    } else if (e == cudaSuccess) {
        e = mixture_properties(x, false);
    }
    if (c.dtmodel == 1) {
        RedArgs r;
        memset(&r, 0, sizeof r);
        r.kind = RED_DT0; r.nx = nx; r.ny = ny;
        r.u = f.u; r.v = f.v; r.Jp = f.Jp;
        run(launch_reduce(r, x->part, x->P, st));
        run(cudaMemcpyAsync(&h.dt0, x->P, sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    run(cudaMemsetAsync(x->P, 0, N * sizeof(double), st));
    run(cudaStreamSynchronize(st));
    return e;
}

extern "C" int m2d_create(const m2d_case *c, int device, m2d_ctx **out)
{
    if (!c || !out) return ctx_fail(M2D_ERR_ARG, "m2d_create: null argument");
    *out = nullptr;
    if (c->nxr < 3 || c->nyr < 3) return ctx_fail(M2D_ERR_ARG, "m2d_create: need at least 3x3 real volumes");
    if (c->solver != 1 && c->nyr + 2 > msi_max_ny()) return ctx_fail(M2D_ERR_TOO_LARGE, "m2d_create: ny exceeds m2d_msi_max_ny()");
    if (c->ktm != 0 && c->ktm != 1) return ctx_fail(M2D_ERR_ARG, "m2d_create: ktm must be 0 (CONSTANT) or 1 (MIXTURE)");
    if (c->modtur != 0 && !(c->modtur == 1 && c->modvis == 1 && c->prt > 0.0 && c->nyr >= 3))
        return ctx_fail(M2D_ERR_ARG, "m2d_create: modtur = 1 needs modvis = 1 and prt > 0");
    if (c->msi_lag < 0) return ctx_fail(M2D_ERR_ARG, "m2d_create: msi_lag must be >= 0");
    if (c->ktm == 1 && (c->mix.ngs < 1 || c->mix.ngs > M2D_MAX_SPECIES || !(c->mix.Rg > 0.0)))
        return ctx_fail(M2D_ERR_ARG, "m2d_create: ktm = 1 needs a mixture from m2d_mixture_init");
    HostInstance h;
    int rc = build_instance(*c, h);
    if (rc) return ctx_fail(rc, "m2d_create: grid set-up failed");
    m2d_ctx *x = new m2d_ctx();
    x->c = *c;
    x->device = device;
    x->nx = h.nx; x->ny = h.ny;
    x->N = (size_t)h.nx * h.ny;
    const size_t N = x->N;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete x; m2d_set_last_error(e, "cudaSetDevice", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    e = cudaStreamCreateWithFlags(&x->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete x; m2d_set_last_error(e, "cudaStreamCreate", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    // one arena: planes + 9N x 3 + 5N + strips + solver scratch + reductions
#define M2D_COUNT(nm) +1
    const size_t nplanes = 0 M2D_PLANES(M2D_COUNT);
#undef M2D_COUNT
    const size_t strips = (size_t)9 * h.ny + 2 * (size_t)h.nx + 64;
    // a third 9-diagonal workspace when the energy equation is solved, so
    // that T keeps its own factors (lagged factorisation)
    const int n9 = (c->modvis == 0 && c->ktm == 0) ? 2 : 3;
    const size_t solver = (size_t)n9 * msi_work_doubles(9, h.nx, h.ny) + msi_work_doubles(5, h.nx, h.ny) + 4 +
                          2 * N + 4 * 32;
    const size_t mixd = (sizeof(m2d_mixture) + sizeof(double) - 1) / sizeof(double);
    const size_t total = nplanes * N + 32 * N + strips + solver + (size_t)kMaxMultiReduce * red_parts() + 72 +
                         S_COUNT + mixd;
    e = cudaMalloc(&x->arena, total * sizeof(double));
    if (e != cudaSuccess) { cudaStreamDestroy(x->st); delete x; m2d_set_last_error(e, "cudaMalloc", __FILE__, __LINE__); return M2D_ERR_NOMEM; }
    cudaMemsetAsync(x->arena, 0, total * sizeof(double), x->st);
    double *cur = x->arena;
    auto take = [&](size_t n) { double *p = cur; cur += n; return p; };
    Fields &f = x->f;
    memset(&f, 0, sizeof f);
    f.nx = h.nx; f.ny = h.ny;
#define M2D_TAKE(nm) f.nm = take(N);
    M2D_PLANES(M2D_TAKE)
#undef M2D_TAKE
    f.au = take(9 * N); f.av = take(9 * N); f.at = take(9 * N); f.ap = take(5 * N);
    f.uin = take(h.ny); f.vin = take(h.ny); f.pin = take(h.ny); f.Tin = take(h.ny);
    f.Mw = take(h.ny); f.plin = take(h.ny); f.pina = take(h.ny); f.Tbe = take(h.ny); f.Tbw = take(h.ny);
    f.Tbn = take(h.nx); f.Tbs = take(h.nx);
    // MSI scratch starts on 256-byte boundaries (one line per warp step)
    auto take_aligned = [&](size_t n) { cur = x->arena + (((size_t)(cur - x->arena) + 31) / 32) * 32; return take(n); };
    x->ws9[2] = nullptr;
    for (int k = 0; k < n9; k++) x->ws9[k] = take_aligned(msi_work_doubles(9, h.nx, h.ny));
    x->ws5 = take_aligned(msi_work_doubles(5, h.nx, h.ny) + 4);   // + the rr words of m2d_msi_workspace_doubles
    x->P = take(N); x->Q = take(N);
    x->part = take((size_t)kMaxMultiReduce * red_parts() + 8);
    x->dsc = take(S_COUNT);
    x->dint = (int *)take(I_COUNT);
    x->dlag = (int *)take(4);   // factor records of ws9[0], ws9[1], ws5, ws9[2] (zeroed: no factors yet)
    x->dmix = (m2d_mixture *)take(mixd);
    if ((size_t)(cur - x->arena) > total) { m2d_destroy(x); return ctx_fail(M2D_ERR_NOMEM, "m2d_create: arena overflow"); }
    e = cudaMallocHost(&x->hsc, S_COUNT * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&x->hint, I_COUNT * sizeof(int));
    if (e != cudaSuccess) { m2d_destroy(x); m2d_set_last_error(e, "cudaMallocHost", __FILE__, __LINE__); return M2D_ERR_NOMEM; }
    e = device_setup(x, *c, h);
    if (e != cudaSuccess) { m2d_destroy(x); m2d_set_last_error(e, "set-up", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    Params &q = x->q;
    memset(&q, 0, sizeof q);
    q.modvis = c->modvis; q.coord = c->coord; q.beta = c->beta; q.Rg = h.Rg; q.gamma = h.gamma;
    q.p0 = c->p0; q.T0 = c->T0; q.Cpref = h.Cpref; q.Href = h.Href; q.Twall = c->Twall;
    x->Href = h.Href; x->Cpref = h.Cpref; x->fm1D = h.fm1D; x->Fd1D = h.Fd1D; x->Fpv1D = h.Fpv1D;
    x->Sg = h.Sg; x->dt = h.dt0;
    *out = x;
    return M2D_OK;
}

extern "C" int m2d_destroy(m2d_ctx *x)
{
    if (!x) return M2D_OK;
    if (x->st) cudaStreamSynchronize(x->st);
    if (x->exec) cudaGraphExecDestroy(x->exec);
    if (x->graph) cudaGraphDestroy(x->graph);
    if (x->st2) cudaStreamDestroy(x->st2);
    if (x->arena) cudaFree(x->arena);
    if (x->hsc) cudaFreeHost(x->hsc);
    if (x->hint) cudaFreeHost(x->hint);
    if (x->hsc_b) cudaFreeHost(x->hsc_b);
    if (x->hint_b) cudaFreeHost(x->hint_b);
    for (cudaEvent_t e : x->ev)
        if (e) cudaEventDestroy(e);
    if (x->st) cudaStreamDestroy(x->st);
    delete x;
    return M2D_OK;
}

extern "C" int m2d_dims(const m2d_ctx *x, int *nx, int *ny)
{
    if (!x) return ctx_fail(M2D_ERR_ARG, "m2d_dims: null context");
    if (nx) *nx = x->nx;
    if (ny) *ny = x->ny;
    return M2D_OK;
}

static RedArgs red(const m2d_ctx *x, int kind)
{
    RedArgs r;
    memset(&r, 0, sizeof r);
    r.kind = kind; r.nx = x->nx; r.ny = x->ny;
    return r;
}

// linear solves of the iteration: solver9d%solve / solver5d%solve, on stream s
static int solve9(m2d_ctx *x, cudaStream_t s, int nsys, double *const *a, double *const *b, double *const *v,
                  const int *islot, const int *rslot)
{
    const m2d_case &c = x->c;
    if (c.solver != 1) {
        MsiLaunch L;
        memset(&L, 0, sizeof L);
        L.nx = x->nx; L.ny = x->ny; L.nitm = c.nitm_u; L.tol = c.tol_u;
        L.prec = (c.solver >= 2) ? 1 : 0;
        L.variant = x->msi_variant;
        L.err = x->dint + I_ERR;
        L.lag_max = L.prec == 1 ? c.msi_lag : 0;
        for (int k = 0; k < nsys; k++) {
            L.s[k].a = a[k]; L.s[k].b = b[k]; L.s[k].x = v[k];
            const bool t_eq = islot[k] == I_NIT_T && x->ws9[2];
            L.s[k].ws = t_eq ? x->ws9[2] : x->ws9[k];
            L.s[k].nit = x->dint + islot[k]; L.s[k].rr = x->dsc + rslot[k];
            L.s[k].lag = x->dlag + (t_eq ? 6 : 2 * k);
            L.s[k].tag = 1 + islot[k];   // the equation (u, v or T) owns the factors
        }
        KL(launch_msi(9, L, nsys, s), msi_last_launch_count());
    } else {
        for (int k = 0; k < nsys; k++)
            KL(launch_tdma(9, x->nx, x->ny, c.nitm_u, a[k], b[k], v[k], x->P, x->Q, s), 4 * c.nitm_u);
    }
    return M2D_OK;
}

static int solve5(m2d_ctx *x, cudaStream_t s)
{
    const m2d_case &c = x->c;
    if (c.solver == 3 || c.solver == 4) {
        // flexible p' solve: the network's correction, then MSI with FP32
        // sweeps; with solver 4 a kept correction that already meets MSI's
        // stopping test is the whole solve
        if (!x->net) return ctx_fail(M2D_ERR_ARG, "m2d_iterate: solvers 3 and 4 need a network (m2d_ctx_set_unet)");
        m2d_learned_report r;
        const int rc = pprime_solve_learned_lagged(x->net, x->nx, x->ny, c.nitm_p, c.tol_p, x->f.ap, x->f.bp,
                                                   x->f.pl, x->f.Jp, x->ws5, c.solver == 4 ? 3 : 1, s, &r,
                                                   x->dlag + 4, 1 + I_NIT_P, c.msi_lag);
        if (rc) return rc;
        x->learned_calls++;
        x->learned_accepted += r.accepted;
        if (r.accepted && r.nit == 0) x->learned_alone++;
        return M2D_OK;
    }
    if (c.solver != 1) {
        MsiLaunch L;
        memset(&L, 0, sizeof L);
        L.nx = x->nx; L.ny = x->ny; L.nitm = c.nitm_p; L.tol = c.tol_p;
        L.prec = (c.solver >= 2) ? 1 : 0;
        L.variant = x->msi_variant;
        L.err = x->dint + I_ERR;
        L.s[0].a = x->f.ap; L.s[0].b = x->f.bp; L.s[0].x = x->f.pl;
        L.s[0].ws = x->ws5;
        L.s[0].nit = x->dint + I_NIT_P; L.s[0].rr = x->dsc + S_RR + 4;
        L.lag_max = L.prec == 1 ? c.msi_lag : 0;
        L.s[0].lag = x->dlag + 4;
        L.s[0].tag = 1 + I_NIT_P;
        KL(launch_msi(5, L, 1, s), msi_last_launch_count());
    } else {
        KL(launch_tdma(5, x->nx, x->ny, c.nitm_p, x->f.ap, x->f.bp, x->f.pl, x->P, x->Q, s), 4 * c.nitm_p);
    }
    return M2D_OK;
}

// ---- end-of-iteration scalars, the same arithmetic on the host and on the
// device: the outer norm (src/mach2d_main.f90:338-395) and the next time step
// (tstepper_dt, mod_tstepper_scarborough.f90:80-123 / the ramp)
__host__ __device__ static inline bool is_nan(double v) { return v != v; }
__host__ __device__ static inline double ctl_max4(double a, double b, double c, double d, int nan_policy)
{
    const double v[4] = {a, b, c, d};
    if (nan_policy == 1) {
        for (int k = 0; k < 4; k++) if (is_nan(v[k])) return v[k];
        double m = a;
        for (int k = 1; k < 4; k++) if (v[k] > m) m = v[k];
        return m;
    }
    double m = 0.0;
    bool have = false;
    for (int k = 0; k < 4; k++) {
        if (is_nan(v[k])) continue;
        if (!have || v[k] > m) { m = v[k]; have = true; }
    }
    return have ? m : a + b + c + d;   // all NaN: a NaN
}
__host__ __device__ static inline double ctl_ramp_dt(int it, const StepCtl &k)
{
    double dt = 0.0;
    if (it + 1 <= k.it1) dt = k.dt1;
    if (it + 1 > k.it1 && it + 1 < k.it2) dt = k.dt1 + (k.dt2 - k.dt1) * (double)(it + 1 - k.it1) / (double)(k.it2 - k.it1);
    if (it + 1 >= k.it2) dt = k.dt2;
    return dt;
}
__host__ __device__ static inline void ctl_finish(const StepCtl &k, const double *hs, int it, double dt, double *norm,
                                                  double *dt_next)
{
    const double eps = 10.0 * 2.220446049250313e-16;
    double n = 0.0;
    n = n + (hs[S_NU_B] > eps ? hs[S_NU_A] / hs[S_NU_B] : hs[S_NU_A]);
    n = n + (hs[S_NV_B] > eps ? hs[S_NV_A] / hs[S_NV_B] : hs[S_NV_A]);
    n = n + hs[S_NP];
    if (k.energy_eq) n = n + (hs[S_NT_B] > eps ? hs[S_NT_A] / hs[S_NT_B] : hs[S_NT_A]);
    *norm = n;
    if (k.dtmodel == 1) {
        const double cc = ctl_max4(hs[S_CC_U], hs[S_CC_V], hs[S_CC_T], hs[S_CC_P], k.nan_policy);
        double hh;
        if (cc < k.mincc) hh = k.h0 * sqrt(1.0 - cc / k.mincc);
        else if (k.maxcc < cc) hh = -(k.h0 * sqrt(cc / k.maxcc - 1.0));
        else hh = 0.0;
        *dt_next = dt * (1.0 + hh);
    } else {
        *dt_next = ctl_ramp_dt(it, k);
    }
}
static StepCtl step_ctl(const m2d_case &c)
{
    StepCtl k;
    k.dtmodel = c.dtmodel; k.nan_policy = c.nan_policy; k.it1 = c.it1; k.it2 = c.it2;
    k.energy_eq = !(c.modvis == 0 && c.ktm == 0); k.itpmax = c.itpmax;
    k.dt1 = c.dt1; k.dt2 = c.dt2; k.h0 = c.h0; k.mincc = c.mincc; k.maxcc = c.maxcc; k.tolm = c.tolm;
    return k;
}

// device control kernels of a captured iteration (one thread each)
__global__ void k_ctx_pavg(double *dsc, int nx, int ny)
{
    dsc[S_PAVG] = dsc[S_PSUM] / ((double)(nx - 2) * (double)(ny - 2));
}
__global__ void k_ctx_itp_reset(int *dint) { dint[I_ITP] = 0; }
// after a p' cycle: normpl = max|p'| / p_avg (src/mach2d_main.f90:307) and the
// loop's exit (normpl < tolm or itpmax cycles) as the WHILE node's condition
__global__ void k_ctx_itp_decide(double *dsc, int *dint, double tolm, int itpmax, cudaGraphConditionalHandle h)
{
    const int itp = dint[I_ITP] + 1;
    dint[I_ITP] = itp;
    dint[I_ITP_TOTAL] += 1;
    const double normpl = dsc[S_MAXPL] / dsc[S_PAVG];
    dsc[S_NORMPL] = normpl;
    cudaGraphSetConditional(h, (normpl < tolm || itp >= itpmax) ? 0u : 1u);
}
__global__ void k_ctx_finish(double *dsc, StepCtl k)
{
    const int it = (int)dsc[S_IT] + 1;
    double norm, dtn;
    ctl_finish(k, dsc, it, dsc[S_DT], &norm, &dtn);
    dsc[S_NORM] = norm;
    dsc[S_DT] = dtn;
    dsc[S_IT] = (double)it;
}

// one p' cycle on stream s: coefficients, boundary rows, source, solve,
// corrections, face densities and max|p'| (src/mach2d_main.f90:259-309)
static int issue_p_cycle(m2d_ctx *x, const Params &q, cudaStream_t s)
{
    Fields &f = x->f;
    Params qc = q;
    qc.maxpl = x->dsc + S_MAXPL;    // zeroed by the coefficient pass, maximised by the update
    KL(launch_p_assembly_bc(f, qc, s), 1);   // coefficients, boundary rows and source
    int rc = solve5(x, s);
    if (rc) return rc;
    // face corrections, boundary faces, p and rho corrections and max|p'|
    // in one pass (bitwise the separate kernels'), then the face densities,
    // which need the corrected rho of the neighbours
    KL(launch_p_cycle_update(f, x->c.modvis, x->dsc + S_MAXPL, s), 1);
    KL(launch_density_at_faces(f, x->c.beta, s), 1);
    return M2D_OK;
}

// during a capture of x->st: a conditional WHILE node whose body (captured on
// x->st2) is one p' cycle followed by k_ctx_itp_decide
static int capture_p_loop(m2d_ctx *x, const Params &q)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    TRY(cudaStreamGetCaptureInfo(x->st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphConditionalHandle h;
    TRY(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    TRY(cudaGraphAddNode(&node, g, deps, nd, &cp));
    TRY(cudaStreamUpdateCaptureDependencies(x->st, &node, 1, cudaStreamSetCaptureDependencies));
    TRY(cudaStreamBeginCaptureToGraph(x->st2, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed));
    const long long l0 = x->launches;
    int rc = issue_p_cycle(x, q, x->st2);
    if (rc == M2D_OK) {
        k_ctx_itp_decide<<<1, 1, 0, x->st2>>>(x->dsc, x->dint, x->c.tolm, x->c.itpmax, h);
        x->launches++;
    }
    cudaGraph_t body = nullptr;
    const cudaError_t e = cudaStreamEndCapture(x->st2, &body);
    x->launches_body = x->launches - l0;
    if (rc) return rc;
    TRY(e);
    TRY(cudaGetLastError());
    return M2D_OK;
}

// the launches of one outer iteration, src/mach2d_main.f90:94-445.  Host mode:
// the p' loop exit is read back after each cycle.  Capture mode: the p' loop
// is captured as a WHILE node, p_avg and the end-of-iteration scalars are
// computed on the device, and nothing is read back.
static int issue_iteration(m2d_ctx *x, bool capture, int *itp_used_out)
{
    const m2d_case &c = x->c;
    Fields &f = x->f;
    Params q = x->q;
    cudaStream_t st = x->st;
    if (capture) q.dtp = x->dsc + S_DT;
    else q.dt = x->dt;
    TRY(cudaMemsetAsync(x->dint, 0, I_COUNT * sizeof(int), st));
    KL(launch_backup(f, st), 1);
    KL(launch_inlet_update(f, q, st), 1);
    if (c.ktm == 1) TRY(mixture_properties(x, true));
    if (c.modvis == 1 && c.modtur == 1) {
        // Baldwin-Lomax eddy viscosity from the previous iteration's flow
        // (blomax.f90:285-490) added to the laminar transport coefficients
        const BlConst blc;
        KL(launch_blomax(x->nx, x->ny, blc, f.x, f.y, f.xp, f.yp, f.xk, f.yk, f.Jp, f.Jn, f.vln, f.ro, f.ron, f.u,
                         f.v, f.vtp, st), 1);
        KL(launch_blomax_fictitious(x->nx, x->ny, f.vtp, st), 1);
        KL(launch_add_eddy(x->nx, x->ny, c.ktm, c.mu, c.kappa, c.prt, f.vtp, f.cp, f.vlp, f.vle, f.vln, f.kp, f.ke,
                           f.kn, st), 1);
    }
    {
        RedArgs r = red(x, RED_SUM_REAL); r.x = f.p;
        KL(launch_reduce(r, x->part, x->dsc + S_PSUM, st), 1);
    }
    KL(launch_g(f, q.Rg, st), 1);
    if (capture) {
        k_ctx_pavg<<<1, 1, 0, st>>>(x->dsc, x->nx, x->ny);
        KL(cudaGetLastError(), 1);
    } else {
        TRY(cudaMemcpyAsync(x->hsc, x->dsc, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    bool have_pavg = false;
    int itp_used = 0;
    for (int itm = 1; itm <= c.itmmax; itm++) {
        // u and v coefficients, sources and boundary rows in one launch
        KL(launch_uv_assembly_bc(f, q, c.modvis, st), 1);
        KL(launch_internal_simplec(f, st), 1);
        KL(launch_boundary_simplec(f, st), 1);
        {
            double *a[2] = {f.au, f.av}, *b[2] = {f.bu, f.bv}, *v[2] = {f.u, f.v};
            int is[2] = {I_NIT_U, I_NIT_V}, rs[2] = {S_RR, S_RR + 2};
            int rc = solve9(x, st, 2, a, b, v, is, rs);
            if (rc) return rc;
        }
        {
            // the u and v norms (norm_l1_9d, norm_l1_b) in one launch
            RedArgs r[4];
            r[0] = red(x, RED_NORM_L1_9D); r[0].a = f.au; r[0].b = f.bu; r[0].x = f.u;
            r[1] = r[0]; r[1].kind = RED_SUM_ABS_B;
            r[2] = red(x, RED_NORM_L1_9D); r[2].a = f.av; r[2].b = f.bv; r[2].x = f.v;
            r[3] = r[2]; r[3].kind = RED_SUM_ABS_B;
            double *out[4] = {x->dsc + S_NU_A, x->dsc + S_NU_B, x->dsc + S_NV_A, x->dsc + S_NV_B};
            KL(launch_reduce_multi(r, out, 4, x->part, st), 1);
        }
        KL(launch_faces_all(f, q.dt, c.modvis, st, q.dtp), 1);   // internal and boundary faces
        TRY(cudaMemsetAsync(f.pl, 0, x->N * sizeof(double), st));
        if (capture) {
            k_ctx_itp_reset<<<1, 1, 0, st>>>(x->dint);
            KL(cudaGetLastError(), 1);
            int rc = capture_p_loop(x, q);
            if (rc) return rc;
        } else {
            for (int itp = 1; itp <= c.itpmax; itp++) {
                itp_used = itp;
                int rc = issue_p_cycle(x, q, st);
                if (rc) return rc;
                TRY(cudaMemcpyAsync(x->hsc + S_MAXPL, x->dsc + S_MAXPL, sizeof(double), cudaMemcpyDeviceToHost, st));
                TRY(cudaStreamSynchronize(st));
                if (!have_pavg) {
                    x->p_avg = x->hsc[S_PSUM] / ((double)(x->nx - 2) * (double)(x->ny - 2));
                    have_pavg = true;
                }
                x->normpl = x->hsc[S_MAXPL] / x->p_avg;
                if (x->normpl < c.tolm) break;
            }
        }
        {
            RedArgs r = red(x, RED_NORM_L1_5D); r.a = f.ap; r.b = f.bp; r.x = f.pl;
            KL(launch_reduce(r, x->part, x->dsc + S_NP, st), 1);
        }
        KL(launch_uv_nodes_correction(f, st), 1);
        KL(launch_extrapolate_uv(f, c.modvis, st), 1);
    }
    {
        RedArgs r = red(x, RED_MASS);
        r.rp = f.rp; r.re = f.re; r.rn = f.rn; r.Jp = f.Jp; r.ro = f.ro; r.roa = f.roa;
        r.ron = f.ron; r.roe = f.roe; r.Uce = f.Uce; r.Vcn = f.Vcn; r.dt = q.dt; r.dtp = q.dtp;
        KL(launch_reduce(r, x->part, x->dsc + S_RMASS, st), 1);
    }
    // T from total-enthalpy conservation for Euler with constant properties
    // only (src/mach2d_main.f90:357-359); otherwise the energy equation
    const bool h_conservation = (c.modvis == 0 && c.ktm == 0);
    if (h_conservation) {
        KL(launch_T_from_H(f, x->Href, x->Cpref, st), 2);
    } else {
        KL(launch_T_assembly(f, q, st), 1);
        KL(launch_set_bcT(f, c.Twall, st), 1);
        double *a[1] = {f.at}, *b[1] = {f.bt}, *v[1] = {f.T};
        int is[1] = {I_NIT_T}, rs[1] = {S_RR + 6};
        int rc = solve9(x, st, 1, a, b, v, is, rs);
        if (rc) return rc;
        RedArgs r[2];
        r[0] = red(x, RED_NORM_L1_9D); r[0].a = f.at; r[0].b = f.bt; r[0].x = f.T;
        r[1] = r[0]; r[1].kind = RED_SUM_ABS_B;
        double *out[2] = {x->dsc + S_NT_A, x->dsc + S_NT_B};
        KL(launch_reduce_multi(r, out, 2, x->part, st), 1);
    }
    KL(launch_density_at_nodes(f, q.Rg, st), 1);
    KL(launch_density_at_faces(f, c.beta, st), 1);
    if (c.dtmodel == 1) {
        // the four mean convergence coefficients (get_mean_cc_9d/5d) in one launch
        RedArgs r[4];
        r[0] = red(x, RED_MEAN_CC_9D); r[0].a = f.au;
        r[1] = r[0]; r[1].a = f.av;
        r[2] = r[0]; r[2].a = f.at;
        r[3] = red(x, RED_MEAN_CC_5D); r[3].a = f.ap;
        double *out[4] = {x->dsc + S_CC_U, x->dsc + S_CC_V, x->dsc + S_CC_T, x->dsc + S_CC_P};
        KL(launch_reduce_multi(r, out, 4, x->part, st), 1);
    }
    KL(launch_mass_flow_thrust(f, x->dsc + S_FMI, st), 1);
    if (capture) {
        k_ctx_finish<<<1, 1, 0, st>>>(x->dsc, step_ctl(c));
        KL(cudaGetLastError(), 1);
    }
    *itp_used_out = itp_used;
    return M2D_OK;
}

// captures issue_iteration once into x->exec
static int build_graph(m2d_ctx *x)
{
    if (!x->st2) TRY(cudaStreamCreateWithFlags(&x->st2, cudaStreamNonBlocking));
    TRY(cudaStreamBeginCapture(x->st, cudaStreamCaptureModeRelaxed));
    const long long l0 = x->launches;
    int itp = 0;
    const int rc = issue_iteration(x, true, &itp);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(x->st, &g);
    const long long captured = x->launches - l0;
    x->launches = l0;                       // capturing launches nothing
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        if (rc) return rc;
        m2d_set_last_error(e, "m2d_iterate: capture", __FILE__, __LINE__);
        return M2D_ERR_CUDA;
    }
    x->launches_fixed = captured - (long long)x->c.itmmax * x->launches_body;
    cudaError_t ei = cudaGraphInstantiate(&x->exec, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        m2d_set_last_error(ei, "m2d_iterate: cudaGraphInstantiate", __FILE__, __LINE__);
        return M2D_ERR_CUDA;
    }
    x->graph = g;
    return M2D_OK;
}

extern "C" int m2d_ctx_set_msi_schedule(m2d_ctx *x, int variant)
{
    if (!x || variant < 0 || variant > 3) return ctx_fail(M2D_ERR_ARG, "m2d_ctx_set_msi_schedule: variant 0..3");
    TRY(cudaSetDevice(x->device));
    if (variant != x->msi_variant && x->exec) {
        // the captured iteration holds the old schedule's launches
        TRY(cudaStreamSynchronize(x->st));
        cudaGraphExecDestroy(x->exec);
        cudaGraphDestroy(x->graph);
        x->exec = nullptr;
        x->graph = nullptr;
    }
    x->msi_variant = variant;
    return M2D_OK;
}

extern "C" int m2d_ctx_set_graph(m2d_ctx *x, int on)
{
    if (!x) return ctx_fail(M2D_ERR_ARG, "m2d_ctx_set_graph: null context");
    if (on && x->c.solver >= 3)
        return ctx_fail(M2D_ERR_ARG, "m2d_ctx_set_graph: solvers 3 and 4 decide on the host and are not captured");
    TRY(cudaSetDevice(x->device));
    if (on && !x->graph_on) {
        // the device copies of dt and of the iteration counter start from the host's
        x->hsc[S_DT] = x->dt;
        x->hsc[S_IT] = (double)x->it;
        TRY(cudaMemcpyAsync(x->dsc + S_DT, x->hsc + S_DT, sizeof(double), cudaMemcpyHostToDevice, x->st));
        TRY(cudaMemcpyAsync(x->dsc + S_IT, x->hsc + S_IT, sizeof(double), cudaMemcpyHostToDevice, x->st));
        TRY(cudaStreamSynchronize(x->st));
    }
    x->graph_on = on != 0;
    return M2D_OK;
}

// The report and the checks that close an iteration, once its scalars are
// in the pinned mirrors (src/mach2d_main.f90:420-443)
static int finish_iteration(m2d_ctx *x, int it, int itp_used, m2d_report *rep)
{
    const m2d_case &c = x->c;
    const double *hs = x->hsc;
    x->rmass = hs[S_RMASS];
    x->itp_used = itp_used;
    if (rep) {
        rep->it = it; rep->dt = x->dt; rep->norm = x->norm; rep->normpl = x->normpl;
        rep->rmass = x->rmass; rep->fmi = hs[S_FMI]; rep->fme = hs[S_FME]; rep->Fd = hs[S_FD];
        rep->itp_used = itp_used;
    }
    if (x->hint[I_ERR] & ERR_SPIN_TIMEOUT) return ctx_fail(M2D_ERR_TIMEOUT, "m2d_iterate: a bounded device-side wait ran out");
    if (x->hint[I_ERR] & ERR_WAIT_TIMEOUT) return ctx_fail(M2D_ERR_TIMEOUT, "m2d_iterate: MSI iteration cap reached");
    if (std::isnan(x->norm)) return ctx_fail(M2D_ERR_NAN, "m2d_iterate: NaN detected");
    if (x->normpl < c.tolt && x->it_stop < 0) x->it_stop = it * 2;
    return M2D_OK;
}

// Captured iterations in two halves, so that a batch can keep every
// instance's iteration in flight at once: the first queues the iteration's
// graph and the copies of its scalars on the instance's stream and returns;
// the second waits for that stream and closes the iteration.  m2d_iterate in
// graph mode is the two back to back.
bool ctx_graph_on(const m2d_ctx *x) { return x && x->graph_on; }

int ctx_iterate_launch(m2d_ctx *x)
{
    TRY(cudaSetDevice(x->device));
    ++x->it;
    if (!x->exec) {
        int rc = build_graph(x);
        if (rc) { x->it--; return rc; }
    }
    cudaStream_t st = x->st;
    TRY(cudaGraphLaunch(x->exec, st));
    TRY(cudaMemcpyAsync(x->hsc, x->dsc, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
    TRY(cudaMemcpyAsync(x->hint, x->dint, I_COUNT * sizeof(int), cudaMemcpyDeviceToHost, st));
    return M2D_OK;
}

int ctx_iterate_complete(m2d_ctx *x, m2d_report *rep)
{
    TRY(cudaSetDevice(x->device));
    TRY(cudaStreamSynchronize(x->st));
    const double *hs = x->hsc;
    const int itp_used = x->hint[I_ITP];
    x->launches += x->launches_fixed + x->launches_body * x->hint[I_ITP_TOTAL];
    x->p_avg = hs[S_PAVG];
    x->normpl = hs[S_NORMPL];
    x->norm = hs[S_NORM];
    x->dt = hs[S_DT];
    return finish_iteration(x, x->it, itp_used, rep);
}

extern "C" int m2d_iterate(m2d_ctx *x, m2d_report *rep)
{
    if (!x) return ctx_fail(M2D_ERR_ARG, "m2d_iterate: null context");
    if (x->graph_on) {
        const int rc = ctx_iterate_launch(x);
        if (rc) return rc;
        return ctx_iterate_complete(x, rep);
    }
    TRY(cudaSetDevice(x->device));
    const m2d_case &c = x->c;
    cudaStream_t st = x->st;
    const int it = ++x->it;
    int itp_used = 0;
    const double *hs = x->hsc;
    int rc = issue_iteration(x, false, &itp_used);
    if (rc) return rc;
    TRY(cudaMemcpyAsync(x->hsc, x->dsc, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
    TRY(cudaMemcpyAsync(x->hint, x->dint, I_COUNT * sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    double norm, dtn;
    ctl_finish(step_ctl(c), hs, it, x->dt, &norm, &dtn);
    x->norm = norm;
    x->dt = dtn;
    return finish_iteration(x, it, itp_used, rep);
}

// m2d_run with captured iterations: two iterations in flight, so that the GPU
// does not wait for the host's turn between them.  Iteration k+1 is queued
// before iteration k's scalars are read; the stop rule's iteration (it_stop
// = 2 it of the first iteration below tolt) is always known an iteration
// ahead, so no iteration past the stop or past itmax starts, and every
// report is the one m2d_iterate gives.  When an iteration fails, the one
// queued behind it still runs before the error returns (the context then
// counts both).
static int run_pipelined(m2d_ctx *x, int itmax, m2d_report *last)
{
    TRY(cudaSetDevice(x->device));
    if (!x->hsc_b) TRY(cudaMallocHost(&x->hsc_b, S_COUNT * sizeof(double)));
    if (!x->hint_b) TRY(cudaMallocHost(&x->hint_b, I_COUNT * sizeof(int)));
    for (cudaEvent_t &e : x->ev)
        if (!e) TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (!x->exec) {
        const int rc = build_graph(x);
        if (rc) return rc;
    }
    double *hs[2] = {x->hsc, x->hsc_b};
    int *hi[2] = {x->hint, x->hint_b};
    cudaStream_t st = x->st;
    auto queue = [&](int slot) -> cudaError_t {
        cudaError_t e = cudaGraphLaunch(x->exec, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hs[slot], x->dsc, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hi[slot], x->dint, I_COUNT * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(x->ev[slot], st);
        return e;
    };
    const int it0 = x->it;
    TRY(queue(0));
    for (int k = 1; k <= itmax; k++) {
        const int slot = (k - 1) & 1, itk = it0 + k;
        const bool more = k < itmax && !(x->it_stop >= 0 && itk >= x->it_stop);
        if (more) {
            const cudaError_t e = queue(slot ^ 1);
            if (e != cudaSuccess) {
                cudaStreamSynchronize(st);
                x->it = itk;
                m2d_set_last_error(e, "m2d_run: queue an iteration", __FILE__, __LINE__);
                return M2D_ERR_CUDA;
            }
        }
        TRY(cudaEventSynchronize(x->ev[slot]));
        x->hsc = hs[slot]; x->hint = hi[slot];
        x->hsc_b = hs[slot ^ 1]; x->hint_b = hi[slot ^ 1];
        x->it = itk;
        const int itp_used = x->hint[I_ITP];
        x->launches += x->launches_fixed + x->launches_body * x->hint[I_ITP_TOTAL];
        x->p_avg = x->hsc[S_PAVG];
        x->normpl = x->hsc[S_NORMPL];
        x->norm = x->hsc[S_NORM];
        x->dt = x->hsc[S_DT];
        const int rc = finish_iteration(x, itk, itp_used, last);
        if (rc) {
            cudaStreamSynchronize(st);
            if (more) x->it = itk + 1;   // the device ran the queued iteration too
            return rc;
        }
        if (!more || x->it_stop == itk) break;
    }
    return M2D_OK;
}

extern "C" int m2d_run(m2d_ctx *x, int itmax, m2d_report *last)
{
    if (!x) return ctx_fail(M2D_ERR_ARG, "m2d_run: null context");
    if (x->graph_on) return itmax > 0 ? run_pipelined(x, itmax, last) : M2D_OK;
    for (int k = 0; k < itmax; k++) {
        int rc = m2d_iterate(x, last);
        if (rc) return rc;
        if (x->it_stop == x->it) break;
    }
    return M2D_OK;
}

extern "C" int m2d_get_field(m2d_ctx *x, const char *name, double *host, long n)
{
    if (!x || !name || !host) return ctx_fail(M2D_ERR_ARG, "m2d_get_field: null argument");
    long len = 0;
    double *d = plane_ptr(x, name, &len);
    if (!d) return ctx_fail(M2D_ERR_ARG, "m2d_get_field: unknown field");
    if (n < len) return ctx_fail(M2D_ERR_ARG, "m2d_get_field: host buffer too small");
    TRY(cudaSetDevice(x->device));
    TRY(cudaMemcpyAsync(host, d, (size_t)len * sizeof(double), cudaMemcpyDeviceToHost, x->st));
    TRY(cudaStreamSynchronize(x->st));
    return M2D_OK;
}

extern "C" int m2d_set_field(m2d_ctx *x, const char *name, const double *host, long n)
{
    if (!x || !name || !host) return ctx_fail(M2D_ERR_ARG, "m2d_set_field: null argument");
    long len = 0;
    double *d = plane_ptr(x, name, &len);
    if (!d) return ctx_fail(M2D_ERR_ARG, "m2d_set_field: unknown field");
    if (n != len) return ctx_fail(M2D_ERR_ARG, "m2d_set_field: size mismatch");
    TRY(cudaSetDevice(x->device));
    TRY(cudaMemcpyAsync(d, host, (size_t)len * sizeof(double), cudaMemcpyHostToDevice, x->st));
    TRY(cudaStreamSynchronize(x->st));
    return M2D_OK;
}

// several fields per call: one asynchronous copy each, one synchronisation
static int copy_fields(m2d_ctx *x, int count, const char *const *names, double *const *host, const long *n,
                       bool to_device)
{
    if (!x || count < 0 || (count > 0 && (!names || !host || !n)))
        return ctx_fail(M2D_ERR_ARG, "m2d_set_fields/m2d_get_fields: null argument");
    TRY(cudaSetDevice(x->device));
    for (int k = 0; k < count; k++) {
        long len = 0;
        double *d = names[k] ? plane_ptr(x, names[k], &len) : nullptr;
        if (!d || !host[k]) return ctx_fail(M2D_ERR_ARG, "m2d_set_fields/m2d_get_fields: unknown field");
        if (to_device ? n[k] != len : n[k] < len)
            return ctx_fail(M2D_ERR_ARG, "m2d_set_fields/m2d_get_fields: size mismatch");
        if (to_device)
            TRY(cudaMemcpyAsync(d, host[k], (size_t)len * sizeof(double), cudaMemcpyHostToDevice, x->st));
        else
            TRY(cudaMemcpyAsync(host[k], d, (size_t)len * sizeof(double), cudaMemcpyDeviceToHost, x->st));
    }
    TRY(cudaStreamSynchronize(x->st));
    return M2D_OK;
}
extern "C" int m2d_set_fields(m2d_ctx *x, int count, const char *const *names, const double *const *host,
                              const long *n)
{ return copy_fields(x, count, names, const_cast<double *const *>(host), n, true); }
extern "C" int m2d_get_fields(m2d_ctx *x, int count, const char *const *names, double *const *host, const long *n)
{ return copy_fields(x, count, names, host, n, false); }

extern "C" int m2d_get_scalar(const m2d_ctx *x, const char *name, double *out)
{
    if (!x || !name || !out) return ctx_fail(M2D_ERR_ARG, "m2d_get_scalar: null argument");
    const struct { const char *nm; double v; } tab[] = {
        {"dt", x->dt}, {"norm", x->norm}, {"normpl", x->normpl}, {"rmass", x->rmass},
        {"p_avg", x->p_avg}, {"Href", x->Href}, {"Cpref", x->Cpref}, {"fm1D", x->fm1D},
        {"Fd1D", x->Fd1D}, {"Fpv1D", x->Fpv1D}, {"Sg", x->Sg}, {"it", (double)x->it},
        {"it_stop", (double)x->it_stop}, {"itp_used", (double)x->itp_used},
        {"launches", (double)x->launches}, {"nit_u", (double)x->hint[I_NIT_U]}, {"nit_v", (double)x->hint[I_NIT_V]},
        {"nit_p", (double)x->hint[I_NIT_P]}, {"nit_T", (double)x->hint[I_NIT_T]},
        {"learned_calls", (double)x->learned_calls}, {"learned_accepted", (double)x->learned_accepted},
        {"learned_alone", (double)x->learned_alone},
        {"solver", (double)x->c.solver}, {"msi_schedule", (double)x->msi_variant}};
    for (auto &t : tab)
        if (!strcmp(name, t.nm)) { *out = t.v; return M2D_OK; }
    return ctx_fail(M2D_ERR_ARG, "m2d_get_scalar: unknown scalar");
}

extern "C" int m2d_ctx_set_unet(m2d_ctx *x, m2d_unet *net)
{
    if (!x) return ctx_fail(M2D_ERR_ARG, "m2d_ctx_set_unet: null context");
    if (net) {
        int H = 0, W = 0;
        m2d_unet_shape(net, nullptr, &H, &W);
        if (x->nx - 2 > W || x->ny - 2 > H) return ctx_fail(M2D_ERR_ARG, "m2d_ctx_set_unet: network images smaller than the grid");
    }
    x->net = net;
    return M2D_OK;
}

extern "C" int m2d_ctx_stream(const m2d_ctx *x, void **stream)
{
    if (!x || !stream) return ctx_fail(M2D_ERR_ARG, "m2d_ctx_stream: null argument");
    *stream = (void *)x->st;
    return M2D_OK;
}

extern "C" int m2d_ctx_field_device(m2d_ctx *x, const char *name, double **dptr, long *n)
{
    if (!x || !name || !dptr) return ctx_fail(M2D_ERR_ARG, "m2d_ctx_field_device: null argument");
    long len = 0;
    double *d = plane_ptr(x, name, &len);
    if (!d) return ctx_fail(M2D_ERR_ARG, "m2d_ctx_field_device: unknown field");
    *dptr = d;
    if (n) *n = len;
    return M2D_OK;
}

extern "C" int m2d_integrals(m2d_ctx *x, double *fmi, double *fme, double *Fd, double *Cd,
                             double *pwall)
{
    if (!x) return ctx_fail(M2D_ERR_ARG, "m2d_integrals: null context");
    TRY(cudaSetDevice(x->device));
    KL(launch_mass_flow_thrust(x->f, x->dsc + S_FMI, x->st), 1);
    TRY(cudaMemcpyAsync(x->hsc + S_FMI, x->dsc + S_FMI, 3 * sizeof(double), cudaMemcpyDeviceToHost, x->st));
    if (pwall)
        TRY(cudaMemcpyAsync(pwall, x->f.p + (size_t)(x->ny - 2) * x->nx, (size_t)x->nx * sizeof(double),
                            cudaMemcpyDeviceToHost, x->st));
    TRY(cudaStreamSynchronize(x->st));
    if (fmi) *fmi = x->hsc[S_FMI];
    if (fme) *fme = x->hsc[S_FME];
    if (Fd) *Fd = x->hsc[S_FD];
    if (Cd) *Cd = x->hsc[S_FME] / x->fm1D;
    return M2D_OK;
}
