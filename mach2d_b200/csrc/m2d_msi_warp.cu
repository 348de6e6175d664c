// m2d_msi_warp.cu -- cluster wavefront MSI kernel (ny <= 1024).
//
// Same arithmetic as k_msi (m2d_msi.cu), spread over a thread-block cluster:
//   * rows are dealt to "wavefront warps", 32 rows per warp, WPC of them per
//     CTA and up to 16 CTAs per cluster, so one SM serves one or two warps;
//   * within a warp the rows advance in lock step and a row's value reaches
//     the row above through one __shfl_up_sync per step (__shfl_down_sync in
//     the backward sweep); the own-row neighbour stays in registers;
//   * global warp g runs kLag steps behind the plain t = i + 2j schedule of
//     warp g-1, so the value its lane 0 needs from lane 31 of warp g-1 was
//     produced in an earlier batch of kLag steps.  It travels through a ring
//     in the consumer's shared memory (a distributed-shared-memory store when
//     the producer sits in another CTA).  Hand-offs are point to point: after
//     each batch the producer publishes a release counter, the consumer waits
//     for it with an acquire load, and the consumer's own counter tells the
//     producer which ring slots are free again.  No warp waits for anything
//     but its two neighbours, and every wait is bounded (on timeout the
//     kernel records ERR_WAIT_TIMEOUT and runs to its end);
//   * coefficients are prefetched D steps ahead into a rotating register
//     buffer, so the loads never sit on the recurrence;
//   * divisions use the divisor's correctly rounded reciprocal and two FMA
//     correction steps (Markstein's method): the correctly rounded quotient,
//     i.e. exactly the result of IEEE division;
//   * the residual passes and the L2 norm of the stopping test use all
//     threads of all CTAs of the cluster; partial sums are combined in a fixed
//     order in CTA 0 and broadcast, so the stopping decision is deterministic.
// A cell outside the grid (before its row starts, after it ends, rows >= ny)
// produces zeros, which is exactly the zero-neighbour rule of the general
// formula, so results stay bitwise equal to the lexicographic reference loop.
#include <cooperative_groups.h>
#include "m2d_solvers.cuh"

namespace cg = cooperative_groups;

namespace m2d {

namespace {
constexpr int kLag = 16;          // steps per batch = per-warp time lag
constexpr int kRing = 128;        // ring slots; a producer may lead its consumer by 5 batches
constexpr int kLead = (kRing - 2 * kLag) / kLag - 1;
constexpr int kThreads = 256;     // threads per CTA (wavefront warps + helpers)
constexpr int kMaxCluster = 16;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxIterUnbounded = 10000;
constexpr long long kSpinLimit = 1LL << 24;
}

#define PL(p, k, np) (p)[(long long)((k) - 1) * N + (np)]

// a / b from y = RN(1/b): q0 = a y, then two corrections q += (a - q b) y
// with exact FMA remainders.  For |b| in [2^-900, 2^900] and |a| < 2^900,
// a = 0 or |a| > 2^-900, the result is the correctly rounded quotient
// (Markstein, IBM J. Res. Dev. 34, 1990), i.e. the IEEE quotient; for a = 0
// the first product a y already is that quotient.  recip_ok tells when it applies,
// and callers fall back to div_ieee outside that range.
__device__ __forceinline__ double div_recip(double a, double b, double y)
{
    const double q0 = a * y;
    const double r0 = fma(-q0, b, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-q1, b, a);
    return (a == 0.0) ? q0 : fma(r1, y, q1);   // a zero quotient keeps the IEEE sign
}
__device__ __forceinline__ bool recip_ok(double a, double b)
{
    const double fa = fabs(a), fb = fabs(b);
    return fb > 0x1p-900 && fb < 0x1p+900 && fa < 0x1p+900 && (fa > 0x1p-900 || fa == 0.0);
}
__device__ __noinline__ double div_ieee(double a, double b) { return a / b; }
__device__ __forceinline__ double qdiv(double a, double b)
{
    return recip_ok(a, b) ? div_recip(a, b, __drcp_rn(b)) : div_ieee(a, b);
}

__device__ __forceinline__ void stamp(const MsiLaunch &L, int rank, int k)
{
    if (L.prof && rank == 0 && threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        L.prof[k] = t;
    }
}

// cluster-scope release store / acquire load on a (possibly remote) counter
__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.cluster.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.cluster.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// one lane waits until *p >= target (bounded); the warp then proceeds together
__device__ __forceinline__ void warp_wait(const int *p, int target, int lane_waiting, bool &timed_out)
{
    if ((threadIdx.x & 31) == lane_waiting && !timed_out) {
        long long k = 0;
        while (ld_acquire(p) < target) {
            if (++k > kSpinLimit) { timed_out = true; break; }
        }
    }
    __syncwarp();
}

// r = A x - b for one cell, in-range neighbours in ascending diagonal order
template <int ND>
__device__ __forceinline__ double residual_cell(const double *__restrict__ a, const double *__restrict__ b,
                                                const double *x, long long np, int nx, int ny, long long N)
{
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
    return v;
}

// r = A x - b over the cluster (this CTA takes a contiguous slice of cells),
// returns the cluster-wide sum of r^2, identical in every thread.  Starts with
// a cluster barrier: x of every row must be final.
template <int ND>
__device__ double cluster_residual(cg::cluster_group &cl, const double *__restrict__ a,
                                   const double *__restrict__ b, const double *x, double *r,
                                   int nx, int ny, double *red, double *part)
{
    cl.sync();
    const long long N = (long long)nx * ny;
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const long long per = (N + C - 1) / C;
    const long long lo = per * rank, hi = (lo + per < N) ? lo + per : N;
    double acc = 0.0;
    for (long long np = lo + threadIdx.x; np < hi; np += kThreads) {
        const double v = residual_cell<ND>(a, b, x, np, nx, ny, N);
        r[np] = v;
        acc = acc + v * v;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double *p0 = cl.map_shared_rank(part, 0);
        p0[rank] = red[0];
    }
    cl.sync();
    if (rank == 0 && threadIdx.x == 0) {
        double s = 0.0;
        for (int c = 0; c < C; c++) s = s + part[c];
        for (int c = 0; c < C; c++) cl.map_shared_rank(part, c)[kMaxCluster] = s;
    }
    cl.sync();
    return part[kMaxCluster];
}

template <int ND, int WPC, int DLU, int DSW>
__global__ void __launch_bounds__(kThreads, 1) k_msi_c(MsiLaunch L)
{
    constexpr int NU = (ND == 9) ? 4 : 3;
    constexpr int NL = (ND == 9) ? 5 : 4;
    static_assert(kLag % DLU == 0 && kLag % DSW == 0, "prefetch distance must divide kLag");
    // per wavefront warp of this CTA: incoming rings and counters
    __shared__ double ring_up[WPC][kRing][NU];   // from the warp below (LU, forward)
    __shared__ double ring_dn[WPC][kRing];       // from the warp above (backward)
    __shared__ int up_ready[WPC], dn_ready[WPC]; // batches delivered to this warp
    __shared__ int up_done[WPC], dn_done[WPC];   // batches of this warp's output consumed
    __shared__ double red[kThreads];
    __shared__ double part[kMaxCluster + 1];
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int sys = blockIdx.x / C;
    const MsiSys S = L.dev ? L.dev[sys] : L.s[sys];
    const int nx = L.nx, ny = L.ny;
    const long long N = (long long)nx * ny;
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const bool front = wl < WPC;                  // wavefront warp?
    const int NWG = C * WPC;                      // wavefront warps in the cluster
    const int wg = rank * WPC + wl;               // global wavefront warp index
    const int j = wg * 32 + lane;
    const bool row_ok = front && j < ny;
    const int nsteps = ((nx + 2 * (ny - 1) + kLag * (NWG - 1) + kLag - 1) / kLag) * kLag;
    const int nbatch = nsteps / kLag;
    const double *__restrict__ a = S.a;
    double *__restrict__ dl = S.dl;
    double *__restrict__ du = S.du;
    double *wk = S.wk;
    double *x = S.x;
    const long long rowbase = (long long)j * nx;

    if (threadIdx.x < WPC) {
        up_ready[threadIdx.x] = 0; dn_ready[threadIdx.x] = 0;
        up_done[threadIdx.x] = 0; dn_done[threadIdx.x] = 0;
    }
    // links of this warp: up channel (LU, forward) feeds warp g+1, down channel
    // (backward) feeds warp g-1; the partner may sit in a neighbouring CTA
    const bool has_below = front && wg > 0, has_above = front && wg < NWG - 1;
    double *up_ring_dst = nullptr, *dn_ring_dst = nullptr;
    int *up_ready_dst = nullptr, *dn_ready_dst = nullptr, *up_done_dst = nullptr, *dn_done_dst = nullptr;
    if (front) {
        if (has_above) {
            const int cw = (wl + 1 < WPC) ? wl + 1 : 0, cr = (wl + 1 < WPC) ? rank : rank + 1;
            up_ring_dst = cl.map_shared_rank(&ring_up[cw][0][0], cr);
            up_ready_dst = cl.map_shared_rank(&up_ready[cw], cr);
            dn_done_dst = cl.map_shared_rank(&dn_done[cw], cr);
        }
        if (has_below) {
            const int pw = (wl > 0) ? wl - 1 : WPC - 1, pr = (wl > 0) ? rank : rank - 1;
            dn_ring_dst = cl.map_shared_rank(&ring_dn[pw][0], pr);
            dn_ready_dst = cl.map_shared_rank(&dn_ready[pw], pr);
            up_done_dst = cl.map_shared_rank(&up_done[pw], pr);
        }
    }
    cl.sync();   // counters initialised before any remote access
    bool bad_pivot = false, timed_out = false;
    int up_base = 0, dn_base = 0;       // batches already run on each channel
    stamp(L, rank, 0);

    // ---- incomplete LU (lu2d9 msi2d9-v03.f90:277-432, lu2d5 msi2d5-v03.f90:247-330)
    if (front) {
        double mw[NU], a1[NU], a2[NU], a3[NU], buf[DLU][ND];
#pragma unroll
        for (int q = 0; q < NU; q++) { mw[q] = 0.0; a1[q] = 0.0; a2[q] = 0.0; a3[q] = 0.0; }
#pragma unroll
        for (int d = 0; d < DLU; d++) {
            const int ic = d - 2 * j - kLag * wg;           // cell of step d
#pragma unroll
            for (int k = 0; k < ND; k++)
                buf[d][k] = (row_ok && ic >= 0 && ic < nx) ? PL(a, k + 1, rowbase + ic) : 0.0;
        }
        for (int b = 0; b < nbatch; b++) {
            const int tb = b * kLag;
            if (has_below) warp_wait(&up_ready[wl], up_base + b, 0, timed_out);
            if (has_above && b > kLead) warp_wait(&up_done[wl], up_base + b - kLead, 31, timed_out);
#pragma unroll
            for (int kk = 0; kk < kLag; kk++) {
                const int tau = tb + kk;
                const int i = tau - 2 * j - kLag * wg;
                const bool valid = row_ok && i >= 0 && i < nx;
                double cb[ND];
#pragma unroll
                for (int k = 0; k < ND; k++) cb[k] = buf[kk % DLU][k];
                if (row_ok && i + DLU >= 0 && i + DLU < nx) {
#pragma unroll
                    for (int k = 0; k < ND; k++) buf[kk % DLU][k] = PL(a, k + 1, rowbase + i + DLU);
                }
                const int src = tau - 1 - kLag;
                const int rs = (int)(((unsigned)up_base * kLag + (unsigned)src) & (kRing - 1));
#pragma unroll
                for (int q = 0; q < NU; q++) {
                    double v = __shfl_up_sync(kFull, mw[q], 1);
                    if (lane == 0) v = (has_below && src >= 0) ? ring_up[wl][rs][q] : 0.0;
                    a3[q] = a2[q]; a2[q] = a1[q]; a1[q] = v;
                }
                double u[NU];
#pragma unroll
                for (int q = 0; q < NU; q++) u[q] = 0.0;
                if (valid) {
                    const long long np = rowbase + i;
                    const double alpha = (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) ? 0.5 : 0.0;
                    // neighbours: W = own previous cell, SE = a1, S = a2, SW = a3
                    if (ND == 9) {
                        const double b1 = cb[0], b2 = cb[1], b3 = cb[2], b4 = cb[3], b5 = cb[4];
                        const double b6 = cb[5], b7 = cb[6], b8 = cb[7], b9 = cb[8];
                        double l5 = b1;
                        double l4 = qdiv(b2 - l5 * a3[0] - alpha * b3 * a1[0], 1.0 - alpha * a2[0] * a1[0]);
                        double l3 = b3 - l4 * a2[0];
                        double l2 = qdiv(b4 - l4 * a2[1] - l5 * a3[2] - 2.0 * alpha * l5 * a3[1], 1 + 2.0 * alpha * mw[1]);
                        double phi1 = l3 * a1[0], phi2 = l5 * a3[1], phi3 = l3 * a1[3], phi4 = l2 * mw[1];
                        double l1 = b5 - l2 * mw[0] - l3 * a1[1] - l4 * a2[2] - l5 * a3[3]
                                  + alpha * (2.0 * phi1 + phi2 + phi3 + 2.0 * phi4);
                        const double n0 = b6 - l3 * a1[2] - l4 * a2[3] - 2.0 * alpha * (phi1 + phi3);
                        const double n1 = b7 - l2 * mw[2];
                        const double n2 = b8 - l2 * mw[3] - alpha * phi4;
                        const double n3 = b9;
                        if (recip_ok(n0, l1) && recip_ok(n1, l1) && recip_ok(n2, l1) && recip_ok(n3, l1)) {
                            const double y = __drcp_rn(l1);
                            u[0] = div_recip(n0, l1, y); u[1] = div_recip(n1, l1, y);
                            u[2] = div_recip(n2, l1, y); u[3] = div_recip(n3, l1, y);
                        } else {
                            u[0] = div_ieee(n0, l1); u[1] = div_ieee(n1, l1);
                            u[2] = div_ieee(n2, l1); u[3] = div_ieee(n3, l1);
                        }
                        if (!(fabs(l1) > 0.0) || !isfinite(l1)) bad_pivot = true;
                        PL(dl, 1, np) = l1; PL(dl, 2, np) = l2; PL(dl, 3, np) = l3; PL(dl, 4, np) = l4; PL(dl, 5, np) = l5;
                    } else {
                        const double b1 = cb[0], b2 = cb[1], b3 = cb[2], b4 = cb[3], b5 = cb[4];
                        double l4 = qdiv(b1, 1.0 - alpha * a2[0] * a1[0]);
                        double l3 = -l4 * a2[0];
                        double l2 = qdiv(b2 - l4 * a2[1], 1.0 + 2.0 * alpha * mw[1]);
                        double phi1 = l3 * a1[0], phi4 = l2 * mw[1];
                        double l1 = b3 - l2 * mw[0] - l3 * a1[1] - l4 * a2[2] + 2.0 * alpha * (phi1 + phi4);
                        const double n0 = b4 - l3 * a1[2] - 2.0 * alpha * phi1;
                        const double n1 = -l2 * mw[2];
                        const double n2 = b5 - alpha * phi4;
                        if (recip_ok(n0, l1) && recip_ok(n1, l1) && recip_ok(n2, l1)) {
                            const double y = __drcp_rn(l1);
                            u[0] = div_recip(n0, l1, y); u[1] = div_recip(n1, l1, y); u[2] = div_recip(n2, l1, y);
                        } else {
                            u[0] = div_ieee(n0, l1); u[1] = div_ieee(n1, l1); u[2] = div_ieee(n2, l1);
                        }
                        if (!(fabs(l1) > 0.0) || !isfinite(l1)) bad_pivot = true;
                        PL(dl, 1, np) = l1; PL(dl, 2, np) = l2; PL(dl, 3, np) = l3; PL(dl, 4, np) = l4;
                    }
#pragma unroll
                    for (int q = 0; q < NU; q++) PL(du, q + 1, np) = u[q];
                }
#pragma unroll
                for (int q = 0; q < NU; q++) mw[q] = u[q];
                if (lane == 31 && has_above) {
                    const int ws = (int)(((unsigned)up_base * kLag + (unsigned)tau) & (kRing - 1));
#pragma unroll
                    for (int q = 0; q < NU; q++) up_ring_dst[ws * NU + q] = u[q];
                }
            }
            if (lane == 31 && has_above) st_release(up_ready_dst, up_base + b + 1);
            if (lane == 0 && has_below) st_release(up_done_dst, up_base + b + 1);
        }
    }
    up_base += nbatch;
    if (bad_pivot && L.err) atomicOr(L.err, ERR_NONFINITE_PIVOT);
    stamp(L, rank, 1);

    // ---- fb2d9 / fb2d5 (msi2d9-v03.f90:42-262, msi2d5-v03.f90:42-233)
    const double rr0 = cluster_residual<ND>(cl, a, S.b, x, wk, nx, ny, red, part);
    stamp(L, rank, 2);
    const double gammarp = L.tol * sqrt(rr0);
    const int cap = (L.nitm > 0) ? L.nitm : kMaxIterUnbounded;
    int nit = 0;
    double rr = rr0;
    for (;;) {
        nit = nit + 1;
        // forward: L w = -r, w overwrites r in wk.  buf[d] = {r, dl1..dlNL}
        if (front) {
            double mine = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, buf[DSW][NL + 1];
#pragma unroll
            for (int d = 0; d < DSW; d++) {
                const int ic = d - 2 * j - kLag * wg;
                const bool ok = row_ok && ic >= 0 && ic < nx;
                buf[d][0] = ok ? wk[rowbase + ic] : 0.0;
#pragma unroll
                for (int k = 0; k < NL; k++) buf[d][k + 1] = ok ? PL(dl, k + 1, rowbase + ic) : 1.0;
            }
            double ycur = __drcp_rn(buf[0][1]);
            for (int b = 0; b < nbatch; b++) {
                const int tb = b * kLag;
                if (has_below) warp_wait(&up_ready[wl], up_base + b, 0, timed_out);
                if (has_above && b > kLead) warp_wait(&up_done[wl], up_base + b - kLead, 31, timed_out);
#pragma unroll
                for (int kk = 0; kk < kLag; kk++) {
                    const int tau = tb + kk;
                    const int i = tau - 2 * j - kLag * wg;
                    const bool valid = row_ok && i >= 0 && i < nx;
                    double c[NL + 1];
#pragma unroll
                    for (int k = 0; k <= NL; k++) c[k] = buf[kk % DSW][k];
                    const double y = ycur;
                    ycur = __drcp_rn(buf[(kk + 1) % DSW][1]);   // next cell's pivot, off the recurrence
                    if (row_ok && i + DSW >= 0 && i + DSW < nx) {
                        buf[kk % DSW][0] = wk[rowbase + i + DSW];
#pragma unroll
                        for (int k = 0; k < NL; k++) buf[kk % DSW][k + 1] = PL(dl, k + 1, rowbase + i + DSW);
                    }
                    const int src = tau - 1 - kLag;
                    double v = __shfl_up_sync(kFull, mine, 1);
                    if (lane == 0)
                        v = (has_below && src >= 0) ? ring_up[wl][((unsigned)up_base * kLag + (unsigned)src) & (kRing - 1)][0] : 0.0;
                    a3 = a2; a2 = a1; a1 = v;
                    double wv = 0.0;
                    if (valid) {
                        // w = -(r + dl2 w_W + dl3 w_SE + dl4 w_S [+ dl5 w_SW]) / dl1
                        double num;
                        if (ND == 9) num = c[0] + c[2] * mine + c[3] * a1 + c[4] * a2 + c[5] * a3;
                        else num = c[0] + c[2] * mine + c[3] * a1 + c[4] * a2;
                        wv = recip_ok(num, c[1]) ? -div_recip(num, c[1], y) : -div_ieee(num, c[1]);
                        wk[rowbase + i] = wv;
                    }
                    mine = wv;
                    if (lane == 31 && has_above)
                        up_ring_dst[(((unsigned)up_base * kLag + (unsigned)tau) & (kRing - 1)) * NU] = wv;
                }
                if (lane == 31 && has_above) st_release(up_ready_dst, up_base + b + 1);
                if (lane == 0 && has_below) st_release(up_done_dst, up_base + b + 1);
            }
        }
        up_base += nbatch;
        if (nit == 1) stamp(L, rank, 3);
        // backward: U z = w, var = z + var; time runs from the top-right
        // corner.  buf[d] = {w, x, du1..duNU}
        if (front) {
            double mine = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, buf[DSW][NU + 2];
            const int wrev = NWG - 1 - wg;
#pragma unroll
            for (int d = 0; d < DSW; d++) {
                const int ic = nx - 1 - (d - 2 * (ny - 1 - j) - kLag * wrev);
                const bool ok = row_ok && ic >= 0 && ic < nx;
                buf[d][0] = ok ? wk[rowbase + ic] : 0.0;
                buf[d][1] = ok ? x[rowbase + ic] : 0.0;
#pragma unroll
                for (int k = 0; k < NU; k++) buf[d][k + 2] = ok ? PL(du, k + 1, rowbase + ic) : 0.0;
            }
            for (int b = 0; b < nbatch; b++) {
                const int tb = b * kLag;
                if (has_above) warp_wait(&dn_ready[wl], dn_base + b, 31, timed_out);
                if (has_below && b > kLead) warp_wait(&dn_done[wl], dn_base + b - kLead, 0, timed_out);
#pragma unroll
                for (int kk = 0; kk < kLag; kk++) {
                    const int tau = tb + kk;
                    const int i = nx - 1 - (tau - 2 * (ny - 1 - j) - kLag * wrev);
                    const bool valid = row_ok && i >= 0 && i < nx;
                    double c[NU + 2];
#pragma unroll
                    for (int k = 0; k < NU + 2; k++) c[k] = buf[kk % DSW][k];
                    if (row_ok && i - DSW >= 0 && i - DSW < nx) {
                        buf[kk % DSW][0] = wk[rowbase + i - DSW];
                        buf[kk % DSW][1] = x[rowbase + i - DSW];
#pragma unroll
                        for (int k = 0; k < NU; k++) buf[kk % DSW][k + 2] = PL(du, k + 1, rowbase + i - DSW);
                    }
                    const int src = tau - 1 - kLag;
                    double v = __shfl_down_sync(kFull, mine, 1);
                    if (lane == 31)
                        v = (has_above && src >= 0) ? ring_dn[wl][((unsigned)dn_base * kLag + (unsigned)src) & (kRing - 1)] : 0.0;
                    a3 = a2; a2 = a1; a1 = v;
                    double z = 0.0;
                    if (valid) {
                        // z = w - du1 z_E - du2 z_NW - du3 z_N [- du4 z_NE]; E = own previous
                        if (ND == 9) z = c[0] - c[2] * mine - c[3] * a1 - c[4] * a2 - c[5] * a3;
                        else z = c[0] - c[2] * mine - c[3] * a1 - c[4] * a2;
                        x[rowbase + i] = z + c[1];
                    }
                    mine = z;
                    if (lane == 0 && has_below)
                        dn_ring_dst[((unsigned)dn_base * kLag + (unsigned)tau) & (kRing - 1)] = z;
                }
                if (lane == 0 && has_below) st_release(dn_ready_dst, dn_base + b + 1);
                if (lane == 31 && has_above) st_release(dn_done_dst, dn_base + b + 1);
            }
        }
        dn_base += nbatch;
        if (nit == 1) stamp(L, rank, 4);
        rr = cluster_residual<ND>(cl, a, S.b, x, wk, nx, ny, red, part);
        if (nit == 1) stamp(L, rank, 5);
        if (sqrt(rr) < gammarp) break;
        if (nit == cap) {
            if (L.nitm <= 0 && L.err && rank == 0 && threadIdx.x == 0) atomicOr(L.err, ERR_WAIT_TIMEOUT);
            break;
        }
    }
    if (timed_out && L.err) atomicOr(L.err, ERR_WAIT_TIMEOUT);
    if (rank == 0 && threadIdx.x == 0) {
        if (S.nit) *S.nit = nit;
        if (S.rr) { S.rr[0] = rr0; S.rr[1] = rr; }
    }
    cl.sync();   // no CTA leaves while another may still write into its shared memory
    stamp(L, rank, 6);
}

bool msi_warp_supported(int ny) { return ny <= 1024; }

// launches one cluster per system if the cluster shape can be scheduled;
// *fits = false (and nothing launched) otherwise
template <int ND, int WPC, int DLU, int DSW>
static cudaError_t launch_cluster(const MsiLaunch &L, int nsys, cudaStream_t st, bool *fits)
{
    *fits = false;
    const int nwarps = (L.ny + 31) / 32;
    const int C = (nwarps + WPC - 1) / WPC;
    if (C > kMaxCluster) return cudaSuccess;
    auto kern = k_msi_c<ND, WPC, DLU, DSW>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(C * nsys));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    e = cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg);
    if (e != cudaSuccess || nclusters < 1) {
        (void)cudaGetLastError();
        return cudaSuccess;
    }
    *fits = true;
    return cudaLaunchKernelEx(&cfg, kern, L);
}

template <int ND>
static cudaError_t launch_nd(const MsiLaunch &L, int nsys, cudaStream_t st)
{
    // fewest wavefront warps per CTA (one SM per warp) whose cluster fits
    bool fits = false;
    cudaError_t e = launch_cluster<ND, 1, (ND == 9 ? 2 : 4), 4>(L, nsys, st, &fits);
    if (e != cudaSuccess || fits) return e;
    e = launch_cluster<ND, 2, (ND == 9 ? 2 : 4), 4>(L, nsys, st, &fits);
    if (e != cudaSuccess || fits) return e;
    e = launch_cluster<ND, 4, (ND == 9 ? 2 : 4), 4>(L, nsys, st, &fits);
    if (e != cudaSuccess || fits) return e;
    return launch_msi_generic(ND, L, nsys, st);
}

cudaError_t launch_msi_warp(int nd, const MsiLaunch &L, int nsys, cudaStream_t st)
{
    return nd == 9 ? launch_nd<9>(L, nsys, st) : launch_nd<5>(L, nsys, st);
}

}  // namespace m2d
