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
//     produced in an earlier batch of kLag steps.  Each batch of such values
//     travels as one bulk shared-to-shared copy into a ring in the consumer's
//     shared memory (distributed shared memory when the producer sits in
//     another CTA), completing on an mbarrier the consumer waits on; the
//     consumer frees ring slots by arriving on the producer's mbarriers.  No
//     warp waits for anything but its two neighbours, and every wait is
//     bounded in %globaltimer time (on timeout the kernel records
//     ERR_SPIN_TIMEOUT and runs to its end);
//   * A (after a transposing pre-pass, k_skew_a), the factors, the residual
//     and the sweep results live in "wavefront-major" planes: the 32 cells a
//     warp touches in one step are one contiguous 256-byte line, so one batch
//     of one plane is a single 4 KB block.  The factorisation and the sweeps
//     stage those blocks into shared memory with bulk asynchronous copies
//     (TMA, completion on an mbarrier) several batches ahead, so no
//     global-memory latency sits on the recurrence;
//   * divisions on the recurrence use the divisor's correctly rounded
//     reciprocal and two FMA corrections (Markstein's method), which yields
//     the IEEE quotient whenever both operands lie in [2^-500, 2^500) (or the
//     dividend is zero).  In the forward sweep a batch in which any cell
//     falls outside that range is recomputed with IEEE division before it is
//     published.  The factorisation tests nothing on the recurrence: the
//     helper warps (those on the SM sub-partitions no wavefront warp uses)
//     refactorise every cell with IEEE division from its stored inputs while
//     the first sweeps run, and any difference repeats the factorisation
//     with IEEE division before x changes;
//   * a step is software-pipelined (critical shuffles first, then the
//     previous step's predicated stores, then the next step's loads), so no
//     branch separates two steps;
//   * the helper warps also compute the initial residual during the
//     factorisation; after each sweep pair x += z and the residual
//     r = A x - b run as cluster-wide passes over all threads, as does the
//     L2 norm of the stopping test (partial sums combined in a fixed order in
//     CTA 0 and broadcast, so the stopping decision is deterministic).
// A cell outside the grid (before its row starts, after it ends, rows >= ny)
// produces zeros, which is exactly the zero-neighbour rule of the general
// formula, so results stay bitwise equal to the lexicographic reference loop.
#include <cstdint>
#include <type_traits>
#include <cooperative_groups.h>
#include "m2d_solvers.cuh"

namespace cg = cooperative_groups;

namespace m2d {

namespace {
constexpr int kRing = 128;        // ring entries per channel (kSlots batches)
constexpr int kThreads = 256;     // threads per CTA (wavefront warps + helpers)
constexpr int kMaxCluster = 16;
constexpr int kSkewPad = 62;      // slots per warp = nx + 62 (slot s = i + 2 lane)
constexpr int kLine = 32;         // values per slot line, one per lane
// Steps per batch = the per-warp time lag (LAG).  FP64: 16.  FP32: 32 on
// grids of kLongLagCells and more, whose short steps and long sweeps made
// the per-batch hand-off and staging show (measured at 514x258: forward
// sweeps 11-12 % and backward sweeps 22-24 % faster with 32-step batches);
// 16 below, where the longer pipeline fill of 32-step batches costs more
// (a sweep of 256 nozzles of 64..512 x 32..128 cells: 7 % slower with 32);
// the FP64 factorisation runs slower with 32-step batches.
template <int LAG> struct Batch {
    static constexpr int kLag = LAG;
    static constexpr int kBlock = kLag * kLine;   // elements of one plane for one batch
    static constexpr int kSlots = kRing / kLag;   // ring slots, one batch each
};
constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxIterUnbounded = 10000;
constexpr unsigned long long kWaitLimitNs = 4000000000ull;   // bound of every wait (4 s of %globaltimer)
}

#define PL(p, k, np) (p)[(long long)((k) - 1) * N + (np)]

// a / b from y = RN(1/b): q0 = a y, then two corrections q += (a - q b) y
// with exact FMA remainders (Markstein, IBM J. Res. Dev. 34, 1990).  With
// |a|, |b| in [2^-500, 2^500) no intermediate leaves the normal range and the
// result is the correctly rounded quotient; for a = 0 the first product a y
// already is the IEEE quotient.  range_bad is 0 when these conditions hold.
__device__ __forceinline__ double div_recip(double a, double b, double y)
{
    const double q0 = a * y;
    const double r0 = fma(-q0, b, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-q1, b, a);
    return (a == 0.0) ? q0 : fma(r1, y, q1);
}
// 1 when |x| lies outside [2^-500, 2^500) (zero, subnormals, Inf and NaN
// included): the biased exponent outside [523, 1522].  Integer arithmetic
// without branches, so the check does not split a recurrence step into
// blocks the scheduler cannot overlap.
__device__ __forceinline__ unsigned exp_out(double x)
{
    const unsigned e = (unsigned)((unsigned long long)__double_as_longlong(x) >> 52) & 0x7ffu;
    return (e - 523u) > 999u ? 1u : 0u;
}
__device__ __forceinline__ unsigned range_bad(double a, double b)
{
    return exp_out(b) | (exp_out(a) & (a != 0.0 ? 1u : 0u));
}


__device__ __forceinline__ void stamp(const MsiLaunch &L, int rank, int k)
{
    if (L.prof && rank == 0 && threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        L.prof[k] = t;
    }
}

// ---- bulk asynchronous copies into shared memory, completion on an mbarrier
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Ordered shared-memory loads and shuffles.  A sweep step's shuffle of the
// previous step's result is its critical input; issued before the next
// step's shared-memory loads, it does not queue behind them.
template <typename T> __device__ __forceinline__ T lds_v(unsigned addr);
template <> __device__ __forceinline__ double lds_v<double>(unsigned addr)
{
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
    return v;
}
template <> __device__ __forceinline__ float lds_v<float>(unsigned addr)
{
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}
__device__ __forceinline__ double shfl_up_v(double x)
{
    double v;
    asm volatile("{\n\t.reg .b32 lo, hi;\n\tmov.b64 {lo, hi}, %1;\n\t"
                 "shfl.sync.up.b32 lo, lo, 1, 0, -1;\n\tshfl.sync.up.b32 hi, hi, 1, 0, -1;\n\t"
                 "mov.b64 %0, {lo, hi};\n\t}" : "=d"(v) : "d"(x));
    return v;
}
// Predicated stores: no branch, so a store of one recurrence step can sit in
// the same block as the next step's first instructions and overlap them.
__device__ __forceinline__ void stg_if(double *p, double v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\t.reg .u64 g;\n\tsetp.ne.u32 q, %2, 0;\n\t"
                 "cvta.to.global.u64 g, %0;\n\t@q st.global.f64 [g], %1;\n\t}"
                 ::"l"(p), "d"(v), "r"((unsigned)c));
}
__device__ __forceinline__ void stg_if(float *p, float v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\t.reg .u64 g;\n\tsetp.ne.u32 q, %2, 0;\n\t"
                 "cvta.to.global.u64 g, %0;\n\t@q st.global.f32 [g], %1;\n\t}"
                 ::"l"(p), "f"(v), "r"((unsigned)c));
}
__device__ __forceinline__ void sts_if(unsigned addr, double v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.shared.f64 [%0], %1;\n\t}"
                 ::"r"(addr), "d"(v), "r"((unsigned)c));
}
__device__ __forceinline__ void sts_if(unsigned addr, float v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.shared.f32 [%0], %1;\n\t}"
                 ::"r"(addr), "f"(v), "r"((unsigned)c));
}
// 1 for a zero or non-finite pivot, from the bits (no branch)
__device__ __forceinline__ unsigned pivot_bad(double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return ((b << 1) == 0ull || ((unsigned)(b >> 52) & 0x7ffu) == 0x7ffu) ? 1u : 0u;
}
__device__ __forceinline__ unsigned pivot_bad(float x)
{
    const unsigned b = (unsigned)__float_as_int(x);
    return ((b << 1) == 0u || ((b >> 23) & 0xffu) == 0xffu) ? 1u : 0u;
}
__device__ __forceinline__ float shfl_up_v(float x)
{
    float v;
    asm volatile("shfl.sync.up.b32 %0, %1, 1, 0, -1;" : "=f"(v) : "f"(x));
    return v;
}
__device__ __forceinline__ float shfl_down_v(float x)
{
    float v;
    asm volatile("shfl.sync.down.b32 %0, %1, 1, 31, -1;" : "=f"(v) : "f"(x));
    return v;
}
__device__ __forceinline__ double shfl_down_v(double x)
{
    double v;
    asm volatile("{\n\t.reg .b32 lo, hi;\n\tmov.b64 {lo, hi}, %1;\n\t"
                 "shfl.sync.down.b32 lo, lo, 1, 31, -1;\n\tshfl.sync.down.b32 hi, hi, 1, 31, -1;\n\t"
                 "mov.b64 %0, {lo, hi};\n\t}" : "=d"(v) : "d"(x));
    return v;
}

// 32-bit shared::cluster address of the same variable in CTA `rank`
__device__ __forceinline__ unsigned cluster_addr(const void *p, int rank)
{
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cluster(unsigned addr, double v)
{
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v));
}
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// true once phase `parity` of the mbarrier has completed; false when
// limit_ns of %globaltimer time passed first
__device__ __forceinline__ bool mbar_wait_for(unsigned long long *bar, unsigned parity, unsigned long long limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    for (;;) {
        for (int k = 0; k < 32; k++)
            if (mbar_try_wait(bar, parity)) return true;
        if (gtimer() - t0 > limit_ns) return false;
    }
}
// all lanes: bounded wait for the completion of phase `parity` (after an
// earlier timeout the warp no longer waits at all)
__device__ __forceinline__ void mbar_wait(unsigned long long *bar, unsigned parity, bool &timed_out)
{
    if (!timed_out && !mbar_wait_for(bar, parity, kWaitLimitNs)) timed_out = true;
    __syncwarp();
}
__device__ __forceinline__ void bulk_s2s(unsigned dst, const void *src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "r"(smem_u32(src)), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void mbar_remote_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(bar) : "memory");
}
// generic-proxy global writes become visible to later bulk copies
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Per wavefront warp: NSTAGE staging blocks of NP planes x kLag lines, one
// mbarrier each.  issued/consumed count staged batches over all phases, so
// block = count % NSTAGE and the mbarrier parity = (count / NSTAGE) & 1.
template <typename TS, int NSTAGE, int PMAX, int LAG>
struct Stager {
    TS *mem;                     // the CTA's staging memory
    int base;                    // this warp's area in it (elements)
    unsigned long long *bar;
    int issued, consumed;
    __device__ int block(int q) const { return base + q * PMAX * Batch<LAG>::kBlock; }
};

// stage slot lines [s_lo, s_lo + kLag) of NP wavefront-major planes (lines
// outside [0, sw) are not copied: every cell on them is invalid)
template <int NP, typename TS, int NSTAGE, int PMAX, int LAG>
__device__ __forceinline__ void stage_issue(Stager<TS, NSTAGE, PMAX, LAG> &st, TS *const *planes,
                                            long long line0, int s_lo, int sw)
{
    static_assert(NP <= 32, "one staged plane per lane");
    const int q = st.issued % NSTAGE;
    const int lane = threadIdx.x & 31;
    const int lo = max(s_lo, 0), hi = min(s_lo + Batch<LAG>::kLag, sw);
    const unsigned bytes = hi > lo ? (unsigned)(hi - lo) * kLine * (unsigned)sizeof(TS) : 0u;
    if (lane == 0) {
        fence_async_shared();   // earlier reads of this block precede the copies into it
        mbar_arrive_tx(&st.bar[q], bytes * NP);
    }
    __syncwarp();
    // one plane per lane: the copies go out in one warp instruction instead of
    // NP single-lane ones on the wavefront warp's path
    if (bytes && lane < NP) {
        fence_async_shared();
        TS *dst = st.mem + st.block(q) + (lo - s_lo) * kLine + lane * Batch<LAG>::kBlock;
        bulk_g2s(dst, planes[lane] + (line0 + lo) * kLine, bytes, &st.bar[q]);
    }
    st.issued++;
}
// waits for the next staged batch; returns its block's offset in st.mem
template <typename TS, int NSTAGE, int PMAX, int LAG>
__device__ __forceinline__ int stage_wait(Stager<TS, NSTAGE, PMAX, LAG> &st, bool &timed_out)
{
    const int q = st.consumed % NSTAGE;
    const unsigned parity = (unsigned)(st.consumed / NSTAGE) & 1u;
    if (!mbar_wait_for(&st.bar[q], parity, kWaitLimitNs)) timed_out = true;
    __syncwarp();
    st.consumed++;
    return st.block(q);
}

// ---- warp-to-warp hand-off (one channel = one direction between two warps)
// The producer stages the values of its batch n (its lane 31 for the warp
// above, lane 0 for the warp below) in slot n % kSlots of a local buffer and
// ships the slot with one bulk shared-to-shared copy into the same slot of the
// consumer's ring; the copy completes on the consumer's "full" barrier of that
// slot.  The consumer frees the slot by arriving on the producer's "empty"
// barrier.  Batch numbers n count over all phases of a channel, so the k-th
// use of a slot is phase k of its barriers.
template <int LAG>
__device__ __forceinline__ void chan_recv(unsigned long long *full, int n, unsigned bytes, bool &timed_out)
{
    constexpr int kSlots = Batch<LAG>::kSlots;
    unsigned long long *bar = &full[n & (kSlots - 1)];
    if ((threadIdx.x & 31) == 0) mbar_arrive_tx(bar, bytes);
    __syncwarp();
    mbar_wait(bar, (unsigned)(n / kSlots) & 1u, timed_out);
}
// producer, before staging batch n: the consumer has released batch n - kSlots
template <int LAG>
__device__ __forceinline__ void chan_slot_free(unsigned long long *empty, int n, bool &timed_out)
{
    constexpr int kSlots = Batch<LAG>::kSlots;
    if (n >= kSlots) mbar_wait(&empty[n & (kSlots - 1)], (unsigned)(n / kSlots - 1) & 1u, timed_out);
}
// producer lane that staged the values: ship batch n (vals elements)
template <typename TS, int LAG>
__device__ __forceinline__ void chan_send(unsigned ring_dst, unsigned full_dst, const TS *out, int n, int vals)
{
    const int slot = n & (Batch<LAG>::kSlots - 1);
    fence_async_shared();   // the staged values become visible to the bulk copy
    bulk_s2s(ring_dst + (unsigned)(slot * vals) * (unsigned)sizeof(TS), out + slot * vals,
             (unsigned)vals * (unsigned)sizeof(TS), full_dst + (unsigned)slot * 8u);
}
template <int LAG>
__device__ __forceinline__ void chan_release(unsigned empty_dst, int n)
{
    mbar_remote_arrive(empty_dst + (unsigned)(n & (Batch<LAG>::kSlots - 1)) * 8u);
}

// wavefront-major slot of cell (i, j): warp j/32, step offset i + 2 (j%32), lane j%32
__device__ __forceinline__ long long skew_slot(int i, int j, int sw)
{
    return ((long long)(j >> 5) * sw + i + 2 * (j & 31)) * kLine + (j & 31);
}

// r = A x - b for one cell, in-range neighbours in ascending diagonal order
template <int ND>
__device__ __forceinline__ double residual_cell(const double *__restrict__ a, const double *__restrict__ b,
                                                const double *__restrict__ x, long long np, int i, int j, int nx,
                                                int ny, long long N)
{
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

__device__ __forceinline__ void named_bar(unsigned id, unsigned count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// The initial residual r = A x - b of this CTA's slice, computed by the
// nhelp helper warps (hw = 0..nhelp-1) while the wavefront warps factorise.
// The helpers run the 256 threads of cluster_residual as virtual threads
// (virtual thread t takes cells lo + t + 256 k, in that order) and the same
// tree over their sums, so the norm is bitwise the one cluster_residual
// gives.  The CTA's sum goes to CTA 0's part[rank]; cluster_total combines
// the CTAs after the next cluster barrier.
template <int ND, typename TS>
__device__ void helper_residual(cg::cluster_group &cl, const double *__restrict__ a, const double *__restrict__ b,
                                const double *__restrict__ x, TS *__restrict__ r, int nx, int ny, int sw,
                                double *red, double *part, int nhelp, int hw)
{
    const long long N = (long long)nx * ny;
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const long long per = (N + C - 1) / C;
    const long long lo = per * rank, hi = (lo + per < N) ? lo + per : N;
    const int lane = threadIdx.x & 31;
    const unsigned nthr = (unsigned)nhelp * 32u;
    for (int vw = hw; vw < kThreads / 32; vw += nhelp) {
        const int t = vw * 32 + lane;
        double acc = 0.0;
#pragma unroll 8
        for (long long np = lo + t; np < hi; np += kThreads) {
            const int j = (int)((unsigned)np / (unsigned)nx), i = (int)np - j * nx;   // N < 2^31
            const double v = residual_cell<ND>(a, b, x, np, i, j, nx, ny, N);
            r[skew_slot(i, j, sw)] = (TS)v;
            acc = acc + v * v;
        }
        red[t] = acc;
    }
    fence_async_global();   // the forward sweep reads r with bulk copies
    named_bar(1, nthr);
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        for (int t = hw * 32 + lane; t < s; t += (int)nthr) red[t] = red[t] + red[t + s];
        named_bar(1, nthr);
    }
    if (hw == 0 && lane == 0) {
        double *p0 = cl.map_shared_rank(part, 0);
        p0[rank] = red[0];
    }
}

// r = A x - b over cells lo + threadIdx.x + kThreads k of [lo, hi), stored
// wavefront-major; returns this thread's sum of r^2 in cell order.  Four
// cells per round with their loads issued together.
template <int ND, typename TS>
__device__ __forceinline__ double residual_pass(const double *__restrict__ a, const double *__restrict__ b,
                                                const double *__restrict__ x, TS *__restrict__ r, long long lo,
                                                long long hi, int nx, int ny, int sw)
{
    const long long N = (long long)nx * ny;
    double acc = 0.0;
    long long np = lo + threadIdx.x;
    for (; np + 3 * kThreads < hi; np += 4 * kThreads) {
        double v[4];
        int ii[4], jj[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const long long c = np + q * kThreads;
            jj[q] = (int)((unsigned)c / (unsigned)nx);   // N < 2^31
            ii[q] = (int)c - jj[q] * nx;
            v[q] = residual_cell<ND>(a, b, x, c, ii[q], jj[q], nx, ny, N);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            r[skew_slot(ii[q], jj[q], sw)] = (TS)v[q];
            acc = acc + v[q] * v[q];
        }
    }
    for (; np < hi; np += kThreads) {
        const int j = (int)((unsigned)np / (unsigned)nx), i = (int)np - j * nx;
        const double v = residual_cell<ND>(a, b, x, np, i, j, nx, ny, N);
        r[skew_slot(i, j, sw)] = (TS)v;
        acc = acc + v * v;
    }
    return acc;
}

// After a cluster barrier: the sum of the CTAs' part[] in rank order,
// identical in every thread
__device__ double cluster_total(cg::cluster_group &cl, double *part)
{
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    cl.sync();
    if (rank == 0 && threadIdx.x == 0) {
        double s = 0.0;
        for (int c = 0; c < C; c++) s = s + part[c];
        for (int c = 0; c < C; c++) cl.map_shared_rank(part, c)[kMaxCluster] = s;
    }
    cl.sync();
    return part[kMaxCluster];
}

// Cluster-wide pass (this CTA takes a contiguous slice of cells): first
// x += z when z (wavefront-major) is given, then r = A x - b stored
// wavefront-major.  Returns the cluster-wide sum of r^2, identical in every
// thread.  Starts with a cluster barrier: every row's sweep must be final.
template <int ND, typename TS>
__device__ double cluster_residual(cg::cluster_group &cl, const double *__restrict__ a,
                                   const double *__restrict__ b, double *x, const TS *z, TS *r,
                                   int nx, int ny, int sw, double *red, double *part)
{
    cl.sync();
    const long long N = (long long)nx * ny;
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const long long per = (N + C - 1) / C;
    const long long lo = per * rank, hi = (lo + per < N) ? lo + per : N;
    if (z) {
        double *__restrict__ xw = x;
        const TS *__restrict__ zr = z;
#pragma unroll 8
        for (long long np = lo + threadIdx.x; np < hi; np += kThreads) {
            const int j = (int)((unsigned)np / (unsigned)nx), i = (int)np - j * nx;   // N < 2^31
            xw[np] = (double)zr[skew_slot(i, j, sw)] + xw[np];
        }
        cl.sync();
    }
    // x is final (read-only) from here on, and r is separate workspace
    const double acc = residual_pass<ND, TS>(a, b, x, r, lo, hi, nx, ny, sw);
    fence_async_global();   // the forward sweep reads r with bulk copies
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

// One factorisation step of one cell (lu2d9 / lu2d5).  cb is the row of A
// (a unit row for an invalid cell), mw the own row's previous u, a1/a2/a3
// the row below's u at SE/S/SW.  FAST divides with Markstein quotients
// (checked against IEEE division afterwards, verify_factors); otherwise it
// divides with '/'.
template <int ND, bool FAST>
__device__ __forceinline__ void lu_cell(const double (&cb)[ND], double alpha, const double *mw,
                                        const double *a1, const double *a2, const double *a3, double *l,
                                        double *u, double &y1)
{
    auto dv = [&](double n, double d) -> double { return FAST ? div_recip(n, d, __drcp_rn(d)) : n / d; };
    if (ND == 9) {
        const double b1 = cb[0], b2 = cb[1], b3 = cb[2], b4 = cb[3], b5 = cb[4];
        const double b6 = cb[5], b7 = cb[6], b8 = cb[7], b9 = cb[8];
        double l5 = b1;
        double l4 = dv(b2 - l5 * a3[0] - alpha * b3 * a1[0], 1.0 - alpha * a2[0] * a1[0]);
        double l3 = b3 - l4 * a2[0];
        double l2 = dv(b4 - l4 * a2[1] - l5 * a3[2] - 2.0 * alpha * l5 * a3[1], 1 + 2.0 * alpha * mw[1]);
        double phi1 = l3 * a1[0], phi2 = l5 * a3[1], phi3 = l3 * a1[3], phi4 = l2 * mw[1];
        double l1 = b5 - l2 * mw[0] - l3 * a1[1] - l4 * a2[2] - l5 * a3[3]
                  + alpha * (2.0 * phi1 + phi2 + phi3 + 2.0 * phi4);
        const double n0 = b6 - l3 * a1[2] - l4 * a2[3] - 2.0 * alpha * (phi1 + phi3);
        const double n1 = b7 - l2 * mw[2];
        const double n2 = b8 - l2 * mw[3] - alpha * phi4;
        if (FAST) {
            const double y = __drcp_rn(l1);
            y1 = y;
            u[0] = div_recip(n0, l1, y); u[1] = div_recip(n1, l1, y);
            u[2] = div_recip(n2, l1, y); u[3] = div_recip(b9, l1, y);
        } else {
            u[0] = n0 / l1; u[1] = n1 / l1; u[2] = n2 / l1; u[3] = b9 / l1;
            y1 = __drcp_rn(l1);
        }
        l[0] = l1; l[1] = l2; l[2] = l3; l[3] = l4; l[4] = l5;
    } else {
        const double b1 = cb[0], b2 = cb[1], b3 = cb[2], b4 = cb[3], b5 = cb[4];
        double l4 = dv(b1, 1.0 - alpha * a2[0] * a1[0]);
        double l3 = -l4 * a2[0];
        double l2 = dv(b2 - l4 * a2[1], 1.0 + 2.0 * alpha * mw[1]);
        double phi1 = l3 * a1[0], phi4 = l2 * mw[1];
        double l1 = b3 - l2 * mw[0] - l3 * a1[1] - l4 * a2[2] + 2.0 * alpha * (phi1 + phi4);
        const double n0 = b4 - l3 * a1[2] - 2.0 * alpha * phi1;
        const double n1 = -l2 * mw[2];
        const double n2 = b5 - alpha * phi4;
        if (FAST) {
            const double y = __drcp_rn(l1);
            y1 = y;
            u[0] = div_recip(n0, l1, y); u[1] = div_recip(n1, l1, y); u[2] = div_recip(n2, l1, y);
        } else {
            u[0] = n0 / l1; u[1] = n1 / l1; u[2] = n2 / l1;
            y1 = __drcp_rn(l1);
        }
        l[0] = l1; l[1] = l2; l[2] = l3; l[3] = l4;
    }
}

// The same factorisation step in FP32 for the mixed-precision solve.  Its
// factors only precondition an FP64 iteration, so the operation order is
// free: fused multiply-adds and approximate reciprocals; y1 = 1/l1.
template <int ND>
__device__ __forceinline__ void lu_cell_f(const float (&cb)[ND], float alpha, const float *mw,
                                          const float *a1, const float *a2, const float *a3, float *l,
                                          float *u, float &y1)
{
    if (ND == 9) {
        const float b1 = cb[0], b2 = cb[1], b3 = cb[2], b4 = cb[3], b5 = cb[4];
        const float b6 = cb[5], b7 = cb[6], b8 = cb[7], b9 = cb[8];
        const float l5 = b1;
        const float l4 = __fdividef(fmaf(-alpha * b3, a1[0], fmaf(-l5, a3[0], b2)), fmaf(-alpha * a2[0], a1[0], 1.0f));
        const float l3 = fmaf(-l4, a2[0], b3);
        const float l2 = __fdividef(fmaf(-2.0f * alpha * l5, a3[1], fmaf(-l5, a3[2], fmaf(-l4, a2[1], b4))),
                                    fmaf(2.0f * alpha, mw[1], 1.0f));
        const float phi1 = l3 * a1[0], phi2 = l5 * a3[1], phi3 = l3 * a1[3], phi4 = l2 * mw[1];
        const float t = fmaf(-l5, a3[3], fmaf(-l4, a2[2], fmaf(-l3, a1[1], fmaf(-l2, mw[0], b5))));
        const float l1 = fmaf(alpha, 2.0f * phi1 + phi2 + phi3 + 2.0f * phi4, t);
        const float y = __fdividef(1.0f, l1);
        u[0] = fmaf(-2.0f * alpha, phi1 + phi3, fmaf(-l4, a2[3], fmaf(-l3, a1[2], b6))) * y;
        u[1] = fmaf(-l2, mw[2], b7) * y;
        u[2] = fmaf(-alpha, phi4, fmaf(-l2, mw[3], b8)) * y;
        u[3] = b9 * y;
        y1 = y;
        l[0] = l1; l[1] = l2; l[2] = l3; l[3] = l4; l[4] = l5;
    } else {
        const float b1 = cb[0], b2 = cb[1], b3 = cb[2], b4 = cb[3], b5 = cb[4];
        const float l4 = __fdividef(b1, fmaf(-alpha * a2[0], a1[0], 1.0f));
        const float l3 = -l4 * a2[0];
        const float l2 = __fdividef(fmaf(-l4, a2[1], b2), fmaf(2.0f * alpha, mw[1], 1.0f));
        const float phi1 = l3 * a1[0], phi4 = l2 * mw[1];
        const float t = fmaf(-l4, a2[2], fmaf(-l3, a1[1], fmaf(-l2, mw[0], b3)));
        const float l1 = fmaf(2.0f * alpha, phi1 + phi4, t);
        const float y = __fdividef(1.0f, l1);
        u[0] = fmaf(-2.0f * alpha, phi1, fmaf(-l3, a1[2], b4)) * y;
        u[1] = -l2 * mw[2] * y;
        u[2] = fmaf(-alpha, phi4, b5) * y;
        y1 = y;
        l[0] = l1; l[1] = l2; l[2] = l3; l[3] = l4;
    }
}

// factorisations repeated with IEEE division on this device since load
__device__ unsigned long long g_lu_redo = 0;

// The helper warps' check of a Markstein factorisation: every real cell of
// this CTA's row groups is factorised again from its row of A and the stored
// u of its W, S, SE [and SW] neighbours (zero outside the grid, as in the
// wavefront) with IEEE division, and its stored dl, du and 1/dl1 are
// compared bit for bit.  If every cell matches, the stored factors are those
// of the IEEE recurrence (induction over the wavefront order); otherwise
// *vbad is set.  The cells are visited line by line of the wavefront-major
// planes (lane l of line (w, s) is cell (s - 2l, 32w + l)), so the loads are
// whole 256-byte lines: the cell's own factors, A and the W neighbour on the
// line itself, the S, SE and SW neighbours on lines s-2, s-1, s-3 one lane
// down (lane 0: lines s+62, s+63, s+61 of the row group below, lane 31).
template <int ND>
__device__ void verify_factors(const double *asp, const double *dl, const double *du, const double *rl, int nx,
                               int ny, int sw, long long PS, int wg0, int nwg, int nhelp, int hw, unsigned *vbad)
{
    constexpr int NU = (ND == 9) ? 4 : 3;
    constexpr int NL = (ND == 9) ? 5 : 4;
    const int lane = threadIdx.x & 31;
    unsigned diff = 0;
    for (int idx = hw; idx < nwg * sw; idx += nhelp) {
        const int wg = wg0 + idx / sw, s = idx % sw;
        const int j = 32 * wg + lane, i = s - 2 * lane;
        if (j >= ny || i < 0 || i >= nx) continue;
        const long long P = ((long long)wg * sw + s) * kLine + lane;
        double cb[ND];
#pragma unroll
        for (int k = 0; k < ND; k++) cb[k] = asp[k * PS + P];
        const double alpha = (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) ? 0.5 : 0.0;
        // neighbours in the row below: lane - 1 of this group, or lane 31 of the group below
        const long long B = (lane > 0) ? ((long long)wg * sw + s) * kLine + lane - 1
                                       : ((long long)(wg - 1) * sw + s + 64) * kLine + 31;
        const long long pS = B - 2 * kLine, pSE = B - kLine, pSW = B - 3 * kLine, pW = P - kLine;
        double mw[NU], a1[NU], a2[NU], a3[NU];
#pragma unroll
        for (int q = 0; q < NU; q++) {
            mw[q] = (i >= 1) ? du[q * PS + pW] : 0.0;
            a2[q] = (j >= 1) ? du[q * PS + pS] : 0.0;
            a1[q] = (j >= 1 && i + 1 <= nx - 1) ? du[q * PS + pSE] : 0.0;
            a3[q] = (j >= 1 && i >= 1) ? du[q * PS + pSW] : 0.0;
        }
        double l[NL], u[NU], y;
        lu_cell<ND, false>(cb, alpha, mw, a1, a2, a3, l, u, y);
#pragma unroll
        for (int k = 0; k < NL; k++) diff |= (__double_as_longlong(l[k]) != __double_as_longlong(dl[k * PS + P])) ? 1u : 0u;
#pragma unroll
        for (int q = 0; q < NU; q++) diff |= (__double_as_longlong(u[q]) != __double_as_longlong(du[q * PS + P])) ? 1u : 0u;
        diff |= (__double_as_longlong(y) != __double_as_longlong(rl[P])) ? 1u : 0u;
    }
    if (diff) *vbad = 1u;
}

// A (plane-major, cell order) -> wavefront-major planes of element type TS for
// the factorisation's bulk copies: line (w, s) lane l holds cell
// (s - 2 l, 32 w + l).  A CTA transposes one plane's tile of 32 rows x
// (kSkewTile + 62) cells through shared memory into kSkewTile lines; cells
// outside the grid become zeros.  Grid: (line tiles, row groups, systems x ND).
constexpr int kSkewTile = 64;
// lagged factorisation (MsiLaunch::lag_max): does this solve reuse the
// factors in its workspace?  Read by the transpose and by every thread of
// the solve before anything writes the record, so all agree.
template <typename TS>
__device__ __forceinline__ bool lag_reuse(const MsiLaunch &L, const MsiSys &S)
{
    if (std::is_same<TS, double>::value || L.lag_max <= 0 || !S.lag || L.reuse_lu || L.apply_only) return false;
    return S.lag[0] == S.tag && S.lag[1] >= 1 && S.lag[1] < L.lag_max;
}

constexpr int kExtBlocks = 296;
constexpr long long kExtMinCells = 1LL << 16;
constexpr long long kLongLagCells = 1LL << 16;   // FP32 grids from here on use 32-step batches
constexpr int kExtTimedOut = 1, kExtLagged = 2, kExtBadPivot = 4;   // status bits of the first launch

struct ExtWords {
    double *partA, *partB;        // block sums of the initial / new residual
    unsigned *cntA, *cntB;        // finished blocks of each reduction
    int *status;                  // kExt* bits from the first launch
    int *done;                    // the stopping test passed (or the solve must stop)
};
__device__ __forceinline__ ExtWords ext_words(const MsiSys &S, int nd, int nx, int ny)
{
    const long long PS = (long long)((ny + 31) / 32) * (nx + kSkewPad) * kLine;
    double *e = S.ws + (long long)(nd == 9 ? 21 : 15) * PS;
    ExtWords w;
    w.partA = e;
    w.partB = e + kExtBlocks;
    w.cntA = reinterpret_cast<unsigned *>(e + 2 * kExtBlocks);
    w.cntB = reinterpret_cast<unsigned *>(e + 2 * kExtBlocks + 1);
    w.status = reinterpret_cast<int *>(e + 2 * kExtBlocks + 2);
    w.done = reinterpret_cast<int *>(e + 2 * kExtBlocks + 3);
    return w;
}

template <int ND, typename TS>
__global__ void __launch_bounds__(256) k_skew_a(MsiLaunch L)
{
    __shared__ double tile[32][kSkewTile + kSkewPad + 1];
    const int sys = blockIdx.z / ND, k = blockIdx.z - sys * ND;
    const MsiSys S = L.s[sys];
    if (L.ext && k == 0 && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        // the whole-GPU passes start from a clean state
        const ExtWords w = ext_words(S, ND, L.nx, L.ny);
        *w.cntA = 0u;
        *w.status = 0;
        *w.done = 0;
    }
    if (lag_reuse<TS>(L, S)) return;   // the factors are reused: A is not needed
    const int nx = L.nx, ny = L.ny;
    const long long N = (long long)nx * ny;
    const int NL = (ND == 9) ? 5 : 4, NU = (ND == 9) ? 4 : 3;
    const int SW = nx + kSkewPad;
    const long long PS = (long long)((ny + 31) / 32) * SW * kLine;
    TS *as = reinterpret_cast<TS *>(S.ws) + (long long)(NL + NU + 3 + k) * PS;
    const int w = blockIdx.y, c0 = blockIdx.x * kSkewTile;
    constexpr int TW = kSkewTile + kSkewPad;
    for (int idx = threadIdx.x; idx < 32 * TW; idx += blockDim.x) {
        const int r = idx / TW, c = idx - r * TW;
        const int i = c0 - kSkewPad + c, j = 32 * w + r;
        tile[r][c] = (j < ny && i >= 0 && i < nx) ? PL(S.a, k + 1, (long long)j * nx + i) : 0.0;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kSkewTile * 32; idx += blockDim.x) {
        const int t = idx >> 5, l = idx & 31, s = c0 + t;
        if (s < SW) as[((long long)w * SW + s) * kLine + l] = (TS)tile[l][t + kSkewPad - 2 * l];
    }
}

// An application of stored factors (MsiLaunch::apply_only): the residual
// plane of the first forward sweep gets r = -b (the residual of x = 0) in
// wavefront-major order, and afterwards x += z from the sweep-result plane,
// each as one whole-GPU pass.  Grid: (cell blocks, systems).
template <int ND, typename TS>
__global__ void k_skew_rhs(MsiLaunch L)
{
    const MsiSys S = L.s[blockIdx.y];
    const int nx = L.nx, ny = L.ny;
    const int NL = (ND == 9) ? 5 : 4, NU = (ND == 9) ? 4 : 3;
    const int SW = nx + kSkewPad;
    const long long PS = (long long)((ny + 31) / 32) * SW * kLine;
    TS *r = reinterpret_cast<TS *>(S.ws) + (long long)(NL + NU + 1) * PS;
    const long long N = (long long)nx * ny;
    for (long long np = blockIdx.x * (long long)blockDim.x + threadIdx.x; np < N;
         np += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(np / nx), i = (int)(np - (long long)j * nx);
        r[skew_slot(i, j, SW)] = (TS)(-S.b[np]);
    }
}
template <int ND, typename TS>
__global__ void k_unskew_add(MsiLaunch L)
{
    const MsiSys S = L.s[blockIdx.y];
    const int nx = L.nx, ny = L.ny;
    const int NL = (ND == 9) ? 5 : 4, NU = (ND == 9) ? 4 : 3;
    const int SW = nx + kSkewPad;
    const long long PS = (long long)((ny + 31) / 32) * SW * kLine;
    const TS *z = reinterpret_cast<const TS *>(S.ws) + (long long)(NL + NU + 2) * PS;
    const long long N = (long long)nx * ny;
    for (long long np = blockIdx.x * (long long)blockDim.x + threadIdx.x; np < N;
         np += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(np / nx), i = (int)(np - (long long)j * nx);
        S.x[np] = (double)z[skew_slot(i, j, SW)] + S.x[np];
    }
}

// ---- whole-GPU residual passes (MsiLaunch::ext).  On a large grid the
// passes over all cells (the initial residual of a solve with reused
// factors, x += z and the new residual) run on the cluster's 9-16 SMs far
// below what the whole GPU moves, and take a sixth to a quarter of a
// one-iteration solve.  With ext the cluster kernel stops after the first
// sweep pair, these kernels make the passes on every SM, and a
// continuation launch of the cluster kernel iterates further only if the
// stopping test asks for it.  Reductions are deterministic: kExtBlocks
// blocks take fixed contiguous shares, a thread sums its cells in order, a
// block adds its threads' sums by a fixed tree, and the last block to
// finish adds the block sums in index order.
// r = A x - b over block blockIdx.x's share into the wavefront-major plane
// r, and the deterministic sum of r^2: returns the total in thread 0 of the
// last block to finish (last = true there), after resetting the counter
template <int ND, typename TS>
__device__ double ext_residual(const MsiSys &S, int nx, int ny, TS *__restrict__ r, double *part, unsigned *cnt,
                               bool &last)
{
    __shared__ double red[256];
    __shared__ bool is_last;
    const long long N = (long long)nx * ny;
    const int SW = nx + kSkewPad;
    const long long per = (N + kExtBlocks - 1) / kExtBlocks;
    const long long lo = per * blockIdx.x, hi = (lo + per < N) ? lo + per : N;
    double acc = 0.0;
    for (long long np = lo + threadIdx.x; np < hi; np += blockDim.x) {
        const int j = (int)((unsigned)np / (unsigned)nx), i = (int)np - j * nx;   // N < 2^31
        const double v = residual_cell<ND>(S.a, S.b, S.x, np, i, j, nx, ny, N);
        r[skew_slot(i, j, SW)] = (TS)v;
        acc = acc + v * v;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x] = red[0];
        __threadfence();
        is_last = atomicAdd(cnt, 1u) == (unsigned)gridDim.x - 1u;
    }
    __syncthreads();
    last = is_last && threadIdx.x == 0;
    double total = 0.0;
    if (last) {
        __threadfence();
        for (int k = 0; k < (int)gridDim.x; k++) total = total + __ldcg(part + k);
        *cnt = 0u;
    }
    return total;
}

// the initial residual of a solve that reuses its factors (lagged
// factorisation); nothing when the factors are renewed (the helper warps
// compute it behind the factorisation then).  Grid (kExtBlocks, systems).
template <int ND, typename TS>
__global__ void __launch_bounds__(256) k_ext_r0(MsiLaunch L)
{
    const MsiSys S = L.s[blockIdx.y];
    if (!lag_reuse<TS>(L, S)) return;
    const int nx = L.nx, ny = L.ny;
    constexpr int NL = (ND == 9) ? 5 : 4, NU = (ND == 9) ? 4 : 3;
    const long long PS = (long long)((ny + 31) / 32) * (nx + kSkewPad) * kLine;
    TS *rp = reinterpret_cast<TS *>(S.ws) + (long long)(NL + NU + 1) * PS;
    const ExtWords w = ext_words(S, ND, nx, ny);
    bool last;
    const double rr0 = ext_residual<ND, TS>(S, nx, ny, rp, w.partA, w.cntA, last);
    if (last) S.rr[0] = rr0;
}

// x += z after the first sweep pair; zeroes the counter of the next pass.
// Grid (blocks, systems).
template <int ND, typename TS>
__global__ void k_ext_update(MsiLaunch L)
{
    const MsiSys S = L.s[blockIdx.y];
    const int nx = L.nx, ny = L.ny;
    constexpr int NL = (ND == 9) ? 5 : 4, NU = (ND == 9) ? 4 : 3;
    const int SW = nx + kSkewPad;
    const long long PS = (long long)((ny + 31) / 32) * SW * kLine;
    const TS *z = reinterpret_cast<const TS *>(S.ws) + (long long)(NL + NU + 2) * PS;
    if (blockIdx.x == 0 && threadIdx.x == 0) *ext_words(S, ND, nx, ny).cntB = 0u;
    const long long N = (long long)nx * ny;
    for (long long np = blockIdx.x * (long long)blockDim.x + threadIdx.x; np < N;
         np += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(np / nx), i = (int)(np - (long long)j * nx);
        S.x[np] = (double)z[skew_slot(i, j, SW)] + S.x[np];
    }
}

// the new residual, its norm and the stopping test of the first iteration;
// when the solve ends here the last block also writes the factor record.
// Grid (kExtBlocks, systems).
template <int ND, typename TS>
__global__ void __launch_bounds__(256) k_ext_resid(MsiLaunch L)
{
    const MsiSys S = L.s[blockIdx.y];
    const int nx = L.nx, ny = L.ny;
    constexpr int NL = (ND == 9) ? 5 : 4, NU = (ND == 9) ? 4 : 3;
    const long long PS = (long long)((ny + 31) / 32) * (nx + kSkewPad) * kLine;
    TS *rp = reinterpret_cast<TS *>(S.ws) + (long long)(NL + NU + 1) * PS;
    const ExtWords w = ext_words(S, ND, nx, ny);
    bool last;
    const double rr = ext_residual<ND, TS>(S, nx, ny, rp, w.partB, w.cntB, last);
    if (!last) return;
    const double rr0 = S.rr[0];
    S.rr[1] = rr;
    const int st = *w.status;
    const int cap = (L.nitm > 0) ? L.nitm : kMaxIterUnbounded;
    const bool done = (st & kExtTimedOut) || sqrt(rr) < L.tol * sqrt(rr0) || cap == 1;
    *w.done = done ? 1 : 0;
    if (done && !std::is_same<TS, double>::value && L.lag_max > 0 && S.lag) {
        const bool lagged = (st & kExtLagged) != 0;
        const bool renew = (st & (kExtTimedOut | kExtBadPivot)) != 0;
        const int age = S.lag[1];
        S.lag[0] = S.tag;
        S.lag[1] = renew ? L.lag_max : (lagged ? age + 1 : 1);
    }
}

// TS = double: the reference's FP64 algorithm, bitwise.  TS = float: the
// factors and both sweeps in FP32 inside the FP64 iteration (residual, x,
// norm and stopping test stay FP64): iterative refinement preconditioned by
// the FP32 factorisation.
template <int ND, int WPC, int NSTAGE, typename TS, int LAG>
__global__ void __launch_bounds__(kThreads, 1) k_msi_c(MsiLaunch L)
{
    constexpr bool EXACT = std::is_same<TS, double>::value;
    constexpr int NU = (ND == 9) ? 4 : 3;
    constexpr int NL = (ND == 9) ? 5 : 4;
    constexpr int PMAX = (ND > NL + 2) ? ND : NL + 2;   // planes staged per batch
    constexpr int DIAG = (ND == 9) ? 4 : 2;      // index of the main diagonal in a row of A
    constexpr unsigned ES = sizeof(TS);
    constexpr int kLag = LAG, kBlock = Batch<LAG>::kBlock, kSlots = Batch<LAG>::kSlots;
    // per wavefront warp of this CTA.  Consumer side: rings of values from the
    // neighbour warps and their "full" barriers; producer side: staging of the
    // values for the neighbours and the "empty" barriers the neighbours release.
    __shared__ __align__(16) TS ring_up[WPC][kRing * NU];   // from the warp below (LU, forward)
    __shared__ __align__(16) TS out_up[WPC][kRing * NU];    // for the warp above
    __shared__ __align__(16) TS ring_dn[WPC][kRing];        // from the warp above (backward)
    __shared__ __align__(16) TS out_dn[WPC][kRing];         // for the warp below
    __shared__ unsigned long long full_up[WPC][kSlots], empty_up[WPC][kSlots];
    __shared__ unsigned long long full_dn[WPC][kSlots], empty_dn[WPC][kSlots];
    __shared__ unsigned long long stage_bar[WPC][NSTAGE];
    __shared__ unsigned long long idle_bar;       // nothing ever arrives on it (test hook)
    __shared__ unsigned vbad;                     // a factor differs from its IEEE value (helpers)
    __shared__ double red[kThreads];
    __shared__ double part[kMaxCluster + 1];
    extern __shared__ __align__(128) double stage_raw[];   // WPC x NSTAGE x PMAX x kBlock elements
    TS *stage_mem = reinterpret_cast<TS *>(stage_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int sys = blockIdx.x / C;
    const MsiSys S = L.dev ? L.dev[sys] : L.s[sys];
    const int nx = L.nx, ny = L.ny;
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const bool front = wl < WPC;                  // wavefront warp?
    const int fw = front ? wl : 0;               // this warp's per-warp arrays (helpers: unused)
    const int NWG = C * WPC;                      // wavefront warps in the cluster
    const int wg = rank * WPC + wl;               // global wavefront warp index
    const int j = wg * 32 + lane;
    const bool row_ok = front && j < ny;
    const int nsteps = ((nx + 2 * (ny - 1) + kLag * (NWG - 1) + kLag - 1) / kLag) * kLag;
    const int nbatch = nsteps / kLag;
    const int SW = nx + kSkewPad;                 // slots per warp
    const long long PS = (long long)((ny + 31) / 32) * SW * kLine;   // one wavefront-major plane
    const int soff = (64 + kLag) * wg;            // step at which this warp's slot 0 comes up
    const double *__restrict__ a = S.a;
    double *x = S.x;
    // wavefront-major planes of TS: dl1..dlNL, du1..duNU, 1/dl1, residual,
    // sweep result, then A (written by k_skew_a)
    TS *dlp = reinterpret_cast<TS *>(S.ws);
    TS *dup = dlp + NL * PS;
    TS *rl1 = dup + NU * PS;
    TS *rp = rl1 + PS;
    TS *wp = rp + PS;
    TS *asp = wp + PS;
    // a wavefront warp past the last row group (possible when WPC > 1) owns no
    // slots: it reads group 0 (values unused, all its cells are invalid) and
    // stores nothing
    const bool has_rows = front && wg * 32 < ny;
    const long long line0 = (long long)(has_rows ? wg : 0) * SW;
    const long long wbase = line0 * kLine + lane;
#define SK(p, s) (p)[wbase + (long long)(s) * kLine]

    // the continuation launch of a solve with whole-GPU passes: nothing to do
    // when the first iteration already met the stopping test (every CTA of a
    // cluster reads the same word, so all return before any cluster barrier)
    const bool cont = L.ext == 2;
    if (cont) {
        stamp(L, rank, 5);
        if (*ext_words(S, ND, nx, ny).done) {
            stamp(L, rank, 6);
            return;
        }
    }
    if (threadIdx.x == 0) {
        vbad = 0u;
        mbar_init(&idle_bar, 1);
    }
    if (threadIdx.x < WPC) {
        for (int q = 0; q < kSlots; q++) {
            mbar_init(&full_up[threadIdx.x][q], 1); mbar_init(&empty_up[threadIdx.x][q], 1);
            mbar_init(&full_dn[threadIdx.x][q], 1); mbar_init(&empty_dn[threadIdx.x][q], 1);
        }
        for (int q = 0; q < NSTAGE; q++) mbar_init(&stage_bar[threadIdx.x][q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const unsigned sbase = smem_u32(stage_mem);
    const unsigned rup = smem_u32(&ring_up[fw][0]), rdn = smem_u32(&ring_dn[fw][0]);
    const unsigned oup1 = smem_u32(&out_up[fw][0]), odn1 = smem_u32(&out_dn[fw][0]);   // sweeps: one value per slot
    Stager<TS, NSTAGE, PMAX, LAG> st;
    st.mem = stage_mem;
    st.base = fw * NSTAGE * PMAX * kBlock;
    st.bar = &stage_bar[fw][0];
    st.issued = 0;
    st.consumed = 0;
    // links: the up channel (LU, forward) feeds warp g+1, the down channel
    // (backward) feeds warp g-1; the partner may sit in a neighbouring CTA
    const bool has_below = front && wg > 0, has_above = front && wg < NWG - 1;
    unsigned up_ring_dst = 0, up_full_dst = 0, dn_empty_dst = 0;   // partner above
    unsigned dn_ring_dst = 0, dn_full_dst = 0, up_empty_dst = 0;   // partner below
    if (has_above) {
        const int cw = (wl + 1 < WPC) ? wl + 1 : 0, cr = (wl + 1 < WPC) ? rank : rank + 1;
        up_ring_dst = cluster_addr(&ring_up[cw][0], cr);
        up_full_dst = cluster_addr(&full_up[cw][0], cr);
        dn_empty_dst = cluster_addr(&empty_dn[cw][0], cr);
    }
    if (has_below) {
        const int pw = (wl > 0) ? wl - 1 : WPC - 1, pr = (wl > 0) ? rank : rank - 1;
        dn_ring_dst = cluster_addr(&ring_dn[pw][0], pr);
        dn_full_dst = cluster_addr(&full_dn[pw][0], pr);
        up_empty_dst = cluster_addr(&empty_up[pw][0], pr);
    }
    // lagged factorisation: reuse the workspace's factors (decided from the
    // record as the launch found it; rank 0 rewrites it at the end)
    const bool lagged = lag_reuse<TS>(L, S);
    const int lag_age = lagged ? S.lag[1] : 0;
    const bool reuse = L.reuse_lu || lagged || cont;
    // with whole-GPU passes the initial residual of a lagged solve comes from
    // k_ext_r0, and a continuation starts from the first iteration's state
    const bool given_r0 = (L.ext == 1 && lagged) || cont;
    cl.sync();   // mbarriers initialised before any use; A staged by k_skew_a
    bool bad_pivot = false, timed_out = false, hook_ran_out = false;
    int up_base = 0, dn_base = 0;       // batches sent so far on each channel
    stamp(L, rank, 0);

    // ---- incomplete LU (lu2d9 msi2d9-v03.f90:277-432, lu2d5 msi2d5-v03.f90:247-330)
    // run by the wavefront warps; IEEE = true divides with '/', false (FP64)
    // with Markstein quotients, which the helper warps check afterwards
    auto run_lu = [&](auto ieee_tag) {
        constexpr bool IEEE = decltype(ieee_tag)::value;
        TS *ap[ND];
#pragma unroll
        for (int k = 0; k < ND; k++) ap[k] = asp + k * PS;
        for (int t = 0; t < NSTAGE - 1 && t < nbatch; t++) stage_issue<ND>(st, ap, line0, t * kLag - soff, SW);
        TS mw[NU], a1[NU], a2[NU], a3[NU];
#pragma unroll
        for (int q = 0; q < NU; q++) { mw[q] = 0; a1[q] = 0; a2[q] = 0; a3[q] = 0; }
        unsigned piv = 0;                              // a zero or non-finite pivot was seen
        const unsigned oup = smem_u32(&out_up[fw][0]);
        for (int b = 0; b < nbatch; b++) {
            const int tb = b * kLag;
            const int n = up_base + b;                          // global batch number on the channel
            const bool send = has_above && b <= nbatch - 2;   // the last batch is never read
            if (has_below && b >= 1) chan_recv<LAG>(&full_up[fw][0], n - 1, kLag * NU * ES, timed_out);
            if (send) chan_slot_free<LAG>(&empty_up[fw][0], n, timed_out);
            const int bo = stage_wait(st, timed_out) + lane;
            if (b + NSTAGE - 1 < nbatch) stage_issue<ND>(st, ap, line0, (b + NSTAGE - 1) * kLag - soff, SW);
            const unsigned rbase = (unsigned)up_base * kLag;
            // Software-pipelined steps.  A step first issues its critical
            // inputs (the shuffles of the previous step's u; lane 0's ring
            // values were loaded one step ahead), then the previous step's
            // predicated stores, then the next step's loads, then its
            // arithmetic: no branch separates two steps.
            TS cn[ND], rn[NU];
            auto load_step = [&](int k2) {
#pragma unroll
                for (int k = 0; k < ND; k++)
                    cn[k] = lds_v<TS>(sbase + (unsigned)(bo + k * kBlock + k2 * kLine) * ES);
                const unsigned rs = (rbase + (unsigned)(tb + k2 - 1 - kLag)) & (kRing - 1);
#pragma unroll
                for (int q = 0; q < NU; q++) rn[q] = lds_v<TS>(rup + (rs * NU + (unsigned)q) * ES);
            };
            // the previous step's results, stored during the next step
            TS pl[NL], pu[NU], py = 0;
            long long poff = 0;
            bool pst = false, psend = false;
            unsigned pws = 0;
#pragma unroll
            for (int k = 0; k < NL; k++) pl[k] = 0;
#pragma unroll
            for (int q = 0; q < NU; q++) pu[q] = 0;
            auto store_prev = [&]() {
                // y = 1/dl1 (RN for FP64), the forward sweep's reciprocal pivot
#pragma unroll
                for (int k = 0; k < NL; k++) stg_if(dlp + k * PS + poff, pl[k], pst);
#pragma unroll
                for (int q = 0; q < NU; q++) stg_if(dup + q * PS + poff, pu[q], pst);
                stg_if(rl1 + poff, py, pst);
#pragma unroll
                for (int q = 0; q < NU; q++) sts_if(oup + (pws * NU + (unsigned)q) * ES, pu[q], psend);
            };
            load_step(0);
#pragma unroll
            for (int kk = 0; kk < kLag; kk++) {
                const int tau = tb + kk;
                const int s = tau - soff;
                const int i = s - 2 * lane;
                const bool valid = row_ok && i >= 0 && i < nx;
                const int src = tau - 1 - kLag;
                TS v[NU];
#pragma unroll
                for (int q = 0; q < NU; q++) v[q] = shfl_up_v(mw[q]);
                TS cb[ND];
#pragma unroll
                for (int k = 0; k < ND; k++) cb[k] = valid ? cn[k] : (TS)(k == DIAG ? 1 : 0);
#pragma unroll
                for (int q = 0; q < NU; q++) {
                    if (lane == 0) v[q] = (has_below && src >= 0) ? rn[q] : (TS)0;
                    a3[q] = a2[q]; a2[q] = a1[q]; a1[q] = v[q];
                }
                if (kk > 0) store_prev();
                if (kk + 1 < kLag) load_step(kk + 1);
                // an invalid cell sees a unit row: all its divisions are by 1
                // and its outputs are replaced by zeros below
                const TS alpha = (valid && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) ? (TS)0.5 : (TS)0;
                TS l[NL], u[NU], y;
                if constexpr (EXACT) lu_cell<ND, !IEEE>(cb, alpha, mw, a1, a2, a3, l, u, y);
                else lu_cell_f<ND>(cb, alpha, mw, a1, a2, a3, l, u, y);
                piv |= valid ? pivot_bad(l[0]) : 0u;
#pragma unroll
                for (int q = 0; q < NU; q++) u[q] = valid ? u[q] : (TS)0;
#pragma unroll
                for (int k = 0; k < NL; k++) pl[k] = valid ? l[k] : (TS)0;
#pragma unroll
                for (int q = 0; q < NU; q++) pu[q] = u[q];
                py = valid ? y : (TS)0;
                pst = has_rows && s >= 0 && s < SW;
                poff = wbase + (long long)s * kLine;
                psend = lane == 31 && send;
                pws = (rbase + (unsigned)tau) & (kRing - 1);
#pragma unroll
                for (int q = 0; q < NU; q++) mw[q] = u[q];
            }
            store_prev();
            if (lane == 31 && send) chan_send<TS, LAG>(up_ring_dst, up_full_dst, &out_up[fw][0], n, kLag * NU);
            if (lane == 0 && has_below && b >= 2) chan_release<LAG>(up_empty_dst, n - 2);
        }
        if (lane == 0 && has_below && nbatch >= 2) chan_release<LAG>(up_empty_dst, up_base + nbatch - 2);
        if (piv) bad_pivot = true;
        fence_async_global();   // the sweeps read the factors with bulk copies
    };
    // helper warps: those on the SM sub-partitions (warp w runs on w % 4)
    // that no wavefront warp uses, so that their work does not take issue
    // slots or FP64 units from the recurrence
    static_assert(WPC >= 1 && WPC <= 3, "wavefront warps must leave a sub-partition for the helpers");
    const bool helper = (wl & 3) >= WPC;
    const int nhelp = (kThreads / 32 / 4) * (4 - WPC);
    const int hw = (wl >> 2) * (4 - WPC) + ((wl & 3) - WPC);
    // the initial residual: with a factorisation to run, the helper warps
    // compute it meanwhile; with reused factors every warp takes part (the
    // same per-thread sums and tree, so the same norm).  An application of
    // the factors alone gets r = -b from k_skew_rhs.
    double rr0 = 0.0;
    if (!reuse) {
        if (front) run_lu(std::false_type{});
        else if (helper && !L.apply_only) helper_residual<ND, TS>(cl, a, S.b, x, rp, nx, ny, SW, red, part, nhelp, hw);
        up_base += nbatch - 1;
    }
    if (bad_pivot && L.err) atomicOr(L.err, ERR_NONFINITE_PIVOT);
    stamp(L, rank, 1);

    // ---- fb2d9 / fb2d5 (msi2d9-v03.f90:42-262, msi2d5-v03.f90:42-233)
    // (the cluster barrier of the first residual pass or of cluster_total
    // also makes every row's factors and the residual final before the
    // first forward sweep)
    if (L.apply_only) rr0 = 0.0;
    else if (given_r0) rr0 = S.rr[0];
    else if (reuse) rr0 = cluster_residual<ND, TS>(cl, a, S.b, x, (const TS *)nullptr, rp, nx, ny, SW, red, part);
    else rr0 = cluster_total(cl, part);
    stamp(L, rank, 2);
    const double gammarp = L.tol * sqrt(rr0);
    const int cap = (L.nitm > 0) ? L.nitm : kMaxIterUnbounded;
    // while the first sweeps run, the helper warps check that every stored
    // factor is the IEEE result of its stored inputs; their finding is read
    // before the first correction of x
    if constexpr (EXACT) {
        if (helper && !L.reuse_lu)
            verify_factors<ND>(asp, dlp, dup, rl1, nx, ny, SW, PS, rank * WPC, WPC, nhelp, hw, &vbad);
    }
    bool lu_redone = !EXACT || L.reuse_lu || cont;   // reused factors were checked when they were made
    int nit = cont ? 1 : 0;
    double rr = cont ? S.rr[1] : rr0;
    for (;;) {
        nit = nit + 1;
        // test hook: wavefront warp 0 waits, bounded by L.hook_ns, on a
        // barrier that nothing completes, then goes on as usual (its
        // neighbours' own waits are bounded far above that, so every real
        // hand-off still completes and no copy is left in flight)
        if (L.hook_ns && nit == 1 && rank == 0 && wl == 0) {
            if (!mbar_wait_for(&idle_bar, 0u, L.hook_ns)) hook_ran_out = true;
            __syncwarp();
        }
        // forward: L w = -r.  Staged planes {r, dl1..dlNL, 1/dl1}; step kk of
        // a batch is line kk of its block
        if (front) {
            TS *fp[NL + 2];
            fp[0] = rp;
#pragma unroll
            for (int k = 0; k < NL; k++) fp[k + 1] = dlp + k * PS;
            fp[NL + 1] = rl1;
            for (int t = 0; t < NSTAGE - 1 && t < nbatch; t++) stage_issue<NL + 2>(st, fp, line0, t * kLag - soff, SW);
            TS mine = 0, a1 = 0, a2 = 0, a3 = 0;
            for (int b = 0; b < nbatch; b++) {
                const int tb = b * kLag;
                const int n = up_base + b;
                const bool send = has_above && b <= nbatch - 2;
                if (has_below && b >= 1) chan_recv<LAG>(&full_up[fw][0], n - 1, kLag * ES, timed_out);
                if (send) chan_slot_free<LAG>(&empty_up[fw][0], n, timed_out);
                const int bo = stage_wait(st, timed_out) + lane;
                if (b + NSTAGE - 1 < nbatch) stage_issue<NL + 2>(st, fp, line0, (b + NSTAGE - 1) * kLag - soff, SW);
                const TS m0 = mine, b1 = a1, b2 = a2, b3 = a3;   // state at batch start
                const unsigned rbase = (unsigned)up_base * kLag;   // ring position of step 0
                unsigned bad = 0;
#pragma unroll
                for (int pass = 0; pass < (EXACT ? 2 : 1); pass++) {
                    if (pass == 1) {
                        // some quotient of pass 0 may differ from IEEE division:
                        // the batch again from its start state with IEEE division
                        if (!__any_sync(kFull, bad != 0u)) break;
                        mine = m0; a1 = b1; a2 = b2; a3 = b3;
                    }
                    // c: staged coefficients of the current step, rv: ring value
                    // (lane 0's south-east neighbour); both loaded one step ahead.
                    // Lane 31's value for the warp above is stored during the
                    // next step (predicated, no branch between two steps).
                    TS pw = 0;
                    TS c[NL + 2], rv;
#pragma unroll
                    for (int k = 0; k < NL + 2; k++) c[k] = stage_mem[bo + k * kBlock];
                    rv = ring_up[fw][(rbase + (unsigned)(tb - 1 - kLag)) & (kRing - 1)];
#pragma unroll
                    for (int kk = 0; kk < kLag; kk++) {
                        const int tau = tb + kk;
                        const int s = tau - soff;
                        const int i = s - 2 * lane;
                        const bool valid = row_ok && i >= 0 && i < nx;
                        const int src = tau - 1 - kLag;
                        TS v = shfl_up_v(mine);
                        if (kk > 0) {
                            // the previous step's w: to the warp above and to its slot
                            sts_if(oup1 + ((rbase + (unsigned)(tau - 1)) & (kRing - 1)) * ES, pw, lane == 31 && send);
                            stg_if(wp + wbase + (long long)(s - 1) * kLine, pw, has_rows && s - 1 >= 0 && s - 1 < SW);
                        }
                        TS cn[NL + 2], rvn = 0;
                        if (kk + 1 < kLag) {
#pragma unroll
                            for (int k = 0; k < NL + 2; k++)
                                cn[k] = lds_v<TS>(sbase + (unsigned)(bo + k * kBlock + (kk + 1) * kLine) * ES);
                            rvn = lds_v<TS>(rup + ((rbase + (unsigned)(tau - kLag)) & (kRing - 1)) * ES);
                        }
                        if (lane == 0) v = (has_below && src >= 0) ? rv : (TS)0;
                        a3 = a2; a2 = a1; a1 = v;
                        // w = -(r + dl2 w_W + dl3 w_SE + dl4 w_S [+ dl5 w_SW]) / dl1
                        TS wv;
                        if constexpr (EXACT) {
                            double num;
                            if (ND == 9) num = c[0] + c[2] * mine + c[3] * a1 + c[4] * a2 + c[5] * a3;
                            else num = c[0] + c[2] * mine + c[3] * a1 + c[4] * a2;
                            if (pass == 0) {
                                wv = -div_recip(num, c[1], c[NL + 1]);
                                bad |= valid ? range_bad(num, c[1]) : 0u;
                            } else {
                                wv = -(num / c[1]);
                            }
                        } else {
                            float num = fmaf(c[4], a2, fmaf(c[3], a1, fmaf(c[2], mine, c[0])));
                            if (ND == 9) num = fmaf(c[5], a3, num);
                            wv = -num * c[NL + 1];
                        }
                        wv = valid ? wv : (TS)0;
                        mine = wv;
                        pw = wv;
                        if (kk + 1 < kLag) {
#pragma unroll
                            for (int k = 0; k < NL + 2; k++) c[k] = cn[k];
                            rv = rvn;
                        }
                    }
                    sts_if(oup1 + ((rbase + (unsigned)(tb + kLag - 1)) & (kRing - 1)) * ES, pw, lane == 31 && send);
                    {
                        const int sl = tb + kLag - 1 - soff;
                        stg_if(wp + wbase + (long long)sl * kLine, pw, has_rows && sl >= 0 && sl < SW);
                    }
                }
                if (lane == 31 && send) chan_send<TS, LAG>(up_ring_dst, up_full_dst, &out_up[fw][0], n, kLag);
                if (lane == 0 && has_below && b >= 2) chan_release<LAG>(up_empty_dst, n - 2);
            }
            if (lane == 0 && has_below && nbatch >= 2) chan_release<LAG>(up_empty_dst, up_base + nbatch - 2);
            fence_async_global();   // the backward sweep reads w with bulk copies
            __syncwarp();
        }
        up_base += nbatch - 1;
        if (nit == 1) stamp(L, rank, 3);
        // backward: U z = w; time runs from the top-right corner, so step tau
        // is slot Tmax - tau - soff and step kk of a batch is line kLag-1-kk of
        // its block.  Staged planes {w, du1..duNU}
        if (front) {
            const int Tmax = (nx - 1) + 2 * (ny - 1) + kLag * (NWG - 1);
            TS *bp[NU + 1];
            bp[0] = wp;
#pragma unroll
            for (int k = 0; k < NU; k++) bp[k + 1] = dup + k * PS;
            for (int t = 0; t < NSTAGE - 1 && t < nbatch; t++)
                stage_issue<NU + 1>(st, bp, line0, Tmax - (t * kLag + kLag - 1) - soff, SW);
            TS mine = 0, a1 = 0, a2 = 0, a3 = 0;
            for (int b = 0; b < nbatch; b++) {
                const int tb = b * kLag;
                const int n = dn_base + b;
                const bool send = has_below && b <= nbatch - 2;
                if (has_above && b >= 1) chan_recv<LAG>(&full_dn[fw][0], n - 1, kLag * ES, timed_out);
                if (send) chan_slot_free<LAG>(&empty_dn[fw][0], n, timed_out);
                const int bo = stage_wait(st, timed_out) + lane;
                if (b + NSTAGE - 1 < nbatch)
                    stage_issue<NU + 1>(st, bp, line0, Tmax - ((b + NSTAGE - 1) * kLag + kLag - 1) - soff, SW);
                const unsigned rbase = (unsigned)dn_base * kLag;
                // c: staged {w, du} of the current step, rv: ring value (lane
                // 31's north-west neighbour); both loaded one step ahead
                TS c[NU + 1], rv;
                TS pz = 0;   // the previous step's z, stored during the next step
#pragma unroll
                for (int k = 0; k < NU + 1; k++) c[k] = stage_mem[bo + k * kBlock + (kLag - 1) * kLine];
                rv = ring_dn[fw][(rbase + (unsigned)(tb - 1 - kLag)) & (kRing - 1)];
#pragma unroll
                for (int kk = 0; kk < kLag; kk++) {
                    const int tau = tb + kk;
                    const int s = Tmax - tau - soff;
                    const int i = s - 2 * lane;
                    const bool valid = row_ok && i >= 0 && i < nx;
                    const int src = tau - 1 - kLag;
                    TS v = shfl_down_v(mine);
                    if (kk > 0) {
                        // the previous step's z: to the warp below and to its slot
                        sts_if(odn1 + ((rbase + (unsigned)(tau - 1)) & (kRing - 1)) * ES, pz, lane == 0 && send);
                        stg_if(wp + wbase + (long long)(s + 1) * kLine, pz, has_rows && s + 1 >= 0 && s + 1 < SW);
                    }
                    TS cn[NU + 1], rvn = 0;
                    if (kk + 1 < kLag) {
#pragma unroll
                        for (int k = 0; k < NU + 1; k++)
                            cn[k] = lds_v<TS>(sbase + (unsigned)(bo + k * kBlock + (kLag - 2 - kk) * kLine) * ES);
                        rvn = lds_v<TS>(rdn + ((rbase + (unsigned)(tau - kLag)) & (kRing - 1)) * ES);
                    }
                    if (lane == 31) v = (has_above && src >= 0) ? rv : (TS)0;
                    a3 = a2; a2 = a1; a1 = v;
                    // z = w - du1 z_E - du2 z_NW - du3 z_N [- du4 z_NE]; E = own previous
                    TS z;
                    if constexpr (EXACT) {
                        if (ND == 9) z = c[0] - c[1] * mine - c[2] * a1 - c[3] * a2 - c[4] * a3;
                        else z = c[0] - c[1] * mine - c[2] * a1 - c[3] * a2;
                    } else {
                        z = fmaf(-c[3], a2, fmaf(-c[2], a1, fmaf(-c[1], mine, c[0])));
                        if (ND == 9) z = fmaf(-c[4], a3, z);
                    }
                    z = valid ? z : (TS)0;
                    mine = z;
                    pz = z;
                    if (kk + 1 < kLag) {
#pragma unroll
                        for (int k = 0; k < NU + 1; k++) c[k] = cn[k];
                        rv = rvn;
                    }
                }
                sts_if(odn1 + ((rbase + (unsigned)(tb + kLag - 1)) & (kRing - 1)) * ES, pz, lane == 0 && send);
                {
                    const int sl = Tmax - (tb + kLag - 1) - soff;
                    stg_if(wp + wbase + (long long)sl * kLine, pz, has_rows && sl >= 0 && sl < SW);
                }
                if (lane == 0 && send) chan_send<TS, LAG>(dn_ring_dst, dn_full_dst, &out_dn[fw][0], n, kLag);
                if (lane == 31 && has_above && b >= 2) chan_release<LAG>(dn_empty_dst, n - 2);
            }
            if (lane == 31 && has_above && nbatch >= 2) chan_release<LAG>(dn_empty_dst, dn_base + nbatch - 2);
        }
        dn_base += nbatch - 1;
        if (nit == 1) stamp(L, rank, 4);
        // var = z + var, then the new residual
        if (!lu_redone) {
            // the helpers' finding on the Markstein factorisation: if any
            // factor differs from IEEE division, factorise again with IEEE
            // division and repeat the first iteration (x is still untouched)
            cl.sync();
            unsigned any = 0;
            for (int c = 0; c < C; c++) any |= *cl.map_shared_rank(&vbad, c);
            lu_redone = true;
            if (any) {
                if (rank == 0 && threadIdx.x == 0) atomicAdd(&g_lu_redo, 1ull);
                cl.sync();   // every CTA has read the findings
                if (front) run_lu(std::true_type{});
                up_base += nbatch - 1;
                if (bad_pivot && L.err) atomicOr(L.err, ERR_NONFINITE_PIVOT);
                cl.sync();   // every row's factors are final
                nit = 0;
                continue;
            }
        }
        if (L.apply_only) break;   // x += z by k_unskew_add after the launch
        if (L.ext == 1) break;     // x += z, the residual and the test on the whole GPU
        rr = cluster_residual<ND, TS>(cl, a, S.b, x, wp, rp, nx, ny, SW, red, part);
        if (nit == 1) stamp(L, rank, 5);
        if (sqrt(rr) < gammarp) break;
        if (nit == cap) {
            if (L.nitm <= 0 && L.err && rank == 0 && threadIdx.x == 0) atomicOr(L.err, ERR_WAIT_TIMEOUT);
            break;
        }
    }
#undef SK
    if (front && st.consumed < st.issued) {
        // only after a timed-out wait: let the copies still in flight land
        // before this CTA's shared memory goes away (bounded)
        bool again = false;
        while (st.consumed < st.issued) (void)stage_wait(st, again);
    }
    if ((timed_out || hook_ran_out) && L.err) atomicOr(L.err, ERR_SPIN_TIMEOUT);
    if (L.ext == 1) {
        // what the whole-GPU passes and the continuation need to know
        int* status = ext_words(S, ND, nx, ny).status;
        if (timed_out || hook_ran_out) atomicOr(status, kExtTimedOut);
        if (bad_pivot) atomicOr(status, kExtBadPivot);
        if (lagged && rank == 0 && threadIdx.x == 0) atomicOr(status, kExtLagged);
    }
    if (rank == 0 && threadIdx.x == 0 && !L.apply_only) {
        if (S.nit) *S.nit = nit;
        if (S.rr) { S.rr[0] = rr0; if (L.ext != 1) S.rr[1] = rr; }
        if (!EXACT && L.lag_max > 0 && S.lag && !L.reuse_lu && L.ext != 1) {
            // the record for the next solve: fresh factors are one solve old;
            // reused ones age, and are renewed next time once they needed a
            // second iteration (or anything went wrong)
            const int st = cont ? *ext_words(S, ND, nx, ny).status : 0;
            const bool lag_solve = cont ? (st & kExtLagged) != 0 : lagged;
            const bool renew = timed_out || hook_ran_out || bad_pivot || (st & (kExtTimedOut | kExtBadPivot)) ||
                               (lag_solve && nit > 1);
            S.lag[0] = S.tag;
            S.lag[1] = renew ? L.lag_max : (lag_solve ? lag_age + 1 : 1);
        }
    }
    cl.sync();   // no CTA leaves while another may still write into its shared memory
    stamp(L, rank, 6);
}

bool msi_warp_supported(int ny) { return ny <= 1024; }

long long msi_lu_redo_count()
{
    unsigned long long v = 0;
    if (cudaMemcpyFromSymbol(&v, g_lu_redo, sizeof v) != cudaSuccess) return -1;
    return (long long)v;
}

template <int ND, int WPC, int NSTAGE, typename TS, int LAG>
static size_t stage_bytes()
{
    constexpr int NL = (ND == 9) ? 5 : 4;
    constexpr int PMAX = (ND > NL + 2) ? ND : NL + 2;
    return (size_t)WPC * NSTAGE * PMAX * Batch<LAG>::kBlock * sizeof(TS);
}

// launches one cluster per system if the cluster shape can be scheduled;
// *fits = false (and nothing launched) otherwise
template <int ND, int WPC, int NSTAGE, typename TS, int LAG>
static cudaError_t launch_cluster(const MsiLaunch &L, int nsys, cudaStream_t st, bool *fits)
{
    *fits = false;
    const int nwarps = (L.ny + 31) / 32;
    const int C = (nwarps + WPC - 1) / WPC;
    if (C > kMaxCluster) return cudaSuccess;
    auto kern = k_msi_c<ND, WPC, NSTAGE, TS, LAG>;
    const size_t smem = stage_bytes<ND, WPC, NSTAGE, TS, LAG>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(C * nsys));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
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
    // A into wavefront-major order first (all systems, whole GPU), unless the
    // factors (made from that copy) are reused
    const bool apply = L.apply_only && L.reuse_lu && L.dev == nullptr && nsys <= 2;
    const long long N = (long long)L.nx * L.ny;
    const dim3 cg((unsigned)((N + 255) / 256 < 1184 ? (N + 255) / 256 : 1184), (unsigned)nsys);
    // the passes over all cells on the whole GPU (grids of kExtMinCells and
    // more, where they outweigh three extra launches)
    bool ext = !L.apply_only && !L.reuse_lu && L.dev == nullptr && nsys <= 2 && N >= kExtMinCells;
    for (int k = 0; k < nsys && ext; k++) ext = L.s[k].rr != nullptr && L.s[k].nit != nullptr;
    MsiLaunch La = L;
    La.apply_only = apply ? 1 : 0;
    if (apply) La.nitm = 1;
    La.ext = ext ? 1 : 0;
    const bool lag_r0 = ext && L.lag_max > 0 && !std::is_same<TS, double>::value;
    int launches = 1;
    if (!L.reuse_lu) {
        const dim3 sg((unsigned)((L.nx + kSkewPad + kSkewTile - 1) / kSkewTile), (unsigned)nwarps,
                      (unsigned)(nsys * ND));
        k_skew_a<ND, TS><<<sg, 256, 0, st>>>(La);
        launches++;
        if (lag_r0) {
            k_ext_r0<ND, TS><<<dim3(kExtBlocks, (unsigned)nsys), 256, 0, st>>>(La);
            launches++;
        }
    } else if (apply) {
        k_skew_rhs<ND, TS><<<cg, 256, 0, st>>>(La);
        launches++;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaLaunchKernelEx(&cfg, kern, La);
    if (e != cudaSuccess) return e;
    if (apply) {
        k_unskew_add<ND, TS><<<cg, 256, 0, st>>>(La);
        launches++;
    } else if (ext) {
        k_ext_update<ND, TS><<<cg, 256, 0, st>>>(La);
        k_ext_resid<ND, TS><<<dim3(kExtBlocks, (unsigned)nsys), 256, 0, st>>>(La);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        MsiLaunch Lc = La;
        Lc.ext = 2;
        e = cudaLaunchKernelEx(&cfg, kern, Lc);
        launches += 3;
    }
    msi_note_launches(launches);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// fewest wavefront warps per CTA (one SM per warp) whose cluster fits,
// unless the caller asked for one schedule
template <int ND, typename TS, int LAG>
static cudaError_t launch_schedules(const MsiLaunch &L, int nsys, cudaStream_t st, bool *done)
{
    cudaError_t e = cudaSuccess;
    if (L.variant != 2) {
        e = launch_cluster<ND, 1, 4, TS, LAG>(L, nsys, st, done);
        if (e != cudaSuccess || *done || L.variant == 1) return e;
    }
    return launch_cluster<ND, 2, 2, TS, LAG>(L, nsys, st, done);
}

template <int ND, typename TS>
static cudaError_t launch_nd(const MsiLaunch &L, int nsys, cudaStream_t st, bool *done)
{
    // the bulk copies need 16-byte aligned scratch (systems given through a
    // device array cannot be checked here) and the wavefront-major layout
    // must fit in the scratch
    *done = false;
    bool aligned = L.dev == nullptr;
    for (int k = 0; k < nsys && aligned; k++) aligned = ((uintptr_t)L.s[k].ws % 16) == 0;
    const bool room = L.ws_cap == 0 || L.ws_cap >= msi_cluster_work_doubles(ND, L.nx, L.ny);
    const bool small = (long long)L.nx * L.ny < (1LL << 31);   // 32-bit cell indices in the passes
    if (!(aligned && room && small)) return cudaSuccess;
    if constexpr (std::is_same<TS, float>::value) {
        if ((long long)L.nx * L.ny >= kLongLagCells) return launch_schedules<ND, TS, 32>(L, nsys, st, done);
    }
    return launch_schedules<ND, TS, 16>(L, nsys, st, done);
}

// m2d_test_wait_hook's setting for the cluster kernel (0: off)
static unsigned long long g_msi_hook_ns = 0;
void set_msi_wait_hook(unsigned long long ns) { g_msi_hook_ns = ns; }

cudaError_t launch_msi_warp(int nd, const MsiLaunch &L0, int nsys, cudaStream_t st)
{
    MsiLaunch L = L0;
    L.hook_ns = g_msi_hook_ns;
    bool done = false;
    cudaError_t e;
    if (L.prec == 1)
        e = nd == 9 ? launch_nd<9, float>(L, nsys, st, &done) : launch_nd<5, float>(L, nsys, st, &done);
    else
        e = nd == 9 ? launch_nd<9, double>(L, nsys, st, &done) : launch_nd<5, double>(L, nsys, st, &done);
    if (e != cudaSuccess || done) return e;
    return launch_msi_generic(nd, L0, nsys, st);
}

}  // namespace m2d
