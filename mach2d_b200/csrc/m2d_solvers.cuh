// m2d_solvers.cuh -- MSI (Schneider-Zedan strongly implicit) and line-TDMA
// solvers for the 9- and 5-diagonal systems of MACH-2D.
#pragma once
#include "m2d_common.cuh"

namespace m2d {

// One linear system A x = b.  A is plane-major (ND planes of N doubles).
// ws is msi_work_doubles(ND, nx, ny) doubles of scratch holding the
// incomplete factors (5+4 planes for ND=9, 4+3 for ND=5) and the residual;
// its layout belongs to the kernel that runs.
struct MsiSys {
    const double *a;
    const double *b;
    double *x;
    double *ws;
    int *nit;          // iterations performed (device int)
    double *rr;        // [0] = |r0|^2, [1] = |r_final|^2 (device doubles)
    int *lag;          // MsiLaunch::lag_max > 0: the workspace's factor record (device ints):
                       // [0] tag of the system whose factors ws holds, [1] solves since they were
                       // made; may be null (factorise every solve)
    int tag;           // this system's tag (nonzero)
};

// scratch doubles one system needs (the larger of the two kernels' layouts),
// and what each layout needs on its own: launch_msi uses the cluster kernel
// only when ws_cap leaves room for its layout
size_t msi_work_doubles(int nd, int nx, int ny);
size_t msi_generic_work_doubles(int nd, int nx, int ny);
size_t msi_cluster_work_doubles(int nd, int nx, int ny);
// the cluster kernel's factor planes are "wavefront-major": slot
// ((j/32) * (nx + 62) + i + 2 (j%32)) * 32 + j%32 holds cell (i, j), so the
// 32 rows a warp sweeps read and write one contiguous 256-byte line per step
size_t msi_skew_plane(int nx, int ny);

// doubles after the wavefront-major planes of a cluster-kernel workspace:
// block partial sums, counters and flags of the whole-GPU residual passes
constexpr int kMsiExtScratch = 1024;

struct MsiLaunch {
    int nx, ny, nitm;
    double tol;
    MsiSys s[2];               // up to two systems passed by value ...
    const MsiSys *dev;         // ... or an array of gridDim.x systems in device memory
    int *err;                  // device error word (ERR_* bits), may be null
    unsigned long long *prof;  // optional phase timestamps (ns, %globaltimer), may be null:
                               // start, after LU, after r0, first forward, first backward,
                               // first residual, end
    size_t ws_cap;             // doubles each ws holds; 0 = at least msi_work_doubles()
    int prec;                  // 0: FP64 throughout (bitwise reference); 1: FP32 factors and
                               // sweeps inside the FP64 iteration (cluster kernel only)
    unsigned long long hook_ns;  // test hook of the cluster kernel (set by launch_msi_warp from
                                 // m2d_test_wait_hook; 0: off)
    int reuse_lu;              // 1: the workspaces already hold these systems' incomplete factors
                               // (an earlier launch on the same A, sizes, precision and schedule,
                               // workspace untouched since): the cluster kernel skips the transpose
                               // of A and the factorisation.  The one-CTA kernel always factorises;
                               // the results are the same either way.
    int apply_only;            // with reuse_lu = 1 and nitm = 1 (cluster kernel): x += (LU)^-1 b,
                               // the preconditioner application of a Krylov method -- the right
                               // side enters the sweeps directly (r = -b, as for x = 0) and no
                               // residual or norm is computed; S.nit and S.rr are not written
    int lag_max;               // > 0 (FP32 factors, cluster kernel): lagged factorisation.  A system
                               // whose workspace holds its own factors from fewer than lag_max solves
                               // ago, and whose last solve took one iteration, reuses them (no
                               // transpose of A, no factorisation); the iteration, its FP64 residual
                               // and stopping test are unchanged, so only the preconditioner is
                               // older.  A stale solve that needs a second iteration marks the
                               // factors for renewal at the next solve.  0: factorise every solve.
    int ext;                   // set by the cluster launcher, not by callers: 0 the residual passes
                               // run inside the cluster kernel; 1 the first launch of a solve whose
                               // passes run on the whole GPU (it stops after the first sweep pair);
                               // 2 the continuation launch (further iterations, if any are needed)
    int variant;               // wavefront schedule: 0 automatic (one wavefront warp per SM when the
                               // cluster fits, else two), 1 one warp per SM (4 staging stages),
                               // 2 two warps per SM (2 stages), 3 the one-CTA kernel (FP64 only);
                               // a schedule that cannot run falls back to the one-CTA kernel.  Every
                               // schedule gives the same iterates.
};

}  // namespace m2d
struct m2d_unet;
struct m2d_learned_report;
namespace m2d {
// the learned p' solve (m2d_pprime_solve_learned) whose MSI iteration may
// reuse lagged FP32 factors (m2d_unet.cu)
int pprime_solve_learned_lagged(::m2d_unet *n, int nx, int ny, int nitm, double tol, const double *d_a,
                                const double *d_b, double *d_x, const double *d_Jp, double *d_work, int prec,
                                void *stream, ::m2d_learned_report *rep, int *lag_rec, int lag_tag, int lag_max);

// kernels the last launch_msi on this host thread issued (transposes and
// whole-GPU passes included)
int msi_last_launch_count();
void msi_note_launches(int n);

// Largest ny the one-CTA wavefront kernel accepts (its shared-memory ring
// holds 4 steps x 4 factor values per row).
int msi_max_ny();
int msi_block_threads(int ny);
size_t msi_smem_bytes(int nd, int ny);

// Solves gridDim.x = nsys systems, one CTA each: LU factorisation (lu2d9 /
// lu2d5) followed by the fb2d9 / fb2d5 iteration, all inside one launch.
cudaError_t launch_msi(int nd, const MsiLaunch &L, int nsys, cudaStream_t st);
// the warp-synchronous kernel used by launch_msi for ny <= 1024 (m2d_msi_warp.cu)
bool msi_warp_supported(int ny);
// factorisations the cluster kernel repeated with IEEE division (current device)
long long msi_lu_redo_count();
cudaError_t launch_msi_warp(int nd, const MsiLaunch &L, int nsys, cudaStream_t st);
// the one-step-per-barrier kernel, any ny <= msi_max_ny() (m2d_msi.cu)
cudaError_t launch_msi_generic(int nd, const MsiLaunch &L, int nsys, cudaStream_t st);

// tdma2d9 / tdma2d5: nitm x (x-line sweep, y-line sweep).  P, Q: N doubles each.
cudaError_t launch_tdma(int nd, int nx, int ny, int nitm, const double *a, const double *b,
                        double *x, double *P, double *Q, cudaStream_t st);

// independent tridiagonal lines, line l element i at l*n + i (the x-line
// layout of tdma2d9): aw, ap, ae, d -> x
cudaError_t launch_tdma_lines(int n, int nlines, const double *aw, const double *ap,
                              const double *ae, const double *d, double *x, double *P,
                              double *Q, cudaStream_t st);
// the same lines by parallel cyclic reduction, one CTA per line (n <= 2048);
// not bitwise equal to the sequential recurrence
bool tdma_lines_pcr_supported(int n);
cudaError_t launch_tdma_lines_pcr(int n, int nlines, const double *aw, const double *ap, const double *ae,
                                  const double *d, double *x, cudaStream_t st);

}  // namespace m2d
