// m2d_noalloc.cu -- MSI solve on device arrays without any device allocation.
//
// Some callers cannot allocate device memory when they call the solver: a
// host program that has handed all device memory to its own pool up front
// (an OpenACC or CUDA Fortran runtime, or a framework's caching allocator),
// or one whose time-critical loop must not call cudaMalloc / cudaFree because
// those calls synchronise the device.  m2d_msi_solve_device needs a
// caller-allocated workspace; this variant takes its workspace from a fixed
// array in the library's own device memory instead.
//
// The array is a file-scope __device__ variable of kNoallocScratchDoubles
// doubles (12 MiB): every GPU that loads the library holds it until the
// process exits.  Host code cannot pass the symbol itself to a kernel (on the
// host it names a host-side stand-in, not a device address), so every call,
// with the caller's device current, looks up the device address with
// cudaGetSymbolAddress and passes that pointer on.  The first call on a
// device also loads the library's device code there, so make it before any
// stream capture.  Because the address is looked up again on every call, a
// device reset between two calls (which reloads the device code, possibly at
// another address) does not leave a stale pointer behind.  All calls on a
// device share the one array and it keeps the last call's contents: the
// solver writes every scratch word before it reads it (factors, residual,
// norms), so nothing needs clearing, but calls that overlap on the GPU (two
// streams, or two host threads) race on it and must be serialised by the
// caller.  The cluster kernel runs only while its wavefront-major layout fits
// in the array, that is while 32*ceil(ny/32) * (nx + 62) is at most 74,849
// (9 diagonals) or 104,789 (5 diagonals); otherwise the one-CTA kernel,
// bitwise equal but slower, runs.  At 514 x 258 (512 x 256 real cells) the
// 9-diagonal solve therefore takes the one-CTA kernel.
#include "m2d_solvers.cuh"
#include "../../include/mach2d_b200.h"

namespace {

const long kNoallocScratchDoubles = 1572864;   // 12 MiB

__device__ __align__(256) double g_msi_scratch[kNoallocScratchDoubles];

}  // namespace

extern void m2d_set_last_error_msg(const char *);
extern "C" int m2d_msi_solve_device_ws(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                                   const double *d_b, double *d_x, double *d_work, long work_doubles,
                                   void *stream, int *d_nit, unsigned long long *d_times, int prec);

extern "C" long m2d_msi_noalloc_max_cells(int nd)
{
    if (nd != 9 && nd != 5) return -1;
    return (kNoallocScratchDoubles - 4) / (nd == 9 ? 10 : 8);
}

extern "C" int m2d_msi_solve_device_noalloc(int nd, int nx, int ny, int nitm, double tol,
                                            const double *d_a, const double *d_b, double *d_x,
                                            void *stream, int *d_nit)
{
    if ((nd != 9 && nd != 5) || nx < 4 || ny < 4 || !d_a || !d_b || !d_x) {
        m2d_set_last_error_msg("msi_solve_device_noalloc: bad arguments");
        return M2D_ERR_ARG;
    }
    // the plain-layout kernel must fit; the wavefront-major one is used when
    // it fits as well
    const long need = (long)m2d::msi_generic_work_doubles(nd, nx, ny) + 4;
    if (ny > m2d::msi_max_ny()) {
        m2d_set_last_error_msg("msi_solve_device_noalloc: ny exceeds m2d_msi_max_ny()");
        return M2D_ERR_TOO_LARGE;
    }
    if (need > kNoallocScratchDoubles) {
        m2d_set_last_error_msg(nd == 9
            ? "msi_solve_device_noalloc: nx*ny exceeds the maximum of 157286 cells for the 9-diagonal solve"
            : "msi_solve_device_noalloc: nx*ny exceeds the maximum of 196607 cells for the 5-diagonal solve");
        return M2D_ERR_TOO_LARGE;
    }
    // the device address of the array on the current device (looked up on
    // every call: it allocates nothing and stays right across device resets)
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_msi_scratch);
    if (e != cudaSuccess || !ptr) {
        m2d_set_last_error(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
        return M2D_ERR_CUDA;
    }
    double *work = (double *)ptr;
    return m2d_msi_solve_device_ws(nd, nx, ny, nitm, tol, d_a, d_b, d_x, work, kNoallocScratchDoubles, stream,
                                   d_nit, nullptr, 0);
}
