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
// host it names a host-side stand-in, not a device address), so the first
// call on each device, with that device current, resolves the device address
// with cudaGetSymbolAddress and caches it; make that first call before any
// stream capture.  All calls on a device share the one array and it keeps
// the last call's contents: the solver writes every scratch word before it
// reads it (factors, residual, norms), so nothing needs clearing, but calls
// that overlap on the GPU (two streams, or two host threads) race on it and
// must be serialised by the caller.
#include <mutex>
#include "m2d_solvers.cuh"
#include "../../include/mach2d_b200.h"

namespace {

const long kNoallocScratchDoubles = 1572864;   // 12 MiB
const int kMaxDevices = 64;

__device__ __align__(256) double g_msi_scratch[kNoallocScratchDoubles];

std::mutex g_mutex;
double *g_scratch_addr[kMaxDevices] = {nullptr};

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
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        m2d_set_last_error(e, "cudaGetDevice", __FILE__, __LINE__);
        return M2D_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        m2d_set_last_error_msg("msi_solve_device_noalloc: device ordinal out of range");
        return M2D_ERR_ARG;
    }
    double *work = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_scratch_addr[dev]) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_msi_scratch);
            if (e != cudaSuccess || !ptr) {
                m2d_set_last_error(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
                return M2D_ERR_CUDA;
            }
            g_scratch_addr[dev] = (double *)ptr;
        }
        work = g_scratch_addr[dev];
    }
    return m2d_msi_solve_device_ws(nd, nx, ny, nitm, tol, d_a, d_b, d_x, work, kNoallocScratchDoubles, stream,
                                   d_nit, nullptr, 0);
}
