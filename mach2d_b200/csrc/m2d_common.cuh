// m2d_common.cuh -- shared definitions for the MACH-2D B200 kernels.
//
// Layout (identical to the reference's Fortran arrays, so host buffers of a
// Fortran caller can be copied without repacking):
//   nx, ny   volumes per direction including the ghost ring, N = nx*ny
//   cell (i,j), 1-based, lives at offset (j-1)*nx + (i-1)
//   a 9-diagonal matrix a(N,9) is plane-major: diagonal k (1..9, order
//   SW,S,SE,W,P,E,NW,N,NE) occupies [(k-1)N, kN); 5-diagonal order S,W,P,E,N.
// Every plane is contiguous along i, so a warp reading 32 consecutive cells of
// one row issues one coalesced 256-byte request.
//
// FP64 kernels are compiled with -fmad=false: every a*b+c is rounded twice, as
// the reference's x86-64 build evaluates it, so stencil results are bitwise
// equal to the CPU restatement.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cmath>

namespace m2d {

struct Dims {
    int nx, ny;
    long long N;
};

__host__ __device__ __forceinline__ long long cell(int nx, int i, int j)
{
    return (long long)(j - 1) * nx + (i - 1);
}

// SIGN(0.5, x) of Fortran, as gfortran implements it (copysign)
__device__ __forceinline__ double sgn05(double x) { return copysign(0.5, x); }

// status codes shared with the C ABI
enum {
    ST_OK = 0,
    ST_CUDA = 1,
    ST_ARG = 2,
    ST_NAN = 3,
    ST_TIMEOUT = 4,
    ST_NOMEM = 5,
    ST_TOO_LARGE = 6,
};

// device-side error word bits (written by kernels, read by the host)
enum {
    ERR_NONFINITE_PIVOT = 1,
    ERR_WAIT_TIMEOUT = 2,      // an unbounded MSI iteration (nitm <= 0) reached its cap
    ERR_BAD_SHAPE = 4,
    ERR_SPIN_TIMEOUT = 8,      // a bounded device-side wait (mbarrier, hand-off) ran out
};

// Test hooks (m2d_test_wait_hook): the next launches of the MSI cluster
// kernel / the tcgen05 convolution make one extra wait, bounded by ns
// nanoseconds, on an mbarrier that nothing completes (0 switches it off).
void set_msi_wait_hook(unsigned long long ns);
void set_conv_wait_hook(unsigned long long ns);

}  // namespace m2d

#define M2D_CUDA_TRY(expr)                                    \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) { m2d_set_last_error(_e, #expr, __FILE__, __LINE__); return m2d::ST_CUDA; } \
    } while (0)

void m2d_set_last_error(cudaError_t e, const char *what, const char *file, int line);
