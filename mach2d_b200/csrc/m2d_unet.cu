// m2d_unet.cu -- the learned p' preconditioner: a 4-level U-Net (channels
// 16/32/64/128, 3x3 convolutions, GELU, BF16 weights and activations, FP32
// accumulation) with hand-written forward, backward and Adam kernels.
// No counterpart in the reference: it maps (p' residual, the nine
// coefficient planes, the Jacobian) to a p' correction that the flexible
// pressure-correction solve (m2d_pprime_solve_learned) tries before the MSI
// iteration, keeping plain MSI as the fallback and the arbiter.
//
// Layout: activations are pixel-major (NHWC), a pixel's channels contiguous,
// so the K slice of one 3x3 tap is one 32-byte row per 16 channels.  Images
// are the real cells of the p' system (pixel (y, x) = cell (x+2, y+2)),
// zero-padded to multiples of 8.  Every convolution is an implicit GEMM
// (M = 8x16 pixel tile, N = output channels, K = 9 taps x input channels)
// on the tensor cores (mma.sync m16n8k16 BF16 -> FP32) from shared-memory
// tiles read with ldmatrix; the halo tile is XOR-swizzled so that the eight
// rows of every ldmatrix fall in distinct banks.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cmath>
#include <cstring>
#include <vector>
#include "m2d_common.cuh"
#include "m2d_solvers.cuh"
#include "../../include/mach2d_b200.h"

using bf16 = __nv_bfloat16;

void m2d_set_last_error_msg(const char *);

namespace {

constexpr int kLevels = 4;
constexpr int kChan[kLevels] = {16, 32, 64, 128};
constexpr int kInPlanes = 11;     // residual, 9 coefficients, Jacobian
constexpr int kInChan = 16;       // padded to the MMA K step
constexpr int kConvs = 14;

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
__device__ __forceinline__ float gelu(float x)
{
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float x)
{
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x * x);
}

// ------------------------------------------------------------- convolution
// Halo tile of one 8x16 pixel tile: 10 x 18 pixels x 16 channels (32 B per
// pixel); the two 16-byte halves of pixel hp are swapped when bit 2 of hp is
// set, which puts any 8 consecutive pixels in distinct banks.
constexpr int kTileH = 8, kTileW = 16, kHaloW = kTileW + 2, kHaloPix = (kTileH + 2) * kHaloW;
constexpr int kWRow = 304;        // bytes per output channel of a weight chunk (9 x 32 + 16 pad)

__device__ __forceinline__ int halo_off(int hp, int half) { return hp * 32 + ((half ^ ((hp >> 2) & 1)) << 4); }

struct ConvArgs {
    const bf16 *x; int ldx;        // input view (channel 0 of the slice), channel stride
    const bf16 *w;                 // [cout][9][cin]
    const float *bias;             // [cout] or null
    float *z;                      // pre-activation [pixel][cout], or null
    bf16 *y; int ldy;              // activation view, or null
    float *yf; int ldyf;           // FP32 output view (input gradients), or null
    int accumulate;                // yf += result
    int act;                       // 1: y = gelu(result)
    int nimg, H, W, cin, cout;
    int *err;                      // device error word (ERR_SPIN_TIMEOUT), may be null
    const bf16 *wtc;               // the weights in the tcgen05 staging order, or null
    unsigned long long hook_ns;    // test hook: CTA 0's extra wait on an idle barrier (0: none)
};

template <int NT>
__global__ void __launch_bounds__(128) k_conv3x3(ConvArgs a)
{
    __shared__ __align__(128) unsigned char s_halo[kHaloPix * 32];
    __shared__ __align__(128) unsigned char s_w[NT * kWRow];
    const int tilesx = (a.W + kTileW - 1) / kTileW;
    const int ty0 = (blockIdx.x / tilesx) * kTileH, tx0 = (blockIdx.x % tilesx) * kTileW;
    const int co0 = blockIdx.y * NT;
    const int img = blockIdx.z;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float acc[2][NT / 8][4];
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
        for (int n = 0; n < NT / 8; n++) acc[m][n][0] = acc[m][n][1] = acc[m][n][2] = acc[m][n][3] = 0.f;
    const uint32_t sh = smem_u32(s_halo), sw = smem_u32(s_w);
    for (int c0 = 0; c0 < a.cin; c0 += 16) {
        for (int q = threadIdx.x; q < kHaloPix * 2; q += 128) {
            const int hp = q >> 1, h = q & 1;
            const int hy = hp / kHaloW, hx = hp - hy * kHaloW;
            const int gy = ty0 + hy - 1, gx = tx0 + hx - 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < a.H && gx >= 0 && gx < a.W)
                v = *reinterpret_cast<const uint4 *>(a.x + ((long long)(img * a.H + gy) * a.W + gx) * a.ldx + c0 + h * 8);
            *reinterpret_cast<uint4 *>(s_halo + halo_off(hp, h)) = v;
        }
        for (int q = threadIdx.x; q < NT * 18; q += 128) {
            const int n = q / 18, r = q - n * 18, tap = r >> 1, h = r & 1;
            const uint4 v = *reinterpret_cast<const uint4 *>(a.w + ((long long)(co0 + n) * 9 + tap) * a.cin + c0 + h * 8);
            *reinterpret_cast<uint4 *>(s_w + n * kWRow + tap * 32 + h * 16) = v;
        }
        __syncthreads();
#pragma unroll 1
        for (int tap = 0; tap < 9; tap++) {
            const int dy = tap / 3, dx = tap - dy * 3;
            uint32_t af[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                const int col = (lane & 7) + ((lane >> 3) & 1) * 8, half = lane >> 4;
                const int hp = (warp * 2 + mt + dy) * kHaloW + col + dx;
                ldsm_x4(sh + halo_off(hp, half), af[mt]);
            }
#pragma unroll
            for (int np = 0; np < NT / 16; np++) {
                const int n = np * 16 + (lane & 7) + (lane >> 4) * 8, kh = (lane >> 3) & 1;
                uint32_t bfr[4];
                ldsm_x4(sw + n * kWRow + tap * 32 + kh * 16, bfr);
#pragma unroll
                for (int mt = 0; mt < 2; mt++) {
                    mma_bf16(acc[mt][2 * np], af[mt], bfr[0], bfr[1]);
                    mma_bf16(acc[mt][2 * np + 1], af[mt], bfr[2], bfr[3]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < NT / 8; nt++)
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                const int gy = ty0 + warp * 2 + mt, gx = tx0 + (lane >> 2) + hh * 8;
                if (gy >= a.H || gx >= a.W) continue;
                const long long p = (long long)(img * a.H + gy) * a.W + gx;
                const int co = co0 + nt * 8 + (lane & 3) * 2;
                float v0 = acc[mt][nt][hh * 2], v1 = acc[mt][nt][hh * 2 + 1];
                if (a.bias) { v0 += a.bias[co]; v1 += a.bias[co + 1]; }
                if (a.z) *reinterpret_cast<float2 *>(a.z + p * a.cout + co) = make_float2(v0, v1);
                if (a.yf) {
                    float2 *d = reinterpret_cast<float2 *>(a.yf + p * a.ldyf + co);
                    if (a.accumulate) { const float2 o = *d; v0 += o.x; v1 += o.y; }
                    *d = make_float2(v0, v1);
                }
                if (a.y) {
                    if (a.act) { v0 = gelu(v0); v1 = gelu(v1); }
                    *reinterpret_cast<__nv_bfloat162 *>(a.y + p * a.ldy + co) = __floats2bfloat162_rn(v0, v1);
                }
            }
}

// ---- the same convolution on the 5th-generation tensor cores (tcgen05)
// One CTA computes two 128-pixel row segments (image rows gy0, gy0 + 1, the
// same columns) for all output channels: for row r, D_r[128 x N] (FP32, in
// tensor memory columns [rN, rN + N)) = sum over 16-channel chunks and the 9
// taps of A_{r,tap}[128 x 16] * B_tap[N x 16]^T, each one tcgen05.mma of
// M = 128, N = cout, K = 16 issued by one thread; the two rows share the
// staged weights.  Operands sit in shared memory in the K-major layout
// without swizzle: 8-row core matrices of 16-byte rows, the two 8-channel
// halves of K `lbo` bytes apart, consecutive groups of 8 rows 128 bytes
// apart.  A chunk's halo is stored [K half][4 rows][130 pixels][8 channels],
// so the A operand of (row r, tap (dy, dx)) is that layout started
// (130 (r + dy) + dx) pixels in; the weights are stored
// [tap][K half][n][8 channels].  Two stages filled with cp.async: the
// threads fill one while the tensor cores read the other, and a
// tcgen05.commit on the stage's mbarrier frees it.  The epilogue reads the
// accumulators with tcgen05.ld (warp w owns tensor-memory lanes
// 32w..32w+31, i.e. pixels 32w..32w+31 of each segment).  Used when W is a
// multiple of 128 and H is even.
constexpr int kTcPix = 128, kTcHaloW = kTcPix + 2, kTcRows = 2, kTcHaloRows = kTcRows + 2;
constexpr int kTcHaloBytes = 2 * kTcHaloRows * kTcHaloW * 16;
constexpr int kTcMaxN = 256;
constexpr unsigned long long kTcWaitNs = 4000000000ull;   // bound of every wait (4 s of %globaltimer)

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    // start, leading and stride byte offsets in 16-byte units; version 1; no swizzle
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ uint32_t umma_idesc_bf16_f32(int M, int N)
{
    // D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both K-major,
    // N >> 3 at bit 17, M >> 4 at bit 24
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// bounded wait for the completion of phase `parity`: false when limit_ns of
// %globaltimer time passed first, or when *abort (may be null) became nonzero
__device__ __forceinline__ bool tc_mbar_wait(unsigned long long *b, uint32_t parity, unsigned long long limit_ns,
                                             const volatile int *abort)
{
    const uint32_t addr = smem_u32(b);
    unsigned long long t0 = 0;
    for (unsigned it = 0;; it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
        if ((it & 63u) == 0u) {
            if (abort && *abort) return false;
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (it == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
}

// Test hook (no counterpart in the reference): when nonzero, CTA 0 of the
// next tcgen05 convolutions first waits on an mbarrier that nothing
// completes, bounded by this many nanoseconds, before it issues any copy; the
// wait runs out, the CTA sets ERR_SPIN_TIMEOUT and stops, and the host reads
// M2D_ERR_TIMEOUT from m2d_unet_status.  Set by m2d_test_wait_hook.
unsigned long long g_conv_hook_ns = 0;

// ---- persistent, warp-specialised tcgen05 convolution fed by TMA
// Each CTA loops over tiles (two 128-pixel row segments, as above).  One
// lane of warp 8 stages (tile, chunk) items into a ring of S shared-memory
// stages: two 4-D tensor-map loads (cp.async.bulk.tensor) bring the halo's two
// 8-channel halves, each box [4 rows][130 pixels][8 channels] landing exactly
// in the K-major operand layout (out-of-image pixels zero-filled), and one
// bulk copy brings the chunk's weights from their staging-order copy; all
// complete on the stage's `full` mbarrier.  One lane of warp 9 issues the
// tile's MMAs into one of NB tensor-memory accumulator buffers and commits
// each stage to its `empty` barrier and each finished tile to `tfull`.
// Warps 0-7 run the epilogue: warp w reads tensor-memory lanes 32(w%4) ..
// +31 of row w/4 and releases the buffer on `tempty`.  So the loads of the
// next items, the MMAs of the current tile and the epilogue of the previous
// one overlap.  Every wait is bounded; when one runs out the CTA sets the
// error word and all roles stop.
constexpr int kTcpThreads = 320;
constexpr int kTcpSmemBudget = 200 * 1024;                   // staging ring
constexpr int kTcpSmemMax = kTcpSmemBudget;    // two stages of the widest N fit: 2 x (kTcHaloBytes + 288 kTcMaxN)
static_assert(2 * (kTcHaloBytes + 9 * 2 * kTcMaxN * 16) <= kTcpSmemBudget, "two stages must fit");
constexpr int kTcHalfBytes = kTcHaloRows * kTcHaloW * 16;   // one 8-channel half of a halo chunk

__device__ __forceinline__ void tc_mbar_init_n(unsigned long long *b, unsigned n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void tc_mbar_arrive(unsigned long long *b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void tc_mbar_expect(unsigned long long *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            unsigned long long *bar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                 ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
                 "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

struct TcpShape {
    int nstage, nbuf;      // staging ring depth, accumulator buffers
    int tiles;             // tiles over all images
};

__global__ void __launch_bounds__(kTcpThreads, 1) k_conv3x3_tcp(ConvArgs a, TcpShape sh,
                                                               const __grid_constant__ CUtensorMap xmap)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long full[4], empty[4], tfull[2], tempty[2], mdone, idle;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int s_abort;
    const int N = a.cout, S = sh.nstage, NB = sh.nbuf;
    const int stage_bytes = kTcHaloBytes + 9 * 2 * N * 16;
    const int segs = a.W / kTcPix, rows2 = a.H / kTcRows;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nchunks = a.cin / 16;
    const int cols = NB * kTcRows * N;
    const uint32_t ncols = cols <= 32 ? 32u : (cols <= 64 ? 64u : (cols <= 128 ? 128u : (cols <= 256 ? 256u : 512u)));
    if (warp == 9) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_slot)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int q = 0; q < S; q++) { tc_mbar_init_n(&full[q], 1); tc_mbar_init_n(&empty[q], 1); }
        for (int q = 0; q < NB; q++) { tc_mbar_init_n(&tfull[q], 1); tc_mbar_init_n(&tempty[q], 8); }
        tc_mbar_init_n(&mdone, 1);
        tc_mbar_init_n(&idle, 1);   // nothing ever arrives on it (test hook)
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t base = smem_u32(tc_smem);
    auto wait = [&](unsigned long long *b, uint32_t parity) {
        if (s_abort) return false;
        if (tc_mbar_wait(b, parity, kTcWaitNs, &s_abort)) return true;
        if (!s_abort) {
            s_abort = 1;
            if (a.err) atomicOr(a.err, m2d::ERR_SPIN_TIMEOUT);
        }
        return false;
    };
    auto tile_origin = [&](int t, int &img, int &gy0, int &gx0) {
        img = t / (rows2 * segs);
        const int r = t - img * rows2 * segs;
        gy0 = (r / segs) * kTcRows;
        gx0 = (r % segs) * kTcPix;
    };

    if (warp == 8) {
        // ---- staging (one lane): items (tile, chunk) in order, S in flight
        if (lane == 0 && a.hook_ns && blockIdx.x == 0) {
            // test hook: a wait that runs out before any copy is issued, so
            // no copy is in flight when the CTA stops
            if (!tc_mbar_wait(&idle, 0u, a.hook_ns, nullptr)) {
                s_abort = 1;
                if (a.err) atomicOr(a.err, m2d::ERR_SPIN_TIMEOUT);
            }
        }
        if (lane == 0) {
            const uint32_t item_bytes = (uint32_t)(2 * kTcHalfBytes + 9 * 2 * N * 16);
            long long it = 0;
            for (int t = blockIdx.x; t < sh.tiles && !s_abort; t += gridDim.x) {
                int img, gy0, gx0;
                tile_origin(t, img, gy0, gx0);
                for (int c = 0; c < nchunks; c++, it++) {
                    const int stg = (int)(it % S);
                    const long long use = it / S;
                    if (use >= 1 && !wait(&empty[stg], (uint32_t)((use - 1) & 1))) break;
                    const uint32_t sb = base + (uint32_t)(stg * stage_bytes);
                    tc_mbar_expect(&full[stg], item_bytes);
                    tma_load_4d(sb, &xmap, c * 16, gx0 - 1, gy0 - 1, img, &full[stg]);
                    tma_load_4d(sb + kTcHalfBytes, &xmap, c * 16 + 8, gx0 - 1, gy0 - 1, img, &full[stg]);
                    bulk_load(sb + kTcHaloBytes, a.wtc + (long long)c * 9 * 2 * N * 8, (uint32_t)(9 * 2 * N * 16),
                              &full[stg]);
                }
            }
        }
        __syncwarp();
    } else if (warp == 9) {
        // ---- MMA issue (one lane)
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_bf16_f32(kTcPix, N);
            long long it = 0, tl = 0;
            for (int t = blockIdx.x; t < sh.tiles && !s_abort; t += gridDim.x, tl++) {
                const int bsel = (int)(tl % NB);
                const long long v = tl / NB;
                if (v >= 1 && !wait(&tempty[bsel], (uint32_t)((v - 1) & 1))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_base = tmem + (uint32_t)(bsel * kTcRows * N);
                bool ok = true;
                for (int c = 0; c < nchunks; c++, it++) {
                    const int stg = (int)(it % S);
                    if (!wait(&full[stg], (uint32_t)((it / S) & 1))) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = base + (uint32_t)(stg * stage_bytes), sw = sa + kTcHaloBytes;
#pragma unroll 1
                    for (int tap = 0; tap < 9; tap++) {
                        const int dy = tap / 3, dx = tap - dy * 3;
                        const uint64_t bd = umma_desc(sw + (uint32_t)tap * 2u * (uint32_t)N * 16u, (uint32_t)N * 16u, 128u);
                        const uint32_t acc = (c > 0 || tap > 0) ? 1u : 0u;
#pragma unroll
                        for (int r = 0; r < kTcRows; r++) {
                            const uint64_t ad = umma_desc(sa + (uint32_t)((r + dy) * kTcHaloW + dx) * 16u,
                                                          (uint32_t)kTcHalfBytes, 128u);
                            asm volatile("{\n\t.reg .pred p;\n\t"
                                         "setp.ne.b32 p, %4, 0;\n\t"
                                         "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                         ::"r"(acc_base + (uint32_t)(r * N)), "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                                         : "memory");
                        }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                 ::"r"(smem_u32(&empty[stg])) : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(smem_u32(&tfull[bsel])) : "memory");
            }
            // every MMA this thread issued has completed before tensor memory is released
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&mdone)) : "memory");
            if (!tc_mbar_wait(&mdone, 0u, kTcWaitNs, nullptr) && a.err) atomicOr(a.err, m2d::ERR_SPIN_TIMEOUT);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 of row w / 4
        long long tl = 0;
        const int q = warp & 3, r = warp >> 2;
        const int pl = q * 32 + lane;
        for (int t = blockIdx.x; t < sh.tiles; t += gridDim.x, tl++) {
            const int bsel = (int)(tl % NB);
            // warp-uniform: the tensor-memory loads below are warp-collective
            if (!__all_sync(0xffffffffu, wait(&tfull[bsel], (uint32_t)((tl / NB) & 1)))) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int img, gy0, gx0;
            tile_origin(t, img, gy0, gx0);
            const uint32_t tlane = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(bsel * kTcRows * N + r * N);
            const long long p = (long long)(img * a.H + gy0 + r) * a.W + gx0 + pl;
            for (int cc = 0; cc < N; cc += 16) {
                uint32_t v[16];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                             "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                               "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                               "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                             : "r"(tlane + (uint32_t)cc));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                // the pixel's 16 channels with 16-byte stores (all offsets are
                // multiples of 8 elements)
                float f[16];
#pragma unroll
                for (int k = 0; k < 16; k++) f[k] = __uint_as_float(v[k]) + (a.bias ? a.bias[cc + k] : 0.f);
                if (a.z) {
                    float4 *d = reinterpret_cast<float4 *>(a.z + p * a.cout + cc);
#pragma unroll
                    for (int k = 0; k < 4; k++) d[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
                }
                if (a.yf) {
                    float4 *d = reinterpret_cast<float4 *>(a.yf + p * a.ldyf + cc);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (a.accumulate) o = d[k];
                        d[k] = make_float4(f[4 * k] + o.x, f[4 * k + 1] + o.y, f[4 * k + 2] + o.z, f[4 * k + 3] + o.w);
                    }
                }
                if (a.y) {
                    uint32_t h[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        float v0 = f[2 * k], v1 = f[2 * k + 1];
                        if (a.act) { v0 = gelu(v0); v1 = gelu(v1); }
                        const __nv_bfloat162 hb = __floats2bfloat162_rn(v0, v1);
                        h[k] = *reinterpret_cast<const uint32_t *>(&hb);
                    }
                    uint4 *d = reinterpret_cast<uint4 *>(a.y + p * a.ldy + cc);
                    d[0] = make_uint4(h[0], h[1], h[2], h[3]);
                    d[1] = make_uint4(h[4], h[5], h[6], h[7]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) tc_mbar_arrive(&tempty[bsel]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 9)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// dW[co][tap][ci] += sum over pixels of dZ[p][co] X[p + tap offset][ci]:
// a GEMM with M = output channels (64 per CTA, 16 per warp), N = 9 taps x 16
// input channels, K = pixels (16 per step, one tile row).  Both operands come
// from pixel-major tiles through ldmatrix.trans.
struct WgradArgs {
    const bf16 *x; int ldx;        // layer input view
    const bf16 *dz;                // [pixel][cout]
    float *dw;                     // [cout][9][cin], accumulated with atomics
    int nimg, H, W, cin, cout;
};

__global__ void __launch_bounds__(128) k_conv3x3_wgrad(WgradArgs a)
{
    __shared__ __align__(128) unsigned char s_dz[kTileH * kTileW * 128];   // 128 pixels x 64 channels
    __shared__ __align__(128) unsigned char s_halo[kHaloPix * 32];
    const int c0 = blockIdx.x * 16, co0 = blockIdx.y * 64;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // warps along the output channels of the tile (1, 2 or 4); the rest of
    // the warps split the tile's pixel rows (each adds its own partial sums)
    const int rem = a.cout - co0;
    const int nco = rem > 32 ? 4 : (rem > 16 ? 2 : 1);
    const int wco = (warp % nco) * 16, row0 = warp / nco, rstep = 4 / nco;
    const bool active = co0 + wco < a.cout;
    float acc[18][4];
#pragma unroll
    for (int n = 0; n < 18; n++) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
    const int tilesx = (a.W + kTileW - 1) / kTileW, tilesy = (a.H + kTileH - 1) / kTileH;
    const int ntiles = a.nimg * tilesx * tilesy;
    const uint32_t sd = smem_u32(s_dz), sh = smem_u32(s_halo);
    for (int t = blockIdx.z; t < ntiles; t += gridDim.z) {
        const int img = t / (tilesx * tilesy), tt = t - img * tilesx * tilesy;
        const int ty0 = (tt / tilesx) * kTileH, tx0 = (tt % tilesx) * kTileW;
        for (int q = threadIdx.x; q < kTileH * kTileW * 8; q += 128) {
            const int pl = q >> 3, s = q & 7;
            const int gy = ty0 + (pl >> 4), gx = tx0 + (pl & 15);
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy < a.H && gx < a.W && co0 + s * 8 < a.cout)
                v = *reinterpret_cast<const uint4 *>(a.dz + ((long long)(img * a.H + gy) * a.W + gx) * a.cout + co0 + s * 8);
            *reinterpret_cast<uint4 *>(s_dz + pl * 128 + ((s ^ (pl & 7)) << 4)) = v;
        }
        for (int q = threadIdx.x; q < kHaloPix * 2; q += 128) {
            const int hp = q >> 1, h = q & 1;
            const int hy = hp / kHaloW, hx = hp - hy * kHaloW;
            const int gy = ty0 + hy - 1, gx = tx0 + hx - 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < a.H && gx >= 0 && gx < a.W)
                v = *reinterpret_cast<const uint4 *>(a.x + ((long long)(img * a.H + gy) * a.W + gx) * a.ldx + c0 + h * 8);
            *reinterpret_cast<uint4 *>(s_halo + halo_off(hp, h)) = v;
        }
        __syncthreads();
        if (active) {
#pragma unroll 1
            for (int yy = row0; yy < kTileH; yy += rstep) {
                uint32_t af[4];
                {
                    const int mi = lane >> 3, r = lane & 7;
                    const int pl = yy * 16 + r + 8 * (mi >> 1);
                    const int seg = (wco + (mi & 1) * 8) >> 3;
                    ldsm_x4_t(sd + pl * 128 + ((seg ^ (pl & 7)) << 4), af);
                }
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    const int dy = tap / 3, dx = tap - dy * 3;
                    const int mi = lane >> 3, r = lane & 7;
                    const int hp = (yy + dy) * kHaloW + r + 8 * (mi & 1) + dx;
                    uint32_t bfr[4];
                    ldsm_x4_t(sh + halo_off(hp, mi >> 1), bfr);
                    mma_bf16(acc[tap * 2], af, bfr[0], bfr[1]);
                    mma_bf16(acc[tap * 2 + 1], af, bfr[2], bfr[3]);
                }
            }
        }
        __syncthreads();
    }
    if (!active) return;
#pragma unroll
    for (int n = 0; n < 18; n++) {
        const int tap = n >> 1, ci = c0 + (n & 1) * 8 + (lane & 3) * 2;
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            const int co = co0 + wco + (lane >> 2) + hh * 8;
            if (co >= a.cout) continue;
            float *d = a.dw + ((long long)co * 9 + tap) * a.cin + ci;
            atomicAdd(d, acc[n][hh * 2]);
            atomicAdd(d + 1, acc[n][hh * 2 + 1]);
        }
    }
}

// dZ = bf16(dA * gelu'(Z)); db[c] += sum of dZ over pixels (before rounding).
// 256 threads, cout divides 256: every element a thread visits has channel
// threadIdx.x % cout, so the bias sums stay in registers until one block
// reduction per channel
constexpr int kEltBlock = 256;
__global__ void __launch_bounds__(kEltBlock) k_gelu_bwd(long long npix, int cout, const float *dA, int lda,
                                                        const float *z, bf16 *dz, float *db)
{
    __shared__ float s_part[kEltBlock];
    const long long n = npix * cout;
    const int c = threadIdx.x % cout;
    float acc = 0.f;
    for (long long e = (long long)blockIdx.x * kEltBlock + threadIdx.x; e < n; e += (long long)gridDim.x * kEltBlock) {
        const long long p = e / cout;
        const float g = dA[p * lda + c] * gelu_grad(z[e]);
        dz[e] = __float2bfloat16_rn(g);
        acc += g;
    }
    s_part[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < cout) {
        float t = 0.f;
        for (int k = threadIdx.x; k < kEltBlock; k += cout) t += s_part[k];
        atomicAdd(&db[threadIdx.x], t);
    }
}

// 2x2 mean (outputs rounded to bf16) and its adjoint (added into dX)
__global__ void k_pool(int nimg, int H, int W, int C, const bf16 *x, int ldx, bf16 *y)
{
    const int Ho = H / 2, Wo = W / 2;
    const long long n = (long long)nimg * Ho * Wo * C;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long p = e / C;
        const int c = (int)(e - p * C);
        const int img = (int)(p / ((long long)Ho * Wo));
        const int r = (int)(p - (long long)img * Ho * Wo), yo = r / Wo, xo = r - yo * Wo;
        const long long q = ((long long)img * H + 2 * yo) * W + 2 * xo;
        const float s = __bfloat162float(x[q * ldx + c]) + __bfloat162float(x[(q + 1) * ldx + c]) +
                        __bfloat162float(x[(q + W) * ldx + c]) + __bfloat162float(x[(q + W + 1) * ldx + c]);
        y[e] = __float2bfloat16_rn(0.25f * s);
    }
}
__global__ void k_pool_bwd(int nimg, int H, int W, int C, const float *dy, float *dx, int lddx)
{
    const long long n = (long long)nimg * H * W * C;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long p = e / C;
        const int c = (int)(e - p * C);
        const int img = (int)(p / ((long long)H * W));
        const int r = (int)(p - (long long)img * H * W), yy = r / W, xx = r - yy * W;
        const long long q = ((long long)img * (H / 2) + yy / 2) * (W / 2) + xx / 2;
        dx[p * lddx + c] += 0.25f * dy[q * C + c];
    }
}
// nearest 2x upsampling into a channel slice, and its adjoint
__global__ void k_up(int nimg, int Ho, int Wo, int C, const bf16 *x, bf16 *y, int ldy)
{
    const int C8 = C / 8;      // 16-byte groups of channels
    const long long n = (long long)nimg * Ho * Wo * C8;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long p = e / C8;
        const int c = (int)(e - p * C8) * 8;
        const int img = (int)(p / ((long long)Ho * Wo));
        const int r = (int)(p - (long long)img * Ho * Wo), yy = r / Wo, xx = r - yy * Wo;
        const long long q = ((long long)img * (Ho / 2) + yy / 2) * (Wo / 2) + xx / 2;
        *reinterpret_cast<uint4 *>(y + p * ldy + c) = *reinterpret_cast<const uint4 *>(x + q * C + c);
    }
}
__global__ void k_up_bwd(int nimg, int Hi, int Wi, int C, const float *dy, int lddy, float *dx)
{
    const int Ho = Hi * 2, Wo = Wi * 2;
    const long long n = (long long)nimg * Hi * Wi * C;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long p = e / C;
        const int c = (int)(e - p * C);
        const int img = (int)(p / ((long long)Hi * Wi));
        const int r = (int)(p - (long long)img * Hi * Wi), yy = r / Wi, xx = r - yy * Wi;
        const long long q = ((long long)img * Ho + 2 * yy) * Wo + 2 * xx;
        dx[e] = dy[q * lddy + c] + dy[(q + 1) * lddy + c] + dy[(q + Wo) * lddy + c] + dy[(q + Wo + 1) * lddy + c];
    }
}

// planar FP32 input [img][11][H][W] -> pixel-major bf16 with 16 channels
__global__ void k_pack_input(int nimg, int H, int W, const float *in, bf16 *x)
{
    const long long n = (long long)nimg * H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int img = (int)(p / ((long long)H * W));
        const long long r = p - (long long)img * H * W;
        __align__(16) bf16 v[kInChan];
#pragma unroll
        for (int c = 0; c < kInChan; c++)
            v[c] = __float2bfloat16_rn(c < kInPlanes ? in[((long long)img * kInPlanes + c) * H * W + r] : 0.f);
        uint4 *d = reinterpret_cast<uint4 *>(x + p * kInChan);
        d[0] = reinterpret_cast<const uint4 *>(v)[0];
        d[1] = reinterpret_cast<const uint4 *>(v)[1];
    }
}

// 1x1 head: out = sum_c U[p][c] wh[c] + bh
__global__ void k_head(long long npix, const bf16 *u, const float *wh, float *out)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
#pragma unroll
        for (int c = 0; c < 16; c++) s += __bfloat162float(u[p * 16 + c]) * wh[c];
        out[p] = s + wh[16];
    }
}
// loss = scale * sum mask (out - t)^2, dout = 2 scale mask (out - t)
__global__ void k_loss(long long npix, const float *out, const float *t, const float *mask, float scale, float *dout,
                       float *loss)
{
    float s = 0.f;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        const float m = mask ? mask[p] : 1.f;
        const float d = (out[p] - t[p]) * m;
        s += d * d;
        dout[p] = 2.f * scale * d;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * scale);
}
// head adjoint: dU[p][c] = dout[p] wh[c]; dwh[c] += sum dout U; dbh += sum dout
__global__ void __launch_bounds__(kEltBlock) k_head_bwd(long long npix, const bf16 *u, const float *wh,
                                                        const float *dout, float *du, float *dwh)
{
    __shared__ float s_g[kEltBlock / 32][17];
    float g[17];
#pragma unroll
    for (int c = 0; c < 17; c++) g[c] = 0.f;
    for (long long p = (long long)blockIdx.x * kEltBlock + threadIdx.x; p < npix; p += (long long)gridDim.x * kEltBlock) {
        const float d = dout[p];
#pragma unroll
        for (int c = 0; c < 16; c++) {
            du[p * 16 + c] = d * wh[c];
            g[c] += d * __bfloat162float(u[p * 16 + c]);
        }
        g[16] += d;
    }
    const int w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 17; c++) {
        float v = g[c];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) s_g[w][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < 17) {
        float t = 0.f;
        for (int k = 0; k < kEltBlock / 32; k++) t += s_g[k][threadIdx.x];
        atomicAdd(&dwh[threadIdx.x], t);
    }
}

__global__ void k_adam(long long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi; v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}
// bf16 copies of one layer's weights: W [cout][9][cin], the adjoint kernel
// WT [cin][9][cout] with the taps reversed, and both in the tcgen05 kernel's
// staging order: per 16-channel chunk of the K dimension, [tap][K half][n][8]
// (one contiguous block of 288 n bytes per chunk, copied with one bulk copy)
__global__ void k_sync_weights(int cin, int cout, const float *w, bf16 *wb, bf16 *wt, bf16 *wbtc, bf16 *wttc)
{
    const int n = cout * 9 * cin;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int co = e / (9 * cin), r = e - co * 9 * cin, tap = r / cin, ci = r - tap * cin;
        const bf16 v = __float2bfloat16_rn(w[e]);
        wb[e] = v;
        wt[((long long)ci * 9 + (8 - tap)) * cout + co] = v;
        // forward: K = ci, N = co
        wbtc[(((long long)(ci >> 4) * 9 + tap) * 2 + ((ci >> 3) & 1)) * cout * 8 + co * 8 + (ci & 7)] = v;
        // adjoint: K = co, N = ci, tap reversed
        wttc[(((long long)(co >> 4) * 9 + (8 - tap)) * 2 + ((co >> 3) & 1)) * cin * 8 + ci * 8 + (co & 7)] = v;
    }
}

inline unsigned grid_for(long long n, int block = 256)
{
    long long g = (n + block - 1) / block;
    if (g > 148LL * 16) g = 148LL * 16;
    return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

namespace m2d {
void set_conv_wait_hook(unsigned long long ns) { g_conv_hook_ns = ns; }
}  // namespace m2d

// ------------------------------------------------------------------ network
struct ConvLayer {
    int cin, cout, level;
    long long woff, boff;      // offsets into the FP32 parameter array
    bf16 *wb = nullptr, *wt = nullptr, *wbtc = nullptr, *wttc = nullptr;
    // forward views
    const bf16 *x = nullptr; int ldx = 0;
    bf16 *y = nullptr; int ldy = 0;
    float *z = nullptr;
    // backward views: gradient of the output (FP32, same layout as y) and of the input
    float *dy = nullptr; int lddy = 0;
    float *dx = nullptr; int lddx = 0;   // null: input gradient not needed
};

struct m2d_unet {
    int device = 0, bmax = 0, H = 0, W = 0;
    long long P[kLevels];
    long long nparam = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    std::vector<void *> allocs;
    ConvLayer L[kConvs];
    bf16 *in0 = nullptr, *D[3] = {}, *pooled[3] = {}, *U[3] = {}, *e3b = nullptr;
    float *out = nullptr, *dout = nullptr, *dU0 = nullptr, *loss = nullptr;
    float *dD[3] = {}, *dpool[3] = {};
    bf16 *dz = nullptr;
    int adam_step = 0;
    // scratch of the flexible p' solve (one image)
    float *feat = nullptr, *yout = nullptr;
    double *r = nullptr, *x1 = nullptr, *stats = nullptr;
    int *nit = nullptr;
    int *err = nullptr;        // device error word of the tensor-core kernels
};

namespace {

int unet_fail(int code, const char *msg)
{
    m2d_set_last_error_msg(msg);
    return code;
}

template <typename T>
T *dalloc(m2d_unet *n, long long count, cudaError_t &e)
{
    void *p = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&p, (size_t)count * sizeof(T));
    if (e == cudaSuccess) { n->allocs.push_back(p); e = cudaMemset(p, 0, (size_t)count * sizeof(T)); }
    return (T *)p;
}

// tcgen05 kernel policy (m2d_unet_set_tensor_path): 0 never (mma.sync for
// every convolution); 1 (default) and 2: wherever the image shape fits (even
// height, width a multiple of 128), where it measured faster on every layer
int g_tensor_tc = 1;

// the 4-D tensor map of an activation view [img][H][W][channels 0..cin) with
// `ldx` channels per pixel, box [1][4][130][8] (one K half of a halo chunk)
bool encode_halo_map(CUtensorMap *map, const bf16 *x, int ldx, int cin, int nimg, int H, int W)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        (void)cudaGetLastError();
    }
    if (!encode || ((uintptr_t)x % 16) != 0 || (ldx * 2) % 16 != 0 || cin % 16 != 0) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)ldx * 2, (cuuint64_t)W * ldx * 2, (cuuint64_t)H * W * ldx * 2};
    const cuuint32_t box[4] = {8, (cuuint32_t)kTcHaloW, (cuuint32_t)kTcHaloRows, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(x), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_conv(int nimg, int H, int W, const bf16 *x, int ldx, const bf16 *w, const bf16 *wtc, int cin,
                        int cout, const float *bias, float *z, bf16 *y, int ldy, float *yf, int ldyf, int accumulate,
                        int act, int *err, cudaStream_t st)
{
    ConvArgs a;
    a.x = x; a.ldx = ldx; a.w = w; a.bias = bias; a.z = z; a.y = y; a.ldy = ldy; a.yf = yf; a.ldyf = ldyf;
    a.accumulate = accumulate; a.act = act; a.nimg = nimg; a.H = H; a.W = W; a.cin = cin; a.cout = cout;
    a.err = err;
    a.wtc = wtc;
    a.hook_ns = g_conv_hook_ns;
    const bool tc_shape = W % kTcPix == 0 && H % kTcRows == 0 && cout % 16 == 0 && cout <= kTcMaxN && cin % 16 == 0;
    CUtensorMap xmap;
    if (tc_shape && wtc && g_tensor_tc != 0 &&
        encode_halo_map(&xmap, x, ldx, cin, nimg, H, W)) {
        static int attr_device = -1;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (attr_device != dev) {
            e = cudaFuncSetAttribute(k_conv3x3_tcp, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcpSmemMax);
            if (e != cudaSuccess) return e;
            attr_device = dev;
        }
        const int stage = kTcHaloBytes + 9 * 2 * cout * 16;
        TcpShape sh;
        sh.nstage = kTcpSmemBudget / stage;
        if (sh.nstage > 4) sh.nstage = 4;
        if (sh.nstage < 2) sh.nstage = 2;
        sh.nbuf = (4 * cout <= 512) ? 2 : 1;
        sh.tiles = nimg * (H / kTcRows) * (W / kTcPix);
        const int smem = sh.nstage * stage;
        const int cols = sh.nbuf * kTcRows * cout;
        const int ncols = cols <= 32 ? 32 : (cols <= 64 ? 64 : (cols <= 128 ? 128 : (cols <= 256 ? 256 : 512)));
        // CTAs per SM: shared memory (227 KB per SM, 1 KB reserved per CTA),
        // tensor-memory columns (512 per SM), at most 2
        int per_sm = (227 * 1024) / (smem + 2048);
        if (per_sm > 512 / ncols) per_sm = 512 / ncols;
        if (per_sm > 2) per_sm = 2;
        if (per_sm < 1) per_sm = 1;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int grid = sms * per_sm;
        if (grid > sh.tiles) grid = sh.tiles;
        k_conv3x3_tcp<<<grid, kTcpThreads, smem, st>>>(a, sh, xmap);
        return cudaGetLastError();
    }
    const unsigned tiles = (unsigned)(((H + kTileH - 1) / kTileH) * ((W + kTileW - 1) / kTileW));
    if (cout % 64 == 0) k_conv3x3<64><<<dim3(tiles, cout / 64, nimg), 128, 0, st>>>(a);
    else if (cout % 32 == 0) k_conv3x3<32><<<dim3(tiles, cout / 32, nimg), 128, 0, st>>>(a);
    else k_conv3x3<16><<<dim3(tiles, cout / 16, nimg), 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_wgrad(int nimg, int H, int W, const bf16 *x, int ldx, const bf16 *dz, float *dw, int cin, int cout,
                         cudaStream_t st)
{
    WgradArgs a;
    a.x = x; a.ldx = ldx; a.dz = dz; a.dw = dw; a.nimg = nimg; a.H = H; a.W = W; a.cin = cin; a.cout = cout;
    const int ntiles = nimg * ((H + kTileH - 1) / kTileH) * ((W + kTileW - 1) / kTileW);
    const int cx = cin / 16, cy = (cout + 63) / 64;
    int z = (148 * 4 + cx * cy - 1) / (cx * cy);
    if (z > ntiles) z = ntiles;
    if (z < 1) z = 1;
    k_conv3x3_wgrad<<<dim3(cx, cy, z), 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

extern "C" long m2d_unet_param_count(void)
{
    // conv layers in network order (input channels, output channels)
    static const int io[kConvs][2] = {{16, 16}, {16, 16}, {16, 32}, {32, 32}, {32, 64}, {64, 64}, {64, 128},
                                      {128, 128}, {192, 64}, {64, 64}, {96, 32}, {32, 32}, {48, 16}, {16, 16}};
    long n = 0;
    for (auto &l : io) n += (long)l[1] * 9 * l[0] + l[1];
    return n + 17;
}

extern "C" int m2d_unet_create(int bmax, int H, int W, int device, m2d_unet **out)
{
    if (!out || bmax < 1 || H < 8 || W < 8 || H % 8 || W % 8)
        return unet_fail(M2D_ERR_ARG, "m2d_unet_create: need batch >= 1 and H, W multiples of 8");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { m2d_set_last_error(e, "cudaSetDevice", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    m2d_unet *n = new m2d_unet();
    n->device = device; n->bmax = bmax; n->H = H; n->W = W;
    for (int l = 0; l < kLevels; l++) n->P[l] = (long long)bmax * (H >> l) * (W >> l);
    static const int io[kConvs][3] = {{16, 16, 0}, {16, 16, 0}, {16, 32, 1}, {32, 32, 1}, {32, 64, 2}, {64, 64, 2},
                                      {64, 128, 3}, {128, 128, 3}, {192, 64, 2}, {64, 64, 2}, {96, 32, 1}, {32, 32, 1},
                                      {48, 16, 0}, {16, 16, 0}};
    long long off = 0;
    for (int k = 0; k < kConvs; k++) {
        ConvLayer &c = n->L[k];
        c.cin = io[k][0]; c.cout = io[k][1]; c.level = io[k][2];
        c.woff = off; off += (long long)c.cout * 9 * c.cin;
        c.boff = off; off += c.cout;
    }
    n->nparam = off + 17;     // head: 16 weights + bias
    const long long *P = n->P;
    n->params = dalloc<float>(n, n->nparam, e);
    n->grads = dalloc<float>(n, n->nparam, e);
    n->adam_m = dalloc<float>(n, n->nparam, e);
    n->adam_v = dalloc<float>(n, n->nparam, e);
    for (int k = 0; k < kConvs; k++) {
        ConvLayer &c = n->L[k];
        c.wb = dalloc<bf16>(n, (long long)c.cout * 9 * c.cin, e);
        c.wt = dalloc<bf16>(n, (long long)c.cout * 9 * c.cin, e);
        c.wbtc = dalloc<bf16>(n, (long long)c.cout * 9 * c.cin, e);
        c.wttc = dalloc<bf16>(n, (long long)c.cout * 9 * c.cin, e);
        c.z = dalloc<float>(n, P[c.level] * c.cout, e);
    }
    // activations: D[l] = [up from level l+1 | skip of level l]
    const int dch[3] = {48, 96, 192}, upch[3] = {32, 64, 128};
    n->in0 = dalloc<bf16>(n, P[0] * 16, e);
    for (int l = 0; l < 3; l++) {
        n->D[l] = dalloc<bf16>(n, P[l] * dch[l], e);
        n->pooled[l] = dalloc<bf16>(n, P[l + 1] * kChan[l], e);
        n->U[l] = dalloc<bf16>(n, P[l] * kChan[l], e);
        n->dD[l] = dalloc<float>(n, P[l] * dch[l], e);
        n->dpool[l] = dalloc<float>(n, P[l + 1] * kChan[l], e);
    }
    n->e3b = dalloc<bf16>(n, P[3] * 128, e);
    bf16 *ea[4], *da[3];
    float *dea[4], *dda[3], *dU[3], *de3b;
    for (int l = 0; l < 4; l++) { ea[l] = dalloc<bf16>(n, P[l] * kChan[l], e); dea[l] = dalloc<float>(n, P[l] * kChan[l], e); }
    for (int l = 0; l < 3; l++) {
        da[l] = dalloc<bf16>(n, P[l] * kChan[l], e); dda[l] = dalloc<float>(n, P[l] * kChan[l], e);
        dU[l] = dalloc<float>(n, P[l] * kChan[l], e);
    }
    de3b = dalloc<float>(n, P[3] * 128, e);
    n->out = dalloc<float>(n, P[0], e);
    n->dout = dalloc<float>(n, P[0], e);
    n->loss = dalloc<float>(n, 1, e);
    n->dz = dalloc<bf16>(n, P[0] * 16 > P[3] * 128 ? P[0] * 16 : P[3] * 128, e);
    n->dU0 = dU[0];
    const long long cells = (long long)(H + 2) * (W + 2);
    n->feat = dalloc<float>(n, (long long)kInPlanes * H * W, e);
    n->yout = dalloc<float>(n, (long long)H * W, e);
    n->r = dalloc<double>(n, cells, e);
    n->x1 = dalloc<double>(n, cells, e);
    n->stats = dalloc<double>(n, 16, e);
    n->nit = dalloc<int>(n, 4, e);
    n->err = dalloc<int>(n, 1, e);
    if (e != cudaSuccess) {
        m2d_set_last_error(e, "m2d_unet_create: allocation", __FILE__, __LINE__);
        m2d_unet_destroy(n);
        return M2D_ERR_NOMEM;
    }
    // wiring (see the file comment for the level structure)
    auto enc = [&](int k1, int l, const bf16 *xin, int ldxin, float *dxin) {
        ConvLayer &a = n->L[k1], &b = n->L[k1 + 1];
        a.x = xin; a.ldx = ldxin; a.y = ea[l]; a.ldy = kChan[l]; a.dy = dea[l]; a.lddy = kChan[l];
        a.dx = dxin; a.lddx = a.cin;
        b.x = ea[l]; b.ldx = kChan[l]; b.dx = dea[l]; b.lddx = kChan[l];
        if (l < 3) {
            b.y = n->D[l] + upch[l]; b.ldy = dch[l]; b.dy = n->dD[l] + upch[l]; b.lddy = dch[l];
        } else {
            b.y = n->e3b; b.ldy = 128; b.dy = de3b; b.lddy = 128;
        }
    };
    enc(0, 0, n->in0, 16, nullptr);
    enc(2, 1, n->pooled[0], 16, n->dpool[0]);
    enc(4, 2, n->pooled[1], 32, n->dpool[1]);
    enc(6, 3, n->pooled[2], 64, n->dpool[2]);
    auto dec = [&](int k1, int l) {
        ConvLayer &a = n->L[k1], &b = n->L[k1 + 1];
        a.x = n->D[l]; a.ldx = dch[l]; a.y = da[l]; a.ldy = kChan[l]; a.dy = dda[l]; a.lddy = kChan[l];
        a.dx = n->dD[l]; a.lddx = dch[l];
        b.x = da[l]; b.ldx = kChan[l]; b.y = n->U[l]; b.ldy = kChan[l]; b.dy = dU[l]; b.lddy = kChan[l];
        b.dx = dda[l]; b.lddx = kChan[l];
    };
    dec(8, 2);
    dec(10, 1);
    dec(12, 0);
    *out = n;
    return M2D_OK;
}

extern "C" int m2d_unet_destroy(m2d_unet *n)
{
    if (!n) return M2D_OK;
    cudaSetDevice(n->device);
    cudaDeviceSynchronize();
    for (void *p : n->allocs) cudaFree(p);
    delete n;
    return M2D_OK;
}

static cudaError_t sync_weights(m2d_unet *n, cudaStream_t st)
{
    for (int k = 0; k < kConvs; k++) {
        ConvLayer &c = n->L[k];
        k_sync_weights<<<grid_for((long long)c.cout * 9 * c.cin), 256, 0, st>>>(c.cin, c.cout, n->params + c.woff, c.wb, c.wt,
                                                                             c.wbtc, c.wttc);
    }
    return cudaGetLastError();
}

extern "C" int m2d_unet_set_params(m2d_unet *n, const float *host, long count)
{
    if (!n || !host || count != n->nparam) return unet_fail(M2D_ERR_ARG, "m2d_unet_set_params: size mismatch");
    cudaSetDevice(n->device);
    cudaError_t e = cudaMemcpy(n->params, host, (size_t)count * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(n->adam_m, 0, (size_t)count * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(n->adam_v, 0, (size_t)count * sizeof(float));
    if (e == cudaSuccess) e = sync_weights(n, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    n->adam_step = 0;
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_unet_set_params", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

static int copy_out(m2d_unet *n, const float *src, float *host, long count, const char *what)
{
    if (!n || !host || count != n->nparam) return unet_fail(M2D_ERR_ARG, what);
    cudaSetDevice(n->device);
    cudaError_t e = cudaMemcpy(host, src, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { m2d_set_last_error(e, what, __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}
extern "C" int m2d_unet_get_params(m2d_unet *n, float *host, long count)
{ return copy_out(n, n ? n->params : nullptr, host, count, "m2d_unet_get_params"); }
extern "C" int m2d_unet_get_grads(m2d_unet *n, float *host, long count)
{ return copy_out(n, n ? n->grads : nullptr, host, count, "m2d_unet_get_grads"); }

// forward pass of nimg images; d_in: [img][11][H][W] FP32 planes; d_out: [img][H][W]
static cudaError_t forward(m2d_unet *n, int nimg, const float *d_in, float *d_out, bool train, cudaStream_t st)
{
    const int H = n->H, W = n->W;
    k_pack_input<<<grid_for((long long)nimg * H * W), 256, 0, st>>>(nimg, H, W, d_in, n->in0);
    cudaError_t e = cudaGetLastError();
    auto conv = [&](int k) {
        ConvLayer &c = n->L[k];
        const int lh = H >> c.level, lw = W >> c.level;
        if (e == cudaSuccess)
            e = launch_conv(nimg, lh, lw, c.x, c.ldx, c.wb, c.wbtc, c.cin, c.cout, n->params + c.boff, train ? c.z : nullptr,
                            c.y, c.ldy, nullptr, 0, 0, 1, n->err, st);
    };
    const int upch[3] = {32, 64, 128}, dch[3] = {48, 96, 192};
    for (int l = 0; l < 4; l++) {
        conv(2 * l);
        conv(2 * l + 1);
        if (l < 3 && e == cudaSuccess) {
            const int lh = H >> l, lw = W >> l;
            k_pool<<<grid_for((long long)nimg * (lh / 2) * (lw / 2) * kChan[l]), 256, 0, st>>>(
                nimg, lh, lw, kChan[l], n->D[l] + upch[l], dch[l], n->pooled[l]);
            e = cudaGetLastError();
        }
    }
    for (int l = 2; l >= 0; l--) {
        const bf16 *src = (l == 2) ? n->e3b : n->U[l + 1];
        const int lh = H >> l, lw = W >> l;
        if (e == cudaSuccess) {
            k_up<<<grid_for((long long)nimg * lh * lw * upch[l] / 8), 256, 0, st>>>(nimg, lh, lw, upch[l], src, n->D[l],
                                                                                    dch[l]);
            e = cudaGetLastError();
        }
        conv(8 + 2 * (2 - l));
        conv(9 + 2 * (2 - l));
    }
    if (e == cudaSuccess) {
        k_head<<<grid_for((long long)nimg * H * W), 256, 0, st>>>((long long)nimg * H * W, n->U[0],
                                                                 n->params + (n->nparam - 17), d_out);
        e = cudaGetLastError();
    }
    return e;
}

extern "C" int m2d_unet_forward(m2d_unet *n, int nimg, const float *d_in, float *d_out, void *stream)
{
    if (!n || !d_in || !d_out || nimg < 1 || nimg > n->bmax) return unet_fail(M2D_ERR_ARG, "m2d_unet_forward: bad arguments");
    cudaError_t e = forward(n, nimg, d_in, d_out, false, (cudaStream_t)stream);
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_unet_forward", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

// one training step's gradients: forward, MSE loss against d_target over
// d_mask (may be null), backward into the gradient array (zeroed first)
extern "C" int m2d_unet_loss_grad(m2d_unet *n, int nimg, const float *d_in, const float *d_target, const float *d_mask,
                                  float loss_scale, float *loss_host, void *stream)
{
    if (!n || !d_in || !d_target || nimg < 1 || nimg > n->bmax)
        return unet_fail(M2D_ERR_ARG, "m2d_unet_loss_grad: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const int H = n->H, W = n->W;
    const long long P0 = (long long)nimg * H * W;
    cudaError_t e = forward(n, nimg, d_in, n->out, true, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->grads, 0, (size_t)n->nparam * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->loss, 0, sizeof(float), st);
    if (e == cudaSuccess) {
        k_loss<<<grid_for(P0), 256, 0, st>>>(P0, n->out, d_target, d_mask, loss_scale, n->dout, n->loss);
        k_head_bwd<<<grid_for(P0), kEltBlock, 0, st>>>(P0, n->U[0], n->params + (n->nparam - 17), n->dout, n->dU0,
                                                 n->grads + (n->nparam - 17));
        e = cudaGetLastError();
    }
    const int upch[3] = {32, 64, 128}, dch[3] = {48, 96, 192};
    // one conv layer backwards: dZ, dW, db, and dX when the layer has an input gradient
    auto back = [&](int k) {
        ConvLayer &c = n->L[k];
        const int lh = H >> c.level, lw = W >> c.level;
        const long long np = (long long)nimg * lh * lw;
        if (e != cudaSuccess) return;
        k_gelu_bwd<<<grid_for(np * c.cout), kEltBlock, 0, st>>>(np, c.cout, c.dy, c.lddy, c.z, n->dz, n->grads + c.boff);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = launch_wgrad(nimg, lh, lw, c.x, c.ldx, n->dz, n->grads + c.woff, c.cin, c.cout, st);
        if (e == cudaSuccess && c.dx)
            e = launch_conv(nimg, lh, lw, n->dz, c.cout, c.wt, c.wttc, c.cout, c.cin, nullptr, nullptr, nullptr, 0, c.dx,
                            c.lddx, 0, 0, n->err, st);
    };
    for (int l = 0; l < 3; l++) {          // decoder, finest level first
        back(13 - 2 * l);
        back(12 - 2 * l);
        // dD[l][:, 0:upch] -> gradient of the upsampled tensor
        const int li = l + 1, lh = H >> li, lw = W >> li;
        float *dsrc = (l == 2) ? n->L[7].dy : n->L[11 - 2 * l].dy;
        if (e == cudaSuccess) {
            k_up_bwd<<<grid_for((long long)nimg * lh * lw * upch[l]), 256, 0, st>>>(nimg, lh, lw, upch[l], n->dD[l],
                                                                                    dch[l], dsrc);
            e = cudaGetLastError();
        }
    }
    for (int l = 3; l >= 0; l--) {         // encoder, coarsest level first
        back(2 * l + 1);
        back(2 * l);
        if (l > 0 && e == cudaSuccess) {
            // pooled[l-1] gradient -> skip slice of D[l-1]
            const int lh = H >> (l - 1), lw = W >> (l - 1);
            k_pool_bwd<<<grid_for((long long)nimg * lh * lw * kChan[l - 1]), 256, 0, st>>>(
                nimg, lh, lw, kChan[l - 1], n->dpool[l - 1], n->dD[l - 1] + upch[l - 1], dch[l - 1]);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && loss_host) {
        e = cudaMemcpyAsync(loss_host, n->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_unet_loss_grad", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

extern "C" int m2d_unet_adam(m2d_unet *n, float lr, float beta1, float beta2, float eps, void *stream)
{
    if (!n || !(lr > 0.f)) return unet_fail(M2D_ERR_ARG, "m2d_unet_adam: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    n->adam_step++;
    const float c1 = 1.f - powf(beta1, (float)n->adam_step), c2 = 1.f - powf(beta2, (float)n->adam_step);
    k_adam<<<grid_for(n->nparam), 256, 0, st>>>(n->nparam, n->params, n->grads, n->adam_m, n->adam_v, lr, beta1, beta2,
                                                eps, c1, c2);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = sync_weights(n, st);
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_unet_adam", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

extern "C" int m2d_unet_shape(const m2d_unet *n, int *bmax, int *H, int *W)
{
    if (!n) return unet_fail(M2D_ERR_ARG, "m2d_unet_shape: null network");
    if (bmax) *bmax = n->bmax;
    if (H) *H = n->H;
    if (W) *W = n->W;
    return M2D_OK;
}

// ------------------------------------------------- p' system <-> network images
// Pixel (y, x) of an H x W image is real cell (i, j) = (x + 2, y + 2) of an
// nx x ny system (nx - 2 <= W, ny - 2 <= H); pixels outside are zero.
namespace {

constexpr int kStatThreads = 1024;

// one block: deterministic sums.  s[0] = sum of r^2 over every cell (the
// norm the MSI stopping test uses, msi2d5-v03.f90:68-120); mode 1 also sums
// (r/aP)^2, log Jp, (log Jp)^2 over the real cells into s[1..3] and stores
// sigma, the mean and the standard deviation of log Jp in s[4..6]
__global__ void __launch_bounds__(kStatThreads) k_sys_stats(int nx, int ny, const double *a5, const double *r,
                                                            const double *Jp, double *s, int mode)
{
    __shared__ double red[4][kStatThreads / 32];
    const long long N = (long long)nx * ny;
    const long long nreal = (long long)(nx - 2) * (ny - 2);
    double v[4] = {0, 0, 0, 0};
    for (long long k = threadIdx.x; k < N; k += kStatThreads) v[0] += r[k] * r[k];
    if (mode)
        for (long long k = threadIdx.x; k < nreal; k += kStatThreads) {
            const int j = (int)(k / (nx - 2)) + 2, i = (int)(k % (nx - 2)) + 2;
            const long long np = (long long)(j - 1) * nx + (i - 1);
            const double rh = r[np] / a5[2 * N + np];
            const double lj = log(Jp[np]);
            v[1] += rh * rh; v[2] += lj; v[3] += lj * lj;
        }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int q = 0; q < 4; q++) {
        double t = v[q];
        for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (l == 0) red[q][w] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[4] = {0, 0, 0, 0};
        for (int q = 0; q < 4; q++)
            for (int k = 0; k < kStatThreads / 32; k++) t[q] += red[q][k];
        s[0] = t[0];
        if (mode) {
            s[1] = t[1]; s[2] = t[2]; s[3] = t[3];
            const double sig = sqrt(t[1] / (double)nreal);
            const double mean = t[2] / (double)nreal;
            const double var = t[3] / (double)nreal - mean * mean;
            s[4] = sig > 0.0 ? sig : 1.0;
            s[5] = mean;
            s[6] = var > 1e-24 ? sqrt(var) : 1.0;
        }
    }
}

// r = b - A x on every cell (5 diagonals S, W, P, E, N); a neighbour outside
// the grid contributes nothing, as in the residual of msi2d5-v03.f90:68-120
__global__ void k_residual5(int nx, int ny, const double *a5, const double *b, const double *x, double *r)
{
    const long long N = (long long)nx * ny;
    for (long long np = (long long)blockIdx.x * blockDim.x + threadIdx.x; np < N; np += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(np / nx) + 1, i = (int)(np - (long long)(j - 1) * nx) + 1;
        double ax = a5[2 * N + np] * x[np];
        if (j > 1) ax += a5[np] * x[np - nx];
        if (i > 1) ax += a5[N + np] * x[np - 1];
        if (i < nx) ax += a5[3 * N + np] * x[np + 1];
        if (j < ny) ax += a5[4 * N + np] * x[np + nx];
        r[np] = b[np] - ax;
    }
}

// the 11 input planes: r / (aP sigma), the nine coefficients over aP
// (SW, S, SE, W, P, E, NW, N, NE; corners zero for a 5-diagonal system) and
// the standardised log Jp
__global__ void k_features(int nx, int ny, int H, int W, const double *a5, const double *r, const double *Jp,
                           const double *s, float *feat)
{
    const long long N = (long long)nx * ny, HW = (long long)H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < HW; p += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(p / W), x = (int)(p - (long long)y * W);
        float f[11];
#pragma unroll
        for (int c = 0; c < 11; c++) f[c] = 0.f;
        if (x < nx - 2 && y < ny - 2) {
            const long long np = (long long)(y + 1) * nx + (x + 1);
            const double ap = a5[2 * N + np];
            f[0] = (float)(r[np] / ap / s[4]);
            f[2] = (float)(a5[np] / ap);
            f[4] = (float)(a5[N + np] / ap);
            f[5] = 1.f;
            f[6] = (float)(a5[3 * N + np] / ap);
            f[8] = (float)(a5[4 * N + np] / ap);
            f[10] = (float)((log(Jp[np]) - s[5]) / s[6]);
        }
#pragma unroll
        for (int c = 0; c < 11; c++) feat[c * HW + p] = f[c];
    }
}

// xout = x + sigma y on the real cells; on the ghost ring, the value that
// satisfies the cell's own row of A x = b given its neighbours (the real ones
// already corrected, the ghost ones as they were), so that the boundary rows
// carry no residual after the correction
__global__ void k_apply(int nx, int ny, int H, int W, const double *a5, const double *b, const float *y,
                        const double *s, const double *x, double *xout)
{
    const long long N = (long long)nx * ny;
    const double sg = s[4];
    auto corrected = [&](long long q) {
        const int jq = (int)(q / nx) + 1, iq = (int)(q - (long long)(jq - 1) * nx) + 1;
        double v = x[q];
        if (iq > 1 && iq < nx && jq > 1 && jq < ny) v += sg * (double)y[(long long)(jq - 2) * W + (iq - 2)];
        return v;
    };
    for (long long np = (long long)blockIdx.x * blockDim.x + threadIdx.x; np < N; np += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(np / nx) + 1, i = (int)(np - (long long)(j - 1) * nx) + 1;
        if (i > 1 && i < nx && j > 1 && j < ny) { xout[np] = corrected(np); continue; }
        const double ap = a5[2 * N + np];
        if (ap == 0.0) { xout[np] = x[np]; continue; }
        double v = b[np];
        if (j > 1) v -= a5[np] * corrected(np - nx);
        if (i > 1) v -= a5[N + np] * corrected(np - 1);
        if (i < nx) v -= a5[3 * N + np] * corrected(np + 1);
        if (j < ny) v -= a5[4 * N + np] * corrected(np + nx);
        xout[np] = v / ap;
    }
}

// training target t = delta / sigma and mask (1 on real cells)
__global__ void k_target(int nx, int ny, int H, int W, const double *delta, const double *s, float *t, float *mask)
{
    const long long HW = (long long)H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < HW; p += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(p / W), x = (int)(p - (long long)y * W);
        const bool in = x < nx - 2 && y < ny - 2;
        t[p] = in ? (float)(delta[(long long)(y + 1) * nx + (x + 1)] / s[4]) : 0.f;
        if (mask) mask[p] = in ? 1.f : 0.f;
    }
}

bool image_fits(int nx, int ny, int H, int W) { return nx >= 4 && ny >= 4 && nx - 2 <= W && ny - 2 <= H; }

}  // namespace

extern "C" int m2d_residual5(int nx, int ny, const double *d_a, const double *d_b, const double *d_x, double *d_r,
                             double *d_rr, void *stream)
{
    if (nx < 3 || ny < 3 || !d_a || !d_b || !d_x || !d_r) return unet_fail(M2D_ERR_ARG, "m2d_residual5: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    k_residual5<<<grid_for((long long)nx * ny), 256, 0, st>>>(nx, ny, d_a, d_b, d_x, d_r);
    if (d_rr) k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, d_r, nullptr, d_rr, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_residual5", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

extern "C" int m2d_pprime_features(int nx, int ny, int H, int W, const double *d_a, const double *d_r,
                                   const double *d_Jp, float *d_feat, double *d_stats, void *stream)
{
    if (!image_fits(nx, ny, H, W) || !d_a || !d_r || !d_Jp || !d_feat || !d_stats)
        return unet_fail(M2D_ERR_ARG, "m2d_pprime_features: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, d_r, d_Jp, d_stats, 1);
    k_features<<<grid_for((long long)H * W), 256, 0, st>>>(nx, ny, H, W, d_a, d_r, d_Jp, d_stats, d_feat);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_pprime_features", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

extern "C" int m2d_pprime_apply(int nx, int ny, int H, int W, const double *d_a, const double *d_b, const float *d_y,
                                const double *d_stats, const double *d_x, double *d_xout, void *stream)
{
    if (!image_fits(nx, ny, H, W) || !d_a || !d_b || !d_y || !d_stats || !d_x || !d_xout || d_x == d_xout)
        return unet_fail(M2D_ERR_ARG, "m2d_pprime_apply: bad arguments");
    k_apply<<<grid_for((long long)nx * ny), 256, 0, (cudaStream_t)stream>>>(nx, ny, H, W, d_a, d_b, d_y, d_stats, d_x,
                                                                           d_xout);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_pprime_apply", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

extern "C" int m2d_pprime_target(int nx, int ny, int H, int W, const double *d_delta, const double *d_stats,
                                 float *d_t, float *d_mask, void *stream)
{
    if (!image_fits(nx, ny, H, W) || !d_delta || !d_stats || !d_t)
        return unet_fail(M2D_ERR_ARG, "m2d_pprime_target: bad arguments");
    k_target<<<grid_for((long long)H * W), 256, 0, (cudaStream_t)stream>>>(nx, ny, H, W, d_delta, d_stats, d_t, d_mask);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_pprime_target", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return M2D_OK;
}

extern "C" int m2d_msi_solve_device_ws(int nd, int nx, int ny, int nitm, double tol, const double *d_a,
                                       const double *d_b, double *d_x, double *d_work, long work_doubles,
                                       void *stream, int *d_nit, unsigned long long *d_times, int prec);
extern "C" long m2d_msi_workspace_doubles(int nd, int nx, int ny);

// Flexible pressure-correction solve: the network's correction first, kept
// only if it lowers |b - A x|; then the MSI iteration (at least one, as in
// plain MSI), whose stopping test stays relative to the residual before the
// correction.
namespace m2d {
// x_out = x + the network's correction for the 5-diagonal system A x = b
// (features of r = b - A x), with no acceptance test: the preconditioner of
// the flexible GMRES (m2d_krylov.cu).  x_out must not alias x.
cudaError_t unet_correct(m2d_unet *n, int nx, int ny, const double *d_a, const double *d_b, const double *d_x,
                         double *d_xout, const double *d_Jp, cudaStream_t st)
{
    if (!image_fits(nx, ny, n->H, n->W)) return cudaErrorInvalidValue;
    const int H = n->H, W = n->W;
    const long long N = (long long)nx * ny;
    double *s = n->stats;
    k_residual5<<<grid_for(N), 256, 0, st>>>(nx, ny, d_a, d_b, d_x, n->r);
    k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, n->r, d_Jp, s, 1);
    k_features<<<grid_for((long long)H * W), 256, 0, st>>>(nx, ny, H, W, d_a, n->r, d_Jp, s, n->feat);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = forward(n, 1, n->feat, n->yout, false, st);
    if (e == cudaSuccess) {
        k_apply<<<grid_for(N), 256, 0, st>>>(nx, ny, H, W, d_a, d_b, n->yout, s, d_x, d_xout);
        e = cudaGetLastError();
    }
    return e;
}
}  // namespace m2d

// m2d_pprime_solve_learned, and for the context's p' solve with lagged FP32
// factors (lag_max > 0, prec bit 0): the MSI iteration after the correction
// reuses the workspace's factors as MsiLaunch::lag_max describes, with the
// factor record lag_rec and the equation's tag
int m2d::pprime_solve_learned_lagged(m2d_unet *n, int nx, int ny, int nitm, double tol, const double *d_a,
                                     const double *d_b, double *d_x, const double *d_Jp, double *d_work, int prec,
                                     void *stream, m2d_learned_report *rep, int *lag_rec, int lag_tag, int lag_max)
{
    if (!n || !image_fits(nx, ny, n->H, n->W) || !d_a || !d_b || !d_x || !d_Jp || !d_work || nitm < 1)
        return unet_fail(M2D_ERR_ARG, "m2d_pprime_solve_learned: bad arguments");
    // prec bit 0: FP32 factors and sweeps; bit 1: a kept correction that
    // already meets the MSI stopping test |r| < tol |r0| stands alone
    const bool alone = (prec & 2) != 0;
    prec &= 1;
    cudaStream_t st = (cudaStream_t)stream;
    const int H = n->H, W = n->W;
    const long long N = (long long)nx * ny;
    double *s = n->stats;       // s[0..6] features, s[8] |r0|^2, s[9] |r1|^2
    k_residual5<<<grid_for(N), 256, 0, st>>>(nx, ny, d_a, d_b, d_x, n->r);
    k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, n->r, d_Jp, s, 1);
    k_features<<<grid_for((long long)H * W), 256, 0, st>>>(nx, ny, H, W, d_a, n->r, d_Jp, s, n->feat);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = forward(n, 1, n->feat, n->yout, false, st);
    if (e == cudaSuccess) {
        k_apply<<<grid_for(N), 256, 0, st>>>(nx, ny, H, W, d_a, d_b, n->yout, s, d_x, n->x1);
        k_residual5<<<grid_for(N), 256, 0, st>>>(nx, ny, d_a, d_b, n->x1, n->r);
        k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, n->r, nullptr, s + 9, 0);
        e = cudaGetLastError();
    }
    double hs[10];
    if (e == cudaSuccess) e = cudaMemcpyAsync(hs, s, sizeof hs, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_pprime_solve_learned", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    const double r0 = std::sqrt(hs[0]), r1 = std::sqrt(hs[9]);
    const bool accept = std::isfinite(r1) && r1 < r0;
    double tol_eff = tol;
    if (accept) {
        e = cudaMemcpyAsync(d_x, n->x1, (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, st);
        tol_eff = r1 > 0.0 ? tol * r0 / r1 : 1.0;
    }
    int nit = 0;
    // at least one MSI iteration, as the arbiter of the correction -- unless the
    // corrected residual, measured in FP64, already passes MSI's own stopping
    // test and the caller allows the correction to stand alone
    const bool skip_msi = alone && accept && r1 < tol * r0;
    if (e == cudaSuccess && !skip_msi) {
        const long wd = m2d_msi_workspace_doubles(5, nx, ny);
        if (lag_rec && lag_max > 0 && prec == 1) {
            MsiLaunch L;
            memset(&L, 0, sizeof L);
            L.nx = nx; L.ny = ny; L.nitm = nitm; L.tol = tol_eff;
            L.prec = 1;
            L.lag_max = lag_max;
            L.ws_cap = (size_t)(wd - 4);
            MsiSys &S = L.s[0];
            S.a = d_a; S.b = d_b; S.x = d_x;
            S.ws = d_work;
            S.rr = d_work + (wd - 4);
            S.nit = n->nit;
            S.lag = lag_rec;
            S.tag = lag_tag;
            e = launch_msi(5, L, 1, st);
            if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_pprime_solve_learned: MSI", __FILE__, __LINE__); return M2D_ERR_CUDA; }
        } else {
            const int rc = m2d_msi_solve_device_ws(5, nx, ny, nitm, tol_eff, d_a, d_b, d_x, d_work, wd, stream,
                                                   n->nit, nullptr, prec);
            if (rc) return rc;
        }
        e = cudaMemcpyAsync(&nit, n->nit, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    } else if (e == cudaSuccess) {
        e = cudaStreamSynchronize(st);   // the copy of the kept correction
    }
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_pprime_solve_learned", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    if (rep) { rep->accepted = accept ? 1 : 0; rep->r0 = r0; rep->r1 = r1; rep->nit = nit; }
    return M2D_OK;
}

extern "C" int m2d_pprime_solve_learned(m2d_unet *n, int nx, int ny, int nitm, double tol, const double *d_a,
                                        const double *d_b, double *d_x, const double *d_Jp, double *d_work, int prec,
                                        void *stream, m2d_learned_report *rep)
{
    return m2d::pprime_solve_learned_lagged(n, nx, ny, nitm, tol, d_a, d_b, d_x, d_Jp, d_work, prec, stream, rep,
                                            nullptr, 0, 0);
}

// Two-level cycles: the network's correction (kept only if it lowers |r|)
// alternating with m MSI iterations, until |r| <= tol |r0| or max_cycles.
// rep->nit counts all MSI iterations, rep->accepted the kept corrections,
// rep->r0 and rep->r1 the initial and final |r|.
extern "C" int m2d_pprime_solve_cycles(m2d_unet *n, int nx, int ny, int m, int max_cycles, double tol,
                                       const double *d_a, const double *d_b, double *d_x, const double *d_Jp,
                                       double *d_work, int prec, void *stream, m2d_learned_report *rep)
{
    if (!n || !image_fits(nx, ny, n->H, n->W) || !d_a || !d_b || !d_x || !d_Jp || !d_work || m < 1 || max_cycles < 1)
        return unet_fail(M2D_ERR_ARG, "m2d_pprime_solve_cycles: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const int H = n->H, W = n->W;
    const long long N = (long long)nx * ny;
    double *s = n->stats;
    const long wd = m2d_msi_workspace_doubles(5, nx, ny);
    const double *rr = d_work + (wd - 4);      // the MSI call's |r0|^2, |r|^2
    auto fail_cuda = [&](cudaError_t e) {
        m2d_set_last_error(e, "m2d_pprime_solve_cycles", __FILE__, __LINE__);
        return M2D_ERR_CUDA;
    };
    k_residual5<<<grid_for(N), 256, 0, st>>>(nx, ny, d_a, d_b, d_x, n->r);
    k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, n->r, nullptr, s + 8, 0);
    double h;
    cudaError_t e = cudaMemcpyAsync(&h, s + 8, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda(e);
    const double r0 = std::sqrt(h), goal = tol * r0;
    double rcur = r0;
    int accepted = 0, nit_total = 0;
    for (int cyc = 0; cyc < max_cycles && rcur > goal; cyc++) {
        // n->r holds b - A x here
        k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, n->r, d_Jp, s, 1);
        k_features<<<grid_for((long long)H * W), 256, 0, st>>>(nx, ny, H, W, d_a, n->r, d_Jp, s, n->feat);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = forward(n, 1, n->feat, n->yout, false, st);
        if (e != cudaSuccess) return fail_cuda(e);
        k_apply<<<grid_for(N), 256, 0, st>>>(nx, ny, H, W, d_a, d_b, n->yout, s, d_x, n->x1);
        k_residual5<<<grid_for(N), 256, 0, st>>>(nx, ny, d_a, d_b, n->x1, n->r);
        k_sys_stats<<<1, kStatThreads, 0, st>>>(nx, ny, d_a, n->r, nullptr, s + 9, 0);
        e = cudaMemcpyAsync(&h, s + 9, sizeof h, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail_cuda(e);
        const double r1 = std::sqrt(h);
        if (std::isfinite(r1) && r1 < rcur) {
            e = cudaMemcpyAsync(d_x, n->x1, (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return fail_cuda(e);
            rcur = r1;
            accepted++;
        }
        const int rc = m2d_msi_solve_device_ws(5, nx, ny, m, goal / rcur, d_a, d_b, d_x, d_work, wd, stream, n->nit,
                                               nullptr, prec);
        if (rc) return rc;
        int nit = 0;
        double rrh[2];
        e = cudaMemcpyAsync(&nit, n->nit, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(rrh, rr, sizeof rrh, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail_cuda(e);
        nit_total += nit;
        rcur = std::sqrt(rrh[1]);
        if (rcur > goal && cyc + 1 < max_cycles) {
            k_residual5<<<grid_for(N), 256, 0, st>>>(nx, ny, d_a, d_b, d_x, n->r);
            e = cudaGetLastError();
            if (e != cudaSuccess) return fail_cuda(e);
        }
    }
    if (rep) { rep->accepted = accepted; rep->r0 = r0; rep->r1 = rcur; rep->nit = nit_total; }
    return M2D_OK;
}

extern "C" int m2d_unet_set_tensor_path(int mode)
{
    if (mode < 0 || mode > 2) return unet_fail(M2D_ERR_ARG, "m2d_unet_set_tensor_path: mode 0, 1 or 2");
    g_tensor_tc = mode;
    return M2D_OK;
}

extern "C" int m2d_unet_status(m2d_unet *n, int *flags)
{
    if (!n || !flags) return unet_fail(M2D_ERR_ARG, "m2d_unet_status: null argument");
    cudaSetDevice(n->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(flags, n->err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && *flags) e = cudaMemset(n->err, 0, sizeof(int));   // read and clear
    if (e != cudaSuccess) { m2d_set_last_error(e, "m2d_unet_status", __FILE__, __LINE__); return M2D_ERR_CUDA; }
    return *flags ? M2D_ERR_TIMEOUT : M2D_OK;
}
