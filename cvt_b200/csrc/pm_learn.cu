// Learned plane proposal: a BF16 CNN whose per-pixel (disparity, nx, ny) replaces the random
// initialisation of PMHuberStereo::disparityMap through its initdisparity and initnormalmap
// arguments (PMHuberStereo.cpp:92-93, :469-470 -> pmhstereo_init_disparity_normal,
// pmhstereo.cl:802-828, which builds each pixel's plane with nd_state_from_disparity_normal,
// :99-106).
//
// Network, at 1 / scale of the image resolution (W4 = W / scale, H4 = H / scale, floor;
// "feature pixels"):
//   input   6 channels: the left and right images' RGB, means of scale x scale blocks of
//           k / 255, minus 0.5, padded with zeros to 16 channels (BF16, NHWC)
//   8 convs 3x3, channels 16(6) -> 32 -> 32 -> 64 -> 64 -> 64 -> 64 -> 32 -> 16(3), dilations
//           1, 1, 2, 4, 8, 16, 1, 1 (a receptive field of 69 feature pixels), BF16 weights and
//           activations, FP32 accumulation, bias and ReLU after the first seven; the eighth
//           gives (d, nx, ny) in FP32: disparity in feature pixels and the normal's x and y
//   output  bilinear upsampling to full resolution: disparity d * scale, normal (nx, ny,
//           sqrt(max(1 - nx^2 - ny^2, 0.01)))
// The right view's proposal is the network applied to the mirrored, swapped pair (the right
// image flipped left-right as the first view): its disparities are the right view's, and
// its normal (nx', ny') becomes (nx', -ny') in the convention pmhstereo_init_disparity_normal
// uses for the right view (there nx / nz is the x-slope of the right disparity, for the left
// view minus the x-slope of the left one).
//
// Tensor cores (tcgen05, kind::f16, BF16 x BF16 -> FP32 in TMEM):
//   k_conv_tc   forward and data gradient: an implicit GEMM, 128-pixel tiles (M) x COUT (N),
//               K = 9 taps x CIN; persistent (one CTA per SM), warp-specialised: TMA loads of
//               each tap's shifted 16 x 8-pixel box (zero padding by the TMA) through a ring of
//               shared-memory buffers, one thread issuing the MMAs into two TMEM accumulators,
//               four warps reading TMEM (tcgen05.ld 32x32b) for the epilogue and storing
//               through shared memory, coalesced.  The data gradient is the same kernel with
//               the layer's transposed, tap-mirrored weights and the ReLU mask of the layer's
//               input in the epilogue.
//   k_wgrad_tc  weight gradient: D[(tap, ci)][co] = sum over pixels of x[p + tap][ci] dy[p][co]
//               as MMAs of M128 (tap, ci rows) x N COUT x K16 (pixels), both operands MN-major
//               (16-byte NHWC channel groups are the core-matrix rows, so cp.async copies them
//               unchanged), a row of ones in A gives the bias gradient; two shared-memory
//               stages so that the copies of 64 pixels overlap the MMAs of the previous 64;
//               per-CTA partial sums reduced in CTA order (deterministic).
// Every wait on an mbarrier is bounded by clock (about two seconds); past the limit the kernel
// raises the error flag that the host reads.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/cvtpm.h"

namespace pm {
namespace lpp {

constexpr int NL = 8;
constexpr int LCIN[NL] = {16, 32, 32, 64, 64, 64, 64, 32};
constexpr int LCOUT[NL] = {32, 32, 64, 64, 64, 64, 32, 16};
constexpr int LDIL[NL] = {1, 1, 2, 4, 8, 16, 1, 1};
constexpr int IN_CH = 16, OUT_CH = 16, MAX_CH = 64;
constexpr int TM = 128;                           // pixels per CTA (conv)
constexpr long long WAIT_CYCLES = 4000000000ll;   // about two seconds at the B200's clock

enum { EPI_RELU_BF16 = 0, EPI_BIAS_F32 = 1, EPI_MASK_BF16 = 2 };

__host__ __device__ constexpr int tmem_cols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor (sm100): start >> 4 in bits 0-13, LBO >> 4 in 16-29,
// SBO >> 4 in 32-45, version 1 in 46-47, no swizzle (layout type 0 in 61-63)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// A and B MN-major when the flags are set (bits 15, 16), N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t idesc(int M, int N, bool a_mn, bool b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of the 16-byte chunk `c` (8 K elements) of row `r` in a canonical K-major tile of
// `rows` rows: 8-row x 16-byte core matrices, row groups 128 bytes apart (SBO), K chunks a
// whole column of core matrices apart (LBO = rows / 8 * 128)
__device__ __forceinline__ uint32_t canon(int c, int r, int rows) { return (uint32_t)(c * (rows / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16); }

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t id, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem), "l"(ad), "l"(bd), "r"(id), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

// non-blocking test of an mbarrier phase
__device__ __forceinline__ bool mbar_test(uint32_t addr, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(phase)
        : "memory");
    return ok != 0;
}

// spin on the phase for at most `cycles` SM clocks
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t phase, long long cycles)
{
    const long long t0 = clock64();
    while (!mbar_test(addr, phase))
        if (clock64() - t0 > cycles) return false;
    return true;
}

// 16 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
}

// 16-byte asynchronous copy global -> shared; zeros when !ok (the source is then not read)
__device__ __forceinline__ void cp16(void* dst, const void* src, bool ok)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(ok ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, int cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t tmem, int cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

// pixel m of a B x H x W batch shifted by tap t (3x3, dilation dil): its linear index, or -1
// outside the image (zero padding)
__device__ __forceinline__ int tap_pixel(int m, int M, int H, int W, int t, int dil)
{
    if (m >= M) return -1;
    const int HW = H * W;
    const int b = m / HW, rem = m - b * HW, y = rem / W, x = rem - y * W;
    const int yy = y + (t / 3 - 1) * dil, xx = x + (t % 3 - 1) * dil;
    if (yy < 0 || yy >= H || xx < 0 || xx >= W) return -1;
    return b * HW + yy * W + xx;
}

// the convolution's pixel tiles: TX x TY pixels of one image, x fastest (the MMA's M rows)
constexpr int TX = 16, TY = 8;
constexpr int CONV_THREADS = 224;   // warps 0-3 epilogue, 4 loads (TMA), 5 MMAs, 6 waits for 5
constexpr int CONV_LOADERS = 8;     // lanes of warp 4 that issue the loads, one step each in turn

template <int CIN, int COUT, int EPI>
struct ConvShape {
    static constexpr int A_STAGE = TM * CIN * 2;          // one tap's 128 pixels x CIN, BF16
    static constexpr int B_BYTES = COUT * 9 * CIN * 2;    // all the weights
    static constexpr int RB = COUT * (EPI == EPI_BIAS_F32 ? 4 : 2);   // output bytes per pixel
    static constexpr int STG = 4 * 32 * RB;               // the epilogue warps' staging rows
    static constexpr int FIT = (225 * 1024 - B_BYTES - STG - 1024) / A_STAGE / CONV_LOADERS * CONV_LOADERS;
    static constexpr int STAGES = FIT > 16 ? 16 : FIT;   // a multiple of CONV_LOADERS
    static constexpr int SMEM = STAGES * A_STAGE + B_BYTES + STG + 1024;   // + alignment of the ring to 1024
    static_assert(STAGES >= CONV_LOADERS && STAGES % CONV_LOADERS == 0, "shared memory");
    static_assert(RB == 32 || RB == 64 || RB == 128, "staging row");
};

// epilogue of one warp's 32 pixels of a tile (lane = TMEM lane = pixel p of the warp: tile row
// 2 warp + p / TX, column p % TX; rows y0.., columns x0.. of image b), per EPI (see k_conv_tc).
// The accumulator row is read from TMEM (tcgen05.ld 32x32b), finished in registers and written
// to the warp's staging rows in shared memory (16-byte chunk q of pixel p at chunk
// q ^ ((p / (128 / RB)) % (RB / 16)), so that 32 lanes writing one chunk each hit distinct
// banks); then the warp stores the rows with consecutive lanes on consecutive 16-byte chunks
// (two image rows of TX pixels, each contiguous in NHWC).  The ReLU mask of the data gradient
// comes in the same way, coalesced, before the accumulator is read.
template <int COUT, int EPI>
struct EpiGeom {
    static constexpr int ES = EPI == EPI_BIAS_F32 ? 4 : 2, RB = COUT * ES, NQ = RB / 16, PPR = 128 / RB;
    // pixel p of warp `warp` in the tile at (b, y0, x0): its linear index, or -1 outside the image
    __device__ __forceinline__ static long long pixel(int p, int warp, int b, int y0, int x0, int H, int W)
    {
        const int y = y0 + 2 * warp + p / TX, x = x0 + p % TX;
        return (y < H && x < W) ? ((long long)b * H + y) * W + x : -1;
    }
    __device__ __forceinline__ static uint8_t* chunk(uint8_t* stg, int p, int q) { return stg + p * RB + ((q ^ ((p / PPR) % NQ)) << 4); }
};

// this lane's share of the warp's 32 pixels' mask rows (chunk c = lane + 32 i), loaded coalesced;
// issued before the accumulator wait so that the loads are in flight meanwhile
template <int COUT>
__device__ __forceinline__ void conv_mask_load(uint4 (&mk)[COUT * 2 / 16], int warp, int lane, int b, int y0, int x0, int H,
                                               int W, const __nv_bfloat16* __restrict__ mask)
{
    using G = EpiGeom<COUT, EPI_MASK_BF16>;
#pragma unroll
    for (int i = 0; i < G::NQ; i++) {
        const int c = lane + 32 * i, p = c / G::NQ, q = c % G::NQ;
        const long long m = G::pixel(p, warp, b, y0, x0, H, W);
        mk[i] = m >= 0 ? *reinterpret_cast<const uint4*>(reinterpret_cast<const uint8_t*>(mask) + m * G::RB + q * 16)
                       : make_uint4(0u, 0u, 0u, 0u);
    }
}

template <int COUT, int EPI>
__device__ __forceinline__ void conv_epilogue(uint32_t tacc, int warp, int lane, uint8_t* stg, int b, int y0, int x0,
                                              int H, int W, const float* __restrict__ sbias, const uint4* mkreg,
                                              void* __restrict__ out)
{
    using G = EpiGeom<COUT, EPI>;
    constexpr int RB = G::RB, NQ = G::NQ;
    auto pixel = [&](int p) { return G::pixel(p, warp, b, y0, x0, H, W); };
    auto chunk = [&](int p, int q) { return G::chunk(stg, p, q); };
    if (EPI == EPI_MASK_BF16) {
#pragma unroll
        for (int i = 0; i < NQ; i++) {
            const int c = lane + 32 * i;
            *reinterpret_cast<uint4*>(chunk(c / NQ, c % NQ)) = mkreg[i];
        }
        __syncwarp();
    }
    uint32_t r[COUT];
#pragma unroll
    for (int j0 = 0; j0 < COUT; j0 += 16) tmem_ld16(tacc + ((uint32_t)(warp * 32) << 16) + j0, *reinterpret_cast<uint32_t(*)[16]>(r + j0));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int p = lane;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        uint4* dst = reinterpret_cast<uint4*>(chunk(p, q));
        if (EPI == EPI_BIAS_F32) {
            const int j = 4 * q;
            *reinterpret_cast<float4*>(dst) =
                make_float4(__uint_as_float(r[j]) + sbias[j], __uint_as_float(r[j + 1]) + sbias[j + 1],
                            __uint_as_float(r[j + 2]) + sbias[j + 2], __uint_as_float(r[j + 3]) + sbias[j + 3]);
        } else {
            const int j = 8 * q;
            __align__(16) __nv_bfloat162 v[4];
            __align__(16) __nv_bfloat162 mk[4];
            if (EPI == EPI_MASK_BF16) *reinterpret_cast<uint4*>(mk) = *dst;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                float x0v = __uint_as_float(r[j + 2 * i]), x1v = __uint_as_float(r[j + 2 * i + 1]);
                if (EPI == EPI_RELU_BF16) {
                    x0v = fmaxf(x0v + sbias[j + 2 * i], 0.0f);
                    x1v = fmaxf(x1v + sbias[j + 2 * i + 1], 0.0f);
                } else {
                    x0v = __low2float(mk[i]) > 0.0f ? x0v : 0.0f;
                    x1v = __high2float(mk[i]) > 0.0f ? x1v : 0.0f;
                }
                v[i] = __floats2bfloat162_rn(x0v, x1v);
            }
            *dst = *reinterpret_cast<const uint4*>(v);
        }
    }
    __syncwarp();
#pragma unroll
    for (int c = lane; c < 32 * NQ; c += 32) {
        const int pp = c / NQ, q = c % NQ;
        const long long m = pixel(pp);
        if (m >= 0) *reinterpret_cast<uint4*>(static_cast<uint8_t*>(out) + m * RB + q * 16) = *reinterpret_cast<const uint4*>(chunk(pp, q));
    }
    __syncwarp();
}

// shared-memory descriptor of a K-major operand whose rows (row = 32, 64 or 128 bytes) are
// swizzled at their own width, as the TMA writes them: 8-row atoms SBO = 8 row apart, layout
// type 6 (32B), 4 (64B) or 2 (128B) in bits 61-63; the leading offset is unused (1)
__device__ __forceinline__ uint64_t smem_desc_sw(uint32_t addr, int row)
{
    const uint64_t lt = row == 128 ? 2u : row == 64 ? 4u : 6u;
    return (uint64_t)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(((8 * row) >> 4) & 0x3FFF) << 32) |
           (1ull << 46) | (lt << 61);
}

__device__ __forceinline__ void mbar_init(uint64_t* b, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
}

// tiled TMA load of one box of a 4-D tensor map into this CTA's shared memory; completion is
// counted in bytes on the mbarrier
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t mbar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(mbar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

// mbarrier.try_wait: the thread may sleep in it until the phase completes or a short,
// hardware-chosen time passes; true once the phase has completed
__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v)
{
    asm volatile("st.release.cta.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}

// wait for an mbarrier phase for at most WAIT_CYCLES, giving up early once another role of the
// CTA has given up (*abort); a timeout sets *abort.  The common case (the phase completes within
// the first try_wait) reads neither the clock nor the flag.
__device__ __forceinline__ bool mbar_wait_role(uint32_t addr, uint32_t phase, volatile int* abort)
{
    if (mbar_try(addr, phase)) return true;
    const long long t0 = clock64();
    while (!mbar_try(addr, phase)) {
        if (*abort) return false;
        if (clock64() - t0 > WAIT_CYCLES) {
            *abort = 1;
            return false;
        }
    }
    return true;
}

// out[m][n] = sum over taps t and channels c of in[pixel m shifted by tap t][c] * wmat[n][t][c],
// 3x3 taps (dy, dx) = ((t / 3 - 1) dil, (t % 3 - 1) dil) with zero padding, then per EPI:
//   EPI_RELU_BF16  + bias, ReLU, BF16 out          (forward, hidden layers)
//   EPI_BIAS_F32   + bias, FP32 out                (forward, last layer)
//   EPI_MASK_BF16  times (mask[m][n] > 0), BF16 out (data gradient through the ReLU)
// Persistent and warp-specialised; CTA c takes tiles c, c + grid, ... of TX x TY pixels.  The
// weights (B, canonical K-major without swizzle, K = 9 CIN) are copied into shared memory once.
// A step is one (tile, tap): its A operand is one TMA box (CIN, TX, TY, 1) of the NHWC input
// at the tile's corner shifted by the tap, which the TMA fills with zeros outside the image
// (the padding), written with the swizzle of a CIN * 2-byte row so that it is the MMA's K-major
// swizzled layout as it lands.  Roles:
//   warp 4, lanes 0..CONV_LOADERS-1: the loads, into a ring of STAGES buffers, lane l taking
//     steps l, l + CONV_LOADERS, ... (one thread can have only a few boxes in issue at a time);
//     a full barrier per buffer counts the bytes, an empty barrier per buffer is the MMAs'
//   warp 6: tests the next 8 steps' full barriers (and, at a tile's first step, whether the
//     epilogue has released the tile's accumulator) and publishes the count of ready steps
//   warp 5, lane 0: issues each ready step's CIN / 16 MMAs (M128, N COUT, K16) into one of two
//     TMEM accumulators, alternating per tile, commits them to the buffer's empty barrier and,
//     after the ninth tap, to the accumulator's full barrier; it reads the published count
//     instead of waiting on mbarriers, whose round trip would stall it
//   warps 0-3: the epilogue (conv_epilogue), then release of the accumulator
// So loads, MMAs and the previous tile's epilogue overlap.  Every wait is bounded; a role that
// times out raises the CTA's abort flag and the error flag, the others stop at their next wait,
// and the CTA waits (bounded) for the loads and MMAs it has in flight before it frees TMEM.
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(CONV_THREADS, 1)
    k_conv_tc(const __grid_constant__ CUtensorMap xmap, const __nv_bfloat16* __restrict__ wmat,
              const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask, void* __restrict__ out, int B,
              int H, int W, int dil, int* err)
{
    using Sh = ConvShape<CIN, COUT, EPI>;
    constexpr int S = Sh::STAGES, A_STAGE = Sh::A_STAGE, ROW = CIN * 2;
    constexpr int KTOT = 9 * CIN, KC = KTOT / 8;
    constexpr uint32_t B_LBO = (COUT / 8) * 128;
    constexpr int TCOLS = tmem_cols(2 * COUT);
    constexpr uint32_t ID = idesc(TM, COUT, false, false);
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full[S], empty[S], accf[2], acce[2];
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag, n_loaded[CONV_LOADERS], n_consumed, n_committed, n_ready;
    __shared__ float sbias[COUT];
    volatile int* abort = &abort_flag;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t sA = (raw + 1023u) & ~1023u;   // swizzle atoms need 1024-byte alignment
    uint8_t* sBp = smem_raw + (sA - raw) + S * A_STAGE;
    const uint32_t sB = smem_u32(sBp);
    uint8_t* stg = sBp + Sh::B_BYTES;   // 4 x 32 x RB bytes
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int txn = (W + TX - 1) / TX, tyn = (H + TY - 1) / TY, per_img = txn * tyn;
    const int ntiles = B * per_img;
    const int mine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int nsteps = 9 * mine;

    for (int i = tid; i < COUT * KC; i += CONV_THREADS) {
        const int n = i / KC, c = i - n * KC;
        cp16(sBp + canon(c, n, COUT), reinterpret_cast<const uint4*>(wmat + (size_t)n * KTOT) + c, true);
    }
    cp_commit();
    if (tid < COUT) sbias[tid] = (EPI == EPI_MASK_BF16) ? 0.0f : bias[tid];
    if (warp == 4) tmem_alloc(&tmem_base, TCOLS);
    if (tid == 0) {
        for (int i = 0; i < S; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&accf[i], 1);
            mbar_init(&acce[i], 4);
        }
        abort_flag = 0;
        for (int i = 0; i < CONV_LOADERS; i++) n_loaded[i] = 0;
        n_consumed = 0;
        n_committed = 0;
        n_ready = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cp_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the weights, for the tensor cores
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    if (warp == 4) {
        // loads: lane l issues steps l, l + CONV_LOADERS, ... (a TMA issue holds its thread for
        // a while, so several lanes keep more boxes in flight); step k's buffer k % S belongs to
        // one lane, as S is a multiple of CONV_LOADERS
        if (lane < CONV_LOADERS) {
            int k = lane;
            for (; k < nsteps; k += CONV_LOADERS) {
                const int s = k % S, use = k / S;
                if (use > 0 && !mbar_wait_role(smem_u32(&empty[s]), (use - 1) & 1, abort)) break;
                const int t = (int)blockIdx.x + (k / 9) * (int)gridDim.x, tap = k % 9;
                const int b = t / per_img, r = t - b * per_img, ty = r / txn, tx = r - ty * txn;
                mbar_expect_tx(smem_u32(&full[s]), A_STAGE);
                tma_load_4d(sA + s * A_STAGE, &xmap, smem_u32(&full[s]), 0, tx * TX + (tap % 3 - 1) * dil,
                            ty * TY + (tap / 3 - 1) * dil, b);
            }
            n_loaded[lane] = k;   // the first step this lane did not issue
        }
    } else if (warp == 5) {
        if (lane == 0) {   // MMAs
            // The MMA thread never waits on an mbarrier: such a wait, issued behind MMAs, holds
            // the thread for a few hundred cycles, longer than a step's MMAs run at N <= 64.
            // Warp 6 does the waiting and publishes how many steps are ready (their loads
            // landed, their accumulator free); the MMA thread reads that count (acquire) only
            // when it has used up the steps it knew of.
            const uint64_t adesc0 = smem_desc_sw(sA, ROW), bdesc0 = smem_desc(sB, B_LBO, 128);
            const uint32_t empty0 = smem_u32(&empty[0]);
            int avail = 0, k = 0, s = 0;   // s = k % S
            bool ok = true;
            for (int i = 0; i < mine && ok; i++) {
                const uint32_t acc = tmem + (uint32_t)((i & 1) * COUT);
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    if (k >= avail) {
                        avail = ld_acquire(&n_ready);
                        if (k >= avail) {
                            const long long t0 = clock64();
                            while (k >= avail && !*abort) {
                                if (clock64() - t0 > WAIT_CYCLES) *abort = 1;
                                avail = ld_acquire(&n_ready);
                            }
                            if (k >= avail) {
                                ok = false;
                                break;
                            }
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    }
                    // descriptors advance by address >> 4 in their low bits
                    const uint64_t ad = adesc0 + (uint64_t)(s * (A_STAGE >> 4));
                    const uint64_t bd = bdesc0 + (uint64_t)((tap * (CIN / 8) * B_LBO) >> 4);
#pragma unroll
                    for (int j = 0; j < CIN / 16; j++)
                        mma_f16(acc, ad + (uint64_t)(2 * j), bd + (uint64_t)((2 * j * B_LBO) >> 4), ID,
                                (tap > 0 || j > 0) ? 1u : 0u);
                    mma_commit(empty0 + 8 * s);
                    k++;
                    s = s + 1 == S ? 0 : s + 1;
                }
                if (ok) mma_commit(smem_u32(&accf[i & 1]));
            }
            n_committed = k;
        }
    } else if (warp == 6) {
        // waits for the MMA thread: a step is ready once its load has landed and, for a tile's
        // first step, the tile's accumulator has been released.  Lanes 0..7 test the next 8
        // steps at once (mbarrier.test_wait, each a round trip of a few hundred cycles); the
        // run of ready steps from the first is published.  Testing at most S steps ahead
        // keeps each barrier within one phase of the one tested, so the parity is exact.
        constexpr int WL = 8;
        static_assert(S >= WL, "test window");
        int k = 0;   // steps published
        long long t0 = 0;
        bool waiting = false;
        while (k < nsteps) {
            const int kk = k + lane;
            bool ready = false;
            if (lane < WL && kk < nsteps) {
                ready = mbar_test(smem_u32(&full[kk % S]), (kk / S) & 1);
                const int i = kk / 9;
                if (ready && kk % 9 == 0 && i >= 2) ready = mbar_test(smem_u32(&acce[i & 1]), ((i >> 1) - 1) & 1);
            }
            const unsigned m = __ballot_sync(0xffffffffu, ready);
            const int run = __ffs(~m) - 1;   // ready steps from lane 0 on (at most WL: lanes >= WL vote no)
            if (run > 0) {
                k += run;
                if (lane == 0) st_release(&n_ready, k);
                waiting = false;
            } else {
                if (!waiting) {
                    t0 = clock64();
                    waiting = true;
                }
                int stop = 0;
                if (lane == 0) {
                    if (*abort) stop = 1;
                    else if (clock64() - t0 > WAIT_CYCLES) {
                        *abort = 1;
                        stop = 1;
                    }
                }
                if (__shfl_sync(0xffffffffu, stop, 0)) break;
            }
        }
        if (lane == 0) n_consumed = k;
    } else {   // epilogue, warps 0-3
        for (int i = 0; i < mine; i++) {
            const int a = i & 1;
            const int t = (int)blockIdx.x + i * (int)gridDim.x;
            const int b = t / per_img, r = t - b * per_img, ty = r / txn, tx = r - ty * txn;
            uint4 mk[EPI == EPI_MASK_BF16 ? COUT * 2 / 16 : 1];
            if constexpr (EPI == EPI_MASK_BF16) conv_mask_load<COUT>(mk, warp, lane, b, ty * TY, tx * TX, H, W, mask);
            int ok = 0;
            if (lane == 0) ok = mbar_wait_role(smem_u32(&accf[a]), (i >> 1) & 1, abort);
            if (!__shfl_sync(0xffffffffu, ok, 0)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            conv_epilogue<COUT, EPI>(tmem + (uint32_t)(a * COUT), warp, lane, stg + warp * 32 * Sh::RB, b, ty * TY,
                                     tx * TX, H, W, sbias, mk, out);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[a]);
        }
    }
    __syncthreads();
    bool done = true;
    if (abort_flag) {
        // loads still landing (issued, never waited for by the MMA warp), then the MMAs issued
        // (their last commit covers all of them)
        if (tid == 0) {
            atomicExch(err, 1);
            for (int k = n_consumed; k < n_consumed + S && done; k++)
                if (k < n_loaded[k % CONV_LOADERS])
                    done = mbar_wait_bounded(smem_u32(&full[k % S]), (k / S) & 1, WAIT_CYCLES);
            if (n_committed > 0 && done)
                done = mbar_wait_bounded(smem_u32(&empty[(n_committed - 1) % S]), ((n_committed - 1) / S) & 1, WAIT_CYCLES);
            abort_flag = done ? 1 : 2;
        }
        __syncthreads();
        done = abort_flag == 1;
    }
    if (warp == 4 && done) {
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tmem_free(tmem, TCOLS);
    }
}

// The same convolution on the CUDA cores (FP32 accumulation in tap-channel order): the
// reference the tensor-core kernel is checked against on the device.  One thread per output.
template <int EPI>
__global__ void k_conv_ref(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ wmat,
                           const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask, void* __restrict__ out,
                           int B, int H, int W, int dil, int CIN, int COUT)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int M = B * H * W;
    if (i >= (long long)M * COUT) return;
    const int m = (int)(i / COUT), n = (int)(i - (long long)m * COUT);
    float acc = 0.0f;
    for (int t = 0; t < 9; t++) {
        const int src = tap_pixel(m, M, H, W, t, dil);
        if (src < 0) continue;
        for (int c = 0; c < CIN; c++)
            acc += __bfloat162float(in[(size_t)src * CIN + c]) * __bfloat162float(wmat[(size_t)n * 9 * CIN + t * CIN + c]);
    }
    if (EPI == EPI_BIAS_F32) static_cast<float*>(out)[i] = acc + bias[n];
    else if (EPI == EPI_RELU_BF16) static_cast<__nv_bfloat16*>(out)[i] = __float2bfloat16_rn(fmaxf(acc + bias[n], 0.0f));
    else static_cast<__nv_bfloat16*>(out)[i] = __float2bfloat16_rn(__bfloat162float(mask[i]) > 0.0f ? acc : 0.0f);
}

// Weight gradient on the tensor cores, stage 1: D[r][co] = sum over pixels p of A[r][p] dy[p][co]
// with A[t * CIN + ci][p] = x[p shifted by tap t][ci] and A[9 * CIN][p] = 1 (the bias
// gradient).  Persistent: CTA c sums over units c, c + grid, ... of TX x WG_TY pixels (one
// image's rows) and writes part[c][r][co] for r <= 9 * CIN.  A unit's operands are TMA boxes:
// x at the unit shifted by each tap (box (CIN, TX, WG_TY, 1), zeros outside the image) and dy
// at the unit (zeros outside, so pixels past the image add nothing), each landing as an
// MN-major operand swizzled at its row width (pixel = K row, channels = M or N): an M block of
// 128 rows is 128 / CIN consecutive tap boxes, one swizzle atom per box along M (LBO = a box),
// the last block padded with a box whose first channel is 1 (the row of ones) and zero boxes,
// written once per buffer.  Warp 1, lanes 0..9, issue a unit's 10 boxes into a ring of STAGES
// buffers; warp 0's lane 0 issues its MB x WG_TY MMAs (M128, N COUT, K16) into MB TMEM
// accumulators that persist over all the CTA's units, and commits each unit to its buffer's
// empty barrier; at the end all four warps read TMEM (tcgen05.ld 32x32b) and store the partial
// sums.  Every wait is bounded, as in k_conv_tc.
constexpr int WG_TY = 4;                  // pixel rows of a unit: 16 x 4 = 64 pixels = 4 K steps
constexpr int WG_PX = TX * WG_TY;
constexpr int WG_MAX_CTAS = 160;          // the partial sums' scratch is sized for this many CTAs

template <int CIN, int COUT>
struct WgradShape {
    static constexpr int ROWS = 9 * CIN + 1;          // (tap, ci) rows and the row of ones
    static constexpr int MB = (ROWS + 127) / 128;     // M blocks of 128 rows
    static constexpr int TPB = 128 / CIN;             // boxes per M block
    static constexpr int NBOX = MB * TPB;             // 9 tap boxes, the ones box, zero boxes
    static constexpr int XROW = CIN * 2, DROW = COUT * 2;
    static constexpr int XBOX = WG_PX * XROW, DBOX = WG_PX * DROW;
    static constexpr int STAGE = NBOX * XBOX + DBOX;
    static constexpr int LOADED = 9 * XBOX + DBOX;    // bytes the TMA brings per unit
    static constexpr int FIT = (220 * 1024 - 1024) / STAGE;
    static constexpr int STAGES = FIT > 4 ? 4 : FIT;
    static constexpr int SMEM = STAGES * STAGE + 1024;
    static constexpr int TCOLS = tmem_cols(MB * COUT);
    static_assert(STAGES >= 2 && NBOX >= 10 && MB * COUT <= 512, "weight-gradient shape");
    static_assert(STAGE % 1024 == 0 && XBOX % 1024 == 0, "swizzle atoms stay aligned");
};

// descriptor of an MN-major operand swizzled at its row width (row = 32, 64 or 128 bytes: one
// swizzle atom is 8 K rows of one row width along MN): LBO = the stride between atoms along MN
// (an operand one atom wide passes 8 rows, so that every field stays inside its buffer),
// SBO = the stride between 8-row groups along K
__device__ __forceinline__ uint64_t smem_desc_mn(uint32_t addr, int row, uint32_t lbo)
{
    const uint64_t lt = row == 128 ? 2u : row == 64 ? 4u : 6u;
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(((8 * row) >> 4) & 0x3FFF) << 32) | (1ull << 46) | (lt << 61);
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(128, 1)
    k_wgrad_tc(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap dmap,
               float* __restrict__ part, int B, int H, int W, int dil, int* err)
{
    using S = WgradShape<CIN, COUT>;
    constexpr int NS = S::STAGES;
    constexpr uint32_t ID = idesc(128, COUT, true, true);
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full[NS], empty[NS], done_bar;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag, n_loaded, n_seen, n_committed;
    volatile int* abort = &abort_flag;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t sbase = (raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (sbase - raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int txn = (W + TX - 1) / TX, tyn = (H + WG_TY - 1) / WG_TY, per_img = txn * tyn;
    const int nunits = B * per_img;
    const int mine = (int)blockIdx.x < nunits ? (nunits - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    // the constant boxes 9 .. NBOX - 1 of every buffer: box 9 has 1 in channel 0 of every pixel
    // row (the row of ones; chunk 0 of row r sits at chunk 0 ^ swizzle(r)), the rest zeros
    {
        constexpr int NQ = S::XROW / 16, PPR = 128 / S::XROW, CH = S::XBOX / 16;
        for (int i = tid; i < NS * (S::NBOX - 9) * CH; i += 128) {
            const int st = i / ((S::NBOX - 9) * CH), rem = i - st * ((S::NBOX - 9) * CH);
            const int bx = 9 + rem / CH, c = rem % CH, r = c / NQ, pc = c % NQ;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (bx == 9 && (pc ^ ((r / PPR) % NQ)) == 0) v.x = 0x3F80u;   // BF16 1.0
            *reinterpret_cast<uint4*>(gbase + st * S::STAGE + bx * S::XBOX + c * 16) = v;
        }
    }
    if (warp == 0) tmem_alloc(&tmem_base, S::TCOLS);
    if (tid == 0) {
        for (int i = 0; i < NS; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(&done_bar, 1);
        abort_flag = 0;
        n_loaded = 0;
        n_seen = 0;
        n_committed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the constant boxes, for the tensor cores
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    if (warp == 1) {   // loads: lane b < 9 the box of tap b, lane 9 the dy box
        int k = 0;
        for (; k < mine; k++) {
            const int st = k % NS, use = k / NS;
            int ok = 1;
            if (lane == 0 && use > 0) ok = mbar_wait_role(smem_u32(&empty[st]), (use - 1) & 1, abort);
            if (!__shfl_sync(0xffffffffu, ok, 0)) break;
            const int u = (int)blockIdx.x + k * (int)gridDim.x;
            const int b = u / per_img, r = u - b * per_img, uy = r / txn, ux = r - uy * txn;
            const int x0 = ux * TX, y0 = uy * WG_TY;
            const uint32_t fb = smem_u32(&full[st]), dst = sbase + st * S::STAGE;
            if (lane == 0) mbar_expect_tx(fb, S::LOADED);
            __syncwarp();
            if (lane < 9)
                tma_load_4d(dst + lane * S::XBOX, &xmap, fb, 0, x0 + (lane % 3 - 1) * dil, y0 + (lane / 3 - 1) * dil, b);
            else if (lane == 9)
                tma_load_4d(dst + S::NBOX * S::XBOX, &dmap, fb, 0, x0, y0, b);
        }
        if (lane == 0) n_loaded = k;
    } else if (warp == 0 && lane == 0) {   // MMAs
        int k = 0, committed = 0;
        for (; k < mine; k++) {
            const int st = k % NS;
            if (!mbar_wait_role(smem_u32(&full[st]), (k / NS) & 1, abort)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = sbase + st * S::STAGE, b0 = a0 + S::NBOX * S::XBOX;
#pragma unroll
            for (int ks = 0; ks < WG_TY; ks++)
#pragma unroll
                for (int j = 0; j < S::MB; j++)
                    mma_f16(tmem + j * COUT, smem_desc_mn(a0 + j * S::TPB * S::XBOX + ks * 16 * S::XROW, S::XROW, S::XBOX),
                            smem_desc_mn(b0 + ks * 16 * S::DROW, S::DROW, 8 * S::DROW), ID, (k > 0 || ks > 0) ? 1u : 0u);
            mma_commit(smem_u32(&empty[st]));
            committed = k + 1;
        }
        n_seen = k;
        n_committed = committed;
        if (k == mine) mma_commit(smem_u32(&done_bar));   // covers every MMA of the CTA
    }
    // all four warps: the partial sums
    int ok = 1;
    if (lane == 0) ok = mbar_wait_role(smem_u32(&done_bar), 0, abort);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float* dst = part + (size_t)blockIdx.x * (9 * CIN + 1) * COUT;
#pragma unroll 1
        for (int j = 0; j < S::MB; j++) {
            const int row = j * 128 + warp * 32 + lane;
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                uint32_t r[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + j * COUT + c0, r);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (row <= 9 * CIN) {
                    float4* o = reinterpret_cast<float4*>(dst + (size_t)row * COUT + c0);
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        o[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                           __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
                }
            }
        }
    }
    __syncthreads();
    bool done = true;
    if (abort_flag) {
        // loads still landing (issued, never seen by the MMA thread), then the MMAs issued
        if (tid == 0) {
            atomicExch(err, 1);
            for (int k = n_seen; k < n_loaded && done; k++)
                done = mbar_wait_bounded(smem_u32(&full[k % NS]), (k / NS) & 1, WAIT_CYCLES);
            if (n_committed > 0 && done)
                done = mbar_wait_bounded(smem_u32(&empty[(n_committed - 1) % NS]), ((n_committed - 1) / NS) & 1, WAIT_CYCLES);
            abort_flag = done ? 1 : 2;
        }
        __syncthreads();
        done = abort_flag == 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0 && done) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tmem_free(tmem, S::TCOLS);
    }
}

// weight gradient, stage 2: grad[co][r] (r < 9 CIN) and grad[COUT * 9 CIN + co] (bias) = the sum
// of the CTAs' partials, in a fixed order (deterministic): first WG_SUM_GROUPS groups of
// consecutive CTAs, each summed in CTA order into the group's first partial (in place), then
// the group sums in group order.
constexpr int WG_SUM_GROUPS = 8;
__global__ void k_wgrad_sum_groups(float* __restrict__ part, int nblocks, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, g = blockIdx.y;
    const int per = (nblocks + WG_SUM_GROUPS - 1) / WG_SUM_GROUPS;
    const int b0 = g * per, b1 = b0 + per < nblocks ? b0 + per : nblocks;
    if (i >= n || b0 >= b1) return;
    float s = 0.0f;
#pragma unroll 4
    for (int b = b0; b < b1; b++) s += __ldg(part + (size_t)b * n + i);
    part[(size_t)b0 * n + i] = s;
}
__global__ void k_wgrad_sum(const float* __restrict__ part, float* __restrict__ grad, int nblocks, int CIN, int COUT)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int rows = 9 * CIN + 1, n = rows * COUT;
    if (i >= n) return;
    const int r = i / COUT, co = i - r * COUT;
    const int per = (nblocks + WG_SUM_GROUPS - 1) / WG_SUM_GROUPS;
    float s = 0.0f;
    for (int b = 0; b < nblocks; b += per) s += part[(size_t)b * n + i];
    if (r < 9 * CIN) grad[(size_t)co * 9 * CIN + r] = s;
    else grad[(size_t)COUT * 9 * CIN + co] = s;
}

// the same weight gradient on the CUDA cores, one thread per (co, r) (reference for tests)
__global__ void k_wgrad_ref(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ dy,
                            float* __restrict__ grad, int B, int H, int W, int dil, int CIN, int COUT)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int rows = 9 * CIN + 1, M = B * H * W;
    if (i >= rows * COUT) return;
    const int co = i / rows, r = i - co * rows;
    float s = 0.0f;
    for (int p = 0; p < M; p++) {
        const float g = __bfloat162float(dy[(size_t)p * COUT + co]);
        if (r == 9 * CIN) {
            s += g;
        } else {
            const int t = r / CIN, ci = r - t * CIN;
            const int src = tap_pixel(p, M, H, W, t, dil);
            if (src >= 0) s += __bfloat162float(x[(size_t)src * CIN + ci]) * g;
        }
    }
    if (r < 9 * CIN) grad[(size_t)co * 9 * CIN + r] = s;
    else grad[(size_t)COUT * 9 * CIN + co] = s;
}

// input of the network: 16 BF16 channels per feature pixel, the first view's then the second
// view's RGB as scale x scale block means of k / 255 minus 0.5, then zeros.  right_view: the
// first view is the right image mirrored left-right, the second the left image mirrored.
__global__ void k_input(const uint8_t* __restrict__ left, const uint8_t* __restrict__ right, size_t stride, int W, int sc,
                        int W4, int H4, int right_view, __nv_bfloat16* __restrict__ out)
{
    const int x4 = blockIdx.x * blockDim.x + threadIdx.x, y4 = blockIdx.y * blockDim.y + threadIdx.y;
    if (x4 >= W4 || y4 >= H4) return;
    float acc[6] = {0, 0, 0, 0, 0, 0};
    const uint8_t* first = right_view ? right : left;
    const uint8_t* second = right_view ? left : right;
    for (int dy = 0; dy < sc; dy++)
        for (int dx = 0; dx < sc; dx++) {
            const int xf = x4 * sc + dx;
            const int x = right_view ? W - 1 - xf : xf;
            const size_t o = (size_t)(y4 * sc + dy) * stride + (size_t)x * 4;
            for (int c = 0; c < 3; c++) {
                acc[c] += (float)first[o + c] / 255.0f;
                acc[3 + c] += (float)second[o + c] / 255.0f;
            }
        }
    const float inv = 1.0f / (float)(sc * sc);
    __align__(16) __nv_bfloat16 v[IN_CH];
    for (int c = 0; c < IN_CH; c++) v[c] = __float2bfloat16_rn(c < 6 ? acc[c] * inv - 0.5f : 0.0f);
    uint4* o = reinterpret_cast<uint4*>(out + ((size_t)y4 * W4 + x4) * IN_CH);
    o[0] = reinterpret_cast<const uint4*>(v)[0];
    o[1] = reinterpret_cast<const uint4*>(v)[1];
}

// training target at 1 / sc resolution from plain PatchMatch's final planes of one view
// (planes, float4 a b c cost: the pixel matches a x + b y + c in the other view) and of the
// other view (for the consistency test).  Per pixel: disparity d = x - (a x + b y + c) for the
// left view, (a x + b y + c) - x for the right; normal (a - 1, b, 1) normalised, which is the
// normal pmhstereo_init_disparity_normal turns back into the same a and b for the left view
// (nd_state_from_disparity_normal, pmhstereo.cl:99-106); for the right view the network sees the
// mirrored pair, in which the right view is a left view with normal (a - 1, -b, 1).  A pixel is
// valid when its plane is finite, 0 < d <= dmax, and the other view's disparity at the matched
// column (rounded) is within 1 px of d.  Per feature block (mirrored for the right view): the
// means of d / sc, nx, ny over its valid pixels, and 1 when at least half of it is valid.
__global__ void k_target(const float4* __restrict__ planes, const float4* __restrict__ other, int W, int sc, int W4,
                         int H4, int right_view, float dmax, float4* __restrict__ out)
{
    const int x4 = blockIdx.x * blockDim.x + threadIdx.x, y4 = blockIdx.y * blockDim.y + threadIdx.y;
    if (x4 >= W4 || y4 >= H4) return;
    float d = 0.0f, nx = 0.0f, ny = 0.0f;
    int n = 0;
    for (int dy = 0; dy < sc; dy++)
        for (int dx = 0; dx < sc; dx++) {
            const int y = y4 * sc + dy, xf = x4 * sc + dx;
            const int x = right_view ? W - 1 - xf : xf;
            const float4 s = planes[(size_t)y * W + x];
            if (!(isfinite(s.x) && isfinite(s.y) && isfinite(s.z))) continue;
            const float tx = s.x * (float)x + s.y * (float)y + s.z;
            const float dv = right_view ? tx - (float)x : (float)x - tx;
            if (!(dv > 0.0f && dv <= dmax)) continue;
            const int xo = __float2int_rn(tx);
            if (xo < 0 || xo >= W) continue;
            const float4 o = other[(size_t)y * W + xo];
            const float txo = o.x * (float)xo + o.y * (float)y + o.z;
            const float dov = right_view ? (float)xo - txo : txo - (float)xo;
            if (!(fabsf(dov - dv) <= 1.0f)) continue;
            const float vx = s.x - 1.0f, vy = right_view ? -s.y : s.y;
            const float inv = rsqrtf(vx * vx + vy * vy + 1.0f);
            d += dv;
            nx += vx * inv;
            ny += vy * inv;
            n++;
        }
    const bool ok = 2 * n >= sc * sc && n > 0;
    out[(size_t)y4 * W4 + x4] = ok ? make_float4(d / (float)n / (float)sc, nx / (float)n, ny / (float)n, 1.0f)
                                   : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// L1 loss of the network output (channels d, nx, ny of OUT_CH) against target (d, nx, ny, valid):
// |d - d*| + wn (|nx - nx*| + |ny - ny*|) over valid pixels, times `scale`; dout = its gradient
// (BF16, zero in the unused channels); parts[block] = the block's loss sum (unscaled)
__global__ void k_loss(const float* __restrict__ outp, const float4* __restrict__ target, float wn, float scale, int M,
                       __nv_bfloat16* __restrict__ dout, float* __restrict__ parts)
{
    __shared__ float red[256];
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (m < M) {
        const float* o = outp + (size_t)m * OUT_CH;
        const float4 t = target[m];
        float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
        if (t.w > 0.0f) {
            const float e0 = o[0] - t.x, e1 = o[1] - t.y, e2 = o[2] - t.z;
            l = fabsf(e0) + wn * (fabsf(e1) + fabsf(e2));
            g0 = scale * (float)((e0 > 0.0f) - (e0 < 0.0f));
            g1 = scale * wn * (float)((e1 > 0.0f) - (e1 < 0.0f));
            g2 = scale * wn * (float)((e2 > 0.0f) - (e2 < 0.0f));
        }
        __align__(16) __nv_bfloat16 v[OUT_CH];
        for (int c = 0; c < OUT_CH; c++) v[c] = __float2bfloat16_rn(c == 0 ? g0 : c == 1 ? g1 : c == 2 ? g2 : 0.0f);
        uint4* d = reinterpret_cast<uint4*>(dout + (size_t)m * OUT_CH);
        d[0] = reinterpret_cast<const uint4*>(v)[0];
        d[1] = reinterpret_cast<const uint4*>(v)[1];
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && parts) parts[blockIdx.x] = red[0];
}

// full-resolution initial disparity and normal map from the network output (W4 x H4 x OUT_CH):
// bilinear in (d, nx, ny) at ((x + 0.5) / sc - 0.5, (y + 0.5) / sc - 0.5), clamped to the map;
// disparity d * sc clamped to [0, dmax], normal (nx, ny, sqrt(max(1 - nx^2 - ny^2, 0.01)), 0).
// right_view: the map is of the mirrored pair, read at the mirrored column, ny negated.
__global__ void k_upsample(const float* __restrict__ o4, int W4, int H4, int W, int H, int sc, int right_view,
                           float dmax, float* __restrict__ disp, float4* __restrict__ normal)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const int xs = right_view ? W - 1 - x : x;
    const float u = fminf(fmaxf(((float)xs + 0.5f) / (float)sc - 0.5f, 0.0f), (float)(W4 - 1));
    const float v = fminf(fmaxf(((float)y + 0.5f) / (float)sc - 0.5f, 0.0f), (float)(H4 - 1));
    const int u0 = (int)u, v0 = (int)v;
    const int u1 = min(u0 + 1, W4 - 1), v1 = min(v0 + 1, H4 - 1);
    const float a = u - (float)u0, b = v - (float)v0;
    float r[3];
    for (int c = 0; c < 3; c++) {
        const float p00 = o4[((size_t)v0 * W4 + u0) * OUT_CH + c], p01 = o4[((size_t)v0 * W4 + u1) * OUT_CH + c];
        const float p10 = o4[((size_t)v1 * W4 + u0) * OUT_CH + c], p11 = o4[((size_t)v1 * W4 + u1) * OUT_CH + c];
        r[c] = (1.0f - b) * ((1.0f - a) * p00 + a * p01) + b * ((1.0f - a) * p10 + a * p11);
    }
    const size_t i = (size_t)y * W + x;
    disp[i] = fminf(fmaxf(r[0] * (float)sc, 0.0f), dmax);
    if (normal) {
        const float nx = r[1], ny = right_view ? -r[2] : r[2];
        normal[i] = make_float4(nx, ny, sqrtf(fmaxf(1.0f - nx * nx - ny * ny, 0.01f)), 0.0f);
    }
}

// Adam on FP32 master parameters (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected)
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1, float* __restrict__ m2,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi, v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    p[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

// BF16 copies of one layer's weights: wmat[co][t][ci] (forward) and wt[ci][8 - t][co] (data
// gradient: the transposed, tap-mirrored convolution)
__global__ void k_weights_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ wmat, __nv_bfloat16* __restrict__ wt,
                               int CIN, int COUT)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int K = 9 * CIN;
    if (i >= COUT * K) return;
    const int co = i / K, k = i - co * K, t = k / CIN, ci = k - t * CIN;
    const __nv_bfloat16 v = __float2bfloat16_rn(p[i]);
    wmat[i] = v;
    if (wt) wt[(size_t)ci * 9 * COUT + (8 - t) * COUT + co] = v;
}

}  // namespace lpp
}  // namespace pm

using namespace pm::lpp;

namespace {
thread_local std::string t_lpp_err;
int lfail(int code, const std::string& msg)
{
    t_lpp_err = msg;
    return code;
}
inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
int check_launch(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return lfail(PM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return PM_OK;
}
int check_dims(int B, int H4, int W4)
{
    if (B <= 0 || H4 <= 0 || W4 <= 0 || (long long)B * H4 * W4 > (1ll << 28)) return lfail(PM_EINVAL_SHAPE, "tensor size out of range");
    return PM_OK;
}
inline bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (the library does not link
// the driver)
EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// the tensor map of a B x H x W x C BF16 NHWC activation for the tensor-core kernels' loads:
// box (C, TX, rows, 1), rows of C * 2 bytes swizzled at that width, zeros outside
int act_map(CUtensorMap* map, const void* x, int C, int B, int H, int W, int rows)
{
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return lfail(PM_ECUDA, "the driver lacks cuTensorMapEncodeTiled");
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    const cuuint32_t box[4] = {(cuuint32_t)C, (cuuint32_t)TX, (cuuint32_t)rows, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapSwizzle sw = C == 64   ? CU_TENSOR_MAP_SWIZZLE_128B
                                  : C == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                            : CU_TENSOR_MAP_SWIZZLE_32B;
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return lfail(PM_ECUDA, "cuTensorMapEncodeTiled failed for an activation");
    return PM_OK;
}

// launch k_conv_tc for a (CIN, COUT) pair that the network has: one CTA per SM (persistent)
template <int CIN, int COUT>
int conv_tc(int epi, const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias, const __nv_bfloat16* mk, void* out,
            int B, int H, int W, int dil, int* err, cudaStream_t st)
{
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            nsm = 148;
    }
    CUtensorMap map;
    int rc = act_map(&map, x, CIN, B, H, W, TY);
    if (rc) return rc;
    const long long ntiles = (long long)B * ((H + TY - 1) / TY) * ((W + TX - 1) / TX);
    const int grid = (int)(ntiles < nsm ? ntiles : nsm);
    if (epi == EPI_RELU_BF16) {
        constexpr int SM = ConvShape<CIN, COUT, EPI_RELU_BF16>::SMEM;
        cudaFuncSetAttribute(k_conv_tc<CIN, COUT, EPI_RELU_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
        k_conv_tc<CIN, COUT, EPI_RELU_BF16><<<grid, CONV_THREADS, SM, st>>>(map, w, bias, mk, out, B, H, W, dil, err);
    } else if (epi == EPI_BIAS_F32) {
        if constexpr (COUT == OUT_CH) {   // the last layer only
            constexpr int SM = ConvShape<CIN, COUT, EPI_BIAS_F32>::SMEM;
            cudaFuncSetAttribute(k_conv_tc<CIN, COUT, EPI_BIAS_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
            k_conv_tc<CIN, COUT, EPI_BIAS_F32><<<grid, CONV_THREADS, SM, st>>>(map, w, bias, mk, out, B, H, W, dil, err);
        } else {
            return lfail(PM_EINVAL_ARG, "an FP32 output is the last layer's only");
        }
    } else {
        constexpr int SM = ConvShape<CIN, COUT, EPI_MASK_BF16>::SMEM;
        cudaFuncSetAttribute(k_conv_tc<CIN, COUT, EPI_MASK_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
        k_conv_tc<CIN, COUT, EPI_MASK_BF16><<<grid, CONV_THREADS, SM, st>>>(map, w, bias, mk, out, B, H, W, dil, err);
    }
    return check_launch("k_conv_tc");
}

int conv_dispatch(int CIN, int COUT, int epi, const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias,
                  const __nv_bfloat16* mk, void* out, int B, int H, int W, int dil, int* err, cudaStream_t st)
{
#define PM_CONV_CASE(A, Bc) \
    if (CIN == A && COUT == Bc) return conv_tc<A, Bc>(epi, x, w, bias, mk, out, B, H, W, dil, err, st);
    PM_CONV_CASE(16, 32) PM_CONV_CASE(32, 32) PM_CONV_CASE(32, 64) PM_CONV_CASE(64, 64) PM_CONV_CASE(64, 32)
    PM_CONV_CASE(32, 16)
#undef PM_CONV_CASE
    return lfail(PM_EINVAL_ARG, "no tensor-core convolution for these channel counts");
}

template <int CIN, int COUT>
int wgrad_tc(const __nv_bfloat16* x, const __nv_bfloat16* dy, float* part, float* grad, int B, int H, int W, int dil,
             int* err, cudaStream_t st)
{
    using Sh = WgradShape<CIN, COUT>;
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            nsm = 148;
    }
    CUtensorMap xm, dm;
    int rc = act_map(&xm, x, CIN, B, H, W, WG_TY);
    if (rc) return rc;
    rc = act_map(&dm, dy, COUT, B, H, W, WG_TY);
    if (rc) return rc;
    const long long units = (long long)B * ((H + WG_TY - 1) / WG_TY) * ((W + TX - 1) / TX);
    long long grid = units < nsm ? units : nsm;
    if (grid > WG_MAX_CTAS) grid = WG_MAX_CTAS;
    cudaFuncSetAttribute(k_wgrad_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::SMEM);
    k_wgrad_tc<CIN, COUT><<<(int)grid, 128, Sh::SMEM, st>>>(xm, dm, part, B, H, W, dil, err);
    rc = check_launch("k_wgrad_tc");
    if (rc) return rc;
    const int n = (9 * CIN + 1) * COUT;
    k_wgrad_sum_groups<<<dim3((n + 255) / 256, WG_SUM_GROUPS), 256, 0, st>>>(part, (int)grid, n);
    rc = check_launch("k_wgrad_sum_groups");
    if (rc) return rc;
    k_wgrad_sum<<<(n + 255) / 256, 256, 0, st>>>(part, grad, (int)grid, CIN, COUT);
    return check_launch("k_wgrad_sum");
}

int check_layer(int l)
{
    if (l < 0 || l >= NL) return lfail(PM_EINVAL_ARG, "layer out of range");
    return PM_OK;
}

size_t layer_params(int l) { return (size_t)LCOUT[l] * 9 * LCIN[l] + LCOUT[l]; }
size_t layer_weights(int l) { return (size_t)LCOUT[l] * 9 * LCIN[l]; }
}  // namespace

extern "C" {

const char* pm_lpp_last_error(void) { return t_lpp_err.c_str(); }

int pm_lpp_layers(void) { return NL; }

int pm_lpp_layer_shape(int layer, int* cin, int* cout, int* dilation)
{
    int rc = check_layer(layer);
    if (rc) return rc;
    if (cin) *cin = LCIN[layer];
    if (cout) *cout = LCOUT[layer];
    if (dilation) *dilation = LDIL[layer];
    return PM_OK;
}

int pm_lpp_conv(int layer, int mode, int tensor_cores, const void* in, const void* w, const float* bias, const void* mask,
                void* out, int B, int H4, int W4, int* err, void* stream)
{
    int rc = check_layer(layer);
    if (rc) return rc;
    rc = check_dims(B, H4, W4);
    if (rc) return rc;
    if (mode != 0 && mode != 1) return lfail(PM_EINVAL_ARG, "mode must be 0 (forward) or 1 (data gradient)");
    if (mode == 1 && layer == 0) return lfail(PM_EINVAL_ARG, "the first layer's input has no gradient");
    const bool last = layer == NL - 1;
    const int epi = mode == 1 ? EPI_MASK_BF16 : last ? EPI_BIAS_F32 : EPI_RELU_BF16;
    if (!in || !w || !out || (epi != EPI_MASK_BF16 && !bias) || (epi == EPI_MASK_BF16 && !mask) || (tensor_cores && !err))
        return lfail(PM_EINVAL_ARG, "null buffer");
    if (!aligned16(in) || !aligned16(w) || !aligned16(out) || (mask && !aligned16(mask)))
        return lfail(PM_EINVAL_ARG, "buffers must be 16-byte aligned");
    // forward: CIN -> COUT; data gradient: COUT -> CIN with the transposed weights
    const int cin = mode ? LCOUT[layer] : LCIN[layer], cout = mode ? LCIN[layer] : LCOUT[layer];
    const auto* x = static_cast<const __nv_bfloat16*>(in);
    const auto* wm = static_cast<const __nv_bfloat16*>(w);
    const auto* mk = static_cast<const __nv_bfloat16*>(mask);
    if (tensor_cores) return conv_dispatch(cin, cout, epi, x, wm, bias, mk, out, B, H4, W4, LDIL[layer], err, S(stream));
    const long long n = (long long)B * H4 * W4 * cout;
    const int grid = (int)((n + 255) / 256);
    if (epi == EPI_RELU_BF16) k_conv_ref<EPI_RELU_BF16><<<grid, 256, 0, S(stream)>>>(x, wm, bias, mk, out, B, H4, W4, LDIL[layer], cin, cout);
    else if (epi == EPI_BIAS_F32) k_conv_ref<EPI_BIAS_F32><<<grid, 256, 0, S(stream)>>>(x, wm, bias, mk, out, B, H4, W4, LDIL[layer], cin, cout);
    else k_conv_ref<EPI_MASK_BF16><<<grid, 256, 0, S(stream)>>>(x, wm, bias, mk, out, B, H4, W4, LDIL[layer], cin, cout);
    return check_launch("k_conv_ref");
}

size_t pm_lpp_wgrad_scratch_floats(int layer, int B, int H4, int W4)
{
    if (layer < 0 || layer >= NL || B <= 0 || H4 <= 0 || W4 <= 0) return 0;
    const long long units = (long long)B * ((H4 + WG_TY - 1) / WG_TY) * ((W4 + TX - 1) / TX);
    return (size_t)(units < WG_MAX_CTAS ? units : WG_MAX_CTAS) * (9 * LCIN[layer] + 1) * LCOUT[layer];
}

int pm_lpp_wgrad(int layer, int tensor_cores, const void* x, const void* dy, float* scratch, float* grad, int B, int H4,
                 int W4, int* err, void* stream)
{
    int rc = check_layer(layer);
    if (rc) return rc;
    rc = check_dims(B, H4, W4);
    if (rc) return rc;
    if (!x || !dy || !grad || (tensor_cores && (!scratch || !err))) return lfail(PM_EINVAL_ARG, "null buffer");
    if (!aligned16(x) || !aligned16(dy) || (scratch && !aligned16(scratch)))
        return lfail(PM_EINVAL_ARG, "buffers must be 16-byte aligned");
    const auto* xb = static_cast<const __nv_bfloat16*>(x);
    const auto* db = static_cast<const __nv_bfloat16*>(dy);
    const int dil = LDIL[layer], cin = LCIN[layer], cout = LCOUT[layer];
    if (!tensor_cores) {
        const int n = (9 * cin + 1) * cout;
        k_wgrad_ref<<<(n + 127) / 128, 128, 0, S(stream)>>>(xb, db, grad, B, H4, W4, dil, cin, cout);
        return check_launch("k_wgrad_ref");
    }
#define PM_WG_CASE(A, Bc) \
    if (cin == A && cout == Bc) return wgrad_tc<A, Bc>(xb, db, scratch, grad, B, H4, W4, dil, err, S(stream));
    PM_WG_CASE(16, 32) PM_WG_CASE(32, 32) PM_WG_CASE(32, 64) PM_WG_CASE(64, 64) PM_WG_CASE(64, 32) PM_WG_CASE(32, 16)
#undef PM_WG_CASE
    return lfail(PM_EINVAL_ARG, "no tensor-core weight gradient for these channel counts");
}

int pm_lpp_input(const uint8_t* left, const uint8_t* right, int W, int H, size_t stride, int scale, int right_view,
                 void* out, void* stream)
{
    if (!left || !right || !out) return lfail(PM_EINVAL_ARG, "null buffer");
    if (scale < 1 || W < scale || H < scale || stride < (size_t)W * 4) return lfail(PM_EINVAL_SHAPE, "bad image size or scale");
    if (!aligned16(out)) return lfail(PM_EINVAL_ARG, "output must be 16-byte aligned");
    const int W4 = W / scale, H4 = H / scale;
    const dim3 b(16, 16), g((W4 + 15) / 16, (H4 + 15) / 16);
    k_input<<<g, b, 0, S(stream)>>>(left, right, stride, W, scale, W4, H4, right_view, static_cast<__nv_bfloat16*>(out));
    return check_launch("k_input");
}

int pm_lpp_target(const float* planes, const float* other, int W, int H, int scale, int right_view, float dmax,
                  float* out, void* stream)
{
    if (!planes || !other || !out) return lfail(PM_EINVAL_ARG, "null buffer");
    if (scale < 1 || W < scale || H < scale) return lfail(PM_EINVAL_SHAPE, "bad image size or scale");
    const int W4 = W / scale, H4 = H / scale;
    const dim3 b(16, 16), g((W4 + 15) / 16, (H4 + 15) / 16);
    k_target<<<g, b, 0, S(stream)>>>(reinterpret_cast<const float4*>(planes), reinterpret_cast<const float4*>(other), W,
                                     scale, W4, H4, right_view, dmax, reinterpret_cast<float4*>(out));
    return check_launch("k_target");
}

int pm_lpp_loss(const float* out, const float* target, float wn, float scale, int M, void* dout, float* parts, void* stream)
{
    if (!out || !target || !dout) return lfail(PM_EINVAL_ARG, "null buffer");
    if (M <= 0) return lfail(PM_EINVAL_SHAPE, "no pixels");
    if (!aligned16(dout) || !aligned16(target)) return lfail(PM_EINVAL_ARG, "buffers must be 16-byte aligned");
    k_loss<<<(M + 255) / 256, 256, 0, S(stream)>>>(out, reinterpret_cast<const float4*>(target), wn, scale, M,
                                                  static_cast<__nv_bfloat16*>(dout), parts);
    return check_launch("k_loss");
}

int pm_lpp_upsample(const float* o4, int W4, int H4, int W, int H, int scale, int right_view, float dmax, float* disp,
                    float* normal, void* stream)
{
    if (!o4 || !disp) return lfail(PM_EINVAL_ARG, "null buffer");
    if (W4 < 1 || H4 < 1 || W < 1 || H < 1 || scale < 1) return lfail(PM_EINVAL_SHAPE, "bad size");
    const dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    k_upsample<<<g, b, 0, S(stream)>>>(o4, W4, H4, W, H, scale, right_view, dmax, disp, reinterpret_cast<float4*>(normal));
    return check_launch("k_upsample");
}

int pm_lpp_adam(float* p, const float* g, float* m1, float* m2, int n, float lr, int step, void* stream)
{
    if (!p || !g || !m1 || !m2 || n <= 0 || step < 1) return lfail(PM_EINVAL_ARG, "bad argument");
    const float b1 = 0.9f, b2 = 0.999f;
    k_adam<<<(n + 255) / 256, 256, 0, S(stream)>>>(p, g, m1, m2, n, lr, b1, b2, 1e-8f, 1.0f - powf(b1, (float)step),
                                                  1.0f - powf(b2, (float)step));
    return check_launch("k_adam");
}

int pm_lpp_weights_bf16(int layer, const float* p, void* wmat, void* wt, void* stream)
{
    int rc = check_layer(layer);
    if (rc) return rc;
    if (!p || !wmat) return lfail(PM_EINVAL_ARG, "null buffer");
    const int n = (int)layer_weights(layer);
    k_weights_bf16<<<(n + 255) / 256, 256, 0, S(stream)>>>(p, static_cast<__nv_bfloat16*>(wmat),
                                                          static_cast<__nv_bfloat16*>(wt), LCIN[layer], LCOUT[layer]);
    return check_launch("k_weights_bf16");
}

size_t pm_lpp_param_count(void)
{
    size_t n = 0;
    for (int l = 0; l < NL; l++) n += layer_params(l);
    return n;
}

size_t pm_lpp_propose_workspace_bytes(int W, int H, int scale)
{
    if (scale < 1 || W < scale || H < scale) return 0;
    const size_t px = (size_t)(W / scale) * (H / scale);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return up(px * IN_CH * 2) + 2 * up(px * MAX_CH * 2) + up(px * OUT_CH * 4);
}

// wall: the BF16 weight matrices of all layers back to back (wmat layout, each starting at a
// 16-byte boundary: layer sizes are multiples of 8 elements); ball: all biases back to back
int pm_lpp_propose_device(const void* wall, const float* ball, int scale, const uint8_t* left, const uint8_t* right, int W,
                          int H, size_t stride, int right_view, float dmax, float* disp, float* normal, void* ws,
                          size_t ws_bytes, int* err, void* stream)
{
    if (!wall || !ball || !left || !right || !disp || !ws || !err) return lfail(PM_EINVAL_ARG, "null buffer");
    if (!aligned16(wall) || ((uintptr_t)ws & 255)) return lfail(PM_EINVAL_ARG, "weights 16-byte, workspace 256-byte aligned");
    const size_t need = pm_lpp_propose_workspace_bytes(W, H, scale);
    if (!need || ws_bytes < need) return lfail(PM_EINVAL_ARG, "workspace too small (pm_lpp_propose_workspace_bytes)");
    const int W4 = W / scale, H4 = H / scale;
    const size_t px = (size_t)W4 * H4;
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    uint8_t* p = static_cast<uint8_t*>(ws);
    void* x0 = p;
    void* act[2] = {p + up(px * IN_CH * 2), p + up(px * IN_CH * 2) + up(px * MAX_CH * 2)};
    float* o4 = reinterpret_cast<float*>(p + up(px * IN_CH * 2) + 2 * up(px * MAX_CH * 2));
    int rc = pm_lpp_input(left, right, W, H, stride, scale, right_view, x0, stream);
    if (rc) return rc;
    const auto* w = static_cast<const __nv_bfloat16*>(wall);
    const float* b = ball;
    const void* cur = x0;
    for (int l = 0; l < NL; l++) {
        void* dst = l == NL - 1 ? static_cast<void*>(o4) : act[l & 1];
        rc = pm_lpp_conv(l, 0, 1, cur, w, b, nullptr, dst, 1, H4, W4, err, stream);
        if (rc) return rc;
        w += layer_weights(l);
        b += LCOUT[l];
        cur = dst;
    }
    return pm_lpp_upsample(o4, W4, H4, W, H, scale, right_view, dmax, disp, normal, stream);
}

}  // extern "C"
