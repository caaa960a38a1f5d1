// Learned plane proposal: a small BF16 CNN whose output replaces the random initialisation
// of PMHuberStereo::disparityMap through its initdisparity argument (PMHuberStereo.cpp:92-93,
// pmhstereo_init_disparity_normal, pmhstereo.cl:802-828; normals then come from
// pmhstereo_disparity_to_normal).
//
// Network, at a quarter (scale 4) or half (scale 2) of the image resolution (W4 = W / scale,
// H4 = H / scale, floor; "feature pixels"):
//   features  grey of scale x scale blocks of both images; a cost volume of D = 32 disparity
//             hypotheses (0, k, .. 31 k feature pixels; at scale 4, k = 1 reaches 124 px and 2
//             reaches 248 px): 3x3 mean of |gL(x, y) - gR(x - k d, y)|, times 8
//   6 convs   3x3, 32 -> 32 channels, BF16 weights and activations, FP32 accumulation; ReLU
//             after the first five; the sixth gives 32 logits per pixel (FP32)
//   output    soft-argmin: disparity = k sum_d d softmax(-(logit_d + skip * cost_d))_d (the
//             network corrects the matching cost); upsampled bilinearly and scaled by `scale`
//             to a full-resolution initial disparity
// Training (cvt_b200/learn.py drives it): smooth-L1 loss against the quarter-resolution mean
// of plain PatchMatch's disparity, hand-written backward kernels (data gradients through the
// same tensor-core kernel with the transposed, mirrored weights; weight gradients on the CUDA
// cores, reduced in a fixed order), and Adam.
//
// Tensor cores.  k_conv_tc is an implicit GEMM on tcgen05: one CTA of 128 threads computes
// 128 pixels x 32 output channels, K = 9 taps x 32 input channels = 288 as 18 MMAs of
// M128 N32 K16 (kind::f16, BF16 A and B, FP32 accumulator in 32 TMEM columns).  A (the 128
// pixels' 3x3 neighbourhoods) and B (the weights) are staged in shared memory in the
// canonical K-major layout without swizzle: 8-row x 16-byte core matrices, the row groups
// 128 bytes apart (SBO), the 8-element K chunks a whole tile apart (LBO).  One thread issues
// the MMAs and commits them to an mbarrier; every warp then reads its 32 TMEM lanes
// (tcgen05.ld 32x32b) for the epilogue.  The wait on the mbarrier is bounded: past the limit
// the kernel raises an error flag that the host reads.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "../../include/cvtpm.h"

namespace pm {
namespace lpp {

constexpr int CH = 32;            // channels of every layer, and disparity hypotheses
constexpr int TAPS = 9;
constexpr int KTOT = CH * TAPS;   // 288
constexpr int TM = 128;           // pixels per CTA
constexpr int A_BYTES = TM * KTOT * 2;
constexpr int B_BYTES = CH * KTOT * 2;
constexpr int CONV_SMEM = A_BYTES + B_BYTES;
constexpr uint32_t A_LBO = (TM / 8) * 128;   // bytes between K chunks of A
constexpr uint32_t B_LBO = (CH / 8) * 128;   // bytes between K chunks of B
// kind::f16 instruction descriptor: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(CH >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
constexpr long long WAIT_CYCLES = 4000000000ll;   // about two seconds at the B200's clock

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor (sm100): start >> 4 in bits 0-13, LBO >> 4 in 16-29,
// SBO >> 4 in 32-45, version 1 in 46-47, no swizzle (layout type 0 in 61-63)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// byte offset of the 16-byte chunk `c` (8 K elements) of row `r` in a canonical K-major tile of
// `rows` rows
__device__ __forceinline__ uint32_t canon(int c, int r, int rows) { return (uint32_t)(c * (rows / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16); }

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

enum { EPI_RELU_BF16 = 0, EPI_BIAS_F32 = 1, EPI_MASK_BF16 = 2 };

// out[m][n] = sum over taps t and channels c of in[pixel m shifted by tap t][c] * wmat[n][t][c],
// 3x3 taps (dy, dx) = (t / 3 - 1, t % 3 - 1) with zero padding, then per EPI:
//   EPI_RELU_BF16  + bias, ReLU, BF16 out          (forward, hidden layers)
//   EPI_BIAS_F32   + bias, FP32 out                (forward, logits)
//   EPI_MASK_BF16  times (mask[m][n] > 0), BF16 out (backward: data gradient through ReLU)
template <int EPI>
__global__ void __launch_bounds__(TM) k_conv_tc(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ wmat,
                                                const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask,
                                                void* __restrict__ out, int B, int H, int W, int* err)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    uint8_t* sA = smem;
    uint8_t* sB = smem + A_BYTES;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int HW = H * W, M = B * HW;
    const int m = blockIdx.x * TM + tid;
    const int b = m / HW, rem = m - b * HW, y = rem / W, x = rem - y * W;
    for (int t = 0; t < TAPS; t++) {
        const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
        const bool ok = m < M && yy >= 0 && yy < H && xx >= 0 && xx < W;
        const uint4* src = ok ? reinterpret_cast<const uint4*>(in + ((size_t)b * HW + (size_t)yy * W + xx) * CH) : nullptr;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint4 v = ok ? __ldg(src + q) : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4*>(sA + canon(t * 4 + q, tid, TM)) = v;
        }
    }
    for (int i = tid; i < CH * (KTOT / 8); i += TM) {
        const int n = i / (KTOT / 8), c = i - n * (KTOT / 8);
        *reinterpret_cast<uint4*>(sB + canon(c, n, CH)) = __ldg(reinterpret_cast<const uint4*>(wmat + (size_t)n * KTOT) + c);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)), "r"(CH));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // staged tiles -> tensor core reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (tid == 0) {
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll 1
        for (int j = 0; j < KTOT / 16; j++) {
            const uint64_t ad = smem_desc(a0 + 2 * j * A_LBO, A_LBO, 128);
            const uint64_t bd = smem_desc(b0 + 2 * j * B_LBO, B_LBO, 128);
            const uint32_t acc = j > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                :
                : "r"(tmem), "l"(ad), "l"(bd), "r"(IDESC), "r"(acc)
                : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&mbar))
                     : "memory");
    }
    bool done = mbar_wait_bounded(smem_u32(&mbar), 0, WAIT_CYCLES);
    if (!done) {
        atomicExch(err, 1);
        // the MMAs of this CTA may still run: wait for them once more before freeing TMEM (a
        // CTA whose MMAs never complete reads nothing and leaves its 32 columns allocated)
        done = mbar_wait_bounded(smem_u32(&mbar), 0, WAIT_CYCLES);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (done) {
        uint32_t r[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
            "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
              "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
              "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
              "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (m < M) {
            if (EPI == EPI_BIAS_F32) {
                float4* o = reinterpret_cast<float4*>(static_cast<float*>(out) + (size_t)m * CH);
#pragma unroll
                for (int j = 0; j < CH; j += 4)
                    o[j / 4] = make_float4(__uint_as_float(r[j]) + bias[j], __uint_as_float(r[j + 1]) + bias[j + 1],
                                           __uint_as_float(r[j + 2]) + bias[j + 2], __uint_as_float(r[j + 3]) + bias[j + 3]);
            } else {
                __nv_bfloat162 v[CH / 2];
                const __nv_bfloat16* mk = mask + (size_t)m * CH;
#pragma unroll
                for (int j = 0; j < CH; j += 2) {
                    float a = __uint_as_float(r[j]), c = __uint_as_float(r[j + 1]);
                    if (EPI == EPI_RELU_BF16) {
                        a = fmaxf(a + bias[j], 0.0f);
                        c = fmaxf(c + bias[j + 1], 0.0f);
                    } else {
                        a = __bfloat162float(mk[j]) > 0.0f ? a : 0.0f;
                        c = __bfloat162float(mk[j + 1]) > 0.0f ? c : 0.0f;
                    }
                    v[j / 2] = __floats2bfloat162_rn(a, c);
                }
                uint4* o = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(out) + (size_t)m * CH);
#pragma unroll
                for (int q = 0; q < 4; q++) o[q] = reinterpret_cast<const uint4*>(v)[q];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0 && done) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CH));
}

// The same convolution on the CUDA cores (FP32 accumulation in tap-channel order): the
// reference the tensor-core kernel is checked against on the device.
template <int EPI>
__global__ void k_conv_ref(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ wmat,
                           const float* __restrict__ bias, const __nv_bfloat16* __restrict__ mask, void* __restrict__ out,
                           int B, int H, int W)
{
    const int HW = H * W, M = B * HW;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const int b = m / HW, rem = m - b * HW, y = rem / W, x = rem - y * W;
    float acc[CH];
#pragma unroll
    for (int n = 0; n < CH; n++) acc[n] = 0.0f;
    for (int t = 0; t < TAPS; t++) {
        const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
        if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
        const __nv_bfloat16* src = in + ((size_t)b * HW + (size_t)yy * W + xx) * CH;
        for (int c = 0; c < CH; c++) {
            const float a = __bfloat162float(src[c]);
#pragma unroll
            for (int n = 0; n < CH; n++) acc[n] = fmaf(a, __bfloat162float(wmat[(size_t)n * KTOT + t * CH + c]), acc[n]);
        }
    }
    if (EPI == EPI_BIAS_F32) {
        float* o = static_cast<float*>(out) + (size_t)m * CH;
        for (int n = 0; n < CH; n++) o[n] = acc[n] + bias[n];
    } else {
        __nv_bfloat16* o = static_cast<__nv_bfloat16*>(out) + (size_t)m * CH;
        for (int n = 0; n < CH; n++) {
            float v = acc[n];
            if (EPI == EPI_RELU_BF16) v = fmaxf(v + bias[n], 0.0f);
            else v = __bfloat162float(mask[(size_t)m * CH + n]) > 0.0f ? v : 0.0f;
            o[n] = __float2bfloat16_rn(v);
        }
    }
}

// weight gradient, stage 1: block `blk` sums over its pixels dW[n][t][c] += dy[m][n] x[m + t][c]
// and db[n] += dy[m][n]; partial sums to part[blk][CH * KTOT + CH]
__global__ void __launch_bounds__(KTOT) k_wgrad_part(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ dy,
                                                     float* __restrict__ part, int B, int H, int W, int per_block)
{
    __shared__ float sdy[CH];
    const int k = threadIdx.x, t = k / CH, c = k - t * CH;
    const int HW = H * W, M = B * HW;
    const int m0 = blockIdx.x * per_block, m1 = min(m0 + per_block, M);
    float acc[CH];
#pragma unroll
    for (int n = 0; n < CH; n++) acc[n] = 0.0f;
    float dbias = 0.0f;
    for (int m = m0; m < m1; m++) {
        __syncthreads();
        if (k < CH) sdy[k] = __bfloat162float(dy[(size_t)m * CH + k]);
        __syncthreads();
        if (k < CH) dbias += sdy[k];
        const int b = m / HW, rem = m - b * HW, y = rem / W, xq = rem - y * W;
        const int yy = y + t / 3 - 1, xx = xq + t % 3 - 1;
        if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
        const float a = __bfloat162float(x[((size_t)b * HW + (size_t)yy * W + xx) * CH + c]);
#pragma unroll
        for (int n = 0; n < CH; n++) acc[n] = fmaf(sdy[n], a, acc[n]);
    }
    float* p = part + (size_t)blockIdx.x * (CH * KTOT + CH);
#pragma unroll
    for (int n = 0; n < CH; n++) p[(size_t)n * KTOT + k] = acc[n];
    if (k < CH) p[CH * KTOT + k] = dbias;
}

// weight gradient, stage 2: sum of the partials in block order (deterministic)
__global__ void k_wgrad_sum(const float* __restrict__ part, float* __restrict__ grad, int nblocks)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CH * KTOT + CH) return;
    float s = 0.0f;
    for (int b = 0; b < nblocks; b++) s += part[(size_t)b * (CH * KTOT + CH) + i];
    grad[i] = s;
}

// grey of the sc x sc blocks of an RGBA8 image (0.2126, 0.7152, 0.0722 weights on k / 255)
__global__ void k_grey(const uint8_t* __restrict__ img, size_t stride, int sc, int W4, int H4, float* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W4) return;
    float s = 0.0f;
    for (int j = 0; j < sc; j++) {
        const uchar4* row = reinterpret_cast<const uchar4*>(img + (size_t)(sc * y + j) * stride) + sc * x;
        for (int i = 0; i < sc; i++) {
            const uchar4 p = __ldg(row + i);
            s += 0.2126f * (float)p.x + 0.7152f * (float)p.y + 0.0722f * (float)p.z;
        }
    }
    out[(size_t)y * W4 + x] = s * (1.0f / ((float)(sc * sc) * 255.0f));
}

// cost volume: channel d = 8 x the 3x3 mean of |g1(x, y) - g2(x + s k d, y)| (hypothesis d at k d
// quarter pixels, k = step), s = -1 for the left view (g1 left, g2 right), +1 for the right view
// (g1 right, g2 left); columns outside the image count as a difference of 1; BF16 NHWC
__global__ void k_costvol(const float* __restrict__ gl, const float* __restrict__ gr, int W4, int H4, int sgn,
                          __nv_bfloat16* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W4) return;
    __nv_bfloat16* o = out + ((size_t)y * W4 + x) * CH;
    for (int d = 0; d < CH; d++) {
        float s = 0.0f;
        int n = 0;
        for (int j = -1; j <= 1; j++) {
            const int yy = y + j;
            if (yy < 0 || yy >= H4) continue;
            for (int i = -1; i <= 1; i++) {
                const int xx = x + i;
                if (xx < 0 || xx >= W4) continue;
                const float a = gl[(size_t)yy * W4 + xx];
                const int xm = xx + sgn * d;
                const float c = xm >= 0 && xm < W4 ? gr[(size_t)yy * W4 + xm] : a + 1.0f;
                s += fabsf(a - c);
                n++;
            }
        }
        o[d] = __float2bfloat16_rn(8.0f * s / (float)n);
    }
}

// soft-argmin over the 32 logits plus `skip` times the input cost volume (the network learns a
// correction to the matching cost), and the smooth-L1 loss against target (quarter pixels; a
// target < 0 is masked): disparity out, dLogits (BF16, scaled by 1 / count) and per-block loss
// sums
__global__ void k_softargmin(const float* __restrict__ logits, const __nv_bfloat16* __restrict__ feats, float skip,
                             float step, const float* __restrict__ target, float* __restrict__ disp,
                             __nv_bfloat16* __restrict__ dlogits, float* __restrict__ loss_part, int M, float inv_count)
{
    __shared__ float red[256];
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (m < M) {
        float lg[CH];
        for (int d = 0; d < CH; d++)
            lg[d] = logits[(size_t)m * CH + d] + (feats ? skip * __bfloat162float(feats[(size_t)m * CH + d]) : 0.0f);
        float mn = lg[0];
        for (int d = 1; d < CH; d++) mn = fminf(mn, lg[d]);
        float p[CH], z = 0.0f;
        for (int d = 0; d < CH; d++) {
            p[d] = __expf(-(lg[d] - mn));
            z += p[d];
        }
        float e = 0.0f;
        for (int d = 0; d < CH; d++) {
            p[d] /= z;
            e += (float)d * p[d];
        }
        e *= step;   // hypotheses are `step` quarter pixels apart
        disp[m] = e;
        if (dlogits) {
            float g = 0.0f;
            const float t = target ? target[m] : -1.0f;
            if (t >= 0.0f) {
                const float r = e - t;
                l = fabsf(r) < 1.0f ? 0.5f * r * r : fabsf(r) - 0.5f;
                g = (fabsf(r) < 1.0f ? r : copysignf(1.0f, r)) * inv_count;
            }
            for (int d = 0; d < CH; d++)
                dlogits[(size_t)m * CH + d] = __float2bfloat16_rn(-p[d] * (step * (float)d - e) * g);
        }
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss_part) loss_part[blockIdx.x] = red[0];
}

// training target at 1 / sc resolution: mean of the valid (> 0) disparities of each sc x sc block
// / sc, -1 when fewer than half are valid
__global__ void k_target(const float* __restrict__ disp, int W, int sc, int W4, int H4, float* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W4) return;
    float s = 0.0f;
    int n = 0;
    for (int j = 0; j < sc; j++)
        for (int i = 0; i < sc; i++) {
            const float v = disp[(size_t)(sc * y + j) * W + sc * x + i];
            if (v > 0.0f) {
                s += v;
                n++;
            }
        }
    out[(size_t)y * W4 + x] = 2 * n >= sc * sc ? s / ((float)sc * (float)n) : -1.0f;
}

// full-resolution initial disparity: bilinear upsampling of the 1 / sc resolution result, times sc
__global__ void k_upsample(const float* __restrict__ d4, int W4, int H4, int W, int H, int sc, float* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const float inv = 1.0f / (float)sc;
    const float u = fminf(fmaxf(((float)x + 0.5f) * inv - 0.5f, 0.0f), (float)(W4 - 1));
    const float v = fminf(fmaxf(((float)y + 0.5f) * inv - 0.5f, 0.0f), (float)(H4 - 1));
    const int x0 = (int)u, y0 = (int)v, x1 = min(x0 + 1, W4 - 1), y1 = min(y0 + 1, H4 - 1);
    const float a = u - (float)x0, b = v - (float)y0;
    const float r0 = (1.0f - a) * d4[(size_t)y0 * W4 + x0] + a * d4[(size_t)y0 * W4 + x1];
    const float r1 = (1.0f - a) * d4[(size_t)y1 * W4 + x0] + a * d4[(size_t)y1 * W4 + x1];
    out[(size_t)y * W + x] = (float)sc * ((1.0f - b) * r0 + b * r1);
}

// Adam on the FP32 master weights of one layer (CH * KTOT weights then CH biases), then the BF16
// copies: wmat[n][t][c] and the data-gradient matrix wt[c][8 - t][n]
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

__global__ void k_weights_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ wmat, __nv_bfloat16* __restrict__ wt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CH * KTOT) return;
    const int n = i / KTOT, k = i - n * KTOT, t = k / CH, c = k - t * CH;
    const __nv_bfloat16 v = __float2bfloat16_rn(p[i]);
    wmat[i] = v;
    wt[(size_t)c * KTOT + (8 - t) * CH + n] = v;
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
}  // namespace

extern "C" {

const char* pm_lpp_last_error(void) { return t_lpp_err.c_str(); }

int pm_lpp_channels(void) { return CH; }

int pm_lpp_conv(int epi, int tensor_cores, const void* in, const void* wmat, const float* bias, const void* mask, void* out,
                int B, int H4, int W4, int* err, void* stream)
{
    int rc = check_dims(B, H4, W4);
    if (rc) return rc;
    if (epi < 0 || epi > 2) return lfail(PM_EINVAL_ARG, "unknown epilogue");
    if (!in || !wmat || !out || (epi != EPI_MASK_BF16 && !bias) || (epi == EPI_MASK_BF16 && !mask) || (tensor_cores && !err))
        return lfail(PM_EINVAL_ARG, "null buffer");
    if (((uintptr_t)in | (uintptr_t)wmat | (uintptr_t)out) & 15) return lfail(PM_EINVAL_ARG, "buffers must be 16-byte aligned");
    const int M = B * H4 * W4;
    const auto* x = static_cast<const __nv_bfloat16*>(in);
    const auto* w = static_cast<const __nv_bfloat16*>(wmat);
    const auto* mk = static_cast<const __nv_bfloat16*>(mask);
    if (tensor_cores) {
        cudaFuncSetAttribute(k_conv_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM);
        cudaFuncSetAttribute(k_conv_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM);
        cudaFuncSetAttribute(k_conv_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM);
        const int grid = (M + TM - 1) / TM;
        if (epi == 0) k_conv_tc<0><<<grid, TM, CONV_SMEM, S(stream)>>>(x, w, bias, mk, out, B, H4, W4, err);
        else if (epi == 1) k_conv_tc<1><<<grid, TM, CONV_SMEM, S(stream)>>>(x, w, bias, mk, out, B, H4, W4, err);
        else k_conv_tc<2><<<grid, TM, CONV_SMEM, S(stream)>>>(x, w, bias, mk, out, B, H4, W4, err);
    } else {
        const int grid = (M + 127) / 128;
        if (epi == 0) k_conv_ref<0><<<grid, 128, 0, S(stream)>>>(x, w, bias, mk, out, B, H4, W4);
        else if (epi == 1) k_conv_ref<1><<<grid, 128, 0, S(stream)>>>(x, w, bias, mk, out, B, H4, W4);
        else k_conv_ref<2><<<grid, 128, 0, S(stream)>>>(x, w, bias, mk, out, B, H4, W4);
    }
    return check_launch("pm_lpp_conv");
}

size_t pm_lpp_wgrad_scratch_floats(int B, int H4, int W4, int per_block)
{
    if (per_block <= 0) return 0;
    const long long M = (long long)B * H4 * W4;
    return (size_t)((M + per_block - 1) / per_block) * (CH * KTOT + CH);
}

int pm_lpp_wgrad(const void* x, const void* dy, float* scratch, float* grad, int B, int H4, int W4, int per_block, void* stream)
{
    int rc = check_dims(B, H4, W4);
    if (rc) return rc;
    if (!x || !dy || !scratch || !grad || per_block <= 0) return lfail(PM_EINVAL_ARG, "bad argument");
    const int M = B * H4 * W4, nb = (M + per_block - 1) / per_block;
    k_wgrad_part<<<nb, KTOT, 0, S(stream)>>>(static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy),
                                              scratch, B, H4, W4, per_block);
    k_wgrad_sum<<<(CH * KTOT + CH + 255) / 256, 256, 0, S(stream)>>>(scratch, grad, nb);
    return check_launch("pm_lpp_wgrad");
}

int pm_lpp_features(const uint8_t* left, const uint8_t* right, int W, int H, size_t stride, int right_view, int step,
                    int scale, float* grey_scratch, void* out, void* stream)
{
    if (scale != 2 && scale != 4) return lfail(PM_EINVAL_ARG, "scale must be 2 or 4");
    if (W < scale || H < scale || W > PM_MAX_WIDTH || H > PM_MAX_HEIGHT) return lfail(PM_EINVAL_SHAPE, "image size out of range");
    if (!left || !right || !grey_scratch || !out || stride < (size_t)W * 4 || stride % 4) return lfail(PM_EINVAL_ARG, "bad argument");
    const int W4 = W / scale, H4 = H / scale;
    const dim3 g((W4 + 127) / 128, H4);
    k_grey<<<g, 128, 0, S(stream)>>>(left, stride, scale, W4, H4, grey_scratch);
    k_grey<<<g, 128, 0, S(stream)>>>(right, stride, scale, W4, H4, grey_scratch + (size_t)W4 * H4);
    float* g0 = grey_scratch;
    float* g1 = grey_scratch + (size_t)W4 * H4;
    if (step < 1 || step > 8) return lfail(PM_EINVAL_ARG, "hypothesis step out of range");
    if (right_view) k_costvol<<<g, 128, 0, S(stream)>>>(g1, g0, W4, H4, step, static_cast<__nv_bfloat16*>(out));
    else k_costvol<<<g, 128, 0, S(stream)>>>(g0, g1, W4, H4, -step, static_cast<__nv_bfloat16*>(out));
    return check_launch("pm_lpp_features");
}

int pm_lpp_softargmin(const float* logits, const void* feats, float skip, float step, const float* target, float* disp,
                      void* dlogits, float* loss_part, int M, float inv_count, void* stream)
{
    if (M <= 0 || !logits || !disp || !(step > 0.0f)) return lfail(PM_EINVAL_ARG, "bad argument");
    k_softargmin<<<(M + 255) / 256, 256, 0, S(stream)>>>(logits, static_cast<const __nv_bfloat16*>(feats), skip, step, target,
                                                          disp,
                                                          static_cast<__nv_bfloat16*>(dlogits), loss_part, M, inv_count);
    return check_launch("pm_lpp_softargmin");
}

int pm_lpp_target(const float* disp, int W, int H, int scale, float* out, void* stream)
{
    if ((scale != 2 && scale != 4) || W < scale || H < scale || !disp || !out) return lfail(PM_EINVAL_ARG, "bad argument");
    const int W4 = W / scale, H4 = H / scale;
    k_target<<<dim3((W4 + 127) / 128, H4), 128, 0, S(stream)>>>(disp, W, scale, W4, H4, out);
    return check_launch("pm_lpp_target");
}

int pm_lpp_upsample(const float* d4, int W4, int H4, int W, int H, int scale, float* out, void* stream)
{
    if (W4 <= 0 || H4 <= 0 || W <= 0 || H <= 0 || scale < 1 || !d4 || !out) return lfail(PM_EINVAL_ARG, "bad argument");
    k_upsample<<<dim3((W + 127) / 128, H), 128, 0, S(stream)>>>(d4, W4, H4, W, H, scale, out);
    return check_launch("pm_lpp_upsample");
}

int pm_lpp_adam(float* p, const float* g, float* m1, float* m2, int n, float lr, int step, void* stream)
{
    if (n <= 0 || step <= 0 || !p || !g || !m1 || !m2) return lfail(PM_EINVAL_ARG, "bad argument");
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, S(stream)>>>(p, g, m1, m2, n, lr, b1, b2, 1e-8f, c1, c2);
    return check_launch("pm_lpp_adam");
}

int pm_lpp_weights_bf16(const float* p, void* wmat, void* wt, void* stream)
{
    if (!p || !wmat || !wt) return lfail(PM_EINVAL_ARG, "bad argument");
    k_weights_bf16<<<(CH * KTOT + 255) / 256, 256, 0, S(stream)>>>(p, static_cast<__nv_bfloat16*>(wmat),
                                                                    static_cast<__nv_bfloat16*>(wt));
    return check_launch("pm_lpp_weights_bf16");
}

size_t pm_lpp_propose_workspace_bytes(int W, int H, int scale)
{
    if ((scale != 2 && scale != 4) || W < scale || H < scale) return 0;
    const size_t M = (size_t)(W / scale) * (H / scale);
    // two grey planes, the features and two BF16 activation buffers, FP32 logits, the quarter
    // disparity
    return 2 * M * 4 + 3 * M * CH * 2 + M * CH * 4 + M * 4 + 6 * 256;
}

int pm_lpp_propose_device(const void* wmats, const float* biases, int nlayers, float skip, int step, int scale,
                          const uint8_t* left, const uint8_t* right, int W, int H, size_t stride, int right_view,
                          float* initdisp, void* workspace, size_t ws_bytes, int* err, void* stream)
{
    if (scale != 2 && scale != 4) return lfail(PM_EINVAL_ARG, "scale must be 2 or 4");
    if (W < scale || H < scale || W > PM_MAX_WIDTH || H > PM_MAX_HEIGHT) return lfail(PM_EINVAL_SHAPE, "image size out of range");
    if (!wmats || !biases || nlayers < 1 || !left || !right || !initdisp || !workspace || !err)
        return lfail(PM_EINVAL_ARG, "null argument");
    if (ws_bytes < pm_lpp_propose_workspace_bytes(W, H, scale)) return lfail(PM_EINVAL_ARG, "workspace too small");
    if (((uintptr_t)workspace | (uintptr_t)wmats) & 255) return lfail(PM_EINVAL_ARG, "workspace and weights must be 256-byte aligned");
    const int W4 = W / scale, H4 = H / scale;
    const size_t M = (size_t)W4 * H4;
    char* ws = static_cast<char*>(workspace);
    float* grey = reinterpret_cast<float*>(ws);
    size_t off = (2 * M * 4 + 255) & ~(size_t)255;
    __nv_bfloat16* feats = reinterpret_cast<__nv_bfloat16*>(ws + off);
    off += (M * CH * 2 + 255) & ~(size_t)255;
    __nv_bfloat16* act[2] = {reinterpret_cast<__nv_bfloat16*>(ws + off), nullptr};
    off += (M * CH * 2 + 255) & ~(size_t)255;
    act[1] = reinterpret_cast<__nv_bfloat16*>(ws + off);
    off += (M * CH * 2 + 255) & ~(size_t)255;
    float* logits = reinterpret_cast<float*>(ws + off);
    off += (M * CH * 4 + 255) & ~(size_t)255;
    float* d4 = reinterpret_cast<float*>(ws + off);
    int rc = pm_lpp_features(left, right, W, H, stride, right_view, step, scale, grey, feats, stream);
    if (rc) return rc;
    const auto* w = static_cast<const __nv_bfloat16*>(wmats);
    const __nv_bfloat16* x = feats;
    for (int l = 0; l < nlayers; l++) {
        const bool last = l == nlayers - 1;
        void* y = last ? static_cast<void*>(logits) : static_cast<void*>(act[l & 1]);
        rc = pm_lpp_conv(last ? EPI_BIAS_F32 : EPI_RELU_BF16, 1, x, w + (size_t)l * CH * KTOT, biases + l * CH, nullptr, y, 1,
                         H4, W4, err, stream);
        if (rc) return rc;
        x = act[l & 1];
    }
    rc = pm_lpp_softargmin(logits, feats, skip, (float)step, nullptr, d4, nullptr, nullptr, (int)M, 0.0f, stream);
    if (rc) return rc;
    return pm_lpp_upsample(d4, W4, H4, W, H, scale, initdisp, stream);
}

}  // extern "C"
