// SVPMFlowCL on sm_100a: PatchMatch optical flow with a TV (primal-dual) pull of
// cvt/vision/SVPMFlowCL.cpp and cvt/cl/kernel/SVPMFlow.cl, behind its own C ABI
// (include/cvtpm.h, "SVPMFlowCL").
//
// A state is (u, v, cost, 0): pixel (x, y) of the first frame moves to (x + u, y + v) in the
// second.  SVPMFlowCL::flow (SVPMFlowCL.cpp:58-89): random init, then passes of
// svpmflow_prop_local_tv_admm, each of which
//   * takes one primal-dual step on the dual field p of the flow's TV (tau 0.1) and pulls
//     the candidates towards u + (lambda / tau) div p with weight 1 / (2 lambda 5) after
//     pass 4,
//   * tests the pulled flow, two random flows, two random neighbours within 5 px, then
//     jump steps of 4, 2, 1 px in the four directions inside the 16x16 work-group (the
//     group's states and a 4-pixel apron in shared memory), then two random refinements.
// The 16x16 work-group is part of the algorithm (which states a jump step sees), so the
// kernel keeps it: one CTA per work-group, every thread of a CTA takes part, including
// those beyond the image, as the reference's padded NDRange does.  The jump steps read the
// cells of the previous step (all reads of a step before its writes, two barriers per step):
// the reference reads and writes the cells in one barrier interval, which OpenCL leaves
// undefined.
//
// Arithmetic is the reference's FP32 sequence (-fmad=false): every result equals the
// restatement in oracle/pm_oracle.cpp bit for bit.  log, sin and cos are the library's own
// (pm_math.cuh), as in the oracle.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "../../include/cvtpm.h"
#include "pm_device.cuh"

namespace pm {
namespace svpm {

constexpr int G = 16;          // work-group edge (SVPMFlowCL.cpp:36-37)
constexpr int OFF = 4;         // apron of the state buffer (SVPMFlow.cl:579)
constexpr int BUF = G + 2 * OFF;
constexpr int PB = G + 2;      // dual buffer: the group and a 1-pixel apron

struct Frames {
    const float4* __restrict__ c1;   // first frame, k / 255
    const float4* __restrict__ c2;   // second frame
    int W, H, r;
};

__device__ __forceinline__ float unorm8(uint32_t v) { return __fdiv_rn((float)v, 255.0f); }

// read_imagef with SAMPLER_BILINEAR, CLK_ADDRESS_CLAMP_TO_EDGE at (u, v), for finite u, v:
// weights (1-a)(1-b), a(1-b), (1-a)b, ab, summed in that order (OpenCL 1.2 s8.2)
__device__ __forceinline__ float3 bilinear(const float4* __restrict__ img, int W, int H, float u, float v)
{
    const float tu = u - 0.5f, tv = v - 0.5f;
    const float fu = floorf(tu), fv = floorf(tv);
    const float a = tu - fu, b = tv - fv;
    const int i0 = (int)fminf(fmaxf(fu, -2.0f), (float)W + 1.0f), j0 = (int)fminf(fmaxf(fv, -2.0f), (float)H + 1.0f);
    const int x0 = min(max(i0, 0), W - 1), x1 = min(max(i0 + 1, 0), W - 1);
    const int y0 = min(max(j0, 0), H - 1), y1 = min(max(j0 + 1, 0), H - 1);
    const float4 T00 = __ldg(img + (size_t)y0 * W + x0), T10 = __ldg(img + (size_t)y0 * W + x1);
    const float4 T01 = __ldg(img + (size_t)y1 * W + x0), T11 = __ldg(img + (size_t)y1 * W + x1);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
    return make_float3(((w00 * T00.x + w10 * T10.x) + w01 * T01.x) + w11 * T11.x,
                       ((w00 * T00.y + w10 * T10.y) + w01 * T01.y) + w11 * T11.y,
                       ((w00 * T00.z + w10 * T10.z) + w01 * T01.z) + w11 * T11.z);
}

// svpmflow_eval_bilateral_trunc_sad (SVPMFlow.cl:170-209) at pixel (x, y), which may lie
// beyond the image (threads of the padded groups).  Taps outside the first frame are skipped
// by the loop bounds, taps whose flow leaves the second frame per tap; the first frame is read
// at whole pixels, where its bilinear read is the texel itself.
template <bool COUNT>
__device__ float eval(const Frames& F, int x, int y, float fx, float fy, unsigned long long& taps)
{
    if (!(fin(fx) && fin(fy))) return 1e10f;
    const int W = F.W, H = F.H;
    const float4 vc = __ldg(F.c1 + (size_t)min(y, H - 1) * W + min(x, W - 1));
    const float cx = (float)x, cy = (float)y;
    float ret = 0.0f, wsum = 0.0f;
    const int ylo = max(y - F.r, 0), yhi = min(y + F.r, H - 1);
    const int xlo = max(x - F.r, 0), xhi = min(x + F.r, W - 1);
    for (int iy = ylo; iy <= yhi; iy++) {
        const float py = cy + (float)(iy - y);
        const float qy = py + fy;
        if (qy < 0 || qy >= (float)H) continue;
        const float4* row = F.c1 + (size_t)iy * W;
        for (int ix = xlo; ix <= xhi; ix++) {
            const float px = cx + (float)(ix - x);
            const float qx = px + fx;
            if (qx < 0 || qx >= (float)W) continue;
            const float4 v1 = __ldg(row + ix);
            const float3 v2 = bilinear(F.c2, W, H, qx + 0.5f, qy + 0.5f);
            const float w = expf_neg(-((fabsf(vc.x - v1.x) + fabsf(vc.y - v1.y)) + fabsf(vc.z - v1.z)) * 2.6f);
            wsum += w;
            ret += w * ((fminf(fabsf(v1.x - v2.x), 0.02f) + fminf(fabsf(v1.y - v2.y), 0.02f)) +
                        fminf(fabsf(v1.z - v2.z), 0.02f));
            if (COUNT) taps++;
        }
    }
    if (wsum < 1.1f) return 1e5f;
    return ret / wsum;
}

// box_mueller (SVPMFlow.cl:38-46); theta = 2.0f * M_PI * y is a double product (M_PI is a double)
__device__ __forceinline__ float2 box_mueller(Rng& g)
{
    const float x = g.next(), y = g.next();
    const float rr = sqrtf(-2.0f * logf_(x));
    const float theta = __double2float_rn(__dmul_rn(2.0 * 3.14159265358979323846, (double)y));
    float s, c;
    sincosf_(theta, &s, &c);
    return make_float2(rr * s, rr * c);
}

// svpmflow_state_init (:48-56)
__device__ __forceinline__ float2 state_init(Rng& g, float flowmax)
{
    const float2 b = box_mueller(g);
    return make_float2(b.x * flowmax * 0.5f, b.y * flowmax * 0.5f);
}

// svpmflow_state_refine (:58-64): its `ret` is read before it is written; taken as zero (the
// value-initialised vector of the reference kernels' host build)
__device__ __forceinline__ float2 state_refine(Rng& g, float refinemax)
{
    const float2 b = box_mueller(g);
    return make_float2(0.0f + b.x * refinemax * 0.5f, 0.0f + b.y * refinemax * 0.5f);
}

// RNG_init(&rng, linpos, k): skip distance (linpos) * k as an int (RNG.cl:54-57)
__device__ __forceinline__ int skip(int linpos, int k) { return (int)((uint32_t)linpos * (uint32_t)k); }

// the colour planes of a frame: k / 255 per channel
__global__ void k_colour(const uint8_t* __restrict__ img, size_t stride, int W, int H, float4* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const uchar4 p = __ldg(reinterpret_cast<const uchar4*>(img + (size_t)y * stride) + x);
    out[(size_t)y * W + x] = f4(unorm8(p.x), unorm8(p.y), unorm8(p.z), unorm8(p.w));
}

// svpmflow_init (:213-233)
__global__ void __launch_bounds__(G* G) k_init(float4* __restrict__ out, Frames F, float flowmax)
{
    const int x = blockIdx.x * G + threadIdx.x, y = blockIdx.y * G + threadIdx.y;
    if (x >= F.W || y >= F.H) return;
    Rng g;
    g.init_skip(skip(y * F.W + x, 2));
    const float2 s = state_init(g, flowmax);
    unsigned long long n = 0;
    out[(size_t)y * F.W + x] = f4(s.x, s.y, eval<false>(F, x, y, s.x, s.y, n), 0.0f);
}

// svpmflow_prop_local_tv_admm (:574-731), one CTA per 16x16 work-group.  counts (COUNT):
// cost-window taps.  Three resident CTAs per SM (80 registers, no spills): 14% faster than
// four at 64 registers with spills, the compiler's choice without a minimum.
template <bool COUNT>
__global__ void __launch_bounds__(G* G, 3) k_prop(float4* __restrict__ out, float4* __restrict__ pout,
                                               const float4* __restrict__ in, const float4* __restrict__ pin, Frames F,
                                               float flowmax, int iter, unsigned long long* counts)
{
    __shared__ float4 buf[BUF][BUF];
    __shared__ float4 bufp[PB][PB];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = blockIdx.x * G + tx, y = blockIdx.y * G + ty;
    const int W = F.W, H = F.H;
    const float tau = 0.1f, lambda0 = 0.01f;
    unsigned long long taps = 0;

    // the group's states and apron, edge-clamped (SAMPLER_NN, :590-594)
    const int bx = blockIdx.x * G - OFF, by = blockIdx.y * G - OFF;
    for (int yy = ty; yy < BUF; yy += G)
        for (int xx = tx; xx < BUF; xx += G) {
            const int sx = min(max(bx + xx, 0), W - 1), sy = min(max(by + yy, 0), H - 1);
            buf[yy][xx] = __ldg(in + (size_t)sy * W + sx);
        }
    __syncthreads();
    // one primal-dual step of the dual field over the group and a 1-pixel apron (:598-613);
    // p outside the image reads as zero (SAMPLER_NN_ZERO)
    const int bpx = blockIdx.x * G - 1, bpy = blockIdx.y * G - 1;
    for (int yy = ty; yy < PB; yy += G)
        for (int xx = tx; xx < PB; xx += G) {
            const int sx = bpx + xx, sy = bpy + yy;
            const float4 p = (sx >= 0 && sx < W && sy >= 0 && sy < H) ? __ldg(pin + (size_t)sy * W + sx) : f4(0, 0, 0, 0);
            const float4 A = buf[yy + OFF - 1][xx + OFF - 1], Bx = buf[yy + OFF - 1][xx + OFF], By = buf[yy + OFF][xx + OFF - 1];
            const float dxx = Bx.x - A.x, dxy = Bx.y - A.y, dyx = By.x - A.x, dyy = By.y - A.y;
            const float4 z = f4(p.x + dxx, p.y + dxy, p.z + dyx, p.w + dyy);
            const float zx = fmaxf(0.0f, 1.0f - tau / fmaxf(sqrtf(z.x * z.x + z.y * z.y), 1e-10f));
            const float zy = fmaxf(0.0f, 1.0f - tau / fmaxf(sqrtf(z.z * z.z + z.w * z.w), 1e-10f));
            const float4 pn = f4((p.x + dxx) - z.x * zx, (p.y + dxy) - z.y * zx, (p.z + dyx) - z.z * zy,
                                 (p.w + dyy) - z.w * zy);
            bufp[yy][xx] = f4(pn.x + 0.5f * (pn.x - p.x), pn.y + 0.5f * (pn.y - p.y), pn.z + 0.5f * (pn.z - p.z),
                              pn.w + 0.5f * (pn.w - p.w));
        }
    __syncthreads();

    // the pull towards the smoothed flow (:616-623)
    const float4 p = iter < 5 ? f4(0, 0, 0, 0) : bufp[ty + 1][tx + 1];
    const float4 Lp = bufp[ty + 1][tx], Up = bufp[ty][tx + 1];
    const float divx = ((p.x - Lp.x) + p.z) - Up.z, divy = ((p.y - Lp.y) + p.w) - Up.w;
    float4 ret = buf[ty + OFF][tx + OFF];
    const float curx = ret.x + (lambda0 / tau) * divx, cury = ret.y + (lambda0 / tau) * divy;
    const float lam = iter < 5 ? 0.0f : 1.0f / (2.0f * lambda0 * 5.0f);
    auto test = [&](float nx, float ny, float cost) {
        const float an = nx - curx, bn = ny - cury, ar = ret.x - curx, br = ret.y - cury;
        if (cost + lam * (an * an + bn * bn) < ret.z + lam * (ar * ar + br * br)) {
            ret.x = nx;
            ret.y = ny;
            ret.z = cost;
        }
    };
    Rng g;
    g.init_skip(skip(y * W + x, 2 * 2 * iter));
    test(curx, cury, eval<COUNT>(F, x, y, curx, cury, taps));
#pragma unroll 1
    for (int k = 0; k < 2; k++) {   // random tries (:637-645)
        const float2 n = state_init(g, flowmax);
        test(n.x, n.y, eval<COUNT>(F, x, y, n.x, n.y, taps));
    }
#pragma unroll 1
    for (int k = 0; k < 2; k++) {   // random neighbours within 5 px (:648-656)
        const float rx = g.next();
        const int ox = (int)((rx - 0.5f) * 2.0f * 5.0f + 0.5f);
        const float ry = g.next();
        const int oy = (int)((ry - 0.5f) * 2.0f * 5.0f + 0.5f);
        const float4 n = __ldg(in + (size_t)min(max(y + oy, 0), H - 1) * W + min(max(x + ox, 0), W - 1));
        test(n.x, n.y, eval<COUNT>(F, x, y, n.x, n.y, taps));
    }
    buf[ty + OFF][tx + OFF] = ret;
    __syncthreads();
    // jump steps 4, 2, 1 in the directions +x, +y, -x, -y (:668-694)
#pragma unroll 1
    for (int step = 4; step >= 1; step >>= 1) {
#pragma unroll 1
        for (int d = 0; d < 4; d++) {
            const int dx = d == 0 ? step : (d == 2 ? -step : 0), dy = d == 1 ? step : (d == 3 ? -step : 0);
            const float4 n = buf[(ty + OFF + dy) % BUF][(tx + OFF + dx) % BUF];
            __syncthreads();
            test(n.x, n.y, eval<COUNT>(F, x, y, n.x, n.y, taps));
            buf[ty + OFF][tx + OFF] = ret;
            __syncthreads();
        }
    }
#pragma unroll 1
    for (int k = 0; k < 2; k++) {   // random refinement (:700-708)
        const float2 n = state_refine(g, 1.0f);
        test(n.x, n.y, eval<COUNT>(F, x, y, n.x, n.y, taps));
    }
    if (x < W && y < H) {
        pout[(size_t)y * W + x] = p;
        out[(size_t)y * W + x] = ret;
    }
    if (COUNT) atomicAdd(counts, taps);
}

// svpmflow_flow (:733-744): (u, v) per pixel
__global__ void k_to_flow(float2* __restrict__ flow, const float4* __restrict__ states, int W, int H)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const float4 s = __ldg(states + (size_t)y * W + x);
    flow[(size_t)y * W + x] = make_float2(s.x, s.y);
}

inline dim3 row_grid(int W, int H) { return dim3((W + 127) / 128, H); }
inline dim3 group_grid(int W, int H) { return dim3((W + G - 1) / G, (H + G - 1) / G); }

void launch_colour(const uint8_t* img, size_t stride, int W, int H, float4* out, cudaStream_t st)
{
    k_colour<<<row_grid(W, H), 128, 0, st>>>(img, stride, W, H, out);
}

void launch_init(float4* out, const Frames& F, float flowmax, cudaStream_t st)
{
    k_init<<<group_grid(F.W, F.H), dim3(G, G), 0, st>>>(out, F, flowmax);
}

void launch_prop(float4* out, float4* pout, const float4* in, const float4* pin, const Frames& F, float flowmax, int iter,
                 unsigned long long* counts, cudaStream_t st)
{
    if (counts) k_prop<true><<<group_grid(F.W, F.H), dim3(G, G), 0, st>>>(out, pout, in, pin, F, flowmax, iter, counts);
    else k_prop<false><<<group_grid(F.W, F.H), dim3(G, G), 0, st>>>(out, pout, in, pin, F, flowmax, iter, nullptr);
}

void launch_to_flow(float2* flow, const float4* states, int W, int H, cudaStream_t st)
{
    k_to_flow<<<row_grid(W, H), 128, 0, st>>>(flow, states, W, H);
}

}  // namespace svpm
}  // namespace pm

using namespace pm;
using namespace pm::svpm;

// An SVPMFlowCL object: a device workspace for one image size.
struct pm_svpm {
    int device = 0;
    std::string err;
    int counting = 0;
    unsigned long long counts[1] = {0};
    void* ws = nullptr;
    size_t ws_bytes = 0;
};

namespace {

thread_local std::string t_svpm_err;

int sfail(pm_svpm* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    t_svpm_err = msg;
    return code;
}

#define SVPM_CUDA(h, call)                                                                         \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return sfail((h), PM_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
inline bool aligned(const void* p, size_t n) { return ((uintptr_t)p % n) == 0; }
inline size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

// workspace: both colour planes, two state and two dual fields, then (host entry) both frames,
// the flow, counters
struct SLayout {
    enum { c1, c2, s0, s1, p0, p1, img0, img1, flow, ctr, COUNT };
    size_t off[COUNT + 1];
    size_t total() const { return off[COUNT]; }
};

SLayout slayout(int W, int H, size_t stride)
{
    const size_t N = (size_t)W * H;
    const size_t sz[SLayout::COUNT] = {16 * N, 16 * N, 16 * N, 16 * N, 16 * N, 16 * N, stride * H, stride * H, 8 * N, 16};
    SLayout L;
    size_t o = 0;
    for (int k = 0; k < SLayout::COUNT; k++) {
        L.off[k] = o;
        o += up256(sz[k]);
    }
    L.off[SLayout::COUNT] = o;
    return L;
}

template <class T> T* sat(void* base, const SLayout& L, int k) { return reinterpret_cast<T*>(static_cast<char*>(base) + L.off[k]); }

int check_common(pm_svpm* h, int W, int H, size_t stride, int r, float flowmax)
{
    if (W <= 0 || H <= 0 || W > PM_MAX_WIDTH || H > PM_MAX_HEIGHT) return sfail(h, PM_EINVAL_SHAPE, "image size out of range");
    if (r < 0 || r > PM_MAX_RADIUS) return sfail(h, PM_EINVAL_SHAPE, "patch size out of range");
    if (stride < (size_t)W * 4 || stride % 4) return sfail(h, PM_EINVAL_SHAPE, "row stride must be >= 4*width and a multiple of 4");
    if (!(flowmax >= 0.0f) || !isfinite(flowmax)) return sfail(h, PM_EINVAL_ARG, "flow range must be finite and >= 0");
    return PM_OK;
}

int ensure_sws(pm_svpm* h, int W, int H, size_t stride)
{
    const size_t need = slayout(W, H, stride).total();
    if (h->ws && h->ws_bytes >= need) return PM_OK;
    if (h->ws) {
        SVPM_CUDA(h, cudaDeviceSynchronize());
        cudaFree(h->ws);
        h->ws = nullptr;
        h->ws_bytes = 0;
    }
    const cudaError_t e = cudaMalloc(&h->ws, need);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->ws = nullptr;
        return sfail(h, PM_ENOMEM, std::string("workspace allocation failed: ") + cudaGetErrorString(e));
    }
    h->ws_bytes = need;
    return PM_OK;
}

// SVPMFlowCL::flow on device buffers: colour planes, init, `iterations` passes, (u, v); the
// final state and dual fields stay in the workspace at the returned index
int run_flow(pm_svpm* h, const uint8_t* img0, const uint8_t* img1, int W, int H, size_t stride, int r, float flowmax,
             int iterations, float* flow, float4* states, float4* duals, cudaStream_t st)
{
    const SLayout L = slayout(W, H, stride);
    float4* c1 = sat<float4>(h->ws, L, SLayout::c1);
    float4* c2 = sat<float4>(h->ws, L, SLayout::c2);
    float4* s[2] = {sat<float4>(h->ws, L, SLayout::s0), sat<float4>(h->ws, L, SLayout::s1)};
    float4* p[2] = {sat<float4>(h->ws, L, SLayout::p0), sat<float4>(h->ws, L, SLayout::p1)};
    unsigned long long* ctr = sat<unsigned long long>(h->ws, L, SLayout::ctr);
    const size_t N = (size_t)W * H;
    launch_colour(img0, stride, W, H, c1, st);
    launch_colour(img1, stride, W, H, c2, st);
    const Frames F = {c1, c2, W, H, r};
    launch_init(s[1], F, flowmax, st);
    SVPM_CUDA(h, cudaMemsetAsync(p[1], 0, N * 16, st));   // clbufp2.fill(0) (SVPMFlowCL.cpp:68)
    if (h->counting) SVPM_CUDA(h, cudaMemsetAsync(ctr, 0, 8, st));
    for (int i = 0; i < iterations; i++) {
        const int swap = i & 1;
        launch_prop(s[swap], p[swap], s[1 - swap], p[1 - swap], F, flowmax, i + 1, h->counting ? ctr : nullptr, st);
    }
    const int last = 1 - (iterations & 1);
    launch_to_flow(reinterpret_cast<float2*>(flow), s[last], W, H, st);
    if (states) SVPM_CUDA(h, cudaMemcpyAsync(states, s[last], N * 16, cudaMemcpyDeviceToDevice, st));
    if (duals) SVPM_CUDA(h, cudaMemcpyAsync(duals, p[last], N * 16, cudaMemcpyDeviceToDevice, st));
    SVPM_CUDA(h, cudaGetLastError());
    if (h->counting) {
        SVPM_CUDA(h, cudaMemcpyAsync(h->counts, ctr, 8, cudaMemcpyDeviceToHost, st));
        SVPM_CUDA(h, cudaStreamSynchronize(st));
    }
    return PM_OK;
}

// the colour planes of both frames for the per-kernel entry points, in stream-ordered scratch
struct SvpmScratch {
    float4* p = nullptr;
    cudaStream_t st = nullptr;
    ~SvpmScratch()
    {
        if (p) cudaFreeAsync(p, st);
    }
    int make(const uint8_t* a, const uint8_t* b, int W, int H, size_t stride, int r, cudaStream_t s, Frames* F)
    {
        st = s;
        const size_t N = (size_t)W * H;
        SVPM_CUDA(nullptr, cudaMallocAsync((void**)&p, 2 * N * sizeof(float4), s));
        launch_colour(a, stride, W, H, p, s);
        launch_colour(b, stride, W, H, p + N, s);
        *F = Frames{p, p + N, W, H, r};
        return PM_OK;
    }
};

}  // namespace

extern "C" {

int pm_svpm_create(pm_svpm** out, int device)
{
    if (!out) return sfail(nullptr, PM_EINVAL_ARG, "null output pointer");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return sfail(nullptr, PM_ENODEV, "no CUDA device");
    }
    if (device < 0 || device >= n) return sfail(nullptr, PM_EINVAL_ARG, "device ordinal out of range");
    pm_svpm* h = new pm_svpm;
    h->device = device;
    *out = h;
    return PM_OK;
}

int pm_svpm_destroy(pm_svpm* h)
{
    if (!h) return PM_OK;
    if (h->ws) {
        cudaSetDevice(h->device);
        cudaDeviceSynchronize();
        cudaFree(h->ws);
    }
    delete h;
    return PM_OK;
}

const char* pm_svpm_last_error(const pm_svpm* h) { return h ? h->err.c_str() : t_svpm_err.c_str(); }

int pm_svpm_set_counting(pm_svpm* h, int on)
{
    if (!h) return sfail(nullptr, PM_EINVAL_ARG, "null handle");
    h->counting = on ? 1 : 0;
    return PM_OK;
}

int pm_svpm_get_counters(pm_svpm* h, uint64_t c[1])
{
    if (!h || !c) return sfail(h, PM_EINVAL_ARG, "null argument");
    c[0] = h->counts[0];
    return PM_OK;
}

int pm_svpm_flow_device(pm_svpm* h, const uint8_t* first, const uint8_t* second, int W, int H, size_t stride,
                        int patchsize, float flowmax, int iterations, float* flow, float* states, float* duals,
                        void* stream)
{
    if (!h) return sfail(nullptr, PM_EINVAL_ARG, "null handle");
    if (!first || !second || !flow) return sfail(h, PM_EINVAL_ARG, "null image");
    int rc = check_common(h, W, H, stride, patchsize, flowmax);
    if (rc) return rc;
    if (iterations < 0) return sfail(h, PM_EINVAL_ARG, "negative iteration count");
    if (!aligned(first, 4) || !aligned(second, 4) || !aligned(flow, 8) || !aligned(states, 16) || !aligned(duals, 16))
        return sfail(h, PM_EINVAL_ARG, "frames must be 4-byte aligned, flow 8-byte, states and duals 16-byte");
    SVPM_CUDA(h, cudaSetDevice(h->device));
    rc = ensure_sws(h, W, H, stride);
    if (rc) return rc;
    return run_flow(h, first, second, W, H, stride, patchsize, flowmax, iterations, flow,
                    reinterpret_cast<float4*>(states), reinterpret_cast<float4*>(duals), S(stream));
}

int pm_svpm_flow(pm_svpm* h, const uint8_t* first, const uint8_t* second, int W, int H, size_t stride, int patchsize,
                 float flowmax, int iterations, float* flow, float* states, float* duals)
{
    if (!h) return sfail(nullptr, PM_EINVAL_ARG, "null handle");
    if (!first || !second || !flow) return sfail(h, PM_EINVAL_ARG, "null image");
    int rc = check_common(h, W, H, stride, patchsize, flowmax);
    if (rc) return rc;
    if (iterations < 0) return sfail(h, PM_EINVAL_ARG, "negative iteration count");
    SVPM_CUDA(h, cudaSetDevice(h->device));
    rc = ensure_sws(h, W, H, stride);
    if (rc) return rc;
    const SLayout L = slayout(W, H, stride);
    const size_t N = (size_t)W * H;
    cudaStream_t st = 0;
    uint8_t* d0 = sat<uint8_t>(h->ws, L, SLayout::img0);
    uint8_t* d1 = sat<uint8_t>(h->ws, L, SLayout::img1);
    float* df = sat<float>(h->ws, L, SLayout::flow);
    SVPM_CUDA(h, cudaMemcpyAsync(d0, first, stride * H, cudaMemcpyHostToDevice, st));
    SVPM_CUDA(h, cudaMemcpyAsync(d1, second, stride * H, cudaMemcpyHostToDevice, st));
    rc = run_flow(h, d0, d1, W, H, stride, patchsize, flowmax, iterations, df, nullptr, nullptr, st);
    if (rc) return rc;
    SVPM_CUDA(h, cudaMemcpyAsync(flow, df, N * 8, cudaMemcpyDeviceToHost, st));
    const int last = 1 - (iterations & 1);
    if (states)
        SVPM_CUDA(h, cudaMemcpyAsync(states, sat<float4>(h->ws, L, last ? SLayout::s1 : SLayout::s0), N * 16,
                                     cudaMemcpyDeviceToHost, st));
    if (duals)
        SVPM_CUDA(h, cudaMemcpyAsync(duals, sat<float4>(h->ws, L, last ? SLayout::p1 : SLayout::p0), N * 16,
                                     cudaMemcpyDeviceToHost, st));
    SVPM_CUDA(h, cudaStreamSynchronize(st));
    return PM_OK;
}

// ---- one reference kernel per call, on device buffers and a stream ---------------------

int pm_k_svpm_init(float* out, const uint8_t* first, const uint8_t* second, int W, int H, size_t stride, int r,
                   float flowmax, void* stream)
{
    int rc = check_common(nullptr, W, H, stride, r, flowmax);
    if (rc) return rc;
    if (!out || !first || !second || !aligned(out, 16) || !aligned(first, 4) || !aligned(second, 4))
        return sfail(nullptr, PM_EINVAL_ARG, "bad buffer");
    SvpmScratch sc;
    Frames F;
    rc = sc.make(first, second, W, H, stride, r, S(stream), &F);
    if (rc) return rc;
    launch_init(reinterpret_cast<float4*>(out), F, flowmax, S(stream));
    SVPM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_svpm_prop(float* out, float* pout, const float* in, const float* pin, const uint8_t* first,
                   const uint8_t* second, int W, int H, size_t stride, int r, float flowmax, int iter, void* stream)
{
    int rc = check_common(nullptr, W, H, stride, r, flowmax);
    if (rc) return rc;
    if (iter < 0) return sfail(nullptr, PM_EINVAL_ARG, "negative pass index");
    if (!out || !pout || !in || !pin || !first || !second || !aligned(out, 16) || !aligned(pout, 16) ||
        !aligned(in, 16) || !aligned(pin, 16) || !aligned(first, 4) || !aligned(second, 4))
        return sfail(nullptr, PM_EINVAL_ARG, "bad buffer");
    SvpmScratch sc;
    Frames F;
    rc = sc.make(first, second, W, H, stride, r, S(stream), &F);
    if (rc) return rc;
    launch_prop(reinterpret_cast<float4*>(out), reinterpret_cast<float4*>(pout), reinterpret_cast<const float4*>(in),
                reinterpret_cast<const float4*>(pin), F, flowmax, iter, nullptr, S(stream));
    SVPM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_svpm_to_flow(float* flow, const float* states, int W, int H, void* stream)
{
    if (W <= 0 || H <= 0 || W > PM_MAX_WIDTH || H > PM_MAX_HEIGHT) return sfail(nullptr, PM_EINVAL_SHAPE, "image size out of range");
    if (!flow || !states || !aligned(flow, 8) || !aligned(states, 16)) return sfail(nullptr, PM_EINVAL_ARG, "bad buffer");
    launch_to_flow(reinterpret_cast<float2*>(flow), reinterpret_cast<const float4*>(states), W, H, S(stream));
    SVPM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

}  // extern "C"
