// CUDA kernels of the PatchMatch-Huber stereo path for sm_100a, and their
// launchers.  One thread handles one pixel; the window loops run in the
// reference's sample order so that every sum rounds exactly as the reference's
// does.  Compile with -fmad=false: the only fused operations are the explicit
// fmaf() of the hot sites (template parameter F).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>

#include "pm_device.cuh"
#include "pm_kernels.h"

namespace pm {

namespace {

__device__ __forceinline__ float u8f(uint8_t v) { return (float)v / 255.0f; }

// RGBA8 texel as read by read_imagef on CL_UNORM_INT8 (value / 255)
__device__ __forceinline__ float4 rgba_at(const uint8_t* __restrict__ img, size_t stride, int x, int y)
{
    const uchar4 c = __ldg(reinterpret_cast<const uchar4*>(img + (size_t)y * stride) + x);
    return f4(u8f(c.x), u8f(c.y), u8f(c.z), u8f(c.w));
}

// grey value dot(rgba, (0.2126, 0.7152, 0.0722, 0)) with CLK_ADDRESS_CLAMP's zero border
// (pmhstereo.cl:1569-1573, PDDiffTensor.cl:41-45)
__device__ __forceinline__ float gray_zero(const uint8_t* __restrict__ img, size_t stride, int W, int H, int x, int y)
{
    if (x < 0 || x >= W || y < 0 || y >= H) return 0.0f;
    const float4 v = rgba_at(img, stride, x, y);
    return v.x * PM_GW_R + v.y * PM_GW_G + v.z * PM_GW_B + v.w * 0.0f;
}

// raw: bw receives the image itself (r, g, b, a), as depthMap hands it to its kernels
// (PMHuberStereo.cpp:203-204), instead of colour and window weight sum; alpha: the diffusion
// tensor's edge weight (24 in disparityMapAll, :416; 12 in depthMap, :152)
template <bool F>
__global__ void k_prep(const uint8_t* __restrict__ img, size_t stride, int W, int H, int r, float4* __restrict__ bw,
                       float4* __restrict__ grad, float4* __restrict__ dt, float alpha, int raw)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * W + x;
    if (bw && raw) {
        bw[i] = rgba_at(img, stride, x, y);
    } else if (bw) {
        // pmhstereo_bilateral_weight_to_alpha (pmhstereo.cl:1462-1498)
        const float4 c = rgba_at(img, stride, x, y);
        float wsum = 0.0f;
        for (int dy = max(-r, -y); dy <= min(r, H - 1 - y); dy++)
            for (int dx = max(-r, -x); dx <= min(r, W - 1 - x); dx++) {
                const float4 v = rgba_at(img, stride, x + dx, y + dy);
                wsum += support_weight<F>(v.x - c.x, v.y - c.y, v.z - c.z);
            }
        bw[i] = f4(c.x, c.y, c.z, wsum);
    }
    const float g = gray_zero(img, stride, W, H, x, y);
    const float gxp = gray_zero(img, stride, W, H, x + 1, y), gyp = gray_zero(img, stride, W, H, x, y + 1);
    if (grad) {
        // pmhstereo_gradxy (:1584-1601)
        const float gxm = gray_zero(img, stride, W, H, x - 1, y), gym = gray_zero(img, stride, W, H, x, y - 1);
        grad[i] = f4(gxp - g, gyp - g, gxp - gxm, gyp - gym);
    }
    if (dt) {
        // PDDiffTensorColor (PDDiffTensor.cl:52-72), beta 1 (PMHuberStereo.cpp:417, :153)
        float dx = gxp - g, dy = gyp - g;
        const float len = sqrtf(dx * dx + dy * dy);
        const float w = expf_(-alpha * len);
        float4 d;
        if (len <= 0.001f) {
            d = f4(1.0f, 0.0f, 0.0f, 1.0f);
        } else {
            dx = dx / len;
            dy = dy / len;
            const float dxo = dy, dyo = -dx;
            d = f4(w * dx * dx + dxo * dxo, w * dx * dy + dxo * dyo, w * dy * dx + dyo * dxo, w * dy * dy + dyo * dyo);
        }
        dt[i] = d;
    }
}

template <bool F, bool CHK>
__global__ void k_init(float4* __restrict__ out, ViewData V, float dmax, int lr, const float* __restrict__ initdisp,
                       const float4* __restrict__ initnormal, int dual)
{
    if (variant_skips<CHK>(V, dual)) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= V.W || y >= V.H) return;
    const size_t i = (size_t)y * V.W + x;
    const float cx = (float)x, cy = (float)y;
    Rng rng;
    rng.init_skip((y * V.W + x) * 3);   // RNG_init(&rng, lin, 3), pmhstereo.cl:766
    float4 ret;
    const float disparity = initdisp ? initdisp[i] : 0.0f;
    if (initdisp && disparity > 0 && lr) {
        const float4 n = initnormal[i];
        ret = from_disparity_normal(cx, cy, disparity, normalize3(make_float3(n.x, n.y, n.z)));
    } else if (initdisp && disparity > 0 && !lr) {
        const float4 n = initnormal[i];
        ret = from_disparity_normal(cx, cy, -disparity, normalize3(make_float3(n.x, n.y, n.z)));
    } else {
        ret = nd_state_init(rng, cx, cy, lr, dmax);
    }
    Counters cnt = {0, 0, 0, 0};
    ret.w = patch_eval<F, false, CHK>(V, x, y, ret, 1e10f, cnt);
    out[i] = ret;
}

template <bool F, bool CHK>
__global__ void k_cost(float* __restrict__ cost, const float4* __restrict__ planes, ViewData V, float mincost,
                       int dual)
{
    if (variant_skips<CHK>(V, dual)) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= V.W || y >= V.H) return;
    const size_t i = (size_t)y * V.W + x;
    Counters cnt = {0, 0, 0, 0};
    cost[i] = patch_eval<F, false, CHK>(V, x, y, planes[i], mincost, cnt);
}

template <bool F, bool CHK>
__global__ void k_klt(float4* __restrict__ out, const float4* __restrict__ planes, ViewData V, int dual)
{
    if (variant_skips<CHK>(V, dual)) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= V.W || y >= V.H) return;
    const size_t i = (size_t)y * V.W + x;
    Counters cnt = {0, 0, 0, 0};
    out[i] = klt2<F, false, CHK>(V, x, y, planes[i], cnt);
}

__device__ __forceinline__ void normal_depth_px(float4* __restrict__ out, const float4* __restrict__ planes, int W,
                                                int H, float dispscale, int lr, int x, int y)
{
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * W + x;
    float4 v = to_ref_normal_depth(planes[i], (float)x, (float)y, lr);   // pmhstereo.cl:1397-1399
    v.w = v.w * dispscale;
    out[i] = v;
}

__global__ void k_normal_depth(float4* __restrict__ out, const float4* __restrict__ planes, int W, int H,
                               float dispscale, int lr)
{
    normal_depth_px(out, planes, W, H, dispscale, lr, blockIdx.x * blockDim.x + threadIdx.x,
                    blockIdx.y * blockDim.y + threadIdx.y);
}

// tensor-weighted, projected dual of PDDROFDiffTensor (PDDROFDiffTensor.cl:72-100) from the
// primal at the pixel (uc), right of it (ux) and below it (uy), the tensor D and the previous dual
struct Dual { float4 lo, hi; };
template <bool HUBER>
__device__ __forceinline__ Dual dual_step(float4 uc, float4 ux, float4 uy, float4 D, float4 plo, float4 phi, float eps)
{
    const float dxv[4] = {uc.x - ux.x, uc.y - ux.y, uc.z - ux.z, uc.w - ux.w};
    const float dyv[4] = {uc.x - uy.x, uc.y - uy.y, uc.z - uy.z, uc.w - uy.w};
    const float pl[4] = {plo.x, plo.y, plo.z, plo.w}, ph[4] = {phi.x, phi.y, phi.z, phi.w};
    float a[4], b[4], nrm[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float DTdx = D.x * dxv[c] + D.z * dyv[c];
        const float DTdy = D.y * dxv[c] + D.w * dyv[c];
        a[c] = pl[c] + 4.0f * DTdx;   // SIGMA
        b[c] = ph[c] + 4.0f * DTdy;
        if (HUBER) {   // PDDHuberDiffTensor.cl:61-63
            a[c] = a[c] / (1.0f + 4.0f * eps);
            b[c] = b[c] / (1.0f + 4.0f * eps);
        }
        nrm[c] = a[c] * a[c] + b[c] * b[c];
    }
    float pr[4];
    if (HUBER) {   // one norm over the four channels (PDDHuberDiffTensor.cl:66-67)
        const float n = sqrtf(nrm[0] * 1.0f + nrm[1] * 1.0f + nrm[2] * 1.0f + nrm[3] * 1.0f);
        pr[0] = pr[1] = pr[2] = pr[3] = fmaxf(1.0f, n);
    } else {
        const float n3 = sqrtf(nrm[0] * 1.0f + nrm[1] * 1.0f + nrm[2] * 1.0f);
        const float n4 = sqrtf(nrm[3]);
        pr[0] = pr[1] = pr[2] = fmaxf(1.0f, n3);
        pr[3] = fmaxf(1.0f, n4);
    }
    float l[4], h[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (pr[c] != 1.0f) {   // x / 1 is x: inside the unit ball the projection divides by 1
            a[c] = a[c] / pr[c];
            b[c] = b[c] / pr[c];
        }
        l[c] = D.x * a[c] + D.z * b[c];
        h[c] = D.y * a[c] + D.w * b[c];
    }
    Dual d;
    d.lo = f4(l[0], l[1], l[2], l[3]);
    d.hi = f4(h[0], h[1], h[2], h[3]);
    return d;
}

// the dual at pixel (x, y) from global fields; the primal is read clamped to the image,
// outside it the tensor and the previous dual read as 0
template <bool HUBER>
__device__ __forceinline__ Dual rof_dual(const float4* __restrict__ u, const float4* __restrict__ p,
                                         const float4* __restrict__ dt, int W, int H, int x, int y, bool first,
                                         float eps)
{
    const int xc = min(max(x, 0), W - 1), yc = min(max(y, 0), H - 1);
    const int xp = min(max(x + 1, 0), W - 1), yp = min(max(y + 1, 0), H - 1);
    const float4 uc = u[(size_t)yc * W + xc], ux = u[(size_t)yc * W + xp], uy = u[(size_t)yp * W + xc];
    const bool inside = x >= 0 && x < W && y >= 0 && y < H;
    const float4 D = inside ? dt[(size_t)y * W + x] : f4(0, 0, 0, 0);
    float4 plo = f4(0, 0, 0, 0), phi = f4(0, 0, 0, 0);
    if (inside && !first) { plo = p[(size_t)y * 2 * W + 2 * x]; phi = p[(size_t)y * 2 * W + 2 * x + 1]; }
    return dual_step<HUBER>(uc, ux, uy, D, plo, phi, eps);
}

// the primal and q updates of one step (PDDROFDiffTensor.cl:102-126) from the divergence of
// the duals at the pixel (c), left of it (l) and above it (t)
__device__ __forceinline__ void primal_step(float4 uu, float4 qq, float4 im, const Dual& c, const Dual& l,
                                            const Dual& t, float4 lam, float4& uout, float4& qout)
{
    const float div[4] = {c.lo.x - l.lo.x + c.hi.x - t.hi.x, c.lo.y - l.lo.y + c.hi.y - t.hi.y,
                          c.lo.z - l.lo.z + c.hi.z - t.hi.z, c.lo.w - l.lo.w + c.hi.w - t.hi.w};
    const float imv[4] = {im.x, im.y, im.z, im.w}, qv[4] = {qq.x, qq.y, qq.z, qq.w}, uv[4] = {uu.x, uu.y, uu.z, uu.w};
    const float lm[4] = {lam.x, lam.y, lam.z, lam.w};
    float on[4], qn[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float o = (uv[k] + 0.05f * (lm[k] * imv[k] - div[k] - qv[k])) / (1.0f + 0.05f * lm[k]);   // TAU
        o = o + 0.5f * (o - uv[k]);                                                               // THETA
        float qn_ = (qv[k] + 8.0f * (o - imv[k])) / (1.0f + 4.0f * 8.0f / lm[k]);                 // ETA
        qn_ = qn_ + 0.5f * (qn_ - qv[k]);
        on[k] = o;
        qn[k] = qn_;
    }
    uout = f4(on[0], on[1], on[2], on[3]);
    qout = f4(qn[0], qn[1], qn[2], qn[3]);
}

constexpr int ROF_BX = 32, ROF_BY = 8;   // k_rof_step block; its duals need a one-pixel apron left and above

// one primal-dual step (PDDROFDiffTensor.cl:102-126; with HUBER PDDHuberDiffTensor.cl:92-106);
// first: p = q = 0.  The divergence at (x, y) needs the duals at (x, y), (x - 1, y) and
// (x, y - 1): the block computes the duals of its tile and of the column left of it and the
// row above it once each, in shared memory, instead of three times per pixel.
template <bool HUBER>
__device__ __forceinline__ void rof_step_tile(float4* __restrict__ unew, float4* __restrict__ pnew,
                                              float4* __restrict__ qnew, const float4* __restrict__ u,
                                              const float4* __restrict__ p, const float4* __restrict__ q,
                                              const float4* __restrict__ img, const float4* __restrict__ dt,
                                              float4 lam, int W, int H, int first, float eps, int x0, int y0)
{
    __shared__ Dual sd[ROF_BY + 1][ROF_BX + 1];
    const int tid = threadIdx.y * ROF_BX + threadIdx.x;
    for (int i = tid; i < (ROF_BX + 1) * (ROF_BY + 1); i += ROF_BX * ROF_BY) {
        const int ex = i % (ROF_BX + 1), ey = i / (ROF_BX + 1);
        sd[ey][ex] = rof_dual<HUBER>(u, p, dt, W, H, x0 - 1 + ex, y0 - 1 + ey, first, eps);
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= W || y >= H) return;
    const Dual c = sd[threadIdx.y + 1][threadIdx.x + 1];
    const Dual l = sd[threadIdx.y + 1][threadIdx.x];
    const Dual t = sd[threadIdx.y][threadIdx.x + 1];
    const size_t i = (size_t)y * W + x;
    float4 un, qn;
    primal_step(u[i], first ? f4(0, 0, 0, 0) : q[i], img[i], c, l, t, lam, un, qn);
    unew[i] = un;
    qnew[i] = qn;
    pnew[(size_t)y * 2 * W + 2 * x] = c.lo;
    pnew[(size_t)y * 2 * W + 2 * x + 1] = c.hi;
}

template <bool HUBER>
__global__ void __launch_bounds__(ROF_BX* ROF_BY) k_rof_step(float4* __restrict__ unew, float4* __restrict__ pnew,
                                                           float4* __restrict__ qnew, const float4* __restrict__ u,
                                                           const float4* __restrict__ p, const float4* __restrict__ q,
                                                           const float4* __restrict__ img,
                                                           const float4* __restrict__ dt, float4 lam, int W, int H,
                                                           int first, float eps)
{
    rof_step_tile<HUBER>(unew, pnew, qnew, u, p, q, img, dt, lam, W, H, first, eps, blockIdx.x * ROF_BX,
                         blockIdx.y * ROF_BY);
}

constexpr int RF_BX = 32, RF_BY = 16, RF_NT = 256;   // k_rof_step2: output tile and threads

// two primal-dual steps in one launch (temporal blocking): the block computes the first
// step's duals over its tile grown by two columns/rows left and above and one right and
// below, the first step's primal over the tile grown by one on every side, and from those
// the second step on its tile.  The fields cross DRAM once per two steps instead of twice;
// every value is formed by the same operations as in k_rof_step, so the result is the same
// bit for bit.  first: p = q = 0 before the first of the two steps.
template <bool HUBER>
__device__ __forceinline__ void rof_step2_tile(float4* __restrict__ unew, float4* __restrict__ pnew,
                                               float4* __restrict__ qnew, const float4* __restrict__ u,
                                               const float4* __restrict__ p, const float4* __restrict__ q,
                                               const float4* __restrict__ img, const float4* __restrict__ dt,
                                               float4 lam, int W, int H, int first, float eps, int x0, int y0)
{
    // duals: first step over x0-2 .. x0+BX, y0-2 .. y0+BY; the second step overwrites the
    // points x0-1 .. x0+BX-1, y0-1 .. y0+BY-1 in place (each point reads only its own first-step dual)
    __shared__ float4 sdl[RF_BY + 3][RF_BX + 3], sdh[RF_BY + 3][RF_BX + 3];
    __shared__ float4 su[RF_BY + 2][RF_BX + 2];   // first-step primal over x0-1 .. x0+BX, y0-1 .. y0+BY (in-image points)
    __shared__ float4 sq[RF_BY][RF_BX];           // first-step q over the tile
    const int tid = threadIdx.x;
    for (int i = tid; i < (RF_BX + 3) * (RF_BY + 3); i += RF_NT) {
        const int ex = i % (RF_BX + 3), ey = i / (RF_BX + 3);
        const Dual d = rof_dual<HUBER>(u, p, dt, W, H, x0 - 2 + ex, y0 - 2 + ey, first, eps);
        sdl[ey][ex] = d.lo;
        sdh[ey][ex] = d.hi;
    }
    __syncthreads();
    for (int i = tid; i < (RF_BX + 2) * (RF_BY + 2); i += RF_NT) {
        const int ex = i % (RF_BX + 2), ey = i / (RF_BX + 2);
        const int x = x0 - 1 + ex, y = y0 - 1 + ey;
        if (x < 0 || x >= W || y < 0 || y >= H) continue;
        const Dual c = {sdl[ey + 1][ex + 1], sdh[ey + 1][ex + 1]};
        const Dual l = {sdl[ey + 1][ex], sdh[ey + 1][ex]};
        const Dual t = {sdl[ey][ex + 1], sdh[ey][ex + 1]};
        const size_t gi = (size_t)y * W + x;
        float4 un, qn;
        primal_step(u[gi], first ? f4(0, 0, 0, 0) : q[gi], img[gi], c, l, t, lam, un, qn);
        su[ey][ex] = un;
        if (ex >= 1 && ex <= RF_BX && ey >= 1 && ey <= RF_BY) sq[ey - 1][ex - 1] = qn;
    }
    __syncthreads();
    // second-step duals; the clamped neighbours of a point of this range lie inside the image
    // and inside su's range
    for (int i = tid; i < (RF_BX + 1) * (RF_BY + 1); i += RF_NT) {
        const int ex = i % (RF_BX + 1), ey = i / (RF_BX + 1);
        const int x = x0 - 1 + ex, y = y0 - 1 + ey;
        const int xc = min(max(x, 0), W - 1) - (x0 - 1), yc = min(max(y, 0), H - 1) - (y0 - 1);
        const int xp = min(max(x + 1, 0), W - 1) - (x0 - 1), yp = min(max(y + 1, 0), H - 1) - (y0 - 1);
        const bool inside = x >= 0 && x < W && y >= 0 && y < H;
        const float4 D = inside ? dt[(size_t)y * W + x] : f4(0, 0, 0, 0);
        const float4 plo = inside ? sdl[ey + 1][ex + 1] : f4(0, 0, 0, 0);
        const float4 phi = inside ? sdh[ey + 1][ex + 1] : f4(0, 0, 0, 0);
        const Dual d = dual_step<HUBER>(su[yc][xc], su[yc][xp], su[yp][xc], D, plo, phi, eps);
        sdl[ey + 1][ex + 1] = d.lo;
        sdh[ey + 1][ex + 1] = d.hi;
    }
    __syncthreads();
    for (int i = tid; i < RF_BX * RF_BY; i += RF_NT) {
        const int ex = i % RF_BX, ey = i / RF_BX;
        const int x = x0 + ex, y = y0 + ey;
        if (x >= W || y >= H) continue;
        const Dual c = {sdl[ey + 2][ex + 2], sdh[ey + 2][ex + 2]};
        const Dual l = {sdl[ey + 2][ex + 1], sdh[ey + 2][ex + 1]};
        const Dual t = {sdl[ey + 1][ex + 2], sdh[ey + 1][ex + 2]};
        const size_t gi = (size_t)y * W + x;
        float4 un, qn;
        primal_step(su[ey + 1][ex + 1], sq[ey][ex], img[gi], c, l, t, lam, un, qn);
        unew[gi] = un;
        qnew[gi] = qn;
        pnew[(size_t)y * 2 * W + 2 * x] = c.lo;
        pnew[(size_t)y * 2 * W + 2 * x + 1] = c.hi;
    }
}

template <bool HUBER>
__global__ void __launch_bounds__(RF_NT) k_rof_step2(float4* __restrict__ unew, float4* __restrict__ pnew,
                                                   float4* __restrict__ qnew, const float4* __restrict__ u,
                                                   const float4* __restrict__ p, const float4* __restrict__ q,
                                                   const float4* __restrict__ img, const float4* __restrict__ dt,
                                                   float4 lam, int W, int H, int first, float eps)
{
    rof_step2_tile<HUBER>(unew, pnew, qnew, u, p, q, img, dt, lam, W, H, first, eps, blockIdx.x * RF_BX,
                          blockIdx.y * RF_BY);
}

static_assert(RF_BX == SMOOTH_TW && RF_BY == SMOOTH_TH16 && ROF_BX == SMOOTH_TW && ROF_BY == SMOOTH_TH8,
              "smoothing job tiles");

// the buffers of launch j of `launches` of a primal-dual run (launch_pd's schedule)
struct PdStep {
    float4 *unew, *pnew, *qnew;
    const float4 *u, *p, *q;
};
__device__ __forceinline__ PdStep pd_step(const SmoothArgs& A, int j, int launches)
{
    const size_t N = (size_t)A.W * A.H;
    float4* ut = A.scratch;
    float4* pp[2] = {ut + N, ut + 3 * N};
    float4* qq[2] = {ut + 5 * N, ut + 6 * N};
    const int pi = j & 1;
    PdStep s;
    s.unew = ((launches - 1 - j) % 2 == 0) ? A.out : ut;
    // the previous launch wrote `out` exactly when this one writes the scratch
    s.u = j == 0 ? A.tmp : (((launches - j) % 2 == 0) ? A.out : ut);
    s.pnew = pp[pi];
    s.qnew = qq[pi];
    s.p = pp[1 - pi];
    s.q = qq[1 - pi];
    return s;
}

// batched smoothing stage (launch_smooth_batch): persistent CTAs over the tiles of all pairs
__global__ void __launch_bounds__(ROF_BX* ROF_BY) k_normal_depth_b(const SmoothArgs* __restrict__ tab, int sel,
                                                                 const uint2* __restrict__ jobs, int njobs,
                                                                 int* next)
{
    for (;;) {
        const int j = grab_job(next);
        if (j >= njobs) return;
        const uint2 job = jobs[j];
        const SmoothArgs& A = tab[job.x];
        normal_depth_px(A.tmp, A.planes[sel], A.W, A.H, A.dispscale, A.lr,
                        (int)(job.y & 0xffffu) * ROF_BX + threadIdx.x, (int)(job.y >> 16) * ROF_BY + threadIdx.y);
    }
}

__global__ void __launch_bounds__(ROF_BX* ROF_BY) k_rof_step_b(const SmoothArgs* __restrict__ tab, float4 lam,
                                                             int launch, int launches,
                                                             const uint2* __restrict__ jobs, int njobs, int* next)
{
    for (;;) {
        const int j = grab_job(next);
        if (j >= njobs) return;
        const uint2 job = jobs[j];
        const SmoothArgs& A = tab[job.x];
        const PdStep s = pd_step(A, launch, launches);
        rof_step_tile<false>(s.unew, s.pnew, s.qnew, s.u, s.p, s.q, A.tmp, A.dt, lam, A.W, A.H, launch == 0, 0.0f,
                             (int)(job.y & 0xffffu) * ROF_BX, (int)(job.y >> 16) * ROF_BY);
    }
}

__global__ void __launch_bounds__(RF_NT) k_rof_step2_b(const SmoothArgs* __restrict__ tab, float4 lam, int launch,
                                                     int launches, const uint2* __restrict__ jobs, int njobs,
                                                     int* next)
{
    for (;;) {
        const int j = grab_job(next);
        if (j >= njobs) return;
        const uint2 job = jobs[j];
        const SmoothArgs& A = tab[job.x];
        const PdStep s = pd_step(A, launch, launches);
        rof_step2_tile<false>(s.unew, s.pnew, s.qnew, s.u, s.p, s.q, A.tmp, A.dt, lam, A.W, A.H, launch == 0, 0.0f,
                              (int)(job.y & 0xffffu) * RF_BX, (int)(job.y >> 16) * RF_BY);
    }
}

__global__ void k_consistency(float4* __restrict__ out, const float4* __restrict__ L, const float4* __restrict__ R,
                              int W, int H, float maxdd, float maxad)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * W + x;
    // pmhstereo_consistency (pmhstereo.cl:1107-1128)
    const float4 sl = L[i];
    const float c2x = transform_x(sl, (float)x, (float)y), c2y = (float)y;
    float4 val = f4(0.0f, 0.0f, 0.0f, -1.0f);
    if (ceilf(c2x) >= 0 && floorf(c2x) < (float)W) {
        const int x1 = min(max(__float2int_rn(floorf(c2x)), 0), W - 1);
        const int x2 = min(max(__float2int_rn(ceilf(c2x)), 0), W - 1);
        const float4 sr = R[(size_t)y * W + x1], sr2 = R[(size_t)y * W + x2];
        const float3 nl = to_normal(sl), n1 = to_normal(viewprop(sr)), n2 = to_normal(viewprop(sr2));
        const float nd = nl.x * n1.x + nl.y * n1.y + nl.z * n1.z;
        const float nd2 = nl.x * n2.x + nl.y * n2.y + nl.z * n2.z;
        const float d1 = fabsf((float)x - transform_x(sr, c2x, c2y));
        const float d2 = fabsf((float)x - transform_x(sr2, c2x, c2y));
        const float lim = maxad / 180.0f;
        if (!(d1 >= maxdd || acospif_(clampf(nd, -1.0f, 1.0f)) >= lim) ||
            !(d2 >= maxdd || acospif_(clampf(nd2, -1.0f, 1.0f)) >= lim))
            val = sl;
    }
    out[i] = val;
}

__device__ __forceinline__ float length3(float4 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }

__global__ void k_to_disparity(float* __restrict__ out, const float4* __restrict__ planes, int W, int H, float scale,
                               int lr)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t i = (size_t)y * W + x;
    // pmhstereo_to_disparity (pmhstereo.cl:1243-1256)
    const float4 s = planes[i];
    const float disp = (transform_x(s, (float)x, (float)y) - (float)x) * (lr ? -1.0f : 1.0f);
    float v;
    if (length3(s) < 1e-4f || disp < 0 || disp > (float)W) v = 0.0f;
    else v = fmaxf(disp, 0.0f);
    out[i] = v * scale;
}

// the row search of pmhstereo_fill_depthmap / pmhstereo_fill_normalmap (:1199-1218, :1271-1290)
__device__ __forceinline__ void fill_neighbours(const float4* __restrict__ row, int W, int x, float cx, float cy,
                                                float4& l, float4& r)
{
    l = f4(0, 0, 0, 0);
    for (int xx = x - 1; length3(l) < 1e-1f && xx >= 0; xx--) l = row[xx];
    r = f4(0, 0, 0, 0);
    for (int xx = x + 1; length3(r) < 1e-1f && xx < W; xx++) r = row[xx];
    if (length3(l) < 1e-1f) { l.x = l.y = l.z = -1e5f; }
    if (length3(r) < 1e-1f) { r.x = r.y = r.z = -1e5f; }
    l.w = -(transform_x(l, cx, cy) - cx);
    r.w = -(transform_x(r, cx, cy) - cx);
}

__global__ void k_fill_depthmap(float* __restrict__ out, const float4* __restrict__ planes, int W, int H, float scale)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float4* row = planes + (size_t)y * W;
    const float4 s = row[x];
    const float cx = (float)x, cy = (float)y;
    float v;
    if (length3(s) < 1e-4f) {
        float4 l, r;
        fill_neighbours(row, W, x, cx, cy, l, r);
        v = fminf(l.w, r.w);
    } else {
        v = fabsf(transform_x(s, cx, cy) - cx);
    }
    out[(size_t)y * W + x] = v * scale;
}

__global__ void k_fill_normalmap(float4* __restrict__ out, const float4* __restrict__ planes, int W, int H)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float4* row = planes + (size_t)y * W;
    const float4 s = row[x];
    const float cx = (float)x, cy = (float)y;
    float3 n;
    if (length3(s) < 1e-1f) {
        float4 l, r;
        fill_neighbours(row, W, x, cx, cy, l, r);
        n = (l.w < r.w) ? to_normal(l) : to_normal(r);
    } else {
        n = to_normal(s);
    }
    out[(size_t)y * W + x] = f4(n.x, n.y, n.z, 0.0f);
}

// Linear sampler, CLK_ADDRESS_CLAMP_TO_EDGE, unnormalised coordinates (OpenCL 1.2 s8.2) at a
// general 2-D point, in FP32 with every product and sum rounded in order: weights
// (1-a)(1-b), a(1-b), (1-a)b, ab, summed left to right.  fetch(x, y) takes clamped texels.
template <class Fetch>
__device__ __forceinline__ float4 sample_linear(Fetch fetch, int w, int h, float cx, float cy)
{
    const float tu = cx - 0.5f, tv = cy - 0.5f;
    const float fu = floorf(tu), fv = floorf(tv);
    const float a = tu - fu, b = tv - fv;
    const int i0 = fu < -2.0f ? -2 : (fu > (float)w + 1.0f ? w + 1 : (int)fu);
    const int j0 = fv < -2.0f ? -2 : (fv > (float)h + 1.0f ? h + 1 : (int)fv);
    const int x0 = min(max(i0, 0), w - 1), x1 = min(max(i0 + 1, 0), w - 1);
    const int y0 = min(max(j0, 0), h - 1), y1 = min(max(j0 + 1, 0), h - 1);
    const float4 T00 = fetch(x0, y0), T10 = fetch(x1, y0), T01 = fetch(x0, y1), T11 = fetch(x1, y1);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
    return f4(w00 * T00.x + w10 * T10.x + w01 * T01.x + w11 * T11.x, w00 * T00.y + w10 * T10.y + w01 * T01.y + w11 * T11.y,
              w00 * T00.z + w10 * T10.z + w01 * T01.z + w11 * T11.z, w00 * T00.w + w10 * T10.w + w01 * T01.w + w11 * T11.w);
}

// write_imagef to a CL_UNORM_INT8 channel: convert_uchar_sat_rte(v * 255) (OpenCL 1.2 s8.3.1.1)
__device__ __forceinline__ unsigned int unorm8(float v)
{
    const float x = v * 255.0f;
    if (!(x > 0.0f)) return 0u;
    if (x >= 255.0f) return 255u;
    return (unsigned int)__float2int_rn(x);
}

// pyrdown (cvt/cl/kernel/pyr/pyrdown.cl:27-46) as CLPyramid::pyrDown runs it
// (cvt/cl/CLPyramid.cpp:73-78): one output texel per thread, the linear sample of the
// RGBA8 input at (Wi/Wo * (x + 0.5), Hi/Ho * (y + 0.5)), written back as RGBA8
__global__ void k_pyrdown(uchar4* __restrict__ out, int Wo, int Ho, const uint8_t* __restrict__ in, size_t stride,
                          int Wi, int Hi)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wo || y >= Ho) return;
    const float incx = (float)Wi / (float)Wo, incy = (float)Hi / (float)Ho;
    auto fetch = [&](int i, int j) {
        const uchar4 p = *reinterpret_cast<const uchar4*>(in + (size_t)j * stride + 4 * (size_t)i);
        return f4(__fdiv_rn((float)p.x, 255.0f), __fdiv_rn((float)p.y, 255.0f), __fdiv_rn((float)p.z, 255.0f),
                  __fdiv_rn((float)p.w, 255.0f));
    };
    const float4 v = sample_linear(fetch, Wi, Hi, incx * ((float)x + 0.5f), incy * ((float)y + 0.5f));
    out[(size_t)y * Wo + x] = make_uchar4(unorm8(v.x), unorm8(v.y), unorm8(v.z), unorm8(v.w));
}

// pyrup_mul4f (cvt/cl/kernel/pyr/pyrupmul.cl:50-71) as PMHuberStereo::pyrUpMul runs it
// (PMHuberStereo.cpp:709-721): mul times the linear sample of a float image of 1 or 4
// channels at (Wi/Wo * (x + 0.5), Hi/Ho * (y + 0.5))
template <int CH>
__global__ void k_pyrup_mul(float* __restrict__ out, int Wo, int Ho, const float* __restrict__ in, int Wi, int Hi,
                            float4 mul)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wo || y >= Ho) return;
    const float incx = (float)Wi / (float)Wo, incy = (float)Hi / (float)Ho;
    auto fetch = [&](int i, int j) {
        const size_t k = (size_t)j * Wi + i;
        if (CH == 1) return f4(in[k], in[k], in[k], in[k]);
        return reinterpret_cast<const float4*>(in)[k];
    };
    const float4 v = sample_linear(fetch, Wi, Hi, incx * ((float)x + 0.5f), incy * ((float)y + 0.5f));
    const size_t o = (size_t)y * Wo + x;
    if (CH == 1) out[o] = mul.x * v.x;
    else reinterpret_cast<float4*>(out)[o] = f4(mul.x * v.x, mul.y * v.y, mul.z * v.z, mul.w * v.w);
}

// float to int as an x86 truncating conversion does it (cvttss2si), which is what the
// reference's implicit float-to-int conversions compile to on its host (pmhstereo.cl:1169-1170
// through the OpenCL-C shim): NaN and values outside the int range give INT_MIN
__device__ __forceinline__ int f2i_x86(float f)
{
    if (!(f > -2147483904.0f && f < 2147483648.0f)) return INT_MIN;
    return (int)f;
}

// pmhstereo_fill_state (pmhstereo.cl:1131-1185): a plane with a negative cost or a disparity
// outside [0, W] takes the valid neighbour of its row (nearest left / right with cost >= 0)
// that gives the smaller positive disparity; out = (normal, depth * dispscale) of the
// reference view
__global__ void k_fill_state(float4* __restrict__ out, const float4* __restrict__ planes, int W, int H,
                             float dispscale, int lr)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float4* row = planes + (size_t)y * W;
    const float4 state = row[x];
    const float cx = (float)x, cy = (float)y;
    const int sidesign = lr ? -1 : 1;
    const float disp = (transform_x(state, cx, cy) - cx) * (float)sidesign;
    float4 val;
    if (state.w < 0 || disp < 0 || disp > (float)W) {
        float4 l = f4(-1.0f, -1.0f, -1.0f, -1.0f), r = l;
        for (int xx = x - 1; l.w < 0 && xx >= 0; xx--) l = row[xx];
        for (int xx = x + 1; r.w < 0 && xx < W; xx++) r = row[xx];
        if (l.w >= 0 && r.w >= 0) {
            int dl = f2i_x86((float)sidesign * (transform_x(l, cx, cy) - cx));
            int dr = f2i_x86((float)sidesign * (transform_x(r, cx, cy) - cx));
            if (dl <= 0) dl = W;
            if (dr <= 0) dr = W;
            val = dl <= dr ? l : r;
        } else {
            val = r.w < 0 ? l : r;
        }
    } else {
        val = state;
    }
    if (!(fin(val.x) && fin(val.y))) { val.x = 0.0f; val.y = 0.0f; }
    float4 nd = to_ref_normal_depth(val, cx, cy, lr);
    nd.w = nd.w * dispscale;
    out[(size_t)y * W + x] = nd;
}

// the top-left Wd x Hd corner of a field with Ws columns (CH floats per texel)
template <int CH>
__global__ void k_crop(float* __restrict__ dst, int Wd, int Hd, const float* __restrict__ src, int Ws)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wd || y >= Hd) return;
#pragma unroll
    for (int c = 0; c < CH; c++) dst[((size_t)y * Wd + x) * CH + c] = src[((size_t)y * Ws + x) * CH + c];
}

__global__ void k_disparity_to_normal(float4* __restrict__ out, const float* __restrict__ d, int W, int H)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    // pmhstereo_disparity_to_normal (pmhstereo.cl:1619-1636), zero border
    auto at = [&](int xx, int yy) { return (xx < 0 || xx >= W || yy < 0 || yy >= H) ? 0.0f : d[(size_t)yy * W + xx]; };
    const float dx = at(x + 1, y) - at(x, y);
    const float dy = at(x, y + 1) - at(x, y);
    const float3 n = normalize3(make_float3(0.0f * dy - dx * 1.0f, dx * 0.0f - 1.0f * dy, 1.0f * 1.0f - 0.0f * 0.0f));
    out[(size_t)y * W + x] = f4(n.x, n.y, n.z, 0.0f);
}

// texel planes of one view (pm_window.cuh): column c in [-2, W+1] of the colour plane
// holds bw, of the gradient plane grad, of the compact plane (bw.rgb, gradient sign
// a finite nonzero colour value below 2^-40 in magnitude (the window loops then need the
// exact-division fallback of ad_sum)
__device__ __forceinline__ bool tiny_colour(float v) { return v != 0.0f && fabsf(v) < 0x1p-40f; }

// bytes), all of column clamp(c, 0, W-1)
__global__ void k_pack_tex(float4* __restrict__ tex, const float4* __restrict__ bw, const float4* __restrict__ grad,
                           int W, int H, int P)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x - TEX_PAD, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (c > W + TEX_PAD - 1 || y >= H) return;
    const int s = min(max(c, 0), W - 1);
    const size_t o = (size_t)y * P + c + TEX_PAD;
    const float4 col = bw[(size_t)y * W + s], g = grad[(size_t)y * W + s];
    tex[o] = col;
    tex[(size_t)H * P + o] = g;
    tex[(size_t)2 * H * P + o] = make_float4(col.x, col.y, col.z, __uint_as_float(sign_bytes(g)));
    if (c == s && (tiny_colour(col.x) || tiny_colour(col.y) || tiny_colour(col.z)))
        atomicOr(reinterpret_cast<int*>(tex + (size_t)3 * H * P), 1);
}

__global__ void k_view_clear(int* __restrict__ count, unsigned long long* __restrict__ src, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        count[i] = 0;
        src[i] = ~0ULL;
    }
}

inline dim3 grid2d(int W, int H, dim3 b) { return dim3((W + b.x - 1) / b.x, (H + b.y - 1) / b.y); }

// 8 independent fma chains per thread: enough instruction-level parallelism to keep
// every FP32 pipe busy; the result is stored so that nothing is optimised away
constexpr int FMA_CHAINS = 8;
constexpr int FMA_UNROLL = 16;
__global__ void k_fma_peak(float* out, int iters)
{
    float a[FMA_CHAINS];
#pragma unroll
    for (int k = 0; k < FMA_CHAINS; k++) a[k] = (float)(threadIdx.x + k) * 1e-3f;
    const float m = 0.999f, c = 1e-4f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < FMA_UNROLL; u++) {
#pragma unroll
            for (int k = 0; k < FMA_CHAINS; k++) a[k] = fmaf(a[k], m, c);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < FMA_CHAINS; k++) s += a[k];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

void launch_fma_peak(float* out, int iters, int blocks, int threads, cudaStream_t st)
{
    k_fma_peak<<<blocks, threads, 0, st>>>(out, iters);
}
double fma_peak_flops_per_iter() { return 2.0 * FMA_CHAINS * FMA_UNROLL; }

// ---- launchers ----------------------------------------------------------------------

void launch_prep(const uint8_t* img, size_t stride, int W, int H, int r, int fused, float4* bw, float4* grad,
                 float4* dt, cudaStream_t st, float alpha, int raw)
{
    const dim3 b(32, 4);
    if (fused) k_prep<true><<<grid2d(W, H, b), b, 0, st>>>(img, stride, W, H, r, bw, grad, dt, alpha, raw);
    else k_prep<false><<<grid2d(W, H, b), b, 0, st>>>(img, stride, W, H, r, bw, grad, dt, alpha, raw);
}

void launch_init(float4* out, const ViewData& V, float dmax, int lr, const float* initdisp, const float4* initnormal,
                 int fused, cudaStream_t st)
{
    const dim3 b(32, 4);
    const dim3 g = grid2d(V.W, V.H, b);
    // both variants; the one that does not apply returns at once (pm_window.cuh)
    if (fused) {
        k_init<true, false><<<g, b, 0, st>>>(out, V, dmax, lr, initdisp, initnormal, 1);
        k_init<true, true><<<g, b, 0, st>>>(out, V, dmax, lr, initdisp, initnormal, 1);
    } else {
        k_init<false, false><<<g, b, 0, st>>>(out, V, dmax, lr, initdisp, initnormal, 1);
        k_init<false, true><<<g, b, 0, st>>>(out, V, dmax, lr, initdisp, initnormal, 1);
    }
}

void launch_cost(float* cost, const float4* planes, const ViewData& V, float mincost, int fused, cudaStream_t st)
{
    const dim3 b(32, 4);
    const dim3 g = grid2d(V.W, V.H, b);
    // both variants; the one that does not apply returns at once (pm_window.cuh)
    if (fused) {
        k_cost<true, false><<<g, b, 0, st>>>(cost, planes, V, mincost, 1);
        k_cost<true, true><<<g, b, 0, st>>>(cost, planes, V, mincost, 1);
    } else {
        k_cost<false, false><<<g, b, 0, st>>>(cost, planes, V, mincost, 1);
        k_cost<false, true><<<g, b, 0, st>>>(cost, planes, V, mincost, 1);
    }
}

void launch_klt(float4* out, const float4* planes, const ViewData& V, int fused, cudaStream_t st)
{
    const dim3 b(32, 4);
    const dim3 g = grid2d(V.W, V.H, b);
    // both variants; the one that does not apply returns at once (pm_window.cuh)
    if (fused) {
        k_klt<true, false><<<g, b, 0, st>>>(out, planes, V, 1);
        k_klt<true, true><<<g, b, 0, st>>>(out, planes, V, 1);
    } else {
        k_klt<false, false><<<g, b, 0, st>>>(out, planes, V, 1);
        k_klt<false, true><<<g, b, 0, st>>>(out, planes, V, 1);
    }
}

void launch_normal_depth(float4* out, const float4* planes, int W, int H, float dispscale, int lr, cudaStream_t st)
{
    const dim3 b(32, 8);
    k_normal_depth<<<grid2d(W, H, b), b, 0, st>>>(out, planes, W, H, dispscale, lr);
}

size_t rof_scratch_bytes(int W, int H) { return (size_t)W * H * sizeof(float4) * (1 + 2 + 2 + 1 + 1); }

namespace {
template <bool HUBER>
void launch_pd(float4* out, const float4* input, const float4* dt, float4 lam, float eps, int iters, int W, int H,
               void* scratch, cudaStream_t st)
{
    const size_t N = (size_t)W * H;
    float4* ut = static_cast<float4*>(scratch);
    float4* p[2] = {ut + N, ut + 3 * N};
    float4* q[2] = {ut + 5 * N, ut + 6 * N};
    // PDOptCL.cpp:1137-1166: `iters` steps, plus one when the last left the result in the scratch image;
    // an odd count (iters = 0) starts with one single step, the rest run two per launch
    const int steps = (iters > 0 && iters % 2 == 0) ? iters : iters + 1;
    const int launches = pd_launch_count(iters);
    const dim3 b1(ROF_BX, ROF_BY), g1 = grid2d(W, H, b1);
    const dim3 b2(RF_NT), g2((W + RF_BX - 1) / RF_BX, (H + RF_BY - 1) / RF_BY);
    // launch j writes `out` when (launches - 1 - j) is even, so that the last lands in `out`
    const float4* ucur = input;
    for (int j = 0; j < launches; j++) {
        float4* unew = ((launches - 1 - j) % 2 == 0) ? out : ut;
        const int pi = j & 1;
        if (j == 0 && steps % 2)
            k_rof_step<HUBER><<<g1, b1, 0, st>>>(unew, p[pi], q[pi], ucur, p[1 - pi], q[1 - pi], input, dt, lam, W, H,
                                                 1, eps);
        else
            k_rof_step2<HUBER><<<g2, b2, 0, st>>>(unew, p[pi], q[pi], ucur, p[1 - pi], q[1 - pi], input, dt, lam, W,
                                                  H, j == 0, eps);
        ucur = unew;
    }
}
}  // namespace

int pd_launch_count(int iters)
{
    const int steps = (iters > 0 && iters % 2 == 0) ? iters : iters + 1;
    return steps % 2 + steps / 2;
}

namespace {
template <class K>
unsigned persistent_grid(K kernel, int threads, int njobs)
{
    int dev = 0, sms = 1, per = 0;
    cudaGetDevice(&dev);
    // a failed query only shrinks the grid; its error is cleared, a pending launch error is not
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        sms = 1;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0) != cudaSuccess) {
        cudaGetLastError();
        per = 1;
    }
    sms = sms < 1 ? 1 : sms;
    per = per < 1 ? 1 : per;
    const long long g = (long long)per * sms;
    return (unsigned)(g < njobs ? g : njobs);
}
}  // namespace

int smooth_batch_launches(int iters) { return 1 + pd_launch_count(iters); }

void launch_smooth_batch(const SmoothArgs* tab, const JobList& j8, const JobList& j16, int sel, float4 lam, int iters,
                         int* next, cudaStream_t st)
{
    if (j8.njobs <= 0) return;
    const dim3 b8(ROF_BX, ROF_BY);
    k_normal_depth_b<<<persistent_grid(k_normal_depth_b, ROF_BX * ROF_BY, j8.njobs), b8, 0, st>>>(
        tab, sel, j8.jobs, j8.njobs, next);
    // launch_pd's schedule: an odd step count starts with one single step, the rest run two per launch
    const int steps = (iters > 0 && iters % 2 == 0) ? iters : iters + 1;
    const int launches = pd_launch_count(iters);
    for (int j = 0; j < launches; j++) {
        if (j == 0 && steps % 2)
            k_rof_step_b<<<persistent_grid(k_rof_step_b, ROF_BX * ROF_BY, j8.njobs), b8, 0, st>>>(
                tab, lam, j, launches, j8.jobs, j8.njobs, next + 1 + j);
        else
            k_rof_step2_b<<<persistent_grid(k_rof_step2_b, RF_NT, j16.njobs), RF_NT, 0, st>>>(
                tab, lam, j, launches, j16.jobs, j16.njobs, next + 1 + j);
    }
}

void launch_rof(float4* out, const float4* input, const float4* dt, float4 lam, int iters, int W, int H, void* scratch,
                cudaStream_t st)
{
    launch_pd<false>(out, input, dt, lam, 0.0f, iters, W, H, scratch, st);
}

// PDOptCL::denoiseDiffusionTensorHuber_PDD (PDOptCL.cpp:1170-1226): the same buffer schedule
void launch_huber(float4* out, const float4* input, const float4* dt, float4 lam, float eps, int iters, int W, int H,
                  void* scratch, cudaStream_t st)
{
    launch_pd<true>(out, input, dt, lam, eps, iters, W, H, scratch, st);
}

void launch_consistency(float4* out, const float4* L, const float4* R, int W, int H, float maxdd, float maxad,
                        cudaStream_t st)
{
    const dim3 b(32, 8);
    k_consistency<<<grid2d(W, H, b), b, 0, st>>>(out, L, R, W, H, maxdd, maxad);
}

void launch_to_disparity(float* out, const float4* planes, int W, int H, float scale, int lr, cudaStream_t st)
{
    const dim3 b(32, 8);
    k_to_disparity<<<grid2d(W, H, b), b, 0, st>>>(out, planes, W, H, scale, lr);
}

void launch_fill_depthmap(float* out, const float4* planes, int W, int H, float scale, cudaStream_t st)
{
    const dim3 b(32, 8);
    k_fill_depthmap<<<grid2d(W, H, b), b, 0, st>>>(out, planes, W, H, scale);
}

void launch_fill_normalmap(float4* out, const float4* planes, int W, int H, cudaStream_t st)
{
    const dim3 b(32, 8);
    k_fill_normalmap<<<grid2d(W, H, b), b, 0, st>>>(out, planes, W, H);
}

void launch_disparity_to_normal(float4* out, const float* d, int W, int H, cudaStream_t st)
{
    const dim3 b(32, 8);
    k_disparity_to_normal<<<grid2d(W, H, b), b, 0, st>>>(out, d, W, H);
}

void launch_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, size_t stride, int Wi, int Hi, cudaStream_t st)
{
    const dim3 b(32, 8);
    k_pyrdown<<<grid2d(Wo, Ho, b), b, 0, st>>>(reinterpret_cast<uchar4*>(out), Wo, Ho, in, stride, Wi, Hi);
}

void launch_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, float4 mul,
                      cudaStream_t st)
{
    const dim3 b(32, 8);
    if (channels == 1) k_pyrup_mul<1><<<grid2d(Wo, Ho, b), b, 0, st>>>(out, Wo, Ho, in, Wi, Hi, mul);
    else k_pyrup_mul<4><<<grid2d(Wo, Ho, b), b, 0, st>>>(out, Wo, Ho, in, Wi, Hi, mul);
}

void launch_fill_state(float4* out, const float4* planes, int W, int H, float dispscale, int lr, cudaStream_t st)
{
    const dim3 b(32, 8);
    k_fill_state<<<grid2d(W, H, b), b, 0, st>>>(out, planes, W, H, dispscale, lr);
}

void launch_crop(float* dst, int Wd, int Hd, const float* src, int Ws, int channels, cudaStream_t st)
{
    const dim3 b(32, 8);
    if (channels == 1) k_crop<1><<<grid2d(Wd, Hd, b), b, 0, st>>>(dst, Wd, Hd, src, Ws);
    else k_crop<4><<<grid2d(Wd, Hd, b), b, 0, st>>>(dst, Wd, Hd, src, Ws);
}

int tex_pitch(int W) { return W + 2 * TEX_PAD; }
size_t tex_bytes(int W, int H) { return ((size_t)tex_pitch(W) * H * 3 + 1) * sizeof(float4); }

void launch_pack_tex(float4* tex, const float4* bw, const float4* grad, int W, int H, cudaStream_t st)
{
    const dim3 b(64, 4);
    cudaMemsetAsync(tex + (size_t)3 * tex_pitch(W) * H, 0, sizeof(float4), st);   // the tiny-colour flag
    k_pack_tex<<<grid2d(tex_pitch(W), H, b), b, 0, st>>>(tex, bw, grad, W, H, tex_pitch(W));
}

void launch_view_clear(int* count, unsigned long long* src, size_t n, cudaStream_t st)
{
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 8);
    k_view_clear<<<blocks > 0 ? blocks : 1, threads, 0, st>>>(count, src, n);
}

}  // namespace pm
