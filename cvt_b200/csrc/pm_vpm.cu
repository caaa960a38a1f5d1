// VPMStereoCL on sm_100a: the simpler one-view slanted-plane PatchMatch of
// cvt/vision/VPMStereoCL.cpp and cvt/cl/kernel/VPMStereo.cl, with the gradient kernel of
// cvt/cl/kernel/gradxy.cl, behind its own C ABI (include/cvtpm.h, "VPMStereoCL").
//
// A plane state is (a, b, c) with x' = a x + b y + c in the second image; the fourth
// component of a stored state is its cost.  disparitySimple (VPMStereoCL.cpp:54-85):
// gradients of both images, init (random fronto-parallel planes, or the caller's
// disparities), `iterations` passes of vpmstereo_iter_simple (a van der Corput candidate,
// eight neighbour states, three Gauss-Newton steps), then |x' - x|.
//
// Texel layout.  The first image is read only at integral texels and only through its colour
// and the signs of its gradient, so it is one float4 plane: (r, g, b, the four gradient sign
// bits as bytes).  The second image is read bilinearly along rows: a colour plane
// (r, g, b, a) and a gradient plane, rows of W float4.  Plane states ping-pong between two
// W*H float4 fields.
//
// Arithmetic is the reference's FP32 sequence (the file is compiled with -fmad=false): every
// result equals the restatement in oracle/pm_oracle.cpp bit for bit.  The one double in the
// source, the 0.25 literal of patch_census_klt (VPMStereo.cl:162), is kept: the tap cost is a
// double sum rounded once to float.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "../../include/cvtpm.h"
#include "pm_window.cuh"

namespace pm {
namespace vpm {

constexpr float ALPHA = 0.05f;       // VPMStereo.cl:130, :210
constexpr float WEIGHT = 8.0f;       // CENSUS_COLOR_WEIGHT (:30)
// iterate / init blocks: a warp spans 32 columns of one row; k_iter asks for 3 resident blocks
// per SM (80 registers): 13% faster than the compiler's 100-register choice at 2 blocks
constexpr int BX = 32, BY = 8;

struct Views {
    const float4* __restrict__ t1;   // first image: (r, g, b, gradient sign bytes)
    const float4* __restrict__ c2;   // second image: colour
    const float4* __restrict__ g2;   // second image: gradient
    int W, H, r;
};

__device__ __forceinline__ float unorm8(uint32_t v) { return __fdiv_rn((float)v, 255.0f); }

// vpmsstate_vanDerCorput2 (:46-54): the five swap steps reverse the 32 bits
__device__ __forceinline__ float vdc2(uint32_t v) { return 2.3283064365386963e-10f * __uint2float_rn(__brev(v)); }

// vpmsstate_from_disparity_normal with the normal (0, 0, 1) (:56-65)
__device__ __forceinline__ float3 fronto(float cx, float cy, float d)
{
    const float nx = 0.0f, ny = 0.0f, nz = 1.0f;
    return make_float3(1.0f - (-nx / nz), 0.0f - (-ny / nz), 0.0f - ((nx * cx + ny * cy) / nz + d));
}

// support weight exp(-|dot(I1(q) - I1(p), gray)| * 8) (:148, :236); the argument lies in
// [-8.0001, 0], inside expf_neg's range
__device__ __forceinline__ float weight(float4 t, float4 ctr)
{
    return expf_neg(-fabsf(gray_dot<false>(t.x - ctr.x, t.y - ctr.y, t.z - ctr.z)) * WEIGHT);
}

// (1 - a) T0 + a T1 per component, each product and the sum rounded once (SAMPLER_BILINEAR
// with the vertical weight 0, as lerp_row)
__device__ __forceinline__ float4 mix(float a, float4 T0, float4 T1)
{
    const float b = 1.0f - a;
    return f4(__fadd_rn(__fmul_rn(b, T0.x), __fmul_rn(a, T1.x)), __fadd_rn(__fmul_rn(b, T0.y), __fmul_rn(a, T1.y)),
              __fadd_rn(__fmul_rn(b, T0.z), __fmul_rn(a, T1.z)), __fadd_rn(__fmul_rn(b, T0.w), __fmul_rn(a, T1.w)));
}

// colour and gradient of the second image at (u, row + 0.5): lerp_row of both planes
__device__ __forceinline__ void sample2(const Views& V, int row, float u, float4& c, float4& g)
{
    const float t = u - 0.5f;
    if (!fin(t)) {
        const float n = qnan();
        c = g = f4(n, n, n, n);
        return;
    }
    float fl = floorf(t);
    const float a = t - fl;
    fl = fminf(fmaxf(fl, -1.0f), (float)V.W);
    const int i0 = (int)fl;
    const int j0 = min(max(i0, 0), V.W - 1), j1 = min(max(i0 + 1, 0), V.W - 1);
    const size_t o = (size_t)row * V.W;
    c = mix(a, __ldg(V.c2 + o + j0), __ldg(V.c2 + o + j1));
    g = mix(a, __ldg(V.g2 + o + j0), __ldg(V.g2 + o + j1));
}

// patch_eval_census (:200-258).  Taps outside the image or mapped outside the second image
// are skipped (:228-231); a centre mapped outside returns 1 (:214-215).
template <bool COUNT>
__device__ float eval(const Views& V, int px, int py, float3 s, unsigned long long& taps)
{
    const float cx = (float)px, cy = (float)py;
    const float c2x = s.x * cx + s.y * cy + s.z;
    if (c2x < 0 || c2x >= (float)V.W) return 1.0f;
    const float4 ctr = __ldg(V.t1 + (size_t)py * V.W + px);
    float wsum = 0.0f, census = 0.0f;
    const int ylo = max(py - V.r, 0), yhi = min(py + V.r, V.H - 1);
    const int xlo = max(px - V.r, 0), xhi = min(px + V.r, V.W - 1);
    for (int iy = ylo; iy <= yhi; iy++) {
        const float qy = cy + (float)(iy - py) * 1.0f;
        const float ry = s.y * qy;
        const float4* row1 = V.t1 + (size_t)iy * V.W;
        for (int ix = xlo; ix <= xhi; ix++) {
            const float qx = cx + (float)(ix - px) * 1.0f;
            const float p2x = (s.x * qx + ry) + s.z;
            if (p2x < 0 || p2x >= (float)V.W) continue;
            const float4 t = __ldg(row1 + ix);
            const float w = weight(t, ctr);
            float4 c, g;
            sample2(V, iy, p2x + 0.5f, c, g);
            census += w * ALPHA * 0.33f * ad_sum<false>(c, t);
            census += w * (1.0f - ALPHA) * 0.25f * (float)sign_mismatch(__float_as_uint(t.w), sign_bytes(g));
            wsum += w;
            if (COUNT) taps++;
        }
    }
    return census / wsum;
}

// the cost of one Gauss-Newton sample (:154-162): k1 = w1 * alpha * 0.33f, kd = w1 * (1 - alpha)
// * 0.25 in double (exact)
__device__ __forceinline__ float klt_tap(float k1, double kd, float4 valin, uint32_t sb1, float4 c, float4 g)
{
    const float C = k1 * ad_sum<false>(c, valin);
    return __double2float_rn(__dadd_rn((double)C, kd * (double)sign_mismatch(sb1, sign_bytes(g))));
}

// patch_census_klt (:117-198): one Gauss-Newton step of the state from the costs at x' - 1,
// x', x' + 1 of every tap; H accumulates w1 (Cxp + Cxm - 2C) p p^T, symmetric, so six sums.
// The three samples of a tap share four texels of each plane when their column indices
// chain (always, except where the clamp to [-1, W] of the floor cuts in, or a coordinate is
// not finite); otherwise each is read on its own.
template <bool COUNT>
__device__ float3 klt(const Views& V, int px, int py, float3 s, unsigned long long& taps)
{
    const float cx = (float)px, cy = (float)py;
    float J0 = 0.0f, J1 = 0.0f, J2 = 0.0f;
    float h00 = 0.0f, h01 = 0.0f, h02 = 0.0f, h11 = 0.0f, h12 = 0.0f, h22 = 0.0f;
    const float4 ctr = __ldg(V.t1 + (size_t)py * V.W + px);
    const int ylo = max(py - V.r, 0), yhi = min(py + V.r, V.H - 1);
    // the taps that reach the cost: inside the image and not in its first or last column (:151)
    const int xlo = max(px - V.r, 1), xhi = min(px + V.r, V.W - 2);
    for (int iy = ylo; iy <= yhi; iy++) {
        const float qy = cy + (float)(iy - py) * 1.0f;
        const float ry = s.y * qy;
        const float4* row1 = V.t1 + (size_t)iy * V.W;
        const size_t o = (size_t)iy * V.W;
        for (int ix = xlo; ix <= xhi; ix++) {
            const float qx = cx + (float)(ix - px) * 1.0f;
            const float4 t = __ldg(row1 + ix);
            const float w1 = weight(t, ctr);
            const float p2x = (s.x * qx + ry) + s.z;
            const float k1 = w1 * ALPHA * 0.33f;
            const double kd = (double)(w1 * (1.0f - ALPHA)) * 0.25;
            const uint32_t sb1 = __float_as_uint(t.w);
            const float t0 = (p2x + 0.5f) - 0.5f, tp = ((p2x + 1.0f) + 0.5f) - 0.5f, tm = ((p2x + -1.0f) + 0.5f) - 0.5f;
            float C, Cxp, Cxm;
            bool done = false;
            if (fin(t0) && fin(tp) && fin(tm)) {
                float f0 = floorf(t0), fp = floorf(tp), fm = floorf(tm);
                const float a0 = t0 - f0, ap = tp - fp, am = tm - fm;
                f0 = fminf(fmaxf(f0, -1.0f), (float)V.W);
                fp = fminf(fmaxf(fp, -1.0f), (float)V.W);
                fm = fminf(fmaxf(fm, -1.0f), (float)V.W);
                const int i0 = (int)f0;
                if ((int)fp == i0 + 1 && (int)fm == i0 - 1) {
                    const int jm = min(max(i0 - 1, 0), V.W - 1), j0 = min(max(i0, 0), V.W - 1);
                    const int j1 = min(max(i0 + 1, 0), V.W - 1), j2 = min(max(i0 + 2, 0), V.W - 1);
                    const float4 cm = __ldg(V.c2 + o + jm), c0 = __ldg(V.c2 + o + j0);
                    const float4 c1 = __ldg(V.c2 + o + j1), c2 = __ldg(V.c2 + o + j2);
                    const float4 gm = __ldg(V.g2 + o + jm), g0 = __ldg(V.g2 + o + j0);
                    const float4 g1 = __ldg(V.g2 + o + j1), g2 = __ldg(V.g2 + o + j2);
                    C = klt_tap(k1, kd, t, sb1, mix(a0, c0, c1), mix(a0, g0, g1));
                    Cxp = klt_tap(k1, kd, t, sb1, mix(ap, c1, c2), mix(ap, g1, g2));
                    Cxm = klt_tap(k1, kd, t, sb1, mix(am, cm, c0), mix(am, gm, g0));
                    done = true;
                }
            }
            if (!done) {
                float4 c, g;
                sample2(V, iy, p2x + 0.5f, c, g);
                C = klt_tap(k1, kd, t, sb1, c, g);
                sample2(V, iy, (p2x + 1.0f) + 0.5f, c, g);
                Cxp = klt_tap(k1, kd, t, sb1, c, g);
                sample2(V, iy, (p2x + -1.0f) + 0.5f, c, g);
                Cxm = klt_tap(k1, kd, t, sb1, c, g);
            }
            const float tj = w1 * (Cxm - Cxp) * 0.5f;
            J0 = J0 + tj * qx;
            J1 = J1 + tj * qy;
            J2 = J2 + tj * 1.0f;
            const float sc = w1 * (Cxp + Cxm - 2.0f * C);
            h00 = h00 + sc * (qx * qx);
            h01 = h01 + sc * (qx * qy);
            h02 = h02 + sc * (qx * 1.0f);
            h11 = h11 + sc * (qy * qy);
            h12 = h12 + sc * (qy * 1.0f);
            h22 = h22 + sc * (1.0f * 1.0f);
            if (COUNT) taps++;
        }
    }
    const float3 d = lusolve(h00, h01, h02, h11, h12, h22, make_float3(J0, J1, J2));
    return make_float3(s.x - d.x, s.y - d.y, s.z - d.z);
}

// Colour texels and gradients of one image (grad_gray_xydiag, gradxy.cl:60-97: central grey
// differences with the zero border of CLK_ADDRESS_CLAMP, the diagonal channels repeating
// them), or the caller's gradient image when gin is given.  Writes any of: the first-image
// compact plane, the colour plane, the gradient plane.
__global__ void k_prep(const uint8_t* __restrict__ img, size_t stride, int W, int H, const float4* __restrict__ gin,
                       float4* __restrict__ compact, float4* __restrict__ colour, float4* __restrict__ grad)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    auto px = [&](int xx, int yy) { return __ldg(reinterpret_cast<const uchar4*>(img + (size_t)yy * stride) + xx); };
    auto gray = [&](int xx, int yy) {
        if (xx < 0 || xx >= W || yy < 0 || yy >= H) return 0.0f;
        const uchar4 p = px(xx, yy);
        return gray_dot<false>(unorm8(p.x), unorm8(p.y), unorm8(p.z));
    };
    const uchar4 p = px(x, y);
    const float4 c = f4(unorm8(p.x), unorm8(p.y), unorm8(p.z), unorm8(p.w));
    float4 g;
    if (gin) {
        g = __ldg(gin + (size_t)y * W + x);
    } else {
        const float dx = gray(x + 1, y) - gray(x - 1, y), dy = gray(x, y + 1) - gray(x, y - 1);
        g = f4(dx, dy, dx, dy);
    }
    const size_t i = (size_t)y * W + x;
    if (compact) compact[i] = f4(c.x, c.y, c.z, __uint_as_float(sign_bytes(g)));
    if (colour) colour[i] = c;
    if (grad) grad[i] = g;
}

// vpmstereo_init / vpmstereo_init_disparity (:260-309)
__global__ void __launch_bounds__(BX* BY) k_init(float4* __restrict__ out, Views V, float dmax,
                                                 const float* __restrict__ initdisp)
{
    const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
    if (x >= V.W || y >= V.H) return;
    const float cx = (float)x, cy = (float)y;
    float3 s;
    const float d = initdisp ? __ldg(initdisp + (size_t)y * V.W + x) : -1.0f;
    if (initdisp && d >= 0 && d < dmax) s = fronto(cx, cy, d);
    else s = fronto(cx, cy, vdc2((uint32_t)x * (uint32_t)V.W + (uint32_t)y) * dmax);
    unsigned long long n = 0;
    out[(size_t)y * V.W + x] = f4(s.x, s.y, s.z, eval<false>(V, x, y, s, n));
}

// vpmstereo_iter_simple (:311-361).  counts (COUNT): cost-window taps, Gauss-Newton taps.
template <bool COUNT>
__global__ void __launch_bounds__(BX* BY, 3) k_iter(float4* __restrict__ out, const float4* __restrict__ in, Views V,
                                                 float dmax, int iter, unsigned long long* counts)
{
    const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
    if (x >= V.W || y >= V.H) return;
    const float cx = (float)x, cy = (float)y;
    unsigned long long ne = 0, nk = 0;
    float4 cur = __ldg(in + (size_t)y * V.W + x);
    float3 s = fronto(cx, cy, vdc2((uint32_t)((x & 7) * (y & 7)) + (uint32_t)iter) * dmax);
    float cost = eval<COUNT>(V, x, y, s, ne);
    if (cost < cur.w) cur = f4(s.x, s.y, s.z, cost);
    // neighbour offsets (:323-332) (1,0) (-1,0) (0,1) (0,-1) (16,0) (-16,0) (0,16) (0,-16), taken
    // from (iter + i) & 7: bit 2 selects the distance, bit 1 the axis, bit 0 the sign; rows and
    // columns clamped to the edge (SAMPLER_NN)
#pragma unroll 1
    for (int i = 0; i < 8; i++) {
        const int k = (iter + i) & 7;
        const int d = ((k & 4) ? 16 : 1) * ((k & 1) ? -1 : 1);
        const int ox = (k & 2) ? 0 : d, oy = (k & 2) ? d : 0;
        const int nx = min(max(x + ox, 0), V.W - 1), ny = min(max(y + oy, 0), V.H - 1);
        const float4 n = __ldg(in + (size_t)ny * V.W + nx);
        s = make_float3(n.x, n.y, n.z);
        cost = eval<COUNT>(V, x, y, s, ne);
        if (cost < cur.w) cur = f4(s.x, s.y, s.z, cost);
    }
    s = klt<COUNT>(V, x, y, make_float3(cur.x, cur.y, cur.z), nk);
#pragma unroll 1
    for (int k = 0; k < 2; k++) s = klt<COUNT>(V, x, y, s, nk);
    cost = eval<COUNT>(V, x, y, s, ne);
    if (cost < cur.w) cur = f4(s.x, s.y, s.z, cost);
    out[(size_t)y * V.W + x] = cur;
    if (COUNT) {
        atomicAdd(counts, ne);
        atomicAdd(counts + 1, nk);
    }
}

// vpmstereo_disparity (:363-377): |x' - x| * scale
__global__ void k_disparity(float* __restrict__ out, const float4* __restrict__ states, int W, int H, float scale)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const float4 s = __ldg(states + (size_t)y * W + x);
    const float cx = (float)x, cy = (float)y;
    out[(size_t)y * W + x] = fabsf(s.x * cx + s.y * cy + s.z - cx) * scale;
}

inline dim3 row_grid(int W, int H) { return dim3((W + 127) / 128, H); }
inline dim3 tile_grid(int W, int H) { return dim3((W + BX - 1) / BX, (H + BY - 1) / BY); }

void launch_prep(const uint8_t* img, size_t stride, int W, int H, const float4* gin, float4* compact, float4* colour,
                 float4* grad, cudaStream_t st)
{
    k_prep<<<row_grid(W, H), 128, 0, st>>>(img, stride, W, H, gin, compact, colour, grad);
}

void launch_init(float4* out, const Views& V, float dmax, const float* initdisp, cudaStream_t st)
{
    k_init<<<tile_grid(V.W, V.H), dim3(BX, BY), 0, st>>>(out, V, dmax, initdisp);
}

void launch_iter(float4* out, const float4* in, const Views& V, float dmax, int iter, unsigned long long* counts,
                 cudaStream_t st)
{
    if (counts) k_iter<true><<<tile_grid(V.W, V.H), dim3(BX, BY), 0, st>>>(out, in, V, dmax, iter, counts);
    else k_iter<false><<<tile_grid(V.W, V.H), dim3(BX, BY), 0, st>>>(out, in, V, dmax, iter, nullptr);
}

void launch_disparity(float* out, const float4* states, int W, int H, float scale, cudaStream_t st)
{
    k_disparity<<<row_grid(W, H), 128, 0, st>>>(out, states, W, H, scale);
}

}  // namespace vpm
}  // namespace pm

using namespace pm;
using namespace pm::vpm;

// A VPMStereoCL object: its three parameters and a device workspace for one image size.
struct pm_vpm {
    int patchsize = 0, iterations = 0;
    float dmax = 0.0f;
    int device = 0;
    std::string err;
    int counting = 0;
    unsigned long long counts[2] = {0, 0};
    int W = 0, H = 0;
    size_t stride = 0;
    void* ws = nullptr;
    size_t ws_bytes = 0;
};

namespace {

thread_local std::string t_vpm_err;

int vfail(pm_vpm* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    t_vpm_err = msg;
    return code;
}

#define VPM_CUDA(h, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return vfail((h), PM_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
inline bool aligned(const void* p, size_t n) { return ((uintptr_t)p % n) == 0; }
inline size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

// workspace: compact plane of image 0, colour and gradient planes of image 1, two state
// fields, then (host entry) both images, the initial disparities, the disparities, counters
struct VLayout {
    enum { t1, c2, g2, s0, s1, img0, img1, initd, disp, ctr, COUNT };
    size_t off[COUNT + 1];
    size_t total() const { return off[COUNT]; }
};

VLayout vlayout(int W, int H, size_t stride)
{
    const size_t N = (size_t)W * H;
    const size_t sz[VLayout::COUNT] = {16 * N, 16 * N, 16 * N, 16 * N, 16 * N, stride * H, stride * H, 4 * N, 4 * N, 16};
    VLayout L;
    size_t o = 0;
    for (int k = 0; k < VLayout::COUNT; k++) {
        L.off[k] = o;
        o += up256(sz[k]);
    }
    L.off[VLayout::COUNT] = o;
    return L;
}

template <class T> T* vat(void* base, const VLayout& L, int k) { return reinterpret_cast<T*>(static_cast<char*>(base) + L.off[k]); }

int check_common(pm_vpm* h, int W, int H, size_t stride, int r, float dmax)
{
    if (W <= 0 || H <= 0 || W > PM_MAX_WIDTH || H > PM_MAX_HEIGHT) return vfail(h, PM_EINVAL_SHAPE, "image size out of range");
    if (r < 0 || r > PM_MAX_RADIUS) return vfail(h, PM_EINVAL_SHAPE, "patch size out of range");
    if (stride < (size_t)W * 4 || stride % 4) return vfail(h, PM_EINVAL_SHAPE, "row stride must be >= 4*width and a multiple of 4");
    if (!(dmax > 0.0f) || !isfinite(dmax)) return vfail(h, PM_EINVAL_ARG, "disparity range must be positive");
    return PM_OK;
}

int ensure_vws(pm_vpm* h, int W, int H, size_t stride)
{
    const size_t need = vlayout(W, H, stride).total();
    if (h->ws && h->ws_bytes >= need) return PM_OK;
    if (h->ws) {
        VPM_CUDA(h, cudaDeviceSynchronize());
        cudaFree(h->ws);
        h->ws = nullptr;
        h->ws_bytes = 0;
    }
    const cudaError_t e = cudaMalloc(&h->ws, need);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->ws = nullptr;
        return vfail(h, PM_ENOMEM, std::string("workspace allocation failed: ") + cudaGetErrorString(e));
    }
    h->ws_bytes = need;
    return PM_OK;
}

// disparitySimple on device buffers in the workspace: gradients, init, iterations, |x' - x|
int run_simple(pm_vpm* h, const uint8_t* img0, const uint8_t* img1, int W, int H, size_t stride, const float* initdisp,
               float* disp, float4* states, cudaStream_t st)
{
    const VLayout L = vlayout(W, H, stride);
    float4* t1 = vat<float4>(h->ws, L, VLayout::t1);
    float4* c2 = vat<float4>(h->ws, L, VLayout::c2);
    float4* g2 = vat<float4>(h->ws, L, VLayout::g2);
    float4* s[2] = {vat<float4>(h->ws, L, VLayout::s0), vat<float4>(h->ws, L, VLayout::s1)};
    unsigned long long* ctr = vat<unsigned long long>(h->ws, L, VLayout::ctr);
    launch_prep(img0, stride, W, H, nullptr, t1, nullptr, nullptr, st);
    launch_prep(img1, stride, W, H, nullptr, nullptr, c2, g2, st);
    const Views V = {t1, c2, g2, W, H, h->patchsize};
    launch_init(s[1], V, h->dmax, initdisp, st);
    if (h->counting) VPM_CUDA(h, cudaMemsetAsync(ctr, 0, 16, st));
    int swap = 0;
    for (int i = 0; i < h->iterations; i++) {
        launch_iter(s[swap], s[1 - swap], V, h->dmax, i, h->counting ? ctr : nullptr, st);
        swap = 1 - swap;
    }
    launch_disparity(disp, s[1 - swap], W, H, 1.0f, st);
    if (states) VPM_CUDA(h, cudaMemcpyAsync(states, s[1 - swap], (size_t)W * H * 16, cudaMemcpyDeviceToDevice, st));
    VPM_CUDA(h, cudaGetLastError());
    if (h->counting) {
        VPM_CUDA(h, cudaMemcpyAsync(h->counts, ctr, 16, cudaMemcpyDeviceToHost, st));
        VPM_CUDA(h, cudaStreamSynchronize(st));
    }
    return PM_OK;
}

// the first-image compact plane and the second image's planes from the reference kernels'
// inputs (RGBA8 colour images and float4 gradient images), in stream-ordered scratch
struct VpmScratch {
    float4* p = nullptr;
    cudaStream_t st = nullptr;
    ~VpmScratch()
    {
        if (p) cudaFreeAsync(p, st);
    }
    int make(const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2, int W, int H, size_t stride, int r,
             cudaStream_t s, Views* V)
    {
        st = s;
        const size_t N = (size_t)W * H;
        VPM_CUDA(nullptr, cudaMallocAsync((void**)&p, 3 * N * sizeof(float4), s));
        launch_prep(c1, stride, W, H, reinterpret_cast<const float4*>(g1), p, nullptr, nullptr, s);
        launch_prep(c2, stride, W, H, reinterpret_cast<const float4*>(g2), nullptr, p + N, p + 2 * N, s);
        *V = Views{p, p + N, p + 2 * N, W, H, r};
        return PM_OK;
    }
};

}  // namespace

extern "C" {

int pm_vpm_create(pm_vpm** out, int patchsize, int iterations, float disparitymax, int device)
{
    if (!out) return vfail(nullptr, PM_EINVAL_ARG, "null output pointer");
    *out = nullptr;
    if (patchsize < 0 || patchsize > PM_MAX_RADIUS) return vfail(nullptr, PM_EINVAL_SHAPE, "patch size out of range");
    if (iterations < 0) return vfail(nullptr, PM_EINVAL_ARG, "negative iteration count");
    if (!(disparitymax > 0.0f) || !isfinite(disparitymax)) return vfail(nullptr, PM_EINVAL_ARG, "disparity range must be positive");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return vfail(nullptr, PM_ENODEV, "no CUDA device");
    }
    if (device < 0 || device >= n) return vfail(nullptr, PM_EINVAL_ARG, "device ordinal out of range");
    pm_vpm* h = new pm_vpm;
    h->patchsize = patchsize;
    h->iterations = iterations;
    h->dmax = disparitymax;
    h->device = device;
    *out = h;
    return PM_OK;
}

int pm_vpm_destroy(pm_vpm* h)
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

const char* pm_vpm_last_error(const pm_vpm* h) { return h ? h->err.c_str() : t_vpm_err.c_str(); }

int pm_vpm_set_counting(pm_vpm* h, int on)
{
    if (!h) return vfail(nullptr, PM_EINVAL_ARG, "null handle");
    h->counting = on ? 1 : 0;
    return PM_OK;
}

int pm_vpm_get_counters(pm_vpm* h, uint64_t c[2])
{
    if (!h || !c) return vfail(h, PM_EINVAL_ARG, "null argument");
    c[0] = h->counts[0];
    c[1] = h->counts[1];
    return PM_OK;
}

int pm_vpm_disparity_simple_device(pm_vpm* h, const uint8_t* image0, const uint8_t* image1, int W, int H,
                                   size_t stride, float* disparity, const float* initdisparity, float* states,
                                   void* stream)
{
    if (!h) return vfail(nullptr, PM_EINVAL_ARG, "null handle");
    if (!image0 || !image1 || !disparity) return vfail(h, PM_EINVAL_ARG, "null image");
    int rc = check_common(h, W, H, stride, h->patchsize, h->dmax);
    if (rc) return rc;
    if (!aligned(image0, 4) || !aligned(image1, 4) || !aligned(disparity, 4) || !aligned(initdisparity, 4) ||
        !aligned(states, 16))
        return vfail(h, PM_EINVAL_ARG, "images must be 4-byte aligned, states 16-byte aligned");
    VPM_CUDA(h, cudaSetDevice(h->device));
    rc = ensure_vws(h, W, H, stride);
    if (rc) return rc;
    return run_simple(h, image0, image1, W, H, stride, initdisparity, disparity, reinterpret_cast<float4*>(states),
                      S(stream));
}

int pm_vpm_disparity_simple(pm_vpm* h, const uint8_t* image0, const uint8_t* image1, int W, int H, size_t stride,
                            float* disparity, const float* initdisparity, float* states)
{
    if (!h) return vfail(nullptr, PM_EINVAL_ARG, "null handle");
    if (!image0 || !image1 || !disparity) return vfail(h, PM_EINVAL_ARG, "null image");
    int rc = check_common(h, W, H, stride, h->patchsize, h->dmax);
    if (rc) return rc;
    VPM_CUDA(h, cudaSetDevice(h->device));
    rc = ensure_vws(h, W, H, stride);
    if (rc) return rc;
    const VLayout L = vlayout(W, H, stride);
    const size_t N = (size_t)W * H;
    cudaStream_t st = 0;
    uint8_t* d0 = vat<uint8_t>(h->ws, L, VLayout::img0);
    uint8_t* d1 = vat<uint8_t>(h->ws, L, VLayout::img1);
    float* di = vat<float>(h->ws, L, VLayout::initd);
    float* dd = vat<float>(h->ws, L, VLayout::disp);
    VPM_CUDA(h, cudaMemcpyAsync(d0, image0, stride * H, cudaMemcpyHostToDevice, st));
    VPM_CUDA(h, cudaMemcpyAsync(d1, image1, stride * H, cudaMemcpyHostToDevice, st));
    if (initdisparity) VPM_CUDA(h, cudaMemcpyAsync(di, initdisparity, N * 4, cudaMemcpyHostToDevice, st));
    rc = run_simple(h, d0, d1, W, H, stride, initdisparity ? di : nullptr, dd, nullptr, st);
    if (rc) return rc;
    VPM_CUDA(h, cudaMemcpyAsync(disparity, dd, N * 4, cudaMemcpyDeviceToHost, st));
    if (states) {
        // after `iterations` passes the result sits in s1 when iterations is even, s0 when odd
        float4* src = vat<float4>(h->ws, L, (h->iterations % 2) ? VLayout::s0 : VLayout::s1);
        VPM_CUDA(h, cudaMemcpyAsync(states, src, N * 16, cudaMemcpyDeviceToHost, st));
    }
    VPM_CUDA(h, cudaStreamSynchronize(st));
    return PM_OK;
}

// ---- one reference kernel per call, on device buffers and a stream ---------------------

int pm_k_vpm_grad(float* out, const uint8_t* img, int W, int H, size_t stride, void* stream)
{
    int rc = check_common(nullptr, W, H, stride, 0, 1.0f);
    if (rc) return rc;
    if (!out || !img || !aligned(out, 16) || !aligned(img, 4)) return vfail(nullptr, PM_EINVAL_ARG, "bad buffer");
    launch_prep(img, stride, W, H, nullptr, nullptr, nullptr, reinterpret_cast<float4*>(out), S(stream));
    VPM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_vpm_init(float* out, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2, int W, int H,
                  size_t stride, int r, float dmax, const float* initdisp, void* stream)
{
    int rc = check_common(nullptr, W, H, stride, r, dmax);
    if (rc) return rc;
    if (!out || !c1 || !g1 || !c2 || !g2 || !aligned(out, 16) || !aligned(g1, 16) || !aligned(g2, 16) ||
        !aligned(c1, 4) || !aligned(c2, 4) || !aligned(initdisp, 4))
        return vfail(nullptr, PM_EINVAL_ARG, "bad buffer");
    VpmScratch sc;
    Views V;
    rc = sc.make(c1, g1, c2, g2, W, H, stride, r, S(stream), &V);
    if (rc) return rc;
    launch_init(reinterpret_cast<float4*>(out), V, dmax, initdisp, S(stream));
    VPM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_vpm_iter(float* out, const float* in, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2,
                  int W, int H, size_t stride, int r, float dmax, int iter, void* stream)
{
    int rc = check_common(nullptr, W, H, stride, r, dmax);
    if (rc) return rc;
    if (iter < 0) return vfail(nullptr, PM_EINVAL_ARG, "negative iteration index");
    if (!out || !in || !c1 || !g1 || !c2 || !g2 || !aligned(out, 16) || !aligned(in, 16) || !aligned(g1, 16) ||
        !aligned(g2, 16) || !aligned(c1, 4) || !aligned(c2, 4))
        return vfail(nullptr, PM_EINVAL_ARG, "bad buffer");
    VpmScratch sc;
    Views V;
    rc = sc.make(c1, g1, c2, g2, W, H, stride, r, S(stream), &V);
    if (rc) return rc;
    launch_iter(reinterpret_cast<float4*>(out), reinterpret_cast<const float4*>(in), V, dmax, iter, nullptr, S(stream));
    VPM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_vpm_disparity(float* out, const float* states, int W, int H, float scale, void* stream)
{
    if (W <= 0 || H <= 0 || W > PM_MAX_WIDTH || H > PM_MAX_HEIGHT) return vfail(nullptr, PM_EINVAL_SHAPE, "image size out of range");
    if (!out || !states || !aligned(out, 4) || !aligned(states, 16)) return vfail(nullptr, PM_EINVAL_ARG, "bad buffer");
    launch_disparity(out, reinterpret_cast<const float4*>(states), W, H, scale, S(stream));
    VPM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

}  // extern "C"
