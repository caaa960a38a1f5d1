// Device functions of the PatchMatch-Huber path: plane-state algebra, support
// weights and the bilinear row read.  Each function names the reference lines it computes
// (cvt/cl/kernel/pmhstereo.cl, Matrix3.cl).  Arithmetic is FP32 with the
// reference's operation order; the file must be compiled with -fmad=false so
// that only the explicit fmaf() calls (the "hot" sites, enabled by the template
// parameter F) are fused.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pm_math.cuh"

namespace pm {

__device__ __forceinline__ float4 f4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
__device__ __forceinline__ bool fin(float v) { return isfinite(v); }
__device__ __forceinline__ float qnan() { return __uint_as_float(0x7fffffffu); }

// OpenCL clamp (fmin(fmax(x, lo), hi))
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// OpenCL 1.2 normalize: a zero vector is returned unchanged, NaN propagates,
// otherwise v / |v| with the squared length kept away from under/overflow
__device__ __forceinline__ float3 normalize3(float3 v)
{
    if (v.x == 0.0f && v.y == 0.0f && v.z == 0.0f) return v;
    if (v.x != v.x || v.y != v.y || v.z != v.z) { const float n = qnan(); return make_float3(n, n, n); }
    if (isinf(v.x) || isinf(v.y) || isinf(v.z)) {
        v.x = isinf(v.x) ? copysignf(1.0f, v.x) : 0.0f * v.x;
        v.y = isinf(v.y) ? copysignf(1.0f, v.y) : 0.0f * v.y;
        v.z = isinf(v.z) ? copysignf(1.0f, v.z) : 0.0f * v.z;
    }
    float d = v.x * v.x + v.y * v.y + v.z * v.z;
    if (d < 7.8886090522101181e-31f) {
        v.x *= 1.8446744073709552e19f; v.y *= 1.8446744073709552e19f; v.z *= 1.8446744073709552e19f;
        d = v.x * v.x + v.y * v.y + v.z * v.z;
    } else if (d > 1.2676506002282294e30f) {
        v.x *= 5.4210108624275222e-20f; v.y *= 5.4210108624275222e-20f; v.z *= 5.4210108624275222e-20f;
        d = v.x * v.x + v.y * v.y + v.z * v.z;
    }
    const float l = sqrtf(d);
    return make_float3(v.x / l, v.y / l, v.z / l);
}

__device__ __forceinline__ float rsqrt_(float x) { return 1.0f / sqrtf(x); }

// nd_state_viewprop (pmhstereo.cl:174-181)
__device__ __forceinline__ float4 viewprop(float4 n)
{
    float4 r = f4(1.0f / n.x, -n.y / n.x, -n.z / n.x, 0.0f);
    if (fabsf(n.x) < 1e-8f) r = f4(0.0f, -n.y, -n.z, 0.0f);
    return r;
}

// nd_state_transform (:183-186), x component
__device__ __forceinline__ float transform_x(float4 s, float cx, float cy) { return s.x * cx + s.y * cy + s.z; }

// nd_state_init (:77-97); azimuth = 2*M_PI*u is formed in double as in the source
__device__ __forceinline__ float4 nd_state_init(Rng& rng, float cx, float cy, int lr, float dmax)
{
    const float z = rng.next() * dmax;
    const float azimuth = (float)(2.0 * 3.14159265358979323846 * (double)rng.next());
    const float u = rng.next() * 0.95f;
    const float w = sqrtf(1.0f - u * u);
    float s, c;
    sincosf_(azimuth, &s, &c);
    float3 n = make_float3(w * c, w * s, u);
    n.z = fmaxf(n.z, 1e-4f);
    n = normalize3(n);
    const float t0 = -n.x / n.z, t1 = -n.y / n.z, t2 = (n.x * cx + n.y * cy) / n.z + z;
    float4 ret = f4(1.0f - t0, 0.0f - t1, 0.0f - t2, 0.0f - 0.0f);
    if (!lr) ret = viewprop(ret);
    return ret;
}

// nd_state_from_disparity_normal (:99-106)
__device__ __forceinline__ float4 from_disparity_normal(float cx, float cy, float disparity, float3 normal)
{
    normal.z = fmaxf(normal.z, 1e-4f);
    normal = normalize3(normal);
    const float t0 = -normal.x / normal.z, t1 = -normal.y / normal.z;
    const float t2 = (normal.x * cx + normal.y * cy) / normal.z + disparity;
    return f4(1.0f - t0, 0.0f - t1, 0.0f - t2, 0.0f - 0.0f);
}

// nd_state_to_ref_normal_depth (:108-127)
__device__ __forceinline__ float4 to_ref_normal_depth(float4 state, float cx, float cy, int lr)
{
    float4 s = state;
    const float sidesign = lr ? -1.0f : 1.0f;
    if (!lr) s = viewprop(state);
    s = f4(1.0f - s.x, 0.0f - s.y, 0.0f - s.z, 0.0f - s.w);
    float4 ret;
    ret.w = (transform_x(state, cx, cy) - cx) * sidesign;
    ret.z = rsqrt_(s.x * s.x + s.y * s.y + 1.0f);
    ret.x = -s.x * ret.z;
    ret.y = -s.y * ret.z;
    if (!(fin(ret.x) && fin(ret.y) && fin(ret.z))) return f4(0.0f, 0.0f, 1.0f, 0.0f);
    return ret;
}

// nd_state_refine (:129-172); for lr == 0 it returns viewprop((1,0,0,0) - viewprop(in)) (:169-170)
__device__ __forceinline__ float4 nd_state_refine(Rng& rng, float4 in, float cx, float cy, float dmax, int lr)
{
    float4 state = in;
    if (!lr) state = viewprop(state);
    state = f4(1.0f - state.x, 0.0f - state.y, 0.0f - state.z, 0.0f - state.w);
    float z = state.x * cx + state.y * cy + state.z;
    float3 n;
    n.z = rsqrt_(state.x * state.x + state.y * state.y + 1.0f);
    n.x = -state.x * n.z;
    n.y = -state.y * n.z;
    z += (rng.next() - 0.5f) * 2.0f * 2.0f;
    z = clampf(z, 0.0f, dmax);
    const float azimuth = (float)(2.0 * 3.14159265358979323846 * (double)rng.next());
    const float u = rng.next() * (1.0f - 0.05f);
    const float w = sqrtf(1.0f - u * u);
    float s, c;
    sincosf_(azimuth, &s, &c);
    const float3 n2 = make_float3(w * c, w * s, u);
    n = make_float3((n.x + n2.x) * 0.5f, (n.y + n2.y) * 0.5f, (n.z + n2.z) * 0.5f);
    n.z = fmaxf(n.z, 1e-4f);
    n = normalize3(n);
    float4 ret = f4(-n.x / n.z, -n.y / n.z, (n.x * cx + n.y * cy) / n.z + z, 0.0f);
    ret = f4(1.0f - ret.x, 0.0f - ret.y, 0.0f - ret.z, 0.0f - ret.w);
    if (!lr) return viewprop(state);
    return ret;
}

// nd_state_to_normal (:201-210)
__device__ __forceinline__ float3 to_normal(float4 st)
{
    const float4 s = f4(1.0f - st.x, 0.0f - st.y, 0.0f - st.z, 0.0f - st.w);
    float3 n;
    n.z = rsqrt_(s.x * s.x + s.y * s.y + 1.0f);
    n.x = -s.x * n.z;
    n.y = -s.y * n.z;
    n.z = sqrtf(1.0f - n.x * n.x - n.y * n.y);
    return n;
}

// one component of smoothDistance (:846-871): the diagonal-weighted squared distance of a
// plane's (normal, depth) to the smoothed field; it does not read the plane's cost
__device__ __forceinline__ float smooth_dist1(float4 s, float4 smooth, float cx, float cy, float dmax, int lr)
{
    const float4 a = to_ref_normal_depth(s, cx, cy, lr);
    const float id2 = 1.0f / (dmax * dmax);
    const float den = id2 + 0.3f;
    const float4 dg = f4(0.1f / den, 0.1f / den, 0.1f / den, id2 / den);
    const float4 da = f4(a.x - smooth.x, a.y - smooth.y, a.z - smooth.z, a.w - smooth.w);
    return da.x * (dg.x * da.x) + da.y * (dg.y * da.y) + da.z * (dg.z * da.z) + da.w * (dg.w * da.w);
}

// smoothDistance (:846-871): returns (distance of a, distance of b)
__device__ __forceinline__ float2 smooth_distance(float4 sa, float4 sb, float4 smooth, float cx, float cy,
                                                  float dmax, int lr)
{
    return make_float2(smooth_dist1(sa, smooth, cx, cy, dmax, lr), smooth_dist1(sb, smooth, cx, cy, dmax, lr));
}

__device__ __forceinline__ uint32_t signbits4(float4 v)
{
    return (__float_as_uint(v.x) >> 31) | ((__float_as_uint(v.y) >> 31) << 1) | ((__float_as_uint(v.z) >> 31) << 2) |
           ((__float_as_uint(v.w) >> 31) << 3);
}

// grey weights of pmhstereo.cl:670
#define PM_GW_R 0.2126f
#define PM_GW_G 0.7152f
#define PM_GW_B 0.0722f

// dot(d, grayWeight) (:701); hot site
template <bool F>
__device__ __forceinline__ float gray_dot(float dx, float dy, float dz)
{
    if (F) return fmaf(dz, PM_GW_B, fmaf(dy, PM_GW_G, dx * PM_GW_R));
    return dx * PM_GW_R + dy * PM_GW_G + dz * PM_GW_B;
}

// expf_ for x in [-87, 0]: the same operations as expf_ on that range, without its NaN /
// overflow / underflow branches, and with rint(x * log2 e) taken by adding 1.5 * 2^23
// (the sum rounds to the nearest integer, ties to even, exactly as rintf) so that the
// integer part comes from the float's bits rather than from two conversions
__device__ __forceinline__ float expf_neg(float x)
{
    const float M = 12582912.0f;   // 1.5 * 2^23
    const float t = __fadd_rn(__fmul_rn(x, 1.44269502162933349609375f), M);
    const float n = __fsub_rn(t, M);
    float r = fmaf(n, -0.693145751953125f, x);
    r = fmaf(n, -1.428606765330187045e-06f, r);
    float p = 1.9841270113829523e-4f;
    p = fmaf(p, r, 1.3888889e-3f);
    p = fmaf(p, r, 8.3333338e-3f);
    p = fmaf(p, r, 4.1666668e-2f);
    p = fmaf(p, r, 1.6666667e-1f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    const int ni = __float_as_int(t) - __float_as_int(M);   // n as an integer, in [-126, 0]
    return p * __int_as_float((ni + 127) << 23);
}

// support weight exp(-|dot(I1(q) - I1(p), gray)| * 12) (:355, :701, :1491).  Colours are
// in [0, 1], so |dot| <= 1 and the argument lies in [-12.0001, 0], inside expf_neg's range.
template <bool F>
__device__ __forceinline__ float support_weight(float dx, float dy, float dz)
{
    return expf_neg(-fabsf(gray_dot<F>(dx, dy, dz)) * 12.0f);
}

// SAMPLER_BILINEAR (:71) read at (u, row + 0.5): OpenCL 1.2 s8.2 with the vertical
// weight exactly 0, i.e. (1-a)*T[i0] + a*T[i0+1], columns clamped to the edge
template <bool F>
__device__ __forceinline__ float4 lerp_row(const float4* __restrict__ row, int W, float u)
{
    const float t = u - 0.5f;
    if (!fin(t)) { const float n = qnan(); return f4(n, n, n, n); }
    float fl = floorf(t);
    const float a = t - fl;
    fl = fminf(fmaxf(fl, -1.0f), (float)W);
    const int i0 = (int)fl;
    const int j0 = min(max(i0, 0), W - 1), j1 = min(max(i0 + 1, 0), W - 1);
    const float4 T0 = __ldg(row + j0), T1 = __ldg(row + j1);
    const float b = 1.0f - a;
    if (F) return f4(fmaf(a, T1.x, b * T0.x), fmaf(a, T1.y, b * T0.y), fmaf(a, T1.z, b * T0.z), fmaf(a, T1.w, b * T0.w));
    return f4(b * T0.x + a * T1.x, b * T0.y + a * T1.y, b * T0.z + a * T1.z, b * T0.w + a * T1.w);
}

}  // namespace pm

