// Device functions of the PatchMatch-Huber path: plane-state algebra and the
// per-pixel window work.  Each function names the reference lines it computes
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

// smoothDistance (:846-871): returns (distance of a, distance of b)
__device__ __forceinline__ float2 smooth_distance(float4 sa, float4 sb, float4 smooth, float cx, float cy,
                                                  float dmax, int lr)
{
    const float4 a = to_ref_normal_depth(sa, cx, cy, lr);
    const float4 b = to_ref_normal_depth(sb, cx, cy, lr);
    const float id2 = 1.0f / (dmax * dmax);
    const float den = id2 + 0.3f;
    const float4 dg = f4(0.1f / den, 0.1f / den, 0.1f / den, id2 / den);
    const float4 da = f4(a.x - smooth.x, a.y - smooth.y, a.z - smooth.z, a.w - smooth.w);
    const float4 db = f4(b.x - smooth.x, b.y - smooth.y, b.z - smooth.z, b.w - smooth.w);
    float2 r;
    r.x = da.x * (dg.x * da.x) + da.y * (dg.y * da.y) + da.z * (dg.z * da.z) + da.w * (dg.w * da.w);
    r.y = db.x * (dg.x * db.x) + db.y * (dg.y * db.y) + db.z * (dg.z * db.z) + db.w * (dg.w * db.w);
    return r;
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

// support weight exp(-|dot(I1(q) - I1(p), gray)| * 12) (:355, :701, :1491)
template <bool F>
__device__ __forceinline__ float support_weight(float dx, float dy, float dz)
{
    return expf_(-fabsf(gray_dot<F>(dx, dy, dz)) * 12.0f);
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

// per-sample cost of patch_eval_census (:707-716)
__device__ __forceinline__ float census_cost(float3 valin, uint32_t sg1, float4 v2, float4 gv2)
{
    const float cx = div005(fminf(fabsf(v2.x - valin.x), 0.05f));
    const float cy = div005(fminf(fabsf(v2.y - valin.y), 0.05f));
    const float cz = div005(fminf(fabsf(v2.z - valin.z), 0.05f));
    const float cad = 0.33f * (cx + cy + cz);
    float cost = 0.125f * cad;
    const float cc = 0.25f * (float)__popc(sg1 ^ signbits4(gv2));
    cost = cost + 0.875f * cc;
    return cost;
}

struct ViewData {
    const float4* __restrict__ bw1;   // first view: rgb + support-weight sum
    const float4* __restrict__ bw2;   // second view
    const float4* __restrict__ g1;
    const float4* __restrict__ g2;
    int W, H, r;
};

struct Counters {
    unsigned long long eval, klt, calls, exits;
};

// patch_eval_census (:661-736).  The early exit `census / bilw >= mincost` is tested as
// census >= exit_threshold(mincost, bilw), which is the same predicate.
template <bool F, bool COUNT>
__device__ float patch_eval(const ViewData& V, int px, int py, float4 s, float mincost, Counters& cnt)
{
    const float cx = (float)px, cy = (float)py;
    const float c2x = transform_x(s, cx, cy);
    if (!(fin(s.x) && fin(s.y) && fin(s.z)) || to_normal(s).z < 1e-4f || c2x < 0 || c2x >= (float)V.W) return 1e5f;
    const float4 in = __ldg(V.bw1 + (size_t)py * V.W + px);
    const float thr = exit_threshold(mincost, in.w);
    float wsum = 0.0f, census = 0.0f;
    if (COUNT) cnt.calls++;
    const int r = V.r;
    const int dy0 = max(-r, -py), dy1 = min(r, V.H - 1 - py);
    const int dx0 = max(-r, -px), dx1 = min(r, V.W - 1 - px);
    // rows and columns outside the image are skipped by the source's own test
    for (int dy = -r; dy <= r; dy++) {
        if (dy < dy0 || dy > dy1) continue;
        const int iy = py + dy;
        const float qy = cy + (float)dy;
        const float byq = s.y * qy;
        const float4* __restrict__ row1 = V.bw1 + (size_t)iy * V.W;
        const float4* __restrict__ rowg1 = V.g1 + (size_t)iy * V.W;
        const float4* __restrict__ row2 = V.bw2 + (size_t)iy * V.W;
        const float4* __restrict__ rowg2 = V.g2 + (size_t)iy * V.W;
        for (int dx = dx0; dx <= dx1; dx++) {
            const float qx = cx + (float)dx;
            const float p2x = F ? fmaf(s.x, qx, byq) + s.z : s.x * qx + byq + s.z;
            if (p2x < 0 || p2x >= (float)V.W) continue;
            const int ix = px + dx;
            const float4 vin = __ldg(row1 + ix);
            const float w = support_weight<F>(vin.x - in.x, vin.y - in.y, vin.z - in.z);
            const float4 gv1 = __ldg(rowg1 + ix);
            const float4 gv2 = lerp_row<F>(rowg2, V.W, p2x + 0.5f);
            const float4 v2 = lerp_row<F>(row2, V.W, p2x + 0.5f);
            const float cost = census_cost(make_float3(vin.x, vin.y, vin.z), signbits4(gv1), v2, gv2);
            census = F ? fmaf(w, cost, census) : census + w * cost;
            wsum += w;
            if (COUNT) cnt.eval++;
            if (census >= thr) { if (COUNT) cnt.exits++; return 1.0f; }
        }
    }
    if (wsum <= 1.0f) return 1.1f;
    return census / wsum;
}

// one tap of patch_census_klt2 (:361-370); the colour term compares against the
// colour difference val1, as in the source.  The double literal in
// `w1 * (1.0f - alpha) * 0.25 * (float)cnt` makes the sum a double-precision one,
// rounded once: formed exactly in double (strict) or with one fma (fused).
template <bool F>
__device__ __forceinline__ float klt_tap(float w1, float3 val1, uint32_t sg1, float4 v2, float4 gv2)
{
    const float cx = div005(fminf(fabsf(v2.x - val1.x), 0.05f));
    const float cy = div005(fminf(fabsf(v2.y - val1.y), 0.05f));
    const float cz = div005(fminf(fabsf(v2.z - val1.z), 0.05f));
    float C = w1 * 0.125f * 0.33f * (cx + cy + cz);
    const int n = __popc(sg1 ^ signbits4(gv2));
    if (F) C = fmaf(w1 * 0.875f * 0.25f, (float)n, C);
    else C = (float)((double)C + (double)(w1 * 0.875f) * 0.25 * (double)(float)n);
    return C;
}

// mat3f_lusolve (Matrix3.cl:286-311) on the symmetric 3x3 H = [h00 h01 h02; h01 h11 h12; h02 h12 h22]
__device__ __forceinline__ float3 lusolve(float h00, float h01, float h02, float h11, float h12, float h22, float3 b)
{
    float m10 = h01, m20 = h02, m11 = h11, m12 = h12, m21 = h12, m22 = h22;
    const float m00 = h00, m01 = h01, m02 = h02;
    m10 /= m00;
    m20 /= m00;
    m11 -= m10 * m01;
    m12 -= m10 * m02;
    m21 -= m20 * m01;
    m22 -= m20 * m02;
    m21 /= m11;
    m22 -= m21 * m12;
    b.y -= m10 * b.x;
    b.z -= m20 * b.x + m21 * b.y;
    float3 ret;
    ret.z = b.z / m22;
    ret.y = (b.y - m12 * ret.z) / m11;
    ret.x = (b.x - (m01 * ret.y + m02 * ret.z)) / m00;
    return ret;
}

// patch_census_klt2 (:326-410), with the in-bounds test on the window position rather
// than the matched one (:358)
template <bool F, bool COUNT>
__device__ float4 klt2(const ViewData& V, int px, int py, float4 s, Counters& cnt)
{
    const float cxf = (float)px, cyf = (float)py;
    float J0 = 0.0f, J1 = 0.0f, J2 = 0.0f;
    float h00 = 0.0f, h01 = 0.0f, h02 = 0.0f, h11 = 0.0f, h12 = 0.0f, h22 = 0.0f;
    const float4 c1 = __ldg(V.bw1 + (size_t)py * V.W + px);
    const int r = V.r;
    const int dy0 = max(-r, -py), dy1 = min(r, V.H - 1 - py);
    // the 3-point cost needs 1 <= qx < W - 1
    const int dx0 = max(-r, 1 - px), dx1 = min(r, V.W - 2 - px);
    for (int dy = dy0; dy <= dy1; dy++) {
        const int iy = py + dy;
        const float qy = cyf + (float)dy;
        const float byq = s.y * qy;
        const float4* __restrict__ row1 = V.bw1 + (size_t)iy * V.W;
        const float4* __restrict__ rowg1 = V.g1 + (size_t)iy * V.W;
        const float4* __restrict__ row2 = V.bw2 + (size_t)iy * V.W;
        const float4* __restrict__ rowg2 = V.g2 + (size_t)iy * V.W;
        for (int dx = dx0; dx <= dx1; dx++) {
            const float qx = cxf + (float)dx;
            const int ix = px + dx;
            const float4 vin = __ldg(row1 + ix);
            const float3 val1 = make_float3(vin.x - c1.x, vin.y - c1.y, vin.z - c1.z);
            const float w1 = support_weight<F>(val1.x, val1.y, val1.z);
            const float p2x = F ? fmaf(s.x, qx, byq) + s.z : s.x * qx + byq + s.z;
            const uint32_t sg1 = signbits4(__ldg(rowg1 + ix));
            const float u0 = p2x + 0.5f;
            const float up = (p2x + 1.0f) + 0.5f;
            const float um = (p2x + -1.0f) + 0.5f;
            const float C = klt_tap<F>(w1, val1, sg1, lerp_row<F>(row2, V.W, u0), lerp_row<F>(rowg2, V.W, u0));
            const float Cxp = klt_tap<F>(w1, val1, sg1, lerp_row<F>(row2, V.W, up), lerp_row<F>(rowg2, V.W, up));
            const float Cxm = klt_tap<F>(w1, val1, sg1, lerp_row<F>(row2, V.W, um), lerp_row<F>(rowg2, V.W, um));
            if (COUNT) cnt.klt++;
            if ((Cxp + Cxm - 2.0f * C) > 0.0f) {
                const float t = w1 * (Cxm - Cxp) * 0.5f;
                const float sc = w1 * (Cxp + Cxm - 2.0f * C);
                const float xx = qx * qx, xy = qx * qy, yy = qy * qy;
                if (F) {
                    J0 = fmaf(t, qx, J0); J1 = fmaf(t, qy, J1); J2 = fmaf(t, 1.0f, J2);
                    h00 = fmaf(sc, xx, h00); h01 = fmaf(sc, xy, h01); h02 = fmaf(sc, qx, h02);
                    h11 = fmaf(sc, yy, h11); h12 = fmaf(sc, qy, h12); h22 = fmaf(sc, 1.0f, h22);
                } else {
                    J0 = J0 + t * qx; J1 = J1 + t * qy; J2 = J2 + t * 1.0f;
                    h00 = h00 + sc * xx; h01 = h01 + sc * xy; h02 = h02 + sc * qx;
                    h11 = h11 + sc * yy; h12 = h12 + sc * qy; h22 = h22 + sc * 1.0f;
                }
            }
        }
    }
    const float3 d = lusolve(h00, h01, h02, h11, h12, h22, make_float3(J0, J1, J2));
    return f4(s.x - d.x, s.y - d.y, s.z - d.z, s.w - 1e5f);
}

}  // namespace pm
