// Window loops of the PatchMatch-Huber path: the adaptive-support-weight cost
// (patch_eval_census, pmhstereo.cl:661-736) and the Gauss-Newton plane step
// (patch_census_klt2, :326-410), one thread per pixel, samples in the
// reference's order.
//
// Texel layout.  Each view is stored as three planes of float4 in rows of W + 4
// texels: columns -2 .. W+1, the four outside ones replicating the edge texel
// (CLK_ADDRESS_CLAMP_TO_EDGE).  Colour (r, g, b, Σw) and gradient (4 components),
// the gradient plane `plane` float4 after the colour plane, serve the second
// view's bilinear taps and the first view's centre texel: a tap pair needs no
// clamping inside the padded range, all loads of a tap come from one index, and
// the lanes of a warp gathering neighbouring texels read 16-byte strided
// addresses.  The compact plane (r, g, b, the four gradient sign bits as bytes),
// `plane` float4 after the gradient plane, holds all that a first-view window
// sample needs, in one load.  (Interleaved 32-byte texels read with 256-bit loads
// measured slower for the Gauss-Newton taps.)  After the three planes, one int:
// set when some colour value is finite, nonzero and below 2^-40 in magnitude (see
// ad_sum).
//
// Blackwell specifics: the 7-channel bilinear reads of the second view and the
// truncated absolute differences run as packed FP32 pairs (FFMA2 / FMUL2,
// sm_100), the sign census packs the four gradient sign bits with byte
// permutes, and the three Gauss-Newton taps at x'-1, x', x'+1 read four shared
// texels whenever their floors chain (checked exactly; each with its own weight
// where the fractional parts differ, near powers of two; otherwise each tap is
// read on its own).  Every packed operation rounds per element exactly like its
// scalar form, so results equal the scalar restatement bit for bit.
#pragma once

#include "pm_device.cuh"

namespace pm {

constexpr int TEX_PAD = 2;   // replicated columns on each side of a texel row

struct ViewData {
    const float4* __restrict__ t1;   // first view: colour plane, gradient plane at + plane, compact at + 2 plane
    const float4* __restrict__ t2;   // second view
    int W, H, r, P;                  // P = W + 2 * TEX_PAD texels per row
    int plane;                       // H * P
    const int* tiny1;                // the views' tiny-colour flags (after the three planes)
    const int* tiny2;
    // colour texel (compact texel) of column 0 of row y
    __device__ __forceinline__ const float4* row1(int y) const { return t1 + (size_t)y * P + TEX_PAD; }
    __device__ __forceinline__ const float4* row1c(int y) const { return t1 + 2 * (size_t)plane + (size_t)y * P + TEX_PAD; }
    __device__ __forceinline__ const float4* row2(int y) const { return t2 + (size_t)y * P + TEX_PAD; }
};

struct Counters {
    unsigned long long eval, klt, calls, exits;
};

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

// bilinear pair: (1-a)*T0 + a*T1 per element; fused contracts a*T1.  The strict form rounds
// the two products (one packed multiply each) and adds them with scalar, explicitly rounded
// adds: packed adds fed by packed multiplies were measured to come out fused, which would
// change the rounding; a packed multiply feeding __fadd_rn does not (the 1280x720 results are
// bit-identical to the all-scalar form, which PM_STRICT_FMUL2=0 selects).
#ifndef PM_STRICT_FMUL2
#define PM_STRICT_FMUL2 1
#endif

template <bool F>
__device__ __forceinline__ float2 lerp2(float2 a2, float2 b2, float2 t0, float2 t1)
{
    if (F) return __ffma2_rn(a2, t1, __fmul2_rn(b2, t0));
#if PM_STRICT_FMUL2
    const float2 p0 = __fmul2_rn(b2, t0), p1 = __fmul2_rn(a2, t1);
    return make_float2(__fadd_rn(p0.x, p1.x), __fadd_rn(p0.y, p1.y));
#else
    return make_float2(__fadd_rn(__fmul_rn(b2.x, t0.x), __fmul_rn(a2.x, t1.x)),
                       __fadd_rn(__fmul_rn(b2.y, t0.y), __fmul_rn(a2.y, t1.y)));
#endif
}

// one texel: colour (r, g, b, w) and gradient (4 components)
struct Texel {
    float4 c, g;
};

__device__ __forceinline__ Texel texel_at(const float4* __restrict__ p, int plane)
{
    Texel t;
    t.c = __ldg(p);
    t.g = __ldg(p + plane);
    return t;
}

template <bool F>
__device__ __forceinline__ Texel lerp_texel(float a, float b, const Texel& t0, const Texel& t1)
{
    const float2 a2 = f2(a, a), b2 = f2(b, b);
    const float2 c01 = lerp2<F>(a2, b2, f2(t0.c.x, t0.c.y), f2(t1.c.x, t1.c.y));
    const float2 c23 = lerp2<F>(a2, b2, f2(t0.c.z, t0.c.w), f2(t1.c.z, t1.c.w));
    const float2 g01 = lerp2<F>(a2, b2, f2(t0.g.x, t0.g.y), f2(t1.g.x, t1.g.y));
    const float2 g23 = lerp2<F>(a2, b2, f2(t0.g.z, t0.g.w), f2(t1.g.z, t1.g.w));
    Texel r;
    r.c = make_float4(c01.x, c01.y, c23.x, c23.y);
    r.g = make_float4(g01.x, g01.y, g23.x, g23.y);
    return r;
}

// SAMPLER_BILINEAR (:71) read at (u, row + 0.5), OpenCL 1.2 s8.2 with the vertical weight
// exactly 0: (1-a)*T[i0] + a*T[i0+1], columns clamped to the edge; a non-finite
// coordinate reads the positive quiet NaN.  General form, for the rare taps the fast
// paths below do not cover.
template <bool F>
__device__ __forceinline__ Texel lerp_texel_at(const float4* __restrict__ row, int plane, int W, float u)
{
    const float t = u - 0.5f;
    if (!fin(t)) {
        const float n = qnan();
        Texel r;
        r.c = f4(n, n, n, n);
        r.g = r.c;
        return r;
    }
    float fl = floorf(t);
    const float a = t - fl;
    fl = fminf(fmaxf(fl, -1.0f), (float)W);
    const int i0 = (int)fl;
    const int j0 = min(max(i0, 0), W - 1), j1 = min(max(i0 + 1, 0), W - 1);
    return lerp_texel<F>(a, 1.0f - a, texel_at(row + j0, plane), texel_at(row + j1, plane));
}

// byte k holds the top byte of component k, so bit 7 of byte k is its sign bit
__device__ __forceinline__ uint32_t sign_bytes(float4 g)
{
    const uint32_t lo = __byte_perm(__float_as_uint(g.x), __float_as_uint(g.y), 0x0073);
    const uint32_t hi = __byte_perm(__float_as_uint(g.z), __float_as_uint(g.w), 0x0073);
    return __byte_perm(lo, hi, 0x5410);
}

// number of gradient components whose signs differ (the census term, :712-715, :367-370)
__device__ __forceinline__ int sign_mismatch(uint32_t a, uint32_t b) { return __popc((a ^ b) & 0x80808080u); }

// Sum over r, g, b of fmin(|v2 - ref|, 0.05) / 0.05 (:707-709, :364-365), divisions exact.
// x / 0.05 is formed as q = 20 x corrected by one fma, exact for every x >= 2^-100 (checked
// exhaustively); below that the division itself is taken (CHK).  The window loops need the
// fallback only for inputs that can make a nonzero |v2 - ref| that small: v2 is a bilinear
// mix of colour values with weights that are multiples of 2^-26 (fractions of coordinates
// formed as (x + 0.5) - 0.5 or x - floor(x)), ref a colour value or a difference of two.
// When every finite nonzero colour value has magnitude >= 2^-40 (its ulp >= 2^-63), all of
// these are multiples of 2^-89, so a nonzero difference is >= 2^-89 and the fallback never
// fires.  k_pack_tex flags any view that breaks this (images read as k/255 never do), and
// only then do the loops run with CHK.
template <bool CHK>
__device__ __forceinline__ float ad_sum(float4 v2, float4 ref)
{
    const float2 d01 = __ffma2_rn(f2(ref.x, ref.y), f2(-1.0f, -1.0f), f2(v2.x, v2.y));   // v2 - ref, exact
    const float d2 = v2.z - ref.z;
    const float m0 = fminf(fabsf(d01.x), 0.05f), m1 = fminf(fabsf(d01.y), 0.05f), m2 = fminf(fabsf(d2), 0.05f);
    const float2 m01 = f2(m0, m1);
    const float2 q01 = __fmul2_rn(m01, f2(20.0f, 20.0f));
    const float2 r01 = __ffma2_rn(q01, f2(-0.05f, -0.05f), m01);
    float2 c01 = __ffma2_rn(r01, f2(20.0f, 20.0f), q01);
    const float q2 = m2 * 20.0f;
    const float r2 = fmaf(q2, -0.05f, m2);
    float c2 = fmaf(r2, 20.0f, q2);
    if (CHK && fminf(fminf(m0, m1), m2) < 7.88860905e-31f) {   // below 2^-100 the fma correction is not exact
        c01 = f2(m0 / 0.05f, m1 / 0.05f);
        c2 = m2 / 0.05f;
    }
    return c01.x + c01.y + c2;
}

// (w1 * 0.125f) * 0.33f and 0.125f * (0.33f * S) as one multiply: the product of 0.125 and
// 0.33f is exact, and scaling by a power of two commutes with rounding
#define PM_K033_8 0.04125000163912773f

// Per-sample weights of a Gauss-Newton window sample for klt_cost: k1 = w1 * 0.125 * 0.33
// (one multiply, see PM_K033_8) and the census weight x = w1 * 0.875f.
struct KltWeights {
    float k1, x;
};

template <bool F>
__device__ __forceinline__ KltWeights klt_weights(float w1)
{
    KltWeights k;
    k.k1 = w1 * PM_K033_8;
    k.x = F ? w1 * 0.21875f : w1 * 0.875f;
    return k;
}

// the cost of one Gauss-Newton tap from its interpolated texel (:361-370).
// `w1 * (1.0f - alpha) * 0.25 * (float)cnt` (:370) carries a double literal, so the sum is a
// double-precision one rounded once: formed exactly in double (strict) or with one fma
// (fused; w1 * 0.875f * 0.25f is one multiply by 0.21875 for the same reason as above).  FP64
// runs at half the FP32 rate on B200, so the strict form costs about as much as a guarded fma.
template <bool F, bool CHK>
__device__ __forceinline__ float klt_cost(const KltWeights& kw, float4 val1, uint32_t sb1, const Texel& t)
{
    float C = kw.k1 * ad_sum<CHK>(t.c, val1);
    const int n = sign_mismatch(sb1, sign_bytes(t.g));
    if (F) C = fmaf(kw.x, (float)n, C);
    else C = (float)((double)C + (double)kw.x * 0.25 * (double)(float)n);
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

// Whether the views carry colour values for which ad_sum needs its fallback.  Kernels that
// run the window loops come in two variants launched back to back: without the fallback
// (returns at once when a flag is set) and with it (returns at once when none is, if
// `dual`); a kernel launched alone has the fallback and dual = 0.
__device__ __forceinline__ bool views_need_check(const ViewData& V) { return (__ldg(V.tiny1) | __ldg(V.tiny2)) != 0; }
template <bool CHK>
__device__ __forceinline__ bool variant_skips(const ViewData& V, int dual)
{
    const bool chk = views_need_check(V);
    return CHK ? (dual && !chk) : chk;
}

// one window sample of patch_eval_census (:690-722) at window position (qx, row of q1) of a
// pixel with centre texel `in`, for the plane s (byq = s.y * qy): accumulates the weighted
// cost into census and the weight into wsum, or returns false when the matched column lies
// outside the image (:693-696)
template <bool F, bool CHK>
__device__ __forceinline__ bool eval_sample(const float4* __restrict__ q1, const float4* __restrict__ row2, int plane,
                                            int W, float fW, float4 in, float4 s, float qx, float byq, float& census,
                                            float& wsum)
{
    const float p2x = F ? fmaf(s.x, qx, byq) + s.z : s.x * qx + byq + s.z;
    if (p2x < 0 || p2x >= fW) return false;
    const float4 q = __ldg(q1);   // compact texel
    const float w = support_weight<F>(q.x - in.x, q.y - in.y, q.z - in.z);
    const float t = (p2x + 0.5f) - 0.5f;
    Texel tx;
    if (fin(t)) {
        // p2x in [0, W) gives t in [0, W]: texels i0, i0 + 1 lie in the padded row
        const float fl = floorf(t);
        const float a = t - fl;
        const float4* __restrict__ b = row2 + (int)fl;
        tx = lerp_texel<F>(a, 1.0f - a, texel_at(b, plane), texel_at(b + 1, plane));
    } else {   // a non-finite coordinate reads the positive quiet NaN (lerp_texel_at)
        const float n = qnan();
        tx.c = f4(n, n, n, n);
        tx.g = tx.c;
    }
    float cost = PM_K033_8 * ad_sum<CHK>(tx.c, q);
    // cost + 0.875f * (0.25f * n): the product 0.21875 n is exact, so one fma rounds the same
    cost = fmaf(0.21875f, (float)sign_mismatch(__float_as_uint(q.w), sign_bytes(tx.g)), cost);
    census = F ? fmaf(w, cost, census) : census + w * cost;
    wsum += w;
    return true;
}

// validity test at the top of patch_eval_census (:675-678): a plane that is not finite,
// too steep, or whose centre matches outside the image costs 1e5 without a window
__device__ __forceinline__ bool plane_usable(float4 s, float cx, float cy, int W)
{
    const float c2x = transform_x(s, cx, cy);
    return fin(s.x) && fin(s.y) && fin(s.z) && !(to_normal(s).z < 1e-4f) && !(c2x < 0) && !(c2x >= (float)W);
}

// patch_eval_census (:661-736).  The early exit `census / bilw >= mincost` (:724) is tested
// as census >= exit_threshold(mincost, bilw), the same predicate without a division.
// Window coordinates run as floats (integers below 2^24 are exact) instead of being
// converted from the loop counters.
template <bool F, bool COUNT, bool CHK>
__device__ __forceinline__ float patch_eval(const ViewData& V, int px, int py, float4 s, float mincost, Counters& cnt)
{
    const float cx = (float)px, cy = (float)py;
    if (!plane_usable(s, cx, cy, V.W)) return 1e5f;
    const int W = V.W, plane = V.plane;
    const float4 in = __ldg(V.row1(py) + px);
    const float thr = exit_threshold(mincost, in.w);
    float wsum = 0.0f, census = 0.0f;
    if (COUNT) cnt.calls++;
    const int r = V.r;
    const int dy0 = max(-r, -py), dy1 = min(r, V.H - 1 - py);
    const int dx0 = max(-r, -px), dx1 = min(r, W - 1 - px);
    const float fW = (float)W;
    const float qx0 = cx + (float)dx0;
    float qy = cy + (float)dy0;
    for (int iy = py + dy0; iy <= py + dy1; iy++, qy += 1.0f) {
        const float byq = s.y * qy;
        const float4* __restrict__ q1 = V.row1c(iy) + px + dx0;
        const float4* __restrict__ row2 = V.row2(iy);
        float qx = qx0;
        for (int n = dx1 - dx0; n >= 0; n--, q1++, qx += 1.0f) {
            if (!eval_sample<F, CHK>(q1, row2, plane, W, fW, in, s, qx, byq, census, wsum)) continue;
            if (COUNT) cnt.eval++;
            if (census >= thr) {
                if (COUNT) cnt.exits++;
                return 1.0f;
            }
        }
    }
    if (wsum <= 1.0f) return 1.1f;
    return census / wsum;
}

// patch_census_klt2 (:326-410), with the in-bounds test on the window position rather than
// the matched one (:358) and the colour term against the colour difference (:352, :364)
template <bool F, bool COUNT, bool CHK>
__device__ __forceinline__ float4 klt2(const ViewData& V, int px, int py, float4 s, Counters& cnt)
{
    const float cxf = (float)px, cyf = (float)py;
    const int W = V.W, plane = V.plane;
    float2 J01 = f2(0.0f, 0.0f);
    float J2 = 0.0f;
    float2 h00_01 = f2(0.0f, 0.0f), h02_11 = f2(0.0f, 0.0f), h12_22 = f2(0.0f, 0.0f);
    const float4 c1 = __ldg(V.row1(py) + px);
    const int r = V.r;
    const int dy0 = max(-r, -py), dy1 = min(r, V.H - 1 - py);
    const int dx0 = max(-r, 1 - px), dx1 = min(r, W - 2 - px);   // the 3-point cost needs 1 <= qx < W - 1
    const float qx0 = cxf + (float)dx0;
    const float fWm2 = (float)(W - 2), fWm1 = (float)(W - 1);
    float qy = cyf + (float)dy0;
    for (int iy = py + dy0; iy <= py + dy1; iy++, qy += 1.0f) {
        const float byq = s.y * qy;
        const float yy = qy * qy;
        const float4* __restrict__ q1 = V.row1c(iy) + px + dx0;
        const float4* __restrict__ row2 = V.row2(iy);
        float qx = qx0;
        for (int n = dx1 - dx0; n >= 0; n--, q1++, qx += 1.0f) {
            const float4 q = __ldg(q1);   // compact texel
            const float4 val1 = make_float4(q.x - c1.x, q.y - c1.y, q.z - c1.z, 0.0f);
            const float w1 = support_weight<F>(val1.x, val1.y, val1.z);
            const uint32_t sb1 = __float_as_uint(q.w);
            const KltWeights kw = klt_weights<F>(w1);
            const float p2x = F ? fmaf(s.x, qx, byq) + s.z : s.x * qx + byq + s.z;
            // The three taps read at t - 1, t, t + 1 (t the tap coordinate minus 0.5, each formed
            // as the source forms it).  Common case: 1 <= p2x < W - 1 and p2x + 1.5 in the binade
            // of p2x; then p2x is a multiple of its ulp (<= 0.5), every +-1 and +-0.5 below is
            // exact, the coordinates are p2x - 1, p2x, p2x + 1 and share the weight
            // p2x - floor(p2x).  Otherwise the coordinates and their floors are formed exactly;
            // when the floors still chain (f0 - 1, f0, f0 + 1) the taps read the same four texels
            // with their own weights, and only then, or off the padded row, each tap is read on
            // its own.  Every path gives the bilinear values lerp_texel_at gives.
            float f0, am, a0, ap;
            bool chain = p2x >= 1.0f && p2x < fWm1 &&
                         ((__float_as_uint(p2x + 1.5f) ^ __float_as_uint(p2x)) < 0x00800000u);
            if (chain) {
                f0 = floorf(p2x);
                a0 = p2x - f0;
                am = a0;
                ap = a0;
            } else {
                const float t0 = (p2x + 0.5f) - 0.5f;
                const float tp = ((p2x + 1.0f) + 0.5f) - 0.5f;
                const float tm = ((p2x + -1.0f) + 0.5f) - 0.5f;
                f0 = floorf(t0);
                const float fp = floorf(tp), fm = floorf(tm);
                a0 = t0 - f0;
                ap = tp - fp;
                am = tm - fm;
                chain = fp == f0 + 1.0f && fm == f0 - 1.0f && f0 >= -1.0f && f0 <= fWm2;
            }
            Texel xm, x0, xp;
            if (chain) {
                // texels f0-1 .. f0+2, inside the padded row
                const float4* __restrict__ b = row2 + ((int)f0 - 1);
                const Texel tA = texel_at(b, plane), tB = texel_at(b + 1, plane);
                const Texel tC = texel_at(b + 2, plane), tD = texel_at(b + 3, plane);
                xm = lerp_texel<F>(am, 1.0f - am, tA, tB);
                x0 = lerp_texel<F>(a0, 1.0f - a0, tB, tC);
                xp = lerp_texel<F>(ap, 1.0f - ap, tC, tD);
            } else {
                xm = lerp_texel_at<F>(row2, plane, W, (p2x + -1.0f) + 0.5f);
                x0 = lerp_texel_at<F>(row2, plane, W, p2x + 0.5f);
                xp = lerp_texel_at<F>(row2, plane, W, (p2x + 1.0f) + 0.5f);
            }
            const float Cxm = klt_cost<F, CHK>(kw, val1, sb1, xm);
            const float C = klt_cost<F, CHK>(kw, val1, sb1, x0);
            const float Cxp = klt_cost<F, CHK>(kw, val1, sb1, xp);
            if (COUNT) cnt.klt++;
            // the update of :394-402 without a branch: a rejected sample adds exact zeros, and
            // no accumulator can be -0, so adding +0 or -0 leaves it unchanged
            const float curv = Cxp + Cxm - 2.0f * C;
            const bool take = curv > 0.0f;
            const float t = take ? w1 * (Cxm - Cxp) * 0.5f : 0.0f;
            const float sc = take ? w1 * curv : 0.0f;
            if (F) {
                const float2 t2 = f2(t, t), s2 = f2(sc, sc);
                J01 = __ffma2_rn(t2, f2(qx, qy), J01);
                J2 = fmaf(t, 1.0f, J2);
                h00_01 = __ffma2_rn(s2, f2(qx * qx, qx * qy), h00_01);
                h02_11 = __ffma2_rn(s2, f2(qx, yy), h02_11);
                h12_22 = __ffma2_rn(s2, f2(qy, 1.0f), h12_22);
            } else {   // scalar, explicitly rounded (see lerp2)
                J01 = f2(__fadd_rn(J01.x, __fmul_rn(t, qx)), __fadd_rn(J01.y, __fmul_rn(t, qy)));
                J2 = J2 + t * 1.0f;
                h00_01 = f2(__fadd_rn(h00_01.x, __fmul_rn(sc, qx * qx)), __fadd_rn(h00_01.y, __fmul_rn(sc, qx * qy)));
                h02_11 = f2(__fadd_rn(h02_11.x, __fmul_rn(sc, qx)), __fadd_rn(h02_11.y, __fmul_rn(sc, yy)));
                h12_22 = f2(__fadd_rn(h12_22.x, __fmul_rn(sc, qy)), __fadd_rn(h12_22.y, __fmul_rn(sc, 1.0f)));
            }
        }
    }
    const float3 d = lusolve(h00_01.x, h00_01.y, h02_11.x, h02_11.y, h12_22.x, h12_22.y, make_float3(J01.x, J01.y, J2));
    return f4(s.x - d.x, s.y - d.y, s.z - d.z, s.w - 1e5f);
}

}  // namespace pm
