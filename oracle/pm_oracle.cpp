/*
 * ORACLE — test infrastructure only (see pm_oracle.h).  Built by
 * oracle/Makefile into oracle/liboracle.so; never linked into the product.
 *
 * A plain CPU restatement of the PatchMatch-Huber stereo path of phheise/cvt.
 * Citations are file:line within the reference project.  Build flags:
 * -O2 -ffp-contract=off -fno-fast-math, so every C operator below rounds once.
 */
#include "pm_oracle.h"
#include "pm_libm.h"
#include "pm_hostloop.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

namespace {

struct F2 { float x, y; };
struct F3 { float x, y, z; };
struct F4 { float x, y, z, w; };

inline F4 f4(float x, float y, float z, float w) { F4 r = {x, y, z, w}; return r; }
inline F3 f3(float x, float y, float z) { F3 r = {x, y, z}; return r; }
inline F3 xyz(const F4& v) { return f3(v.x, v.y, v.z); }

/* ---- arithmetic-mode helpers -------------------------------------------------- */

/* a*b + c, contracted in fused mode (used only at the hot sites named ORC_HOT) */
inline float orc_mad(int fused, float a, float b, float c) { return fused ? fmaf(a, b, c) : a * b + c; }

/* OpenCL dot(float3, float3), left to right (ORC_HOT: contracted in fused mode) */
inline float dot3_hot(int fused, F3 a, F3 b)
{
    if (fused) return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x));
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot4(F4 a, F4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

inline bool isfin(float v) { return isfinite(v) != 0; }
inline bool allfinite3(F3 v) { return isfin(v.x) && isfin(v.y) && isfin(v.z); }

/* OpenCL clamp = fmin(fmax(x, lo), hi) */
inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

/* OpenCL 1.2 normalize: zero vector returned unchanged, NaN propagated, otherwise
 * v / |v| with the squared length rescaled away from under/overflow. */
F3 normalize3(F3 v)
{
    if (v.x == 0.0f && v.y == 0.0f && v.z == 0.0f) return v;
    if (v.x != v.x || v.y != v.y || v.z != v.z) { float n = NAN; return f3(n, n, n); }
    if (isinf(v.x) || isinf(v.y) || isinf(v.z)) {
        v.x = isinf(v.x) ? copysignf(1.0f, v.x) : 0.0f * v.x;
        v.y = isinf(v.y) ? copysignf(1.0f, v.y) : 0.0f * v.y;
        v.z = isinf(v.z) ? copysignf(1.0f, v.z) : 0.0f * v.z;
    }
    float d = dot3(v, v);
    if (d < 7.8886090522101181e-31f) {            /* 2^-100: rescale by 2^64 */
        v.x *= 1.8446744073709552e19f; v.y *= 1.8446744073709552e19f; v.z *= 1.8446744073709552e19f;
        d = dot3(v, v);
    } else if (d > 1.2676506002282294e30f) {      /* 2^100: rescale by 2^-64 */
        v.x *= 5.4210108624275222e-20f; v.y *= 5.4210108624275222e-20f; v.z *= 5.4210108624275222e-20f;
        d = dot3(v, v);
    }
    const float l = sqrtf(d);
    return f3(v.x / l, v.y / l, v.z / l);
}

/* native_rsqrt: 1/sqrt, both correctly rounded */
inline float rsqrt_(float x) { return 1.0f / sqrtf(x); }

/* convert_int_rte / convert_int: NaN -> 0, saturating */
inline int cvt_int_sat(float f)
{
    if (f != f) return 0;
    if (f >= 2147483648.0f) return 2147483647;
    if (f < -2147483648.0f) return (-2147483647 - 1);
    return (int)f;
}
inline int convert_int_rte(float x) { return cvt_int_sat(rintf(x)); }
inline int convert_int_rtz(float x) { return cvt_int_sat(x); }

inline uint32_t signbits4(F4 v)
{
    return (orc_f2bits(v.x) >> 31) | ((orc_f2bits(v.y) >> 31) << 1) | ((orc_f2bits(v.z) >> 31) << 2) |
           ((orc_f2bits(v.w) >> 31) << 3);
}
inline int popc4(uint32_t m) { return (int)((m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1)); }

/* ---- images ------------------------------------------------------------------ */

struct Img4 {
    const float* p; int W, H;
    F4 at(int x, int y) const { const float* q = p + 4 * ((size_t)y * W + x); return f4(q[0], q[1], q[2], q[3]); }
    /* SAMPLER_NN with CLK_ADDRESS_CLAMP_TO_EDGE (pmhstereo.cl:70) */
    F4 edge(int x, int y) const {
        x = x < 0 ? 0 : (x >= W ? W - 1 : x);
        y = y < 0 ? 0 : (y >= H ? H - 1 : y);
        return at(x, y);
    }
    /* CLK_ADDRESS_CLAMP: border colour (0,0,0,0) */
    F4 zero(int x, int y) const {
        if (x < 0 || x >= W || y < 0 || y >= H) return f4(0, 0, 0, 0);
        return at(x, y);
    }
};

/* SAMPLER_BILINEAR (CLK_FILTER_LINEAR, CLK_ADDRESS_CLAMP_TO_EDGE, pmhstereo.cl:71) read
 * at (u, y + 0.5) with integral y, as every call on the path makes it (OpenCL 1.2 s8.2):
 * t = u - 0.5, i0 = floor(t), a = t - floor(t); the vertical weight is exactly 0, so the
 * value is (1-a)*T[i0] + a*T[i0+1] with edge-clamped columns (ORC_HOT: a*T[i0+1] is
 * contracted in fused mode).  A non-finite u yields the positive quiet NaN. */
inline F4 lerp_row(int fused, const Img4& im, float u, int y)
{
    const float t = u - 0.5f;
    if (!isfin(t)) { const float n = orc_bits2f(0x7fffffffu); return f4(n, n, n, n); }
    float fl = floorf(t);
    const float a = t - fl;
    fl = fminf(fmaxf(fl, -1.0f), (float)im.W);
    const int i0 = (int)fl;
    const F4 T0 = im.edge(i0, y), T1 = im.edge(i0 + 1, y);
    const float b = 1.0f - a;
    return f4(orc_mad(fused, a, T1.x, b * T0.x), orc_mad(fused, a, T1.y, b * T0.y),
              orc_mad(fused, a, T1.z, b * T0.z), orc_mad(fused, a, T1.w, b * T0.w));
}

/* ---- MWC64X (MWC64X.cl:36-141, RNG.cl:30-59) --------------------------------- */

const uint64_t MWC_A = 4294883355ULL;
const uint64_t MWC_M = 18446383549859758079ULL;
const uint64_t MWC_BASEID = 4077358422479273989ULL;

inline uint64_t mulmod(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % MWC_M); }
uint64_t powmod(uint64_t a, uint64_t e)
{
    uint64_t acc = 1, sq = a;
    while (e) { if (e & 1) acc = mulmod(acc, sq); sq = mulmod(sq, sq); e >>= 1; }
    return acc;
}

struct Rng {
    uint32_t x, c;
    /* RNG_init(s, linpos, numdraws): MWC64X_SeedStreams(s, 0, 0) starts every stream at
     * MWC_BASEID (stream gap 0), then MWC64X_Skip(s, (linpos) * numdraws).  The macro
     * does not parenthesise numdraws (RNG.cl:54-57), so the distance is the int value of
     * the expanded expression; callers pass it. */
    void init_skip(int32_t dist32) {
        const uint64_t dist = (uint64_t)(int64_t)dist32;
        uint64_t v = mulmod(MWC_BASEID, powmod(MWC_A, dist));
        x = (uint32_t)(v / MWC_A); c = (uint32_t)(v % MWC_A);
    }
    float next() {
        const uint32_t res = x ^ c;
        const uint32_t Xn = (uint32_t)MWC_A * x + c;
        const uint32_t carry = (uint32_t)(Xn < c);
        const uint32_t Cn = (uint32_t)(((uint64_t)(uint32_t)MWC_A * x) >> 32) + carry;
        x = Xn; c = Cn;
        return 2.3283064365386962890625e-10f * (float)res;
    }
};

/* ---- plane state algebra (pmhstereo.cl:74-224) -------------------------------- */

const float GW_R = 0.2126f, GW_G = 0.7152f, GW_B = 0.0722f;

/* nd_state_viewprop (:174-181) */
inline F4 viewprop(F4 n)
{
    F4 r = f4(1.0f / n.x, -n.y / n.x, -n.z / n.x, 0.0f);
    if (fabsf(n.x) < 1e-8f) r = f4(0.0f, -n.y, -n.z, 0.0f);
    return r;
}
/* nd_state_transform (:183-186), x component, strict */
inline float transform_x(F4 s, float cx, float cy) { return s.x * cx + s.y * cy + s.z; }

/* nd_state_init (:77-97) */
F4 nd_state_init(Rng& rng, float cx, float cy, int lr, float dmax)
{
    const float z = rng.next() * dmax;
    const float azimuth = (float)(2.0f * M_PI * (double)rng.next());
    const float u = rng.next() * 0.95f;
    const float w = sqrtf(1.0f - u * u);
    float s, c;
    orc_sincosf(azimuth, &s, &c);
    F3 n = f3(w * c, w * s, u);
    n.z = fmaxf(n.z, 1e-4f);
    n = normalize3(n);
    const float t0 = -n.x / n.z, t1 = -n.y / n.z, t2 = (n.x * cx + n.y * cy) / n.z + z;
    F4 ret = f4(1.0f - t0, 0.0f - t1, 0.0f - t2, 0.0f - 0.0f);
    if (!lr) ret = viewprop(ret);
    return ret;
}

/* nd_state_from_disparity_normal (:99-106) */
F4 from_disparity_normal(float cx, float cy, float disparity, F3 normal)
{
    normal.z = fmaxf(normal.z, 1e-4f);
    normal = normalize3(normal);
    const float t0 = -normal.x / normal.z, t1 = -normal.y / normal.z;
    const float t2 = (normal.x * cx + normal.y * cy) / normal.z + disparity;
    return f4(1.0f - t0, 0.0f - t1, 0.0f - t2, 0.0f - 0.0f);
}

/* nd_state_to_ref_normal_depth (:108-127) */
F4 to_ref_normal_depth(F4 state, float cx, float cy, int lr)
{
    F4 s = state;
    const float sidesign = lr ? -1.0f : 1.0f;
    if (!lr) s = viewprop(state);
    s = f4(1.0f - s.x, 0.0f - s.y, 0.0f - s.z, 0.0f - s.w);
    F4 ret;
    ret.w = (transform_x(state, cx, cy) - cx) * sidesign;
    ret.z = rsqrt_(s.x * s.x + s.y * s.y + 1.0f);
    ret.x = -s.x * ret.z;
    ret.y = -s.y * ret.z;
    if (!allfinite3(xyz(ret))) return f4(0.0f, 0.0f, 1.0f, 0.0f);
    return ret;
}

/* nd_state_refine (:129-172), including the lr == 0 early return at :169-170 */
F4 nd_state_refine(Rng& rng, F4 in, float cx, float cy, float dmax, int lr)
{
    F4 state = in;
    if (!lr) state = viewprop(state);
    state = f4(1.0f - state.x, 0.0f - state.y, 0.0f - state.z, 0.0f - state.w);
    float z = state.x * cx + state.y * cy + state.z;
    F3 n;
    n.z = rsqrt_(state.x * state.x + state.y * state.y + 1.0f);
    n.x = -state.x * n.z;
    n.y = -state.y * n.z;
    z += (rng.next() - 0.5f) * 2.0f * 2.0f;
    z = clampf(z, 0.0f, dmax);
    const float azimuth = (float)(2.0f * M_PI * (double)rng.next());
    const float u = rng.next() * (1.0f - 0.05f);
    const float w = sqrtf(1.0f - u * u);
    float s, c;
    orc_sincosf(azimuth, &s, &c);
    F3 n2 = f3(w * c, w * s, u);
    n = f3((n.x + n2.x) * 0.5f, (n.y + n2.y) * 0.5f, (n.z + n2.z) * 0.5f);
    n.z = fmaxf(n.z, 1e-4f);
    n = normalize3(n);
    F4 ret = f4(-n.x / n.z, -n.y / n.z, (n.x * cx + n.y * cy) / n.z + z, 0.0f);
    ret = f4(1.0f - ret.x, 0.0f - ret.y, 0.0f - ret.z, 0.0f - ret.w);
    if (!lr) return viewprop(state);
    return ret;
}

/* nd_state_to_normal (:201-210) */
F3 to_normal(F4 st)
{
    const F4 s = f4(1.0f - st.x, 0.0f - st.y, 0.0f - st.z, 0.0f - st.w);
    F3 n;
    n.z = rsqrt_(s.x * s.x + s.y * s.y + 1.0f);
    n.x = -s.x * n.z;
    n.y = -s.y * n.z;
    n.z = sqrtf(1.0f - n.x * n.x - n.y * n.y);
    return n;
}

/* smoothDistance (:846-871) */
F2 smooth_distance(F4 sa, F4 sb, F4 smooth, float cx, float cy, float dmax, int lr)
{
    const F4 a = to_ref_normal_depth(sa, cx, cy, lr);
    const F4 b = to_ref_normal_depth(sb, cx, cy, lr);
    const float id2 = 1.0f / (dmax * dmax);
    const float den = id2 + 0.3f;
    const F4 diag = f4(0.1f / den, 0.1f / den, 0.1f / den, id2 / den);
    const F4 da = f4(a.x - smooth.x, a.y - smooth.y, a.z - smooth.z, a.w - smooth.w);
    const F4 db = f4(b.x - smooth.x, b.y - smooth.y, b.z - smooth.z, b.w - smooth.w);
    F2 r;
    r.x = dot4(da, f4(diag.x * da.x, diag.y * da.y, diag.z * da.z, diag.w * da.w));
    r.y = dot4(db, f4(diag.x * db.x, diag.y * db.y, diag.z * db.z, diag.w * db.w));
    return r;
}

/* ---- window kernels ----------------------------------------------------------- */

struct Views {
    Img4 bw1, bw2, g1, g2;  /* first/second: rgb + support-weight sum; gradients */
    int W, H, r;
};

/* support weight exp(-|dot(I1(q) - I1(p), gray)| * 12) (pmhstereo.cl:355, :701, :1491) */
inline float support_weight(int fused, F3 val1)
{
    const float d = dot3_hot(fused, val1, f3(GW_R, GW_G, GW_B));
    return orc_expf(-fabsf(d) * 12.0f);
}

/* per-sample ASW cost terms of patch_eval_census (:698-716) */
inline float census_cost(F3 valin, F4 gval1, F4 v2, F4 gval2)
{
    const float cx = fminf(fabsf(v2.x - valin.x), 0.05f) / 0.05f;
    const float cy = fminf(fabsf(v2.y - valin.y), 0.05f) / 0.05f;
    const float cz = fminf(fabsf(v2.z - valin.z), 0.05f) / 0.05f;
    const float cad = 0.33f * (cx + cy + cz);
    float cost = 0.125f * cad;
    const int cnt = popc4(signbits4(gval1) ^ signbits4(gval2));
    const float cc = 0.25f * (float)cnt;
    cost += 0.875f * cc;
    return cost;
}

/* patch_eval_census (pmhstereo.cl:661-736) */
float patch_eval(const Views& V, int fused, int px, int py, F4 state, float mincost, int64_t* cnt)
{
    const float cx = (float)px, cy = (float)py;
    const float c2x = transform_x(state, cx, cy);
    if (!allfinite3(xyz(state)) || to_normal(state).z < 1e-4f || c2x < 0 || c2x >= (float)V.W) return 1e5f;
    const F4 in = V.bw1.at(px, py);
    const float bilw = in.w;
    const F3 valc1 = xyz(in);
    float wsum = 0.0f, census = 0.0f;
    const int r = V.r;
    if (cnt) cnt[2]++;
    for (int dy = -r; dy <= r; dy++) {
        for (int dx = -r; dx <= r; dx++) {
            const float qx = cx + (float)dx, qy = cy + (float)dy;
            /* ORC_HOT: the transform's a*x is contracted in fused mode */
            const float p2x = orc_mad(fused, state.x, qx, state.y * qy) + state.z;
            if (p2x < 0 || p2x >= (float)V.W || qx < 0 || qx >= (float)V.W || qy < 0 || qy >= (float)V.H) continue;
            const int ix = px + dx, iy = py + dy;
            const F3 valin = xyz(V.bw1.at(ix, iy));
            const F3 val1 = f3(valin.x - valc1.x, valin.y - valc1.y, valin.z - valc1.z);
            const float w = support_weight(fused, val1);
            const F4 gval1 = V.g1.at(ix, iy);
            const F4 gval2 = lerp_row(fused, V.g2, p2x + 0.5f, iy);
            const F4 val2 = lerp_row(fused, V.bw2, p2x + 0.5f, iy);
            const float cost = census_cost(valin, gval1, val2, gval2);
            census = orc_mad(fused, w, cost, census);   /* ORC_HOT */
            wsum += w;
            if (cnt) cnt[0]++;
            if (census / bilw >= mincost) { if (cnt) cnt[3]++; return 1.0f; }
        }
    }
    if (wsum <= 1.0f) return 1.1f;
    return census / wsum;
}

/* cost of one KLT tap: patch_census_klt2 (:361-370) with the colour term taken
 * against the colour difference val1, as the reference does */
inline float klt_tap(int fused, float w1, F3 val1, uint32_t sg1, F4 v2, F4 gv2)
{
    const float cx = fminf(fabsf(v2.x - val1.x), 0.05f) / 0.05f;
    const float cy = fminf(fabsf(v2.y - val1.y), 0.05f) / 0.05f;
    const float cz = fminf(fabsf(v2.z - val1.z), 0.05f) / 0.05f;
    float C = w1 * 0.125f * 0.33f * (cx + cy + cz);
    const int cnt = popc4(sg1 ^ signbits4(gv2));
    /* `w1 * (1.0f - alpha) * 0.25 * (float)cnt` has a double literal: the sum is formed in
     * double and rounded once; fused mode forms the same sum with one fma. */
    if (fused) C = fmaf(w1 * 0.875f * 0.25f, (float)cnt, C);
    else C = (float)((double)C + (double)(w1 * 0.875f) * 0.25 * (double)(float)cnt);
    return C;
}

/* mat3f_lusolve (Matrix3.cl:286-311) on the symmetric H */
F3 lusolve(const float Hm[3][3], F3 b)
{
    float m[3][3];
    memcpy(m, Hm, sizeof(m));
    m[1][0] /= m[0][0];
    m[2][0] /= m[0][0];
    m[1][1] -= m[1][0] * m[0][1];
    m[1][2] -= m[1][0] * m[0][2];
    m[2][1] -= m[2][0] * m[0][1];
    m[2][2] -= m[2][0] * m[0][2];
    m[2][1] /= m[1][1];
    m[2][2] -= m[2][1] * m[1][2];
    b.y -= m[1][0] * b.x;
    b.z -= m[2][0] * b.x + m[2][1] * b.y;
    F3 ret;
    ret.z = b.z / m[2][2];
    ret.y = (b.y - m[1][2] * ret.z) / m[1][1];
    ret.x = (b.x - (m[0][1] * ret.y + m[0][2] * ret.z)) / m[0][0];
    return ret;
}

/* patch_census_klt2 (pmhstereo.cl:326-410), including the in-bounds test on pos rather
 * than pos2 (:358) */
F4 klt2(const Views& V, int fused, int px, int py, F4 state, int64_t* cnt)
{
    const float cxf = (float)px, cyf = (float)py;
    float J[3] = {0, 0, 0};
    float Hm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    const F3 valc1 = xyz(V.bw1.at(px, py));
    const int r = V.r;
    for (int dy = -r; dy <= r; dy++) {
        for (int dx = -r; dx <= r; dx++) {
            const float qx = cxf + (float)dx, qy = cyf + (float)dy;
            if (qx < 0 || qx >= (float)V.W || qy < 0 || qy >= (float)V.H) continue;
            const int ix = px + dx, iy = py + dy;
            const F3 valin = xyz(V.bw1.at(ix, iy));
            const F3 val1 = f3(valin.x - valc1.x, valin.y - valc1.y, valin.z - valc1.z);
            const F4 gval1 = V.g1.at(ix, iy);
            const float w1 = support_weight(fused, val1);
            const float p2x = orc_mad(fused, state.x, qx, state.y * qy) + state.z;   /* ORC_HOT */
            if (qx < 1 || qx >= (float)(V.W - 1)) continue;
            if (cnt) cnt[1]++;
            const uint32_t sg1 = signbits4(gval1);
            const float u0 = p2x + 0.5f;
            const float up = (p2x + 1.0f) + 0.5f;
            const float um = (p2x + -1.0f) + 0.5f;
            const float C = klt_tap(fused, w1, val1, sg1, lerp_row(fused, V.bw2, u0, iy), lerp_row(fused, V.g2, u0, iy));
            const float Cxp = klt_tap(fused, w1, val1, sg1, lerp_row(fused, V.bw2, up, iy), lerp_row(fused, V.g2, up, iy));
            const float Cxm = klt_tap(fused, w1, val1, sg1, lerp_row(fused, V.bw2, um, iy), lerp_row(fused, V.g2, um, iy));
            if ((Cxp + Cxm - 2.0f * C) > 0.0f) {
                const float p[3] = {qx, qy, 1.0f};
                const float t = w1 * (Cxm - Cxp) * 0.5f;
                const float s = w1 * (Cxp + Cxm - 2.0f * C);
                for (int i = 0; i < 3; i++) J[i] = orc_mad(fused, t, p[i], J[i]);           /* ORC_HOT */
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) Hm[i][j] = orc_mad(fused, s, p[i] * p[j], Hm[i][j]); /* ORC_HOT */
            }
        }
    }
    const F3 d = lusolve(Hm, f3(J[0], J[1], J[2]));
    return f4(state.x - d.x, state.y - d.y, state.z - d.z, state.w - 1e5f);
}

/* minimalCost (:873-877) */
inline float minimal_cost(F4 nb, F4 self, F4 smooth, float cx, float cy, float theta, float dmax, int lr)
{
    const F2 sd = smooth_distance(nb, self, smooth, cx, cy, dmax, lr);
    return self.w + theta * sd.y - theta * sd.x;
}

inline bool same_plane(F4 a, F4 b) { return memcmp(&a, &b, 3 * sizeof(float)) == 0; }

/* candidates whose outcome was known without evaluating them, and those of them that
 * changed the state all the same (must stay 0; see try_candidate) */
int64_t g_known = 0, g_known_changed = 0;

/* the select at :976 / :990 / :1002 / :1015 / :1027 / :1052.
 * A candidate whose plane equals the current one bit for bit has the current plane's
 * smoothing distance (smoothDistance reads no cost).  Evaluated without an early exit it
 * returns the current cost and is taken, which changes nothing; with an exit it returns 1
 * and is taken only if 1 + theta d <= cost + theta d.  When that comparison fails the
 * outcome is known: the CUDA kernels skip the evaluation.  Here it is still evaluated, but
 * its window samples are not counted (the counters are the work the kernels do), and a
 * state change by such a candidate is recorded in g_known_changed. */
inline void try_candidate(const Views& V, int fused, int px, int py, F4& self, F4 nb, F4 smooth,
                          float theta, float dmax, int lr, int64_t* cnt)
{
    const float cx = (float)px, cy = (float)py;
    const float mincost = minimal_cost(nb, self, smooth, cx, cy, theta, dmax, lr);
    const F2 sd0 = smooth_distance(nb, self, smooth, cx, cy, dmax, lr);
    const bool known = same_plane(nb, self) && !(1.0f + theta * sd0.y <= self.w + theta * sd0.y);
    const F4 before = self;
    nb.w = patch_eval(V, fused, px, py, nb, mincost, known ? nullptr : cnt);
    const F2 sd = smooth_distance(nb, self, smooth, cx, cy, dmax, lr);
    if (nb.w + theta * sd.x <= self.w + theta * sd.y) self = nb;
    if (known) {
#pragma omp atomic
        g_known++;
        if (memcmp(&self, &before, sizeof(F4)) != 0) {
#pragma omp atomic
            g_known_changed++;
        }
    }
}

struct ScatterReq { int target; int src; F4 value; };

/* pmhstereo_propagate_view body for one pixel (:924-1070) */
F4 propagate_pixel(const Views& V, int fused, const Img4& old, const Img4& smoothimg, float theta,
                   float dmax, int lr, int iter, const int32_t* vin_n, const float* vin_val,
                   int px, int py, ScatterReq* req, int64_t* cnt)
{
    const int W = V.W;
    const float cx = (float)px, cy = (float)py;
    F4 smooth = smoothimg.at(px, py);
    smooth.w = clampf(smooth.w, 0.0f, 1.0f) * dmax;
    F4 self = old.at(px, py);
    self.w = patch_eval(V, fused, px, py, self, 1e10f, cnt);

    Rng rng;
    /* RNG_init(&rng, lin, (((2*PROPSIZE+1)*(2*PROPSIZE+1)-1) + NUMRNDTRIES)*3 + 2*NUMRNDSAMPLE)
     * (:942) expands to (lin) * ((1*1 - 1) + 2) * 3 + 2 * 4 = 6 * lin + 8 */
    const int32_t lin = py * W + px + iter;
    rng.init_skip(lin * 2 * 3 + 2 * 4);

    /* smooth candidate (:968-976) */
    F4 nb = from_disparity_normal(cx, cy, smooth.w * (lr ? -1.0f : 1.0f), normalize3(xyz(smooth)));
    if (!lr) nb = viewprop(nb);
    try_candidate(V, fused, px, py, self, nb, smooth, theta, dmax, lr, cnt);

    /* random neighbourhood (:982-991); the two offsets are drawn x first */
    for (int i = 0; i < 4; i++) {
        const int ox = (int)((rng.next() - 0.5f) * 2.0f * 5.0f + 0.5f);
        const int oy = (int)((rng.next() - 0.5f) * 2.0f * 5.0f + 0.5f);
        nb = old.edge(px + ox, py + oy);
        try_candidate(V, fused, px, py, self, nb, smooth, theta, dmax, lr, cnt);
    }

    /* random plane (:996-1002) */
    nb = nd_state_init(rng, cx, cy, lr, dmax);
    try_candidate(V, fused, px, py, self, nb, smooth, theta, dmax, lr, cnt);

    /* other view (:1007-1016) */
    const size_t idx = (size_t)py * W + px;
    int nview = vin_n ? vin_n[idx] : 0;
    if (nview > 2) nview = 2;
    for (int i = 0; i < nview; i++) {
        const float* v = vin_val + 8 * idx + 4 * i;
        nb = f4(v[0], v[1], v[2], v[3]);
        try_candidate(V, fused, px, py, self, nb, smooth, theta, dmax, lr, cnt);
    }

    /* randomized refinement, NUMRNDTRIES - 1 = 1 (:1021-1028) */
    nb = nd_state_refine(rng, self, cx, cy, dmax, lr);
    try_candidate(V, fused, px, py, self, nb, smooth, theta, dmax, lr, cnt);

    /* KLT step (:1034-1053) */
    nb = klt2(V, fused, px, py, self, cnt);
    for (int k = 0; k < 5; k++) nb = klt2(V, fused, px, py, nb, cnt);
    try_candidate(V, fused, px, py, self, nb, smooth, theta, dmax, lr, cnt);

    /* view scatter (:1060-1067) */
    req->target = -1;
    const float sidesign = lr ? -1.0f : 1.0f;
    const float tx = transform_x(self, cx, cy);
    const int xposview = convert_int_rte(tx);
    const int disp = convert_int_rtz((tx - cx) * sidesign);
    if (xposview >= 0 && xposview < W && disp > 0) {
        req->target = py * W + xposview;
        req->src = px;
        req->value = viewprop(self);
    }
    return self;
}

inline void put4(float* dst, size_t i, F4 v) { dst[4 * i] = v.x; dst[4 * i + 1] = v.y; dst[4 * i + 2] = v.z; dst[4 * i + 3] = v.w; }

std::vector<float> rgba8_to_float(const uint8_t* img, int W, int H, int stride)
{
    std::vector<float> f((size_t)W * H * 4);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int c = 0; c < 4; c++) f[4 * ((size_t)y * W + x) + c] = (float)img[(size_t)y * stride + 4 * x + c] / 255.0f;
    return f;
}

void add_counters(int64_t* dst, const int64_t* src) { if (dst) for (int i = 0; i < ORC_NCOUNTERS; i++) dst[i] += src[i]; }

}  // namespace

extern "C" {

int orc_version(void) { return 1; }
void orc_known_counts(int64_t out[2]) { out[0] = g_known; out[1] = g_known_changed; }

float orc_exp(float x) { return orc_expf(x); }
float orc_log(float x) { return orc_logf(x); }
float orc_sin(float x) { return orc_sinf(x); }
float orc_cos(float x) { return orc_cosf(x); }
float orc_acospi(float x) { return orc_acospif(x); }

int orc_rng_floats(int64_t linpos, int nd, int ndraws, float* out)
{
    Rng r; r.init_skip((int32_t)linpos * nd);
    for (int i = 0; i < ndraws; i++) out[i] = r.next();
    return 0;
}

/* raw: bw holds the image itself (r, g, b, a) instead of the colour and its window weight sum
 * (the images depthMap hands to its kernels, PMHuberStereo.cpp:203-204); alpha: the diffusion
 * tensor's edge weight (24 in disparityMapAll, :416; 12 in depthMap, :152) */
static int prep_impl(const uint8_t* img, int W, int H, int stride, int r, int fused, float* bw, float* grad, float* dt,
                     float alpha, int raw)
{
    const std::vector<float> f = rgba8_to_float(img, W, H, stride);
    const Img4 src = {f.data(), W, H};
    /* grey with the zero border of CLK_ADDRESS_CLAMP (:1569-1573, PDDiffTensor.cl:41-45) */
    auto gray = [&](int x, int y) { return dot4(src.zero(x, y), f4(GW_R, GW_G, GW_B, 0.0f)); };
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            if (bw && raw) {
                put4(bw, i, src.at(x, y));
            } else if (bw) {
                /* pmhstereo_bilateral_weight_to_alpha (:1462-1498) */
                const F3 valc1 = xyz(src.at(x, y));
                float wsum = 0.0f;
                for (int dy = -r; dy <= r; dy++)
                    for (int dx = -r; dx <= r; dx++) {
                        const int qx = x + dx, qy = y + dy;
                        if (qx < 0 || qx >= W || qy < 0 || qy >= H) continue;
                        const F3 v = xyz(src.at(qx, qy));
                        wsum += support_weight(fused, f3(v.x - valc1.x, v.y - valc1.y, v.z - valc1.z));
                    }
                put4(bw, i, f4(valc1.x, valc1.y, valc1.z, wsum));
            }
            const float g = gray(x, y);
            if (grad) {
                /* pmhstereo_gradxy (:1584-1601) */
                put4(grad, i, f4(gray(x + 1, y) - g, gray(x, y + 1) - g, gray(x + 1, y) - gray(x - 1, y),
                                 gray(x, y + 1) - gray(x, y - 1)));
            }
            if (dt) {
                /* PDDiffTensorColor (PDDiffTensor.cl:52-72) with beta = 1 (PMHuberStereo.cpp:417,
                 * :153); pow(len, 1) = len */
                float dx = gray(x + 1, y) - g;
                float dy = gray(x, y + 1) - g;
                const float len = sqrtf(dx * dx + dy * dy);
                const float w = orc_expf(-alpha * len);
                F4 d;
                if (len <= 0.001f) {
                    d = f4(1.0f, 0.0f, 0.0f, 1.0f);
                } else {
                    dx = dx / len;
                    dy = dy / len;
                    const float dxo = dy, dyo = -dx;
                    d = f4(w * dx * dx + dxo * dxo, w * dx * dy + dxo * dyo, w * dy * dx + dyo * dxo,
                           w * dy * dy + dyo * dyo);
                }
                put4(dt, i, d);
            }
        }
    }
    return 0;
}

int orc_prep(const uint8_t* img, int W, int H, int stride, int r, int fused, float* bw, float* grad, float* dt)
{
    return prep_impl(img, W, H, stride, r, fused, bw, grad, dt, 24.0f, 0);
}

int orc_prep_raw(const uint8_t* img, int W, int H, int stride, float alpha, float* colour, float* grad, float* dt)
{
    return prep_impl(img, W, H, stride, 0, 0, colour, grad, dt, alpha, 1);
}

int orc_init(float* out, const float* bw1, const float* bw2, const float* g1, const float* g2,
             int W, int H, int r, float dmax, int lr, const float* initdisp, const float* initnormal, int fused)
{
    const Views V = {{bw1, W, H}, {bw2, W, H}, {g1, W, H}, {g2, W, H}, W, H, r};
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            const float cx = (float)x, cy = (float)y;
            Rng rng;
            rng.init_skip((y * W + x) * 3);   /* RNG_init(&rng, lin, 3) (:766) */
            F4 ret;
            const float disparity = initdisp ? initdisp[i] : 0.0f;
            if (initdisp && disparity > 0 && lr) {
                const F3 n = normalize3(f3(initnormal[4 * i], initnormal[4 * i + 1], initnormal[4 * i + 2]));
                ret = from_disparity_normal(cx, cy, disparity, n);
            } else if (initdisp && disparity > 0 && !lr) {
                const F3 n = normalize3(f3(initnormal[4 * i], initnormal[4 * i + 1], initnormal[4 * i + 2]));
                ret = from_disparity_normal(cx, cy, -disparity, n);
            } else {
                ret = nd_state_init(rng, cx, cy, lr, dmax);
            }
            ret.w = patch_eval(V, fused, x, y, ret, 1e10f, nullptr);
            put4(out, i, ret);
        }
    }
    return 0;
}

int orc_propagate(float* out, const float* old, const float* bw1, const float* bw2,
                  const float* g1, const float* g2, const float* smooth, float theta,
                  int W, int H, int r, float dmax, int lr, int iter,
                  const int32_t* vin_n, const float* vin_val,
                  int32_t* vout_n, float* vout_val, int32_t* vout_src,
                  int fused, int64_t* counters)
{
    const Views V = {{bw1, W, H}, {bw2, W, H}, {g1, W, H}, {g2, W, H}, W, H, r};
    const Img4 oldimg = {old, W, H}, smoothimg = {smooth, W, H};
    std::vector<ScatterReq> req((size_t)W * H);
    int64_t total[ORC_NCOUNTERS] = {0, 0, 0, 0};
#pragma omp parallel
    {
        int64_t local[ORC_NCOUNTERS] = {0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const size_t i = (size_t)y * W + x;
                const F4 s = propagate_pixel(V, fused, oldimg, smoothimg, theta, dmax, lr, iter, vin_n, vin_val,
                                             x, y, &req[i], local);
                put4(out, i, s);
            }
#pragma omp critical
        add_counters(total, local);
    }
    add_counters(counters, total);
    /* append in the order a sequential executor issues atomic_inc: row-major */
    if (vout_n) {
        for (size_t i = 0; i < (size_t)W * H; i++) {
            const ScatterReq& q = req[i];
            if (q.target < 0) continue;
            const int nold = vout_n[q.target]++;
            if (nold < 2) {
                put4(vout_val + 4 * nold, 2 * (size_t)q.target, q.value);
                if (vout_src) vout_src[2 * (size_t)q.target + nold] = q.src;
            }
        }
    }
    return 0;
}

int orc_cost(float* cost, const float* planes, const float* bw1, const float* bw2,
             const float* g1, const float* g2, int W, int H, int r, float mincost, int fused)
{
    const Views V = {{bw1, W, H}, {bw2, W, H}, {g1, W, H}, {g2, W, H}, W, H, r};
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            const F4 s = f4(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], planes[4 * i + 3]);
            cost[i] = patch_eval(V, fused, x, y, s, mincost, nullptr);
        }
    return 0;
}

int orc_klt(float* out, const float* planes, const float* bw1, const float* bw2,
            const float* g1, const float* g2, int W, int H, int r, int fused)
{
    const Views V = {{bw1, W, H}, {bw2, W, H}, {g1, W, H}, {g2, W, H}, W, H, r};
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            const F4 s = f4(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], planes[4 * i + 3]);
            put4(out, i, klt2(V, fused, x, y, s, nullptr));
        }
    return 0;
}

int orc_normal_depth(float* out, const float* planes, int W, int H, float dispscale, int lr)
{
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            const F4 s = f4(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], planes[4 * i + 3]);
            F4 v = to_ref_normal_depth(s, (float)x, (float)y, lr);
            v.w = v.w * dispscale;
            put4(out, i, v);
        }
    return 0;
}

/* The primal-dual steps of PDOptCL::denoiseDiffusionTensorROF_PDD (PDOptCL.cpp:1114-1168, kernel
 * PDDROFDiffTensor.cl:43-127) or, with huber, denoiseDiffusionTensorHuber_PDD (PDOptCL.cpp:1170-1226,
 * kernel PDDHuberDiffTensor.cl:38-107): the Huber dual divides p + SIGMA DT du by 1 + SIGMA eps
 * and projects all four channels with one norm. */
static int pd_tensor(int huber, float eps, float* out, const float* input, const float* dt, const float lambda[4],
                     int iters, int W, int H)
{
    const float SIGMA = 4.0f, TAU = 0.05f, ETA = 8.0f, THETA = 0.5f;   /* PDDROFDiffTensor.cl:35-41 */
    const size_t N = (size_t)W * H;
    std::vector<float> u0(input, input + 4 * N), u1(4 * N);
    std::vector<float> p0(8 * N, 0.0f), p1(8 * N, 0.0f), q0(4 * N, 0.0f), q1(4 * N, 0.0f);
    const float lam[4] = {lambda[0], lambda[1], lambda[2], lambda[3]};
    std::vector<float>* ucur = &u0; std::vector<float>* unew = &u1;
    std::vector<float>* pcur = &p0; std::vector<float>* pnew = &p1;
    std::vector<float>* qcur = &q0; std::vector<float>* qnew = &q1;
    /* the host loop runs iters steps and, when the last one left the result in the
     * scratch image (iters odd, or 0), one more (PDOptCL.cpp:1137-1166) */
    const int steps = (iters > 0 && iters % 2 == 0) ? iters : iters + 1;
    for (int it = 0; it < steps; it++) {
        const Img4 U = {ucur->data(), W, H}, DT = {dt, W, H}, IMG = {input, W, H}, Q = {qcur->data(), W, H};
        const Img4 P = {pcur->data(), 2 * W, H};
        /* projected, tensor-weighted dual at pixel (x, y), zero outside (PDDROFDiffTensor.cl:72-100) */
        auto dual = [&](int x, int y, F4& lo, F4& hi) {
            const F4 uc = U.edge(x, y), ux = U.edge(x + 1, y), uy = U.edge(x, y + 1);
            const F4 D = DT.zero(x, y);
            const float dxv[4] = {uc.x - ux.x, uc.y - ux.y, uc.z - ux.z, uc.w - ux.w};
            const float dyv[4] = {uc.x - uy.x, uc.y - uy.y, uc.z - uy.z, uc.w - uy.w};
            const F4 plo = P.zero(2 * x, y), phi = P.zero(2 * x + 1, y);
            const float pl[4] = {plo.x, plo.y, plo.z, plo.w}, ph[4] = {phi.x, phi.y, phi.z, phi.w};
            float a[4], b[4], nrm[4];
            const float den = 1.0f + SIGMA * eps;
            for (int c = 0; c < 4; c++) {
                const float DTdx = D.x * dxv[c] + D.z * dyv[c];
                const float DTdy = D.y * dxv[c] + D.w * dyv[c];
                a[c] = pl[c] + SIGMA * DTdx;
                b[c] = ph[c] + SIGMA * DTdy;
                if (huber) {
                    a[c] = a[c] / den;
                    b[c] = b[c] / den;
                }
                nrm[c] = a[c] * a[c] + b[c] * b[c];
            }
            float pr[4];
            if (huber) {
                const float n = sqrtf(nrm[0] * 1.0f + nrm[1] * 1.0f + nrm[2] * 1.0f + nrm[3] * 1.0f);
                pr[0] = pr[1] = pr[2] = pr[3] = fmaxf(1.0f, n);
            } else {
                const float n3 = sqrtf(nrm[0] * 1.0f + nrm[1] * 1.0f + nrm[2] * 1.0f);
                const float n4 = sqrtf(nrm[3]);
                pr[0] = pr[1] = pr[2] = fmaxf(1.0f, n3);
                pr[3] = fmaxf(1.0f, n4);
            }
            float l[4], h[4];
            for (int c = 0; c < 4; c++) {
                a[c] = a[c] / pr[c];
                b[c] = b[c] / pr[c];
                l[c] = D.x * a[c] + D.z * b[c];
                h[c] = D.y * a[c] + D.w * b[c];
            }
            lo = f4(l[0], l[1], l[2], l[3]);
            hi = f4(h[0], h[1], h[2], h[3]);
        };
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                F4 lo, hi, llo, lhi, tlo, thi;
                dual(x, y, lo, hi);
                dual(x - 1, y, llo, lhi);
                dual(x, y - 1, tlo, thi);
                const float div[4] = {lo.x - llo.x + hi.x - thi.x, lo.y - llo.y + hi.y - thi.y,
                                      lo.z - llo.z + hi.z - thi.z, lo.w - llo.w + hi.w - thi.w};
                const F4 im = IMG.at(x, y), q = Q.at(x, y), u = U.at(x, y);
                const float imv[4] = {im.x, im.y, im.z, im.w}, qv[4] = {q.x, q.y, q.z, q.w}, uv[4] = {u.x, u.y, u.z, u.w};
                float on[4], qn[4];
                for (int c = 0; c < 4; c++) {
                    float o = (uv[c] + TAU * (lam[c] * imv[c] - div[c] - qv[c])) / (1.0f + TAU * lam[c]);
                    o = o + THETA * (o - uv[c]);
                    float qq = (qv[c] + ETA * (o - imv[c])) / (1.0f + 4.0f * ETA / lam[c]);
                    qq = qq + THETA * (qq - qv[c]);
                    on[c] = o; qn[c] = qq;
                }
                const size_t i = (size_t)y * W + x;
                put4(unew->data(), i, f4(on[0], on[1], on[2], on[3]));
                put4(qnew->data(), i, f4(qn[0], qn[1], qn[2], qn[3]));
                put4(pnew->data(), (size_t)y * 2 * W + 2 * x, lo);
                put4(pnew->data(), (size_t)y * 2 * W + 2 * x + 1, hi);
            }
        std::swap(ucur, unew); std::swap(pcur, pnew); std::swap(qcur, qnew);
    }
    memcpy(out, ucur->data(), 4 * N * sizeof(float));
    return 0;
}

int orc_rof(float* out, const float* input, const float* dt, const float lambda[4], int iters, int W, int H)
{
    return pd_tensor(0, 0.0f, out, input, dt, lambda, iters, W, H);
}

int orc_huber(float* out, const float* input, const float* dt, const float lambda[4], float eps, int iters, int W, int H)
{
    return pd_tensor(1, eps, out, input, dt, lambda, iters, W, H);
}

/* float to int as an x86 truncating conversion does it (cvttss2si), which is what the
 * reference's implicit conversions compile to on the host: NaN and values outside the int
 * range give INT_MIN */
static inline int f2i_x86(float f)
{
    if (!(f > -2147483904.0f && f < 2147483648.0f)) return INT32_MIN;
    return (int)f;
}

/* pmhstereo_fill_state (pmhstereo.cl:1131-1185): planes with a negative cost, or a disparity
 * outside [0, W], take the nearer-disparity valid neighbour of their row; the result as
 * (normal, depth * dispscale) of the reference view */
int orc_fill_state(float* out, const float* planes, int W, int H, float dispscale, int lr)
{
    const Img4 P = {planes, W, H};
    const int sidesign = lr ? -1 : 1;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const F4 state = P.at(x, y);
            const float cx = (float)x, cy = (float)y;
            const float disp = (transform_x(state, cx, cy) - cx) * (float)sidesign;
            F4 val;
            if (state.w < 0 || disp < 0 || disp > (float)W) {
                F4 l = f4(-1.0f, -1.0f, -1.0f, -1.0f), r = f4(-1.0f, -1.0f, -1.0f, -1.0f);
                for (int xx = x - 1; l.w < 0 && xx >= 0; xx--) l = P.at(xx, y);
                for (int xx = x + 1; r.w < 0 && xx < W; xx++) r = P.at(xx, y);
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
            if (!(isfin(val.x) && isfin(val.y))) { val.x = 0.0f; val.y = 0.0f; }
            F4 nd = to_ref_normal_depth(val, cx, cy, lr);
            nd.w = nd.w * dispscale;
            put4(out, (size_t)y * W + x, nd);
        }
    return 0;
}

int orc_consistency(float* out, const float* left, const float* right, int W, int H, float maxdispdiff, float maxanglediff)
{
    const Img4 R = {right, W, H};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            const F4 sl = f4(left[4 * i], left[4 * i + 1], left[4 * i + 2], left[4 * i + 3]);
            const float c2x = transform_x(sl, (float)x, (float)y), c2y = (float)y;
            F4 val = f4(0.0f, 0.0f, 0.0f, -1.0f);
            if (ceilf(c2x) >= 0 && floorf(c2x) < (float)W) {
                const F4 sr = R.edge(convert_int_rte(floorf(c2x)), y);
                const F4 sr2 = R.edge(convert_int_rte(ceilf(c2x)), y);
                const F3 nl = to_normal(sl);
                const float nd = dot3(nl, to_normal(viewprop(sr)));
                const float nd2 = dot3(nl, to_normal(viewprop(sr2)));
                const float d1 = fabsf((float)x - transform_x(sr, c2x, c2y));
                const float d2 = fabsf((float)x - transform_x(sr2, c2x, c2y));
                const float lim = maxanglediff / 180.0f;
                if (!(d1 >= maxdispdiff || orc_acospif(clampf(nd, -1.0f, 1.0f)) >= lim) ||
                    !(d2 >= maxdispdiff || orc_acospif(clampf(nd2, -1.0f, 1.0f)) >= lim))
                    val = sl;
            }
            put4(out, i, val);
        }
    return 0;
}

static inline float length3(F3 v) { return sqrtf(dot3(v, v)); }

int orc_to_disparity(float* out, const float* planes, int W, int H, float scale, int lr)
{
    const float sidesign = lr ? -1.0f : 1.0f;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            const F4 s = f4(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], planes[4 * i + 3]);
            const float disp = (transform_x(s, (float)x, (float)y) - (float)x) * sidesign;
            float v;
            if (length3(xyz(s)) < 1e-4f || disp < 0 || disp > (float)W) v = 0.0f;
            else v = fmaxf(disp, 0.0f);
            out[i] = v * scale;
        }
    return 0;
}

int orc_fill_depthmap(float* out, const float* planes, int W, int H, float scale)
{
    const Img4 P = {planes, W, H};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const F4 s = P.at(x, y);
            const float cx = (float)x, cy = (float)y;
            float v;
            if (length3(xyz(s)) < 1e-4f) {
                F4 l = f4(0, 0, 0, 0);
                for (int xx = x - 1; length3(xyz(l)) < 1e-1f && xx >= 0; xx--) l = P.at(xx, y);
                F4 rr = f4(0, 0, 0, 0);
                for (int xx = x + 1; length3(xyz(rr)) < 1e-1f && xx < W; xx++) rr = P.at(xx, y);
                if (length3(xyz(l)) < 1e-1f) { l.x = l.y = l.z = -1e5f; }
                if (length3(xyz(rr)) < 1e-1f) { rr.x = rr.y = rr.z = -1e5f; }
                l.w = -(transform_x(l, cx, cy) - cx);
                rr.w = -(transform_x(rr, cx, cy) - cx);
                v = fminf(l.w, rr.w);
            } else {
                v = fabsf(transform_x(s, cx, cy) - cx);
            }
            out[(size_t)y * W + x] = v * scale;
        }
    return 0;
}

int orc_fill_normalmap(float* out, const float* planes, int W, int H, int lr)
{
    (void)lr;
    const Img4 P = {planes, W, H};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const F4 s = P.at(x, y);
            const float cx = (float)x, cy = (float)y;
            F3 n;
            if (length3(xyz(s)) < 1e-1f) {
                F4 l = f4(0, 0, 0, 0);
                for (int xx = x - 1; length3(xyz(l)) < 1e-1f && xx >= 0; xx--) l = P.at(xx, y);
                F4 rr = f4(0, 0, 0, 0);
                for (int xx = x + 1; length3(xyz(rr)) < 1e-1f && xx < W; xx++) rr = P.at(xx, y);
                if (length3(xyz(l)) < 1e-1f) { l.x = l.y = l.z = -1e5f; }
                if (length3(xyz(rr)) < 1e-1f) { rr.x = rr.y = rr.z = -1e5f; }
                l.w = -(transform_x(l, cx, cy) - cx);
                rr.w = -(transform_x(rr, cx, cy) - cx);
                n = (l.w < rr.w) ? to_normal(l) : to_normal(rr);
            } else {
                n = to_normal(s);
            }
            put4(out, (size_t)y * W + x, f4(n.x, n.y, n.z, 0.0f));
        }
    return 0;
}

int orc_disparity_to_normal(float* out, const float* disp, int W, int H)
{
    auto d = [&](int x, int y) { return (x < 0 || x >= W || y < 0 || y >= H) ? 0.0f : disp[(size_t)y * W + x]; };
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const float dx = d(x + 1, y) - d(x, y);
            const float dy = d(x, y + 1) - d(x, y);
            /* cross((1,0,dx,0), (0,1,dy,0)) */
            const F3 n = f3(0.0f * dy - dx * 1.0f, dx * 0.0f - 1.0f * dy, 1.0f * 1.0f - 0.0f * 0.0f);
            const F3 nn = normalize3(n);
            put4(out, (size_t)y * W + x, f4(nn.x, nn.y, nn.z, 0.0f));
        }
    return 0;
}

/* Linear sampler, CLK_ADDRESS_CLAMP_TO_EDGE, unnormalised coordinates (OpenCL 1.2 s8.2) in
 * FP32 at a general 2-D point: t = c - 0.5, i0 = floor(t), a = t - floor(t) per axis;
 * T = (1-a)(1-b) T00 + a(1-b) T10 + (1-a)b T01 + ab T11, each weight one product, summed
 * left to right.  fetch(x, y) returns the texel with clamped coordinates. */
extern "C++" {
template <class Fetch>
static F4 sample_linear(Fetch fetch, int w, int h, float cx, float cy)
{
    const float tu = cx - 0.5f, tv = cy - 0.5f;
    const float fu = floorf(tu), fv = floorf(tv);
    const float a = tu - fu, b = tv - fv;
    auto ci = [](float f, int n) { return f < -2.0f ? -2 : (f > (float)n + 1.0f ? n + 1 : (int)f); };
    const int i0 = ci(fu, w), j0 = ci(fv, h);
    auto cl = [](int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); };
    const F4 T00 = fetch(cl(i0, w), cl(j0, h)), T10 = fetch(cl(i0 + 1, w), cl(j0, h));
    const F4 T01 = fetch(cl(i0, w), cl(j0 + 1, h)), T11 = fetch(cl(i0 + 1, w), cl(j0 + 1, h));
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
    return f4(w00 * T00.x + w10 * T10.x + w01 * T01.x + w11 * T11.x, w00 * T00.y + w10 * T10.y + w01 * T01.y + w11 * T11.y,
              w00 * T00.z + w10 * T10.z + w01 * T01.z + w11 * T11.z, w00 * T00.w + w10 * T10.w + w01 * T01.w + w11 * T11.w);
}
}  // extern "C++"

/* write_imagef to a CL_UNORM_INT8 channel: convert_uchar_sat_rte(v * 255) (OpenCL 1.2 s8.3.1.1) */
static uint8_t unorm8(float v)
{
    const float x = v * 255.0f;
    if (!(x > 0.0f)) return 0;
    if (x >= 255.0f) return 255;
    return (uint8_t)rintf(x);
}

/* pyrdown (cvt/cl/kernel/pyr/pyrdown.cl) as CLPyramid::pyrDown runs it (cvt/cl/CLPyramid.cpp:73-78):
 * RGBA8 in (Wi x Hi, tight rows) -> RGBA8 out (Wo x Ho), each output pixel the linear sample
 * at (Wi/Wo * (x + 0.5), Hi/Ho * (y + 0.5)) */
int orc_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, int Wi, int Hi)
{
    const float incx = (float)Wi / (float)Wo, incy = (float)Hi / (float)Ho;
    auto fetch = [&](int x, int y) {
        const uint8_t* p = in + 4 * ((size_t)y * Wi + x);
        return f4((float)p[0] / 255.0f, (float)p[1] / 255.0f, (float)p[2] / 255.0f, (float)p[3] / 255.0f);
    };
#pragma omp parallel for schedule(static)
    for (int y = 0; y < Ho; y++)
        for (int x = 0; x < Wo; x++) {
            const F4 v = sample_linear(fetch, Wi, Hi, incx * ((float)x + 0.5f), incy * ((float)y + 0.5f));
            uint8_t* o = out + 4 * ((size_t)y * Wo + x);
            o[0] = unorm8(v.x); o[1] = unorm8(v.y); o[2] = unorm8(v.z); o[3] = unorm8(v.w);
        }
    return 0;
}

/* pyrup_mul4f (cvt/cl/kernel/pyr/pyrupmul.cl) as PMHuberStereo::pyrUpMul runs it
 * (PMHuberStereo.cpp:709-721): out = mul * linear sample at (Wi/Wo * (x + 0.5), Hi/Ho * (y + 0.5)),
 * per component; channels 1 (a grey float image, the sample's .x) or 4 */
int orc_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, const float mul[4])
{
    if (channels != 1 && channels != 4) return -1;
    const float incx = (float)Wi / (float)Wo, incy = (float)Hi / (float)Ho;
    auto fetch = [&](int x, int y) {
        const size_t i = (size_t)y * Wi + x;
        if (channels == 1) return f4(in[i], in[i], in[i], in[i]);
        return f4(in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]);
    };
#pragma omp parallel for schedule(static)
    for (int y = 0; y < Ho; y++)
        for (int x = 0; x < Wo; x++) {
            const F4 v = sample_linear(fetch, Wi, Hi, incx * ((float)x + 0.5f), incy * ((float)y + 0.5f));
            const size_t i = (size_t)y * Wo + x;
            if (channels == 1) {
                out[i] = mul[0] * v.x;
            } else {
                out[4 * i] = mul[0] * v.x; out[4 * i + 1] = mul[1] * v.y;
                out[4 * i + 2] = mul[2] * v.z; out[4 * i + 3] = mul[3] * v.w;
            }
        }
    return 0;
}

/* ---- VPMStereoCL (cvt/vision/VPMStereoCL.cpp, cvt/cl/kernel/VPMStereo.cl) ------------- */
/* A simpler slanted-plane PatchMatch on one view: states (a, b, c) with x' = a x + b y + c,
 * van der Corput candidates, eight fixed neighbour offsets, three Gauss-Newton steps. */

/* grad_gray_xydiag (cvt/cl/kernel/gradxy.cl): central grey differences with a zero border
 * (CLK_ADDRESS_CLAMP); the diagonal channels repeat them */
int orc_vpm_grad(float* out, const uint8_t* img, int W, int H, int stride)
{
    const std::vector<float> f = rgba8_to_float(img, W, H, stride);
    const Img4 src = {f.data(), W, H};
    auto gray = [&](int x, int y) { return dot3(xyz(src.zero(x, y)), f3(GW_R, GW_G, GW_B)); };
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const float dx = gray(x + 1, y) - gray(x - 1, y), dy = gray(x, y + 1) - gray(x, y - 1);
            put4(out, (size_t)y * W + x, f4(dx, dy, dx, dy));
        }
    return 0;
}

static inline float vdc2(uint32_t v)   /* vpmsstate_vanDerCorput2 (VPMStereo.cl:47-55): bit reversal * 2^-32 */
{
    v = (v << 16) | (v >> 16);
    v = ((v & 0x55555555u) << 1) | ((v & 0xAAAAAAAAu) >> 1);
    v = ((v & 0x33333333u) << 2) | ((v & 0xCCCCCCCCu) >> 2);
    v = ((v & 0x0F0F0F0Fu) << 4) | ((v & 0xF0F0F0F0u) >> 4);
    v = ((v & 0x00FF00FFu) << 8) | ((v & 0xFF00FF00u) >> 8);
    return 2.3283064365386963e-10f * (float)v;
}

/* vpmsstate_from_disparity_normal with normal (0, 0, 1) (:57-61, :63-66) */
static inline F3 vpm_fronto(float cx, float cy, float d)
{
    const F3 n = f3(0.0f, 0.0f, 1.0f);
    return f3(1.0f - (-n.x / n.z), 0.0f - (-n.y / n.z), 0.0f - ((n.x * cx + n.y * cy) / n.z + d));
}

struct VpmViews {
    Img4 c1, g1, c2, g2;   /* colours as floats, gradients */
    int W, H, r;
};

/* patch_eval_census of VPMStereo.cl (:203-256): no early exit */
static float vpm_eval(const VpmViews& V, int px, int py, F3 s)
{
    const float cx = (float)px, cy = (float)py;
    const float alpha = 0.05f;
    const float c2x = s.x * cx + s.y * cy + s.z;
    if (c2x < 0 || c2x >= (float)V.W) return 1.0f;
    const F3 valc1 = xyz(V.c1.at(px, py));
    float wsum = 0.0f, census = 0.0f;
    for (int dy = -V.r; dy <= V.r; dy++)
        for (int dx = -V.r; dx <= V.r; dx++) {
            const float qx = cx + (float)dx * 1.0f, qy = cy + (float)dy * 1.0f;
            const float p2x = s.x * qx + s.y * qy + s.z;
            if (p2x < 0 || p2x >= (float)V.W || qx < 0 || qx >= (float)V.W || qy < 0 || qy >= (float)V.H) continue;
            const int ix = px + dx, iy = py + dy;
            const F3 valin = xyz(V.c1.at(ix, iy));
            const F3 val1 = f3(valin.x - valc1.x, valin.y - valc1.y, valin.z - valc1.z);
            const float w = orc_expf(-fabsf(dot3(val1, f3(GW_R, GW_G, GW_B))) * 8.0f);
            const F4 v2 = lerp_row(0, V.c2, p2x + 0.5f, iy);
            const float ccx = fminf(fabsf(v2.x - valin.x), 0.05f) / 0.05f;
            const float ccy = fminf(fabsf(v2.y - valin.y), 0.05f) / 0.05f;
            const float ccz = fminf(fabsf(v2.z - valin.z), 0.05f) / 0.05f;
            census += w * alpha * 0.33f * (ccx + ccy + ccz);
            const F4 gval1 = V.g1.at(ix, iy);
            const F4 gval2 = lerp_row(0, V.g2, p2x + 0.5f, iy);
            census += w * (1.0f - alpha) * 0.25f * (float)popc4(signbits4(gval1) ^ signbits4(gval2));
            wsum += w;
        }
    return census / wsum;
}

/* patch_census_klt of VPMStereo.cl (:113-201): every sample updates J and H (no curvature test) */
static F3 vpm_klt(const VpmViews& V, int px, int py, F3 s)
{
    const float cx = (float)px, cy = (float)py;
    const float alpha = 0.05f;
    float J[3] = {0, 0, 0};
    float Hm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    const F3 valc1 = xyz(V.c1.at(px, py));
    for (float dy = (float)-V.r; dy <= (float)V.r; dy += 1.0f)
        for (float dx = (float)-V.r; dx <= (float)V.r; dx += 1.0f) {
            const float qx = cx + dx * 1.0f, qy = cy + dy * 1.0f;
            if (qx < 0 || qx >= (float)V.W || qy < 0 || qy >= (float)V.H) continue;
            const int ix = (int)qx, iy = (int)qy;
            const F3 valin = xyz(V.c1.at(ix, iy));
            const F3 val1 = f3(valin.x - valc1.x, valin.y - valc1.y, valin.z - valc1.z);
            const F4 gval1 = V.g1.at(ix, iy);
            const float w1 = orc_expf(-fabsf(dot3(val1, f3(GW_R, GW_G, GW_B))) * 8.0f);
            const float p2x = s.x * qx + s.y * qy + s.z;
            if (qx < 1 || qx >= (float)(V.W - 1)) continue;
            const uint32_t sg1 = signbits4(gval1);
            float C3[3];
            const float us[3] = {p2x + 0.5f, (p2x + 1.0f) + 0.5f, (p2x + -1.0f) + 0.5f};
            for (int k = 0; k < 3; k++) {
                const F4 v2 = lerp_row(0, V.c2, us[k], iy);
                const float ccx = fminf(fabsf(v2.x - valin.x), 0.05f) / 0.05f;
                const float ccy = fminf(fabsf(v2.y - valin.y), 0.05f) / 0.05f;
                const float ccz = fminf(fabsf(v2.z - valin.z), 0.05f) / 0.05f;
                float C = w1 * alpha * 0.33f * (ccx + ccy + ccz);
                const F4 g2 = lerp_row(0, V.g2, us[k], iy);
                /* 0.25 is a double literal: the sum is formed in double and rounded once */
                C = (float)((double)C + (double)(w1 * (1.0f - alpha)) * 0.25 * (double)(float)popc4(sg1 ^ signbits4(g2)));
                C3[k] = C;
            }
            const float C = C3[0], Cxp = C3[1], Cxm = C3[2];
            const float p[3] = {qx, qy, 1.0f};
            const float t = w1 * (Cxm - Cxp) * 0.5f;
            const float sc = w1 * (Cxp + Cxm - 2.0f * C);
            for (int i = 0; i < 3; i++) J[i] = J[i] + t * p[i];
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) Hm[i][j] = Hm[i][j] + sc * (p[i] * p[j]);
        }
    const F3 d = lusolve(Hm, f3(J[0], J[1], J[2]));
    return f3(s.x - d.x, s.y - d.y, s.z - d.z);
}

/* vpmstereo_init / vpmstereo_init_disparity (VPMStereo.cl:258-309): initdisp NULL for the
 * first; the van der Corput index is x * W + y as the source forms it */
int orc_vpm_init(float* out, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2, int W, int H,
                 int stride, int r, float dmax, const float* initdisp)
{
    const std::vector<float> f1 = rgba8_to_float(c1, W, H, stride), f2 = rgba8_to_float(c2, W, H, stride);
    const VpmViews V = {{f1.data(), W, H}, {g1, W, H}, {f2.data(), W, H}, {g2, W, H}, W, H, r};
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const float cx = (float)x, cy = (float)y;
            F3 st;
            const float d = initdisp ? initdisp[(size_t)y * W + x] : -1.0f;
            if (initdisp && d >= 0 && d < dmax) st = vpm_fronto(cx, cy, d);
            else st = vpm_fronto(cx, cy, vdc2((uint32_t)x * (uint32_t)W + (uint32_t)y) * dmax);
            put4(out, (size_t)y * W + x, f4(st.x, st.y, st.z, vpm_eval(V, x, y, st)));
        }
    return 0;
}

/* vpmstereo_iter_simple (VPMStereo.cl:311-356) */
int orc_vpm_iter(float* out, const float* in, const uint8_t* c1, const float* g1, const uint8_t* c2,
                 const float* g2, int W, int H, int stride, int r, float dmax, int iter)
{
    const std::vector<float> f1 = rgba8_to_float(c1, W, H, stride), f2 = rgba8_to_float(c2, W, H, stride);
    const VpmViews V = {{f1.data(), W, H}, {g1, W, H}, {f2.data(), W, H}, {g2, W, H}, W, H, r};
    const Img4 I = {in, W, H};
    static const int off[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {16, 0}, {-16, 0}, {0, 16}, {0, -16}};
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const float cx = (float)x, cy = (float)y;
            F4 cur = I.at(x, y);
            F3 st = vpm_fronto(cx, cy, vdc2((uint32_t)((x & 7) * (y & 7)) + (uint32_t)iter) * dmax);
            float cost = vpm_eval(V, x, y, st);
            if (cost < cur.w) cur = f4(st.x, st.y, st.z, cost);
            for (int i = 0; i < 8; i++) {
                const int* o = off[(iter + i) & 7];
                st = xyz(I.edge(x + o[0], y + o[1]));
                cost = vpm_eval(V, x, y, st);
                if (cost < cur.w) cur = f4(st.x, st.y, st.z, cost);
            }
            st = vpm_klt(V, x, y, xyz(cur));
            for (int k = 0; k < 2; k++) st = vpm_klt(V, x, y, st);
            cost = vpm_eval(V, x, y, st);
            if (cost < cur.w) cur = f4(st.x, st.y, st.z, cost);
            put4(out, (size_t)y * W + x, cur);
        }
    return 0;
}

/* vpmstereo_disparity (VPMStereo.cl:358-373): |x' - x| * scale */
int orc_vpm_disparity(float* out, const float* states, int W, int H, float scale)
{
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            const float cx = (float)x, cy = (float)y;
            out[i] = fabsf(states[4 * i] * cx + states[4 * i + 1] * cy + states[4 * i + 2] - cx) * scale;
        }
    return 0;
}

/* VPMStereoCL::disparitySimple (cvt/vision/VPMStereoCL.cpp:54-85) without its debugging block
 * (:74-81: a PNG of every iterate and a wait for a key press; no result depends on it).  The
 * states ping-pong: init writes out1, iteration i reads out[1 - swap] and writes out[swap]. */
int orc_vpm_disparity_simple(float* disparity, float* states, const uint8_t* c1, const uint8_t* c2, int W, int H,
                             int stride, int r, int iterations, float dmax, const float* initdisp)
{
    const size_t N = (size_t)W * H;
    std::vector<float> g1(4 * N), g2(4 * N), s0(4 * N), s1(4 * N);
    orc_vpm_grad(g1.data(), c1, W, H, stride);
    orc_vpm_grad(g2.data(), c2, W, H, stride);
    float* out[2] = {s0.data(), s1.data()};
    orc_vpm_init(out[1], c1, g1.data(), c2, g2.data(), W, H, stride, r, dmax, initdisp);
    int swap = 0;
    for (int i = 0; i < iterations; i++) {
        orc_vpm_iter(out[swap], out[1 - swap], c1, g1.data(), c2, g2.data(), W, H, stride, r, dmax, i);
        swap = 1 - swap;
    }
    orc_vpm_disparity(disparity, out[1 - swap], W, H, 1.0f);
    if (states) memcpy(states, out[1 - swap], 4 * N * sizeof(float));
    return 0;
}

/* ---- SVPMFlowCL (cvt/vision/SVPMFlowCL.cpp, cvt/cl/kernel/SVPMFlow.cl) --------------------
 * PatchMatch optical flow: a state is (u, v, cost, 0); candidates are tested against a
 * quadratic pull towards a TV-smoothed flow (a primal-dual step on a dual field p, ADMM
 * style).  The kernel works on 16x16 work-groups with the states of the group and a 4-pixel
 * apron in local memory; the neighbour tests of a group see each other's updates. */

/* read_imagef with SAMPLER_BILINEAR (CLK_ADDRESS_CLAMP_TO_EDGE) at (u, v), OpenCL 1.2 s8.2:
 * the four weights (1-a)(1-b), a(1-b), (1-a)b, ab and the sum in that order */
static F4 bilinear2d(const Img4& im, float u, float v)
{
    if (!isfin(u) || !isfin(v)) { const float n = orc_bits2f(0x7fffffffu); return f4(n, n, n, n); }
    const float tu = u - 0.5f, tv = v - 0.5f;
    const float fu = floorf(tu), fv = floorf(tv);
    const float a = tu - fu, b = tv - fv;
    const int i0 = (int)fminf(fmaxf(fu, -2.0f), (float)im.W + 1.0f), j0 = (int)fminf(fmaxf(fv, -2.0f), (float)im.H + 1.0f);
    const F4 T00 = im.edge(i0, j0), T10 = im.edge(i0 + 1, j0), T01 = im.edge(i0, j0 + 1), T11 = im.edge(i0 + 1, j0 + 1);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
    return f4(((w00 * T00.x + w10 * T10.x) + w01 * T01.x) + w11 * T11.x,
              ((w00 * T00.y + w10 * T10.y) + w01 * T01.y) + w11 * T11.y,
              ((w00 * T00.z + w10 * T10.z) + w01 * T01.z) + w11 * T11.z,
              ((w00 * T00.w + w10 * T10.w) + w01 * T01.w) + w11 * T11.w);
}

/* svpmflow_eval_bilateral_trunc_sad (SVPMFlow.cl:170-209), the cost svpmflow_eval names (:211) */
static float svpm_eval(const Img4& c1, const Img4& c2, float cx, float cy, float fx, float fy, int r)
{
    if (!(isfin(fx) && isfin(fy))) return 1e10f;
    const int W = c2.W, H = c2.H;
    const F4 vc = bilinear2d(c1, cx + 0.5f, cy + 0.5f);
    float ret = 0.0f, wsum = 0.0f;
    for (float dy = (float)-r; dy <= (float)r; dy += 1.0f)
        for (float dx = (float)-r; dx <= (float)r; dx += 1.0f) {
            const float px = cx + dx, py = cy + dy;
            const float qx = px + fx, qy = py + fy;
            if (px < 0 || px >= W || py < 0 || py >= H || qx < 0 || qx >= W || qy < 0 || qy >= H) continue;
            const F4 v1 = bilinear2d(c1, px + 0.5f, py + 0.5f);
            const F4 v2 = bilinear2d(c2, qx + 0.5f, qy + 0.5f);
            const float w = orc_expf(-((fabsf(vc.x - v1.x) * 1.0f + fabsf(vc.y - v1.y) * 1.0f) + fabsf(vc.z - v1.z) * 1.0f) * 2.6f);
            wsum += w;
            ret += w * ((fminf(fabsf(v1.x - v2.x), 0.02f) * 1.0f + fminf(fabsf(v1.y - v2.y), 0.02f) * 1.0f) +
                        fminf(fabsf(v1.z - v2.z), 0.02f) * 1.0f);
        }
    if (wsum < 1.1f) return 1e5f;
    return ret / wsum;
}

/* box_mueller (:38-46): theta = 2.0f * M_PI * y is formed in double (M_PI is a double) */
static void svpm_box_mueller(Rng& g, float* bx, float* by)
{
    const float x = g.next(), y = g.next();
    const float rr = sqrtf(-2.0f * orc_logf(x));
    const float theta = (float)(2.0 * M_PI * (double)y);
    *bx = rr * orc_sinf(theta);
    *by = rr * orc_cosf(theta);
}

/* svpmflow_state_init (:48-56) */
static F4 svpm_state_init(Rng& g, float flowmax)
{
    float bx, by;
    svpm_box_mueller(g, &bx, &by);
    return f4(bx * flowmax * 0.5f, by * flowmax * 0.5f, 1e10f, 0.0f);
}

/* svpmflow_state_refine (:58-64).  Its `ret` is read before it is written (`ret.xy += ...`);
 * it is taken as zero, the value-initialised vector of the reference kernels' host build, so
 * the candidate is a small flow around zero */
static F4 svpm_state_refine(Rng& g, float refinemax)
{
    float bx, by;
    svpm_box_mueller(g, &bx, &by);
    return f4(0.0f + bx * refinemax * 0.5f, 0.0f + by * refinemax * 0.5f, 1e10f, 0.0f);
}

/* RNG_init(&rng, linpos, 2 * (NUMRNDTRIES) * iter): the macro does not parenthesise its
 * third argument, so the distance is the int product linpos * 2 * 2 * iter (RNG.cl:54-57) */
static int32_t svpm_skip(int linpos, int factor) { return (int32_t)((uint32_t)linpos * (uint32_t)factor); }

/* the flow images of both frames, RGBA8 read as k / 255 */
struct SvpmFrames {
    std::vector<float> f1, f2;
    Img4 c1, c2;
    SvpmFrames(const uint8_t* a, const uint8_t* b, int W, int H, int stride)
        : f1(rgba8_to_float(a, W, H, stride)), f2(rgba8_to_float(b, W, H, stride))
    {
        c1 = {f1.data(), W, H};
        c2 = {f2.data(), W, H};
    }
};

/* svpmflow_init (:213-233) */
int orc_svpm_init(float* out, const uint8_t* img1, const uint8_t* img2, int W, int H, int stride, int r, float flowmax)
{
    const SvpmFrames F(img1, img2, W, H, stride);
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            Rng g;
            g.init_skip(svpm_skip(y * W + x, 2));
            F4 st = svpm_state_init(g, flowmax);
            st.z = svpm_eval(F.c1, F.c2, (float)x, (float)y, st.x, st.y, r);
            put4(out, (size_t)y * W + x, st);
        }
    return 0;
}

/* svpmflow_prop_local_tv_admm (:574-731), one 16x16 work-group at a time.  The neighbour
 * tests (:673-690) read a neighbour's cell of the group buffer while that neighbour may be
 * writing it in the same barrier interval; here every test reads the cells as they were at
 * the interval's start (all reads of a step happen before its writes). */
int orc_svpm_prop(float* out, float* pout, const float* in, const float* pin, const uint8_t* img1,
                  const uint8_t* img2, int W, int H, int stride, int r, float flowmax, int iter)
{
    const SvpmFrames F(img1, img2, W, H, stride);
    const Img4 I = {in, W, H}, P = {pin, W, H};
    const int GX = (W + 15) / 16, GY = (H + 15) / 16;
    const float tau = 0.1f, lambda0 = 0.01f;
#pragma omp parallel for schedule(dynamic, 1)
    for (int gid = 0; gid < GX * GY; gid++) {
        const int gx = gid % GX, gy = gid / GX;
        const int bx = gx * 16 - 4, by = gy * 16 - 4, bpx = gx * 16 - 1, bpy = gy * 16 - 1;
        static thread_local F4 buf[24][24], bufp[18][18];
        for (int y = 0; y < 24; y++)
            for (int x = 0; x < 24; x++) buf[y][x] = I.edge(bx + x, by + y);
        for (int y = 0; y < 18; y++)
            for (int x = 0; x < 18; x++) {
                const F4 p = P.zero(bpx + x, bpy + y);
                const F4 A = buf[y + 3][x + 3], Bx = buf[y + 3][x + 4], By = buf[y + 4][x + 3];
                const float dxx = Bx.x - A.x, dxy = Bx.y - A.y, dyx = By.x - A.x, dyy = By.y - A.y;
                const F4 z = f4(p.x + dxx, p.y + dxy, p.z + dyx, p.w + dyy);
                const float zx = fmaxf(0.0f, 1.0f - tau / fmaxf(sqrtf(z.x * z.x + z.y * z.y), 1e-10f));
                const float zy = fmaxf(0.0f, 1.0f - tau / fmaxf(sqrtf(z.z * z.z + z.w * z.w), 1e-10f));
                const F4 pn = f4((p.x + dxx) - z.x * zx, (p.y + dxy) - z.y * zx, (p.z + dyx) - z.z * zy,
                                 (p.w + dyy) - z.w * zy);
                bufp[y][x] = f4(pn.x + 0.5f * (pn.x - p.x), pn.y + 0.5f * (pn.y - p.y), pn.z + 0.5f * (pn.z - p.z),
                                pn.w + 0.5f * (pn.w - p.w));
            }
        F4 ret[16][16], pw[16][16];
        float curx[16][16], cury[16][16];
        Rng g[16][16];
        const float lam = iter < 5 ? 0.0f : 1.0f / (2.0f * lambda0 * 5.0f);
        auto test = [&](int lx, int ly, float nx, float ny, float cost) {
            F4& R = ret[ly][lx];
            const float cx = curx[ly][lx], cy = cury[ly][lx];
            const float an = nx - cx, bn = ny - cy, ar = R.x - cx, br = R.y - cy;
            if (cost + lam * (an * an + bn * bn) < R.z + lam * (ar * ar + br * br)) {
                R.x = nx;
                R.y = ny;
                R.z = cost;
            }
        };
        for (int ly = 0; ly < 16; ly++)
            for (int lx = 0; lx < 16; lx++) {
                const int x = gx * 16 + lx, y = gy * 16 + ly;
                const float fx = (float)x, fy = (float)y;
                g[ly][lx].init_skip(svpm_skip(y * W + x, 2 * 2 * iter));
                const F4 p = iter < 5 ? f4(0.0f, 0.0f, 0.0f, 0.0f) : bufp[ly + 1][lx + 1];
                const F4 L = bufp[ly + 1][lx], U = bufp[ly][lx + 1];
                const float divx = ((p.x - L.x) + p.z) - U.z, divy = ((p.y - L.y) + p.w) - U.w;
                pw[ly][lx] = p;
                ret[ly][lx] = buf[ly + 4][lx + 4];
                curx[ly][lx] = ret[ly][lx].x + (lambda0 / tau) * divx;
                cury[ly][lx] = ret[ly][lx].y + (lambda0 / tau) * divy;
                test(lx, ly, curx[ly][lx], cury[ly][lx], svpm_eval(F.c1, F.c2, fx, fy, curx[ly][lx], cury[ly][lx], r));
                for (int k = 0; k < 2; k++) {   /* random tries (:637-645) */
                    const F4 n = svpm_state_init(g[ly][lx], flowmax);
                    test(lx, ly, n.x, n.y, svpm_eval(F.c1, F.c2, fx, fy, n.x, n.y, r));
                }
                for (int k = 0; k < 2; k++) {   /* random neighbours within 5 px (:648-656) */
                    const float rx = g[ly][lx].next();
                    const int ox = (int)((rx - 0.5f) * 2.0f * 5.0f + 0.5f);
                    const float ry = g[ly][lx].next();
                    const int oy = (int)((ry - 0.5f) * 2.0f * 5.0f + 0.5f);
                    const F4 n = I.edge(x + ox, y + oy);
                    test(lx, ly, n.x, n.y, svpm_eval(F.c1, F.c2, fx, fy, n.x, n.y, r));
                }
            }
        for (int ly = 0; ly < 16; ly++)
            for (int lx = 0; lx < 16; lx++) buf[ly + 4][lx + 4] = ret[ly][lx];
        /* jump steps 4, 2, 1 in the directions +x, +y, -x, -y (:668-694) */
        for (int step = 4; step >= 1; step >>= 1) {
            const int dirs[4][2] = {{step, 0}, {0, step}, {-step, 0}, {0, -step}};
            for (int d = 0; d < 4; d++) {
                for (int ly = 0; ly < 16; ly++)
                    for (int lx = 0; lx < 16; lx++) {
                        const F4 n = buf[(ly + 4 + dirs[d][1]) % 24][(lx + 4 + dirs[d][0]) % 24];
                        const float fx = (float)(gx * 16 + lx), fy = (float)(gy * 16 + ly);
                        test(lx, ly, n.x, n.y, svpm_eval(F.c1, F.c2, fx, fy, n.x, n.y, r));
                    }
                for (int ly = 0; ly < 16; ly++)
                    for (int lx = 0; lx < 16; lx++) buf[ly + 4][lx + 4] = ret[ly][lx];
            }
        }
        for (int ly = 0; ly < 16; ly++)
            for (int lx = 0; lx < 16; lx++) {
                const int x = gx * 16 + lx, y = gy * 16 + ly;
                for (int k = 0; k < 2; k++) {   /* random refinement (:700-708) */
                    const F4 n = svpm_state_refine(g[ly][lx], 1.0f);
                    test(lx, ly, n.x, n.y, svpm_eval(F.c1, F.c2, (float)x, (float)y, n.x, n.y, r));
                }
                if (x < W && y < H) {
                    put4(pout, (size_t)y * W + x, pw[ly][lx]);
                    put4(out, (size_t)y * W + x, ret[ly][lx]);
                }
            }
    }
    return 0;
}

/* svpmflow_flow (:733-744): (u, v) per pixel */
int orc_svpm_to_flow(float* flow, const float* states, int W, int H)
{
    for (size_t i = 0; i < (size_t)W * H; i++) {
        flow[2 * i] = states[4 * i];
        flow[2 * i + 1] = states[4 * i + 1];
    }
    return 0;
}

/* SVPMFlowCL::flow (SVPMFlowCL.cpp:58-89) with `iterations` passes (the reference runs MAXITER
 * = 200, :40) and without its debugging block (:74-84: AEE print, a colour-coded PNG and a wait
 * for a key press after every pass; no result depends on it).  states / duals (NULL: not
 * returned) get the final state and dual fields. */
int orc_svpm_flow(float* flow, float* states, float* duals, const uint8_t* img1, const uint8_t* img2, int W, int H,
                  int stride, int r, float flowmax, int iterations)
{
    const size_t N = (size_t)W * H;
    std::vector<float> s0(4 * N), s1(4 * N), p0(4 * N, 0.0f), p1(4 * N, 0.0f);
    float* buf[2] = {s0.data(), s1.data()};
    float* bufp[2] = {p0.data(), p1.data()};
    orc_svpm_init(buf[1], img1, img2, W, H, stride, r, flowmax);
    for (int i = 0; i < iterations; i++) {
        const int swap = i & 1;
        orc_svpm_prop(buf[swap], bufp[swap], buf[1 - swap], bufp[1 - swap], img1, img2, W, H, stride, r, flowmax, i + 1);
    }
    const int last = 1 - (iterations & 1);
    orc_svpm_to_flow(flow, buf[last], W, H);
    if (states) memcpy(states, buf[last], 4 * N * sizeof(float));
    if (duals) memcpy(duals, bufp[last], 4 * N * sizeof(float));
    return 0;
}

static const PmKernels ORC_KERNELS = {orc_prep, orc_init, orc_propagate, orc_normal_depth, orc_rof,
                                      orc_consistency, orc_to_disparity, orc_fill_depthmap, orc_fill_normalmap,
                                      orc_disparity_to_normal, orc_pyrdown, orc_pyrup_mul, orc_prep_raw,
                                      orc_fill_state, orc_huber};

int orc_disparity_map(const uint8_t* left, const uint8_t* right, int W, int H, int stride,
                      int r, float dmax, int iterations, int pp, int views,
                      float* dmap, float* normal, const float* initdisp, const float* initnormal,
                      float* planesL, float* planesR, int fused, int64_t* counters)
{
    return pm_host_disparity_map(ORC_KERNELS, left, right, W, H, stride, r, dmax, iterations, pp, views, 1, dmap,
                                 normal, initdisp, initnormal, planesL, planesR, fused, counters, nullptr, nullptr);
}

int orc_disparity_map_dump(const uint8_t* left, const uint8_t* right, int W, int H, int stride,
                           int r, float dmax, int iterations, int pp, int views, int levels,
                           float* dmap, float* normal, const float* initdisp, const float* initnormal,
                           float* planesL, float* planesR, int fused, int64_t* counters, PmDumpFn dump, void* user)
{
    return pm_host_disparity_map(ORC_KERNELS, left, right, W, H, stride, r, dmax, iterations, pp, views, levels,
                                 dmap, normal, initdisp, initnormal, planesL, planesR, fused, counters, dump, user);
}

int orc_depth_map_dump(const uint8_t* left, const uint8_t* right, int W, int H, int stride, int r, float dmax,
                       int iterations, float dscale, int pp, int views, float* dmap, float* normal,
                       const float* initdisp, const float* initnormal, float* planesL, float* planesR, int fused,
                       int64_t* counters, PmDumpFn dump, void* user)
{
    return pm_host_depth_map(ORC_KERNELS, left, right, W, H, stride, r, dmax, iterations, dscale, pp, views, dmap,
                             normal, initdisp, initnormal, planesL, planesR, fused, counters, dump, user);
}

}  // extern "C"
