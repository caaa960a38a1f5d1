// Deterministic FP32 arithmetic shared by the kernels and by their host-side
// self-test entry points.
//
// The reference kernels call OpenCL built-ins whose last bits are
// implementation-defined (exp, sin, cos, acospi, normalize, native_rsqrt;
// cvt/cl/kernel/pmhstereo.cl:86-91, :119, :355, :701, :1123).  This file fixes
// one choice inside OpenCL 1.2's error bounds, built only from IEEE add,
// multiply, fma, sqrt and divide so that host and device agree bit for bit:
//   exp     Cody-Waite reduction by ln2 (two-part constant), degree-7 Taylor
//           polynomial in Horner form, scaling through the exponent field
//           (max error 0.92 ulp on [-40, 0]);
//   sincos  Cody-Waite reduction by pi/2 (three-part constant), Taylor
//           polynomials of degree 9 / 10 on |r| <= pi/4 (1.42 ulp);
//   acospi  arcsine Maclaurin series on |x| <= 1/2, half-angle identity beyond
//           (2.4 ulp);
//   log     (SVPMFlow.cl:42) x = 2^k m, m in [sqrt(1/2), sqrt(2)], s = (m-1)/(m+1),
//           log(m) = 2 atanh(s) by its series to s^11, plus k ln2 (two-part).
// Build with -fmad=false (device) and -ffp-contract=off (host) so that only the
// explicit fmaf calls fuse.
#pragma once

#include <stdint.h>
#include <math.h>
#include <string.h>

#ifdef __CUDACC__
#define PM_HD __host__ __device__ __forceinline__
#else
#define PM_HD inline
#endif

namespace pm {

PM_HD float u2f(uint32_t u)
{
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}
PM_HD uint32_t f2u(float f)
{
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}

PM_HD float pow2i(int n) { return u2f((uint32_t)(n + 127) << 23); }

PM_HD float logf_(float x)
{
    if (x != x) return x;
    if (x < 0.0f) return (x - x) / (x - x);
    if (x == 0.0f) return u2f(0xff800000u);
    if (x == u2f(0x7f800000u)) return x;
    int k = 0;
    uint32_t u = f2u(x);
    if (u < 0x00800000u) {
        x *= 8388608.0f;
        k = -23;
        u = f2u(x);
    }
    k += (int)(u >> 23) - 127;
    u = (u & 0x007fffffu) | 0x3f800000u;
    if (u > 0x3fb504f3u) {
        u -= 0x00800000u;
        k += 1;
    }
    const float f = u2f(u) - 1.0f;
    const float s = f / (2.0f + f);
    const float z = s * s;
    // log(m) = f - (f^2/2 - s (f^2/2 + R)), R = 2 (z/3 + ... + z^5/11) (fdlibm's e_log.c form)
    float R = 1.8181819e-1f;               /* 2/11 */
    R = fmaf(R, z, 2.2222222e-1f);
    R = fmaf(R, z, 2.8571430e-1f);
    R = fmaf(R, z, 4.0000001e-1f);
    R = fmaf(R, z, 6.6666669e-1f);
    R = R * z;
    const float hfsq = (0.5f * f) * f;
    const float kf = (float)k;
    const float lo = fmaf(s, hfsq + R, kf * 1.428606765330187045e-06f);
    return fmaf(kf, 0.693145751953125f, f - (hfsq - lo));
}

PM_HD float expf_(float x)
{
    if (x != x) return x;
    if (x > 88.72283935546875f) return u2f(0x7f800000u);
    if (x < -103.97208404541015625f) return 0.0f;
    const float n = rintf(x * 1.44269502162933349609375f);
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
    const int ni = (int)n;
    if (ni > 127) return (p * pow2i(127)) * 2.0f;
    if (ni < -126) return (p * pow2i(ni + 64)) * 5.42101086242752217e-20f;
    return p * pow2i(ni);
}

PM_HD void sincosf_(float x, float* s, float* c)
{
    if (!(fabsf(x) < 1.0e5f)) { *s = x - x; *c = x - x; return; }
    const float q = rintf(x * 0.636619746685028076171875f);
    float r = fmaf(q, -1.5707963705062866f, x);
    r = fmaf(q, 4.371138828673793e-08f, r);
    r = fmaf(q, 1.7151245100058819e-15f, r);
    const float r2 = r * r;
    float ps = 2.7557319e-6f;
    ps = fmaf(ps, r2, -1.9841270e-4f);
    ps = fmaf(ps, r2, 8.3333338e-3f);
    ps = fmaf(ps, r2, -1.6666667e-1f);
    ps = ps * r2;
    const float sr = fmaf(ps, r, r);
    float pc = -2.7557319e-7f;
    pc = fmaf(pc, r2, 2.4801587e-5f);
    pc = fmaf(pc, r2, -1.3888889e-3f);
    pc = fmaf(pc, r2, 4.1666668e-2f);
    pc = fmaf(pc, r2, -0.5f);
    const float cr = fmaf(pc, r2, 1.0f);
    switch (((int)q) & 3) {
        case 0: *s = sr; *c = cr; break;
        case 1: *s = cr; *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

PM_HD float asin_small_(float x)
{
    const float x2 = x * x;
    float p = 6.447210442274809e-3f;
    p = fmaf(p, x2, 7.3125258e-3f);
    p = fmaf(p, x2, 8.3903358e-3f);
    p = fmaf(p, x2, 9.7616095e-3f);
    p = fmaf(p, x2, 1.1551800e-2f);
    p = fmaf(p, x2, 1.3964844e-2f);
    p = fmaf(p, x2, 1.7352764e-2f);
    p = fmaf(p, x2, 2.2372159e-2f);
    p = fmaf(p, x2, 3.0381944e-2f);
    p = fmaf(p, x2, 4.4642858e-2f);
    p = fmaf(p, x2, 7.5000003e-2f);
    p = fmaf(p, x2, 1.6666667e-1f);
    p = p * x2;
    return fmaf(p, x, x);
}

PM_HD float acospif_(float x)
{
    if (x != x) return x;
    if (x > 1.0f || x < -1.0f) return (x - x) / (x - x);
    float a;
    if (x > 0.5f) a = 2.0f * asin_small_(sqrtf((1.0f - x) * 0.5f));
    else if (x < -0.5f) a = 3.14159274101257324f - 2.0f * asin_small_(sqrtf((1.0f + x) * 0.5f));
    else a = 1.57079637050628662f - asin_small_(x);
    return a * 0.318309873342514038f;
}

// x / 0.05f correctly rounded for 0 <= x <= 0.05: one multiply by RN(1/0.05) = 20 and
// one fma correction (Markstein); verified against IEEE division for every float in
// [2^-103, 0.05] and 0; smaller inputs take the division.
PM_HD float div005(float x)
{
    const float q = x * 20.0f;
    const float r = fmaf(-q, 0.05f, x);
    float res = fmaf(r, 20.0f, q);
    if (x < 7.88860905e-31f) res = x / 0.05f;   // 2^-100
    return res;
}

// Smallest float c >= 0 with RN(c / b) >= m, for finite b >= 1: the cost loop's test
// `census / bilw >= mincost` (pmhstereo.cl:724) is equivalent to census >= threshold
// because c -> RN(c / b) is monotone.  m <= 0 gives -inf (always), NaN m gives NaN
// (never), +inf gives +inf (never).
PM_HD float exit_threshold(float m, float b)
{
    if (m != m) return m;
    if (m <= 0.0f) return -u2f(0x7f800000u);
    if (m == u2f(0x7f800000u)) return m;
    float c = m * b;
    if (c == u2f(0x7f800000u)) c = u2f(0x7f7fffffu);
    int guard = 0;
    while (!(c / b >= m)) {
        c = u2f(f2u(c) + 1u);
        if (++guard > 64 || c == u2f(0x7f800000u)) return u2f(0x7f800000u);
    }
    while (c > 0.0f && guard < 128) {
        const float p = u2f(f2u(c) - 1u);
        if (p / b >= m) c = p; else break;
        ++guard;
    }
    return c;
}

// ---- MWC64X (cvt/cl/kernel/MWC64X.cl:36-141, RNG.cl:30-59) ---------------------------
// RNG_init(s, linpos, nd) = SeedStreams(s, 0, 0) (every stream starts at MWC_BASEID,
// since the stream gap is 0) followed by Skip(s, (linpos) * nd): the state is
// BASEID * A^dist mod M split as (v / A, v % A).  The macro leaves nd unparenthesised
// (RNG.cl:54-57), so dist is the value of the expanded expression at each call site.  The skip uses 64x64->128-bit
// products reduced with 2^64 = K (mod M), K = 83941 * 2^32 + 1, instead of the
// reference's shift-and-add loop; the result is the same integer.
constexpr uint64_t MWC_A = 4294883355ULL;
constexpr uint64_t MWC_M = 18446383549859758079ULL;
constexpr uint64_t MWC_BASEID = 4077358422479273989ULL;
constexpr uint64_t MWC_K = 360523849793537ULL;   // 2^64 mod M = 83941 * 2^32 + 1

PM_HD uint64_t mwc_mulmod(uint64_t a, uint64_t b)
{
    unsigned __int128 p = (unsigned __int128)a * b;
    while ((uint64_t)(p >> 64) != 0) p = (unsigned __int128)(uint64_t)(p >> 64) * MWC_K + (uint64_t)p;
    uint64_t r = (uint64_t)p;
    if (r >= MWC_M) r -= MWC_M;
    return r;
}

PM_HD uint64_t mwc_powmod(uint64_t e)
{
    uint64_t acc = 1, sq = MWC_A;
    while (e) {
        if (e & 1) acc = mwc_mulmod(acc, sq);
        sq = mwc_mulmod(sq, sq);
        e >>= 1;
    }
    return acc;
}

struct Rng {
    uint32_t x, c;
    // state after RNG_init: skip distance `dist` from the common seed
    PM_HD void init_skip(int dist32)
    {
        const uint64_t dist = (uint64_t)(int64_t)dist32;
        const uint64_t v = mwc_mulmod(MWC_BASEID, mwc_powmod(dist));
        x = (uint32_t)(v / MWC_A);
        c = (uint32_t)(v % MWC_A);
    }
    PM_HD float next()
    {
        const uint32_t res = x ^ c;
        const uint32_t xn = (uint32_t)MWC_A * x + c;
        const uint32_t carry = (uint32_t)(xn < c);
        const uint32_t cn = (uint32_t)(((uint64_t)(uint32_t)MWC_A * x) >> 32) + carry;
        x = xn;
        c = cn;
        return 2.3283064365386962890625e-10f * (float)res;
    }
};

}  // namespace pm
