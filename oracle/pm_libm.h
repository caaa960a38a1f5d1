/*
 * ORACLE — test infrastructure only. Never linked into the product library.
 *
 * Deterministic single-precision elementary functions for the CPU oracle.
 *
 * The reference kernels call OpenCL built-ins whose last-bit behaviour is
 * implementation-defined: exp / native_exp (cvt/cl/kernel/pmhstereo.cl:355,
 * :701, :1491; cvt/cl/kernel/PDDiffTensor.cl:58), cos / sin
 * (pmhstereo.cl:86-87, :148-149), acospi (pmhstereo.cl:1123-1124),
 * normalize (pmhstereo.cl:91, :103, :165, :819, :968), native_rsqrt
 * (pmhstereo.cl:119, :137, :205).  OpenCL 1.2 only bounds their error
 * (exp 3 ulp, sin/cos 4 ulp, acospi 5 ulp).  The oracle pins one concrete
 * choice inside those bounds so that it and the CUDA kernels can agree bit for
 * bit; the CUDA side carries an independent copy of the same algorithms
 * (cvt_b200/csrc/pm_math.cuh), and the GPU tests compare the two over every
 * input they meet.
 *
 * Methods (all from textbook numerical analysis, no vendor code):
 *  - exp:    Cody & Waite additive range reduction x = n ln2 + r with a
 *            two-part ln2, |r| <= ln2/2, degree-7 Taylor polynomial of e^r in
 *            Horner form with fused multiply-add, scaling by 2^n through the
 *            exponent field.
 *  - sincos: Cody & Waite reduction by pi/2 (three-part constant), Taylor
 *            polynomials of degree 9 (sin) and 10 (cos) on |r| <= pi/4,
 *            quadrant selection.
 *  - acospi: arcsine Maclaurin series (coefficients (2k)!/(4^k (k!)^2 (2k+1)))
 *            on |x| <= 1/2 and the half-angle identity
 *            acos(x) = 2 asin(sqrt((1-x)/2)) beyond.
 *  - log:    (cvt/cl/kernel/SVPMFlow.cl:42, Box-Muller) x = 2^k m with m in
 *            [sqrt(1/2), sqrt(2)], f = m - 1 (exact), s = f / (2 + f) and
 *            log(m) = 2 atanh(s) = f - (f^2/2 - s (f^2/2 + R)) with R = 2 (s^2/3 + ... + s^10/11)
 *            (the arrangement of fdlibm's e_log.c), |s| <= 0.1716;
 *            log(x) = k ln2 + log(m) with the two-part ln2 of exp.
 * Every operation is an IEEE single-precision add, multiply, fma, sqrt or
 * divide, so the results are the same on any conforming machine.
 */
#ifndef PM_ORACLE_LIBM_H
#define PM_ORACLE_LIBM_H

#include <math.h>
#include <stdint.h>
#include <string.h>

static inline float orc_bits2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t orc_f2bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* 2^n for n in [-126, 127] */
static inline float orc_pow2i(int n) { return orc_bits2f((uint32_t)(n + 127) << 23); }

static inline float orc_expf(float x)
{
    if (x != x) return x;
    if (x > 88.72283935546875f) return INFINITY;
    if (x < -103.97208404541015625f) return 0.0f;
    const float n = rintf(x * 1.44269502162933349609375f);
    float r = fmaf(n, -0.693145751953125f, x);          /* ln2 high part (exact products) */
    r = fmaf(n, -1.428606765330187045e-06f, r);         /* ln2 low part */
    float p = 1.9841270113829523e-4f;                   /* 1/7! */
    p = fmaf(p, r, 1.3888889e-3f);                      /* 1/6! */
    p = fmaf(p, r, 8.3333338e-3f);                      /* 1/5! */
    p = fmaf(p, r, 4.1666668e-2f);                      /* 1/4! */
    p = fmaf(p, r, 1.6666667e-1f);                      /* 1/3! */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    const int ni = (int)n;
    if (ni > 127) return (p * orc_pow2i(127)) * 2.0f;
    if (ni < -126) return (p * orc_pow2i(ni + 64)) * 5.42101086242752217e-20f; /* 2^-64 */
    return p * orc_pow2i(ni);
}

static inline void orc_sincosf(float x, float* s, float* c)
{
    if (!(fabsf(x) < 1.0e5f)) { *s = x - x; *c = x - x; return; }   /* outside the supported domain: NaN */
    const float q = rintf(x * 0.636619746685028076171875f);        /* 2/pi */
    float r = fmaf(q, -1.5707963705062866f, x);                    /* pi/2, three parts */
    r = fmaf(q, 4.371138828673793e-08f, r);
    r = fmaf(q, 1.7151245100058819e-15f, r);
    const float r2 = r * r;
    float ps = 2.7557319e-6f;                                      /* 1/9! */
    ps = fmaf(ps, r2, -1.9841270e-4f);                             /* -1/7! */
    ps = fmaf(ps, r2, 8.3333338e-3f);                              /* 1/5! */
    ps = fmaf(ps, r2, -1.6666667e-1f);                             /* -1/3! */
    ps = ps * r2;
    const float sr = fmaf(ps, r, r);
    float pc = -2.7557319e-7f;                                     /* -1/10! */
    pc = fmaf(pc, r2, 2.4801587e-5f);                              /* 1/8! */
    pc = fmaf(pc, r2, -1.3888889e-3f);                             /* -1/6! */
    pc = fmaf(pc, r2, 4.1666668e-2f);                              /* 1/4! */
    pc = fmaf(pc, r2, -0.5f);
    const float cr = fmaf(pc, r2, 1.0f);
    const int quad = ((int)q) & 3;
    switch (quad) {
        case 0: *s = sr;  *c = cr;  break;
        case 1: *s = cr;  *c = -sr; break;
        case 2: *s = -sr; *c = -cr; break;
        default: *s = -cr; *c = sr; break;
    }
}

static inline float orc_sinf(float x) { float s, c; orc_sincosf(x, &s, &c); return s; }
static inline float orc_cosf(float x) { float s, c; orc_sincosf(x, &s, &c); return c; }

/* asin on |x| <= 1/2 from its Maclaurin series */
static inline float orc_asin_small(float x)
{
    const float x2 = x * x;
    float p = 6.447210442274809e-3f;   /* c12 = 676039/104857600 */
    p = fmaf(p, x2, 7.3125258e-3f);    /* c11 = 88179/12058624 */
    p = fmaf(p, x2, 8.3903358e-3f);    /* c10 = 46189/5505024 */
    p = fmaf(p, x2, 9.7616095e-3f);    /* c9  = 12155/1245184 */
    p = fmaf(p, x2, 1.1551800e-2f);    /* c8  = 6435/557056 */
    p = fmaf(p, x2, 1.3964844e-2f);    /* c7  = 143/10240 */
    p = fmaf(p, x2, 1.7352764e-2f);    /* c6  = 231/13312 */
    p = fmaf(p, x2, 2.2372159e-2f);    /* c5  = 63/2816 */
    p = fmaf(p, x2, 3.0381944e-2f);    /* c4  = 35/1152 */
    p = fmaf(p, x2, 4.4642858e-2f);    /* c3  = 5/112 */
    p = fmaf(p, x2, 7.5000003e-2f);    /* c2  = 3/40 */
    p = fmaf(p, x2, 1.6666667e-1f);    /* c1  = 1/6 */
    p = p * x2;
    return fmaf(p, x, x);
}

static inline float orc_acospif(float x)
{
    const float PI = 3.14159274101257324f;
    const float INV_PI = 0.318309873342514038f;
    if (x != x) return x;
    if (x > 1.0f || x < -1.0f) return (x - x) / (x - x);
    float a;
    if (x > 0.5f) {
        a = 2.0f * orc_asin_small(sqrtf((1.0f - x) * 0.5f));
    } else if (x < -0.5f) {
        a = PI - 2.0f * orc_asin_small(sqrtf((1.0f + x) * 0.5f));
    } else {
        a = 1.57079637050628662f - orc_asin_small(x);
    }
    return a * INV_PI;
}

static inline float orc_logf(float x)
{
    if (x != x) return x;
    if (x < 0.0f) return (x - x) / (x - x);
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    int k = 0;
    uint32_t u = orc_f2bits(x);
    if (u < 0x00800000u) {   /* subnormal: scale by 2^23 */
        x *= 8388608.0f;
        k = -23;
        u = orc_f2bits(x);
    }
    k += (int)(u >> 23) - 127;
    u = (u & 0x007fffffu) | 0x3f800000u;   /* m in [1, 2) */
    if (u > 0x3fb504f3u) {                 /* above sqrt(2): m / 2 */
        u -= 0x00800000u;
        k += 1;
    }
    const float f = orc_bits2f(u) - 1.0f;
    const float s = f / (2.0f + f);
    const float z = s * s;
    /* R = 2 (z/3 + z^2/5 + ... + z^5/11); log(m) = f - (f^2/2 - s (f^2/2 + R)), the form of
     * fdlibm's e_log.c, which keeps the rounding of s out of the leading term */
    float R = 1.8181819e-1f;               /* 2/11 */
    R = fmaf(R, z, 2.2222222e-1f);         /* 2/9 */
    R = fmaf(R, z, 2.8571430e-1f);         /* 2/7 */
    R = fmaf(R, z, 4.0000001e-1f);         /* 2/5 */
    R = fmaf(R, z, 6.6666669e-1f);         /* 2/3 */
    R = R * z;
    const float hfsq = (0.5f * f) * f;
    const float kf = (float)k;
    const float lo = fmaf(s, hfsq + R, kf * 1.428606765330187045e-06f);
    return fmaf(kf, 0.693145751953125f, f - (hfsq - lo));
}

#endif
