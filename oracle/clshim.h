/*
 * ORACLE — test infrastructure only.
 *
 * A minimal OpenCL C 1.2 environment in C++ so that the reference's own kernel
 * sources (cvt/cl/kernel/pmhstereo.cl and the files it #imports,
 * PDDiffTensor.cl, PDDROFDiffTensor.cl) compile on the host after the
 * mechanical rewrite in oracle/translate.py.  The output of that build goes to
 * oracle/_ref/ and is never committed.
 *
 * Semantics pinned here (each is an implementation choice OpenCL allows):
 *  - vector types with the swizzles the sources use (.x .y .z .w, .xy .yz .xyz,
 *    .lo .hi; the multi-letter ones become member calls in the rewrite);
 *  - vector relational results are -1 per true lane, scalar ones 1;
 *  - exp/native_exp, log, sin, cos, acospi come from oracle/pm_libm.h; sqrt, the
 *    division and native_rsqrt (1/sqrt) are correctly rounded; pow(x, 1) = x;
 *    length(v) = sqrt(dot(v, v));
 *  - normalize follows OpenCL 1.2 s6.12.5 (a zero vector is returned as is);
 *  - convert_int*: NaN -> 0, out-of-range values saturate;
 *  - image reads implement OpenCL 1.2 s8.2 in full FP32 (UNORM_INT8 as v/255),
 *    CL_INTENSITY reads return (I, I, I, I); a non-finite coordinate reads the
 *    positive quiet NaN;
 *  - work-groups run one after another per host thread; work items of a group
 *    run as cooperative fibers so that barrier() works.
 */
#ifndef PM_CLSHIM_H
#define PM_CLSHIM_H

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <cstdlib>

#include "pm_libm.h"

#undef signbit
#undef isfinite
#undef isnan
#undef isinf

namespace clk {

typedef unsigned int uint;
typedef unsigned long ulong;
typedef unsigned char uchar;

/* ---------------------------------------------------------------- vectors */

template <class V, class T> struct Swz2 {
    T* a; T* b;
    operator V() const { return V(*a, *b); }
    Swz2& operator=(const V& v) { T x = v.x, y = v.y; *a = x; *b = y; return *this; }
    Swz2& operator=(const Swz2& o) { return *this = (V)o; }
    Swz2& operator+=(const V& v) { return *this = (V)*this + v; }
    Swz2& operator-=(const V& v) { return *this = (V)*this - v; }
    Swz2& operator*=(const V& v) { return *this = (V)*this * v; }
    Swz2& operator*=(T s) { return *this = (V)*this * V(s); }
};
template <class V, class T> struct Swz3 {
    T* a; T* b; T* c;
    operator V() const { return V(*a, *b, *c); }
    Swz3& operator=(const V& v) { T x = v.x, y = v.y, z = v.z; *a = x; *b = y; *c = z; return *this; }
    Swz3& operator=(const Swz3& o) { return *this = (V)o; }
    Swz3& operator+=(const V& v) { return *this = (V)*this + v; }
    Swz3& operator-=(const V& v) { return *this = (V)*this - v; }
    Swz3& operator*=(const V& v) { return *this = (V)*this * v; }
    Swz3& operator*=(T s) { return *this = (V)*this * V(s); }
};
template <class V, class P> struct Half {
    P* a;
    operator V() const { return *a; }
    Half& operator=(const V& v) { *a = v; return *this; }
    Half& operator=(const Half& o) { *a = *o.a; return *this; }
};

#define CL_VEC2(T, N)                                                                  \
    struct N {                                                                         \
        T x, y;                                                                        \
        N() : x(0), y(0) {}                                                            \
        N(T s) : x(s), y(s) {}                                                         \
        N(T x_, T y_) : x(x_), y(y_) {}                                                \
    };
#define CL_VEC3(T, N, N2)                                                              \
    struct N {                                                                         \
        T x, y, z;                                                                     \
        N() : x(0), y(0), z(0) {}                                                      \
        N(T s) : x(s), y(s), z(s) {}                                                   \
        N(T x_, T y_, T z_) : x(x_), y(y_), z(z_) {}                                   \
        N(N2 v, T z_) : x(v.x), y(v.y), z(z_) {}                                       \
        N(T x_, N2 v) : x(x_), y(v.x), z(v.y) {}                                       \
        Swz2<N2, T> xy() { return Swz2<N2, T>{&x, &y}; }                               \
        Swz2<N2, T> yz() { return Swz2<N2, T>{&y, &z}; }                               \
        Swz3<N, T> xyz() { return Swz3<N, T>{&x, &y, &z}; }                            \
        N2 xy() const { return N2(x, y); }                                             \
        N2 yz() const { return N2(y, z); }                                             \
        N xyz() const { return *this; }                                                \
    };
#define CL_VEC4(T, N, N2, N3)                                                          \
    struct N {                                                                         \
        T x, y, z, w;                                                                  \
        N() : x(0), y(0), z(0), w(0) {}                                                \
        N(T s) : x(s), y(s), z(s), w(s) {}                                             \
        N(T x_, T y_, T z_, T w_) : x(x_), y(y_), z(z_), w(w_) {}                      \
        N(N3 v, T w_) : x(v.x), y(v.y), z(v.z), w(w_) {}                               \
        N(T x_, N3 v) : x(x_), y(v.x), z(v.y), w(v.z) {}                               \
        N(N2 a, N2 b) : x(a.x), y(a.y), z(b.x), w(b.y) {}                              \
        N(N2 a, T z_, T w_) : x(a.x), y(a.y), z(z_), w(w_) {}                          \
        Swz2<N2, T> xy() { return Swz2<N2, T>{&x, &y}; }                               \
        Swz2<N2, T> yz() { return Swz2<N2, T>{&y, &z}; }                               \
        Swz3<N3, T> xyz() { return Swz3<N3, T>{&x, &y, &z}; }                          \
        N2 xy() const { return N2(x, y); }                                             \
        N2 yz() const { return N2(y, z); }                                             \
        N3 xyz() const { return N3(x, y, z); }                                         \
        N2 zw() const { return N2(z, w); }                                             \
        N2 lo() const { return N2(x, y); }                                             \
        N2 hi() const { return N2(z, w); }                                             \
    };

CL_VEC2(float, float2)
CL_VEC3(float, float3, float2)
CL_VEC4(float, float4, float2, float3)
CL_VEC2(int, int2)
CL_VEC3(int, int3, int2)
CL_VEC4(int, int4, int2, int3)
CL_VEC2(uint, uint2)
CL_VEC3(uint, uint3, uint2)
CL_VEC4(uint, uint4, uint2, uint3)

struct float8 {
    float4 l, h;
    float8() {}
    float8(float s) : l(s), h(s) {}
    float8(float4 a, float4 b) : l(a), h(b) {}
    Half<float4, float4> lo() { return Half<float4, float4>{&l}; }
    Half<float4, float4> hi() { return Half<float4, float4>{&h}; }
    float4 lo() const { return l; }
    float4 hi() const { return h; }
};

/* elementwise operators, non-template so that swizzle proxies convert implicitly */
#define CL_BINOP2(N, T, OP)                                                                          \
    inline N operator OP(const N& a, const N& b) { return N(a.x OP b.x, a.y OP b.y); }               \
    inline N operator OP(const N& a, T s) { return N(a.x OP s, a.y OP s); }                          \
    inline N operator OP(T s, const N& a) { return N(s OP a.x, s OP a.y); }                          \
    inline N& operator OP##=(N& a, const N& b) { a = a OP b; return a; }                             \
    inline N& operator OP##=(N& a, T s) { a = a OP s; return a; }
#define CL_BINOP3(N, T, OP)                                                                          \
    inline N operator OP(const N& a, const N& b) { return N(a.x OP b.x, a.y OP b.y, a.z OP b.z); }   \
    inline N operator OP(const N& a, T s) { return N(a.x OP s, a.y OP s, a.z OP s); }                \
    inline N operator OP(T s, const N& a) { return N(s OP a.x, s OP a.y, s OP a.z); }                \
    inline N& operator OP##=(N& a, const N& b) { a = a OP b; return a; }                             \
    inline N& operator OP##=(N& a, T s) { a = a OP s; return a; }
#define CL_BINOP4(N, T, OP)                                                                          \
    inline N operator OP(const N& a, const N& b) { return N(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); } \
    inline N operator OP(const N& a, T s) { return N(a.x OP s, a.y OP s, a.z OP s, a.w OP s); }      \
    inline N operator OP(T s, const N& a) { return N(s OP a.x, s OP a.y, s OP a.z, s OP a.w); }      \
    inline N& operator OP##=(N& a, const N& b) { a = a OP b; return a; }                             \
    inline N& operator OP##=(N& a, T s) { a = a OP s; return a; }

#define CL_ARITH(N, T, K) CL_BINOP##K(N, T, +) CL_BINOP##K(N, T, -) CL_BINOP##K(N, T, *) CL_BINOP##K(N, T, /)
CL_ARITH(float2, float, 2) CL_ARITH(float3, float, 3) CL_ARITH(float4, float, 4)
CL_ARITH(int2, int, 2) CL_ARITH(int3, int, 3) CL_ARITH(int4, int, 4)
CL_ARITH(uint2, uint, 2) CL_ARITH(uint3, uint, 3) CL_ARITH(uint4, uint, 4)
CL_BINOP3(uint3, uint, &) CL_BINOP4(uint4, uint, &)
CL_BINOP3(uint3, uint, <<) CL_BINOP4(uint4, uint, <<)
CL_BINOP3(uint3, uint, >>) CL_BINOP4(uint4, uint, >>)

inline float2 operator-(const float2& a) { return float2(-a.x, -a.y); }
inline float3 operator-(const float3& a) { return float3(-a.x, -a.y, -a.z); }
inline float4 operator-(const float4& a) { return float4(-a.x, -a.y, -a.z, -a.w); }
inline int4 operator+(const int4& a, const int4& b);

inline float8 operator/(const float8& a, const float8& b) { return float8(a.l / b.l, a.h / b.h); }

/* ---------------------------------------------------------------- bit casts */
template <class D, class S> inline D bitcast_(S s) { D d; static_assert(sizeof(D) == sizeof(S), "size"); memcpy(&d, &s, sizeof(D)); return d; }
inline uint3 as_uint3(float3 v) { return uint3(bitcast_<uint>(v.x), bitcast_<uint>(v.y), bitcast_<uint>(v.z)); }
inline uint3 as_uint3(int3 v) { return uint3((uint)v.x, (uint)v.y, (uint)v.z); }
inline uint3 as_uint3(uint3 v) { return v; }
inline int3 as_int3(uint3 v) { return int3((int)v.x, (int)v.y, (int)v.z); }
inline uint4 as_uint4(float4 v) { return uint4(bitcast_<uint>(v.x), bitcast_<uint>(v.y), bitcast_<uint>(v.z), bitcast_<uint>(v.w)); }
inline uint4 as_uint4(int4 v) { return uint4((uint)v.x, (uint)v.y, (uint)v.z, (uint)v.w); }
inline uint4 as_uint4(uint4 v) { return v; }
inline int4 as_int4(uint4 v) { return int4((int)v.x, (int)v.y, (int)v.z, (int)v.w); }

/* ---------------------------------------------------------------- scalar math */
inline float fabs(float x) { return std::fabs(x); }
inline double fabs(double x) { return std::fabs(x); }
inline float floor(float x) { return std::floor(x); }
inline float ceil(float x) { return std::ceil(x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline double sqrt(double x) { return std::sqrt(x); }
inline float native_sqrt(float x) { return std::sqrt(x); }
inline float native_rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline float exp(float x) { return orc_expf(x); }
inline float native_exp(float x) { return orc_expf(x); }
inline float log(float x) { return orc_logf(x); }
inline double log(double x) { return std::log(x); }
inline float native_log(float x) { return std::log(x); }
inline float cos(float x) { return orc_cosf(x); }
inline float sin(float x) { return orc_sinf(x); }
inline float acospi(float x) { return orc_acospif(x); }
inline float pow(float x, float y) { return y == 1.0f ? x : std::pow(x, y); }
inline float fmin(float a, float b) { return std::fmin(a, b); }
inline float fmax(float a, float b) { return std::fmax(a, b); }
inline float clamp(float x, float lo, float hi) { return fmin(fmax(x, lo), hi); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline int mad24(int a, int b, int c) { return a * b + c; }
inline int mul24(int a, int b) { return a * b; }   /* exact for the 24-bit operands the kernels pass */
inline uint mad_hi(uint a, uint b, uint c) { return (uint)(((ulong)a * (ulong)b) >> 32) + c; }
inline int isfinite(float x) { return std::isfinite(x) ? 1 : 0; }
inline int convert_int(float f)
{
    if (f != f) return 0;
    if (f >= 2147483648.0f) return 2147483647;
    if (f < -2147483648.0f) return -2147483647 - 1;
    return (int)f;
}
inline int convert_int_rte(float f) { return convert_int(std::rint(f)); }
inline float select(float a, float b, int c) { return c ? b : a; }
inline int select(int a, int b, int c) { return c ? b : a; }
inline int abs(int x) { return x < 0 ? -x : x; }

/* ---------------------------------------------------------------- vector math */
inline float2 fabs(float2 v) { return float2(fabs(v.x), fabs(v.y)); }
inline float3 fabs(float3 v) { return float3(fabs(v.x), fabs(v.y), fabs(v.z)); }
inline float4 fabs(float4 v) { return float4(fabs(v.x), fabs(v.y), fabs(v.z), fabs(v.w)); }
inline float3 fmin(float3 a, float3 b) { return float3(fmin(a.x, b.x), fmin(a.y, b.y), fmin(a.z, b.z)); }
inline float3 fmin(float3 a, float b) { return fmin(a, float3(b)); }
inline float3 fmax(float3 a, float3 b) { return float3(fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z)); }
inline float3 clamp(float3 x, float3 lo, float3 hi) { return fmin(fmax(x, lo), hi); }
inline float2 fmin(float2 a, float2 b) { return float2(fmin(a.x, b.x), fmin(a.y, b.y)); }
inline float2 fmax(float2 a, float2 b) { return float2(fmax(a.x, b.x), fmax(a.y, b.y)); }
inline float4 fmin(float4 a, float4 b) { return float4(fmin(a.x, b.x), fmin(a.y, b.y), fmin(a.z, b.z), fmin(a.w, b.w)); }
inline float4 fmin(float4 a, float b) { return fmin(a, float4(b)); }
inline float4 fmax(float4 a, float4 b) { return float4(fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z), fmax(a.w, b.w)); }
inline float4 fmax(float a, float4 b) { return fmax(float4(a), b); }
inline float4 fmax(float4 a, float b) { return fmax(a, float4(b)); }
inline float3 sqrt(float3 v) { return float3(sqrt(v.x), sqrt(v.y), sqrt(v.z)); }
inline float4 sqrt(float4 v) { return float4(sqrt(v.x), sqrt(v.y), sqrt(v.z), sqrt(v.w)); }
inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float length(float2 v) { return sqrt(dot(v, v)); }
inline float4 xxyy_(float2 v) { return float4(v.x, v.x, v.y, v.y); }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float length(float3 v) { return sqrt(dot(v, v)); }
inline float length(float4 v) { return sqrt(dot(v, v)); }
inline float3 cross(float3 a, float3 b) { return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float4 cross(float4 a, float4 b) { return float4(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f); }
inline float3 normalize(float3 v)
{
    if (v.x == 0.0f && v.y == 0.0f && v.z == 0.0f) return v;
    if (v.x != v.x || v.y != v.y || v.z != v.z) return float3(NAN);
    if (std::isinf(v.x) || std::isinf(v.y) || std::isinf(v.z)) {
        v.x = std::isinf(v.x) ? std::copysign(1.0f, v.x) : 0.0f * v.x;
        v.y = std::isinf(v.y) ? std::copysign(1.0f, v.y) : 0.0f * v.y;
        v.z = std::isinf(v.z) ? std::copysign(1.0f, v.z) : 0.0f * v.z;
    }
    float d = dot(v, v);
    if (d < 7.8886090522101181e-31f) { v = v * 1.8446744073709552e19f; d = dot(v, v); }
    else if (d > 1.2676506002282294e30f) { v = v * 5.4210108624275222e-20f; d = dot(v, v); }
    const float l = std::sqrt(d);
    return float3(v.x / l, v.y / l, v.z / l);
}
inline float3 sincos(float3 x, float3* c)
{
    float3 s;
    orc_sincosf(x.x, &s.x, &c->x); orc_sincosf(x.y, &s.y, &c->y); orc_sincosf(x.z, &s.z, &c->z);
    return s;
}
inline int3 isfinite(float3 v) { return int3(std::isfinite(v.x) ? -1 : 0, std::isfinite(v.y) ? -1 : 0, std::isfinite(v.z) ? -1 : 0); }
inline int2 isfinite(float2 v) { return int2(std::isfinite(v.x) ? -1 : 0, std::isfinite(v.y) ? -1 : 0); }
inline int all(int3 v) { return (v.x < 0) && (v.y < 0) && (v.z < 0); }
inline int all(int2 v) { return (v.x < 0) && (v.y < 0); }
inline int4 signbit(float4 v) { uint4 u = as_uint4(v); return int4(u.x >> 31 ? -1 : 0, u.y >> 31 ? -1 : 0, u.z >> 31 ? -1 : 0, u.w >> 31 ? -1 : 0); }
inline uint3 abs(int3 v) { return uint3((uint)abs(v.x), (uint)abs(v.y), (uint)abs(v.z)); }
inline uint4 abs(int4 v) { return uint4((uint)abs(v.x), (uint)abs(v.y), (uint)abs(v.z), (uint)abs(v.w)); }
inline int3 isgreaterequal(float3 a, float b) { return int3(a.x >= b ? -1 : 0, a.y >= b ? -1 : 0, a.z >= b ? -1 : 0); }
inline int4 isgreaterequal(float4 a, float b) { return int4(a.x >= b ? -1 : 0, a.y >= b ? -1 : 0, a.z >= b ? -1 : 0, a.w >= b ? -1 : 0); }
template <class V, class M> inline V select_lanes(V a, V b, M m);
inline float4 select(float4 a, float4 b, int4 m)
{
    return float4(m.x < 0 ? b.x : a.x, m.y < 0 ? b.y : a.y, m.z < 0 ? b.z : a.z, m.w < 0 ? b.w : a.w);
}
inline float4 select(float4 a, float4 b, uint4 m) { return select(a, b, as_int4(m)); }

/* ---------------------------------------------------------------- work items */
struct WorkItem { size_t gid[2], lid[2], grp[2], lsz[2], gsz[2]; };
extern thread_local WorkItem g_wi;
inline size_t get_global_id(int d) { return g_wi.gid[d]; }
inline size_t get_local_id(int d) { return g_wi.lid[d]; }
inline size_t get_group_id(int d) { return g_wi.grp[d]; }
inline size_t get_local_size(int d) { return g_wi.lsz[d]; }
inline size_t get_global_size(int d) { return g_wi.gsz[d]; }
enum { CLK_LOCAL_MEM_FENCE = 1, CLK_GLOBAL_MEM_FENCE = 2 };
void barrier(int flags);
inline int atomic_inc(volatile int* p) { return __atomic_fetch_add((int*)p, 1, __ATOMIC_SEQ_CST); }

/* ---------------------------------------------------------------- images */
typedef int sampler_t;
enum {
    CLK_NORMALIZED_COORDS_FALSE = 0,
    CLK_ADDRESS_CLAMP_TO_EDGE = 2, CLK_ADDRESS_CLAMP = 4,
    CLK_FILTER_NEAREST = 16, CLK_FILTER_LINEAR = 32
};
enum ImgKind { IMG_RGBA_FLOAT, IMG_RGBA_UNORM8, IMG_INTENSITY_FLOAT };
struct image2d_t {
    void* data; int w, h; ImgKind kind;
};
inline int get_image_width(image2d_t im) { return im.w; }
inline int get_image_height(image2d_t im) { return im.h; }

inline float4 texel_(const image2d_t& im, int x, int y, int addr)
{
    if (addr == CLK_ADDRESS_CLAMP) {
        if (x < 0 || x >= im.w || y < 0 || y >= im.h) return float4(0.0f);
    } else {
        x = x < 0 ? 0 : (x >= im.w ? im.w - 1 : x);
        y = y < 0 ? 0 : (y >= im.h ? im.h - 1 : y);
    }
    const size_t i = (size_t)y * im.w + x;
    switch (im.kind) {
        case IMG_RGBA_FLOAT: { const float* p = (const float*)im.data + 4 * i; return float4(p[0], p[1], p[2], p[3]); }
        case IMG_RGBA_UNORM8: {
            const unsigned char* p = (const unsigned char*)im.data + 4 * i;
            return float4((float)p[0] / 255.0f, (float)p[1] / 255.0f, (float)p[2] / 255.0f, (float)p[3] / 255.0f);
        }
        default: { const float v = ((const float*)im.data)[i]; return float4(v); }
    }
}
inline int clamp_coord_(float f, int n)
{
    /* keep the integer conversion defined; every clamped value addresses the same texel */
    if (f != f) return 0;
    if (f < -2.0f) return -2;
    if (f > (float)n + 1.0f) return n + 1;
    return (int)f;
}
inline float4 read_imagef(image2d_t im, sampler_t s, int2 c) { return texel_(im, c.x, c.y, s & 6); }
inline float4 read_imagef(image2d_t im, sampler_t s, float2 c)
{
    const int addr = s & 6;
    if (!std::isfinite(c.x) || !std::isfinite(c.y)) return float4(bitcast_<float>(0x7fffffffu));
    if (s & CLK_FILTER_LINEAR) {
        const float tu = c.x - 0.5f, tv = c.y - 0.5f;
        const float fu = std::floor(tu), fv = std::floor(tv);
        const float a = tu - fu, b = tv - fv;
        const int i0 = clamp_coord_(fu, im.w), j0 = clamp_coord_(fv, im.h);
        const float4 T00 = texel_(im, i0, j0, addr), T10 = texel_(im, i0 + 1, j0, addr);
        const float4 T01 = texel_(im, i0, j0 + 1, addr), T11 = texel_(im, i0 + 1, j0 + 1, addr);
        return (1.0f - a) * (1.0f - b) * T00 + a * (1.0f - b) * T10 + (1.0f - a) * b * T01 + a * b * T11;
    }
    return texel_(im, clamp_coord_(std::floor(c.x), im.w), clamp_coord_(std::floor(c.y), im.h), addr);
}
inline void write_imagef(image2d_t im, int2 c, float4 v)
{
    if (c.x < 0 || c.x >= im.w || c.y < 0 || c.y >= im.h) return;
    const size_t i = (size_t)c.y * im.w + c.x;
    if (im.kind == IMG_RGBA_FLOAT) { float* p = (float*)im.data + 4 * i; p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w; }
    else if (im.kind == IMG_INTENSITY_FLOAT) { ((float*)im.data)[i] = v.x; }
    else {   /* CL_UNORM_INT8: convert_uchar_sat_rte(v * 255) (OpenCL 1.2 s8.3.1.1) */
        unsigned char* p = (unsigned char*)im.data + 4 * i;
        const float c[4] = {v.x, v.y, v.z, v.w};
        for (int k = 0; k < 4; k++) {
            const float x = c[k] * 255.0f;
            p[k] = !(x > 0.0f) ? 0 : (x >= 255.0f ? 255 : (unsigned char)std::nearbyint(x));
        }
    }
}

}  // namespace clk

#endif
