/*
 * ORACLE — test infrastructure only.
 *
 * Glue around cvt/cl/kernel/pyr/pyrdown.cl and pyrupmul.cl compiled from their own
 * source: CLPyramid::pyrDown (cvt/cl/CLPyramid.cpp:73-78) and PMHuberStereo::pyrUpMul
 * (cvt/vision/PMHuberStereo.cpp:709-721), both with 32x32 work groups.
 */
#include <cstdint>

#include "ref_exec.h"

namespace clk {
namespace pyrd {
#include "_ref/pyrdown.cl.cpp"
}  // namespace pyrd
namespace pyru {
#include "_ref/pyrupmul.cl.cpp"
}  // namespace pyru
}  // namespace clk

using namespace clk;

namespace {
inline int pad32(int v) { return (v + 31) / 32 * 32; }
}

extern "C" {

int ref_k_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, int Wi, int Hi)
{
    image2d_t o{(void*)out, Wo, Ho, IMG_RGBA_UNORM8}, s{(void*)in, Wi, Hi, IMG_RGBA_UNORM8};
    nd_range(pad32(Wo), pad32(Ho), 32, 32, false, [&]() { pyrd::pyrdown(o, s); });
    return 0;
}

int ref_k_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, const float* mul)
{
    if (channels != 1 && channels != 4) return -1;
    const ImgKind k = channels == 1 ? IMG_INTENSITY_FLOAT : IMG_RGBA_FLOAT;
    image2d_t o{(void*)out, Wo, Ho, k}, s{(void*)in, Wi, Hi, k};
    const float4 m(mul[0], mul[1], mul[2], mul[3]);
    nd_range(pad32(Wo), pad32(Ho), 32, 32, false, [&]() { pyru::pyrup_mul4f(o, s, m); });
    return 0;
}

}  // extern "C"
