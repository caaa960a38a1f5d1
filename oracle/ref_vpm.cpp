/*
 * ORACLE — test infrastructure only.
 *
 * Glue around cvt/cl/kernel/VPMStereo.cl and gradxy.cl compiled from their own source
 * (after oracle/translate.py): each ref_vpm_* function launches one reference kernel over
 * the NDRange VPMStereoCL uses, (pad(W,32), pad(H,32)) with 32x32 work-groups
 * (cvt/vision/VPMStereoCL.cpp:31-32, e.g. :98), and ref_vpm_disparity_simple runs
 * VPMStereoCL::disparitySimple (:54-85) without its debugging block (:74-81, which saves a
 * PNG and waits for a key press after every iteration and changes no result).
 */
#include <cstdint>
#include <vector>

#include "ref_exec.h"

namespace clk {
namespace vpm {
#include "_ref/VPMStereo.cl.cpp"
}  // namespace vpm
namespace gxy {
#include "_ref/gradxy.cl.cpp"
}  // namespace gxy
}  // namespace clk

using namespace clk;

namespace {
inline int pad32(int v) { return (v + 31) / 32 * 32; }
inline image2d_t img(const float* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_RGBA_FLOAT}; }
inline image2d_t img1(const float* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_INTENSITY_FLOAT}; }
inline image2d_t img8(const uint8_t* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_RGBA_UNORM8}; }
}  // namespace

extern "C" {

/* grad_gray_xydiag (gradxy.cl:60-97) on a packed RGBA_UINT8 image */
int ref_vpm_grad(float* out, const uint8_t* rgba8, int W, int H)
{
    image2d_t o = img(out, W, H), s = img8(rgba8, W, H);
    nd_range(pad32(W), pad32(H), 32, 32, true, [&]() { gxy::grad_gray_xydiag(o, s); });
    return 0;
}

/* vpmstereo_init, or vpmstereo_init_disparity when initdisp is given (VPMStereo.cl:260-309);
 * c1 / c2 packed RGBA_UINT8 */
int ref_vpm_init(float* out, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2, int W, int H,
                 int r, float dmax, const float* initdisp)
{
    image2d_t o = img(out, W, H), a = img8(c1, W, H), ga = img(g1, W, H), b = img8(c2, W, H), gb = img(g2, W, H);
    if (initdisp) {
        image2d_t d = img1(initdisp, W, H);
        nd_range(pad32(W), pad32(H), 32, 32, false, [&]() { vpm::vpmstereo_init_disparity(o, d, a, ga, b, gb, r, dmax); });
    } else {
        nd_range(pad32(W), pad32(H), 32, 32, false, [&]() { vpm::vpmstereo_init(o, a, ga, b, gb, r, dmax); });
    }
    return 0;
}

/* vpmstereo_iter_simple (VPMStereo.cl:311-361) */
int ref_vpm_iter(float* out, const float* in, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2,
                 int W, int H, int r, float dmax, int iter)
{
    image2d_t o = img(out, W, H), i = img(in, W, H), a = img8(c1, W, H), ga = img(g1, W, H), b = img8(c2, W, H),
              gb = img(g2, W, H);
    nd_range(pad32(W), pad32(H), 32, 32, false, [&]() { vpm::vpmstereo_iter_simple(o, i, a, ga, b, gb, r, dmax, iter); });
    return 0;
}

/* vpmstereo_disparity (VPMStereo.cl:363-377) into a GRAY_FLOAT image */
int ref_vpm_disparity(float* out, const float* states, int W, int H, float scale)
{
    image2d_t o = img1(out, W, H), s = img(states, W, H);
    nd_range(pad32(W), pad32(H), 32, 32, false, [&]() { vpm::vpmstereo_disparity(o, s, scale); });
    return 0;
}

/* VPMStereoCL::disparitySimple (VPMStereoCL.cpp:54-85); states (4*W*H floats, may be NULL)
 * receives the final plane states */
int ref_vpm_disparity_simple(float* disparity, float* states, const uint8_t* c1, const uint8_t* c2, int W, int H,
                             int r, int iterations, float dmax, const float* initdisp)
{
    const size_t N = (size_t)W * H;
    std::vector<float> g1(4 * N), g2(4 * N), s0(4 * N), s1(4 * N);
    ref_vpm_grad(g1.data(), c1, W, H);
    ref_vpm_grad(g2.data(), c2, W, H);
    float* out[2] = {s0.data(), s1.data()};
    ref_vpm_init(out[1], c1, g1.data(), c2, g2.data(), W, H, r, dmax, initdisp);
    int swap = 0;
    for (int i = 0; i < iterations; i++) {
        ref_vpm_iter(out[swap], out[1 - swap], c1, g1.data(), c2, g2.data(), W, H, r, dmax, i);
        swap = 1 - swap;
    }
    ref_vpm_disparity(disparity, out[1 - swap], W, H, 1.0f);
    if (states)
        for (size_t k = 0; k < 4 * N; k++) states[k] = out[1 - swap][k];
    return 0;
}

}  // extern "C"
