/*
 * ORACLE — test infrastructure only.
 *
 * Glue around cvt/cl/kernel/SVPMFlow.cl compiled from its own source (after
 * oracle/translate.py, which also separates the reads and writes of its neighbour tests by a
 * barrier): each ref_svpm_* function launches one reference kernel over the NDRange
 * SVPMFlowCL uses, (pad(W,16), pad(H,16)) with 16x16 work-groups (cvt/vision/SVPMFlowCL.cpp:36-37,
 * e.g. :173), and ref_svpm_flow runs SVPMFlowCL::flow (:58-89) with a given number of passes
 * (the reference: MAXITER = 200) and without its debugging block (:74-84).
 */
#include <cstdint>
#include <cstring>
#include <vector>

#include "ref_exec.h"

namespace clk {
namespace svpm {
#include "_ref/SVPMFlow.cl.cpp"
}  // namespace svpm
}  // namespace clk

using namespace clk;

namespace {
inline int pad16(int v) { return (v + 15) / 16 * 16; }
inline image2d_t img(const float* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_RGBA_FLOAT}; }
inline image2d_t img8(const uint8_t* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_RGBA_UNORM8}; }
}  // namespace

extern "C" {

/* svpmflow_init (SVPMFlow.cl:213-233); images packed RGBA8 */
int ref_svpm_init(float* out, const uint8_t* img1, const uint8_t* img2, int W, int H, int r, float flowmax)
{
    image2d_t o = img(out, W, H), a = img8(img1, W, H), b = img8(img2, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { svpm::svpmflow_init(o, a, b, r, flowmax); });
    return 0;
}

/* svpmflow_prop_local_tv_admm (:574-731) */
int ref_svpm_prop(float* out, float* pout, const float* in, const float* pin, const uint8_t* img1, const uint8_t* img2,
                  int W, int H, int r, float flowmax, int iter)
{
    image2d_t o = img(out, W, H), i = img(in, W, H), po = img(pout, W, H), pi = img(pin, W, H);
    image2d_t a = img8(img1, W, H), b = img8(img2, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, true,
             [&]() { svpm::svpmflow_prop_local_tv_admm(o, i, a, b, po, pi, r, flowmax, iter); });
    return 0;
}

/* svpmflow_flow (:733-744) into a GRAYALPHA_FLOAT (CL_RG) image: (u, v) per pixel */
int ref_svpm_to_flow(float* flow, const float* states, int W, int H)
{
    std::vector<float> tmp((size_t)W * H * 4);
    image2d_t o = img(tmp.data(), W, H), s = img(states, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { svpm::svpmflow_flow(o, s); });
    for (size_t k = 0; k < (size_t)W * H; k++) {
        flow[2 * k] = tmp[4 * k];
        flow[2 * k + 1] = tmp[4 * k + 1];
    }
    return 0;
}

/* SVPMFlowCL::flow (SVPMFlowCL.cpp:58-89) */
int ref_svpm_flow(float* flow, float* states, float* duals, const uint8_t* img1, const uint8_t* img2, int W, int H,
                  int r, float flowmax, int iterations)
{
    const size_t N = (size_t)W * H;
    std::vector<float> s0(4 * N), s1(4 * N), p0(4 * N, 0.0f), p1(4 * N, 0.0f);
    float* buf[2] = {s0.data(), s1.data()};
    float* bufp[2] = {p0.data(), p1.data()};
    ref_svpm_init(buf[1], img1, img2, W, H, r, flowmax);
    for (int i = 0; i < iterations; i++) {
        const int swap = i & 1;
        ref_svpm_prop(buf[swap], bufp[swap], buf[1 - swap], bufp[1 - swap], img1, img2, W, H, r, flowmax, i + 1);
    }
    const int last = 1 - (iterations & 1);
    ref_svpm_to_flow(flow, buf[last], W, H);
    if (states) memcpy(states, buf[last], 4 * N * sizeof(float));
    if (duals) memcpy(duals, bufp[last], 4 * N * sizeof(float));
    return 0;
}

}  // extern "C"
