/*
 * ORACLE — test infrastructure only.
 *
 * Glue around cvt/cl/kernel/PDDiffTensor.cl and PDDROFDiffTensor.cl compiled
 * from their own source: PDOptCL::diffusionTensor (PDOptCL.cpp:134-155) and
 * PDOptCL::denoiseDiffusionTensorROF_PDD (PDOptCL.cpp:1114-1168), including the
 * buffer ping-pong of the latter.
 */
#include <cstdint>
#include <cstring>
#include <vector>

#include "ref_exec.h"

namespace clk {
namespace pdt {
#include "_ref/PDDiffTensor.cl.cpp"
}  // namespace pdt
}  // namespace clk

namespace clk {
namespace rof {
#include "_ref/PDDROFDiffTensor.cl.cpp"
}  // namespace rof
}  // namespace clk

namespace clk {
namespace hub {
#include "_ref/PDDHuberDiffTensor.cl.cpp"
}  // namespace hub
}  // namespace clk

using namespace clk;

namespace {
inline int pad16(int v) { return (v + 15) / 16 * 16; }
inline image2d_t img(const float* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_RGBA_FLOAT}; }
}

extern "C" {

int ref_k_difftensor(const uint8_t* rgba8, int W, int H, float alpha, float beta, float* dt)
{
    image2d_t src{(void*)rgba8, W, H, IMG_RGBA_UNORM8};
    image2d_t o = img(dt, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, true, [&]() { pdt::PDDiffTensorColor(o, src, alpha, beta); });
    return 0;
}

/* PDOptCL::denoiseDiffusionTensorHuber_PDD (PDOptCL.cpp:1170-1226): the buffer ping-pong of the
 * ROF variant below with the PDDHuberDiffTensor kernel */
int ref_k_huber(float* out, const float* input, const float* dt, const float lambda[4], float eps, int iters, int W,
                int H)
{
    const size_t N = (size_t)W * H;
    std::vector<float> tmpu(4 * N, 0.0f), outu(input, input + 4 * N);
    std::vector<float> p1(8 * N, 0.0f), p2(8 * N, 0.0f), q1(4 * N, 0.0f), q2(4 * N, 0.0f);
    image2d_t climg[2] = {img(tmpu.data(), W, H), img(outu.data(), W, H)};
    image2d_t clp[2] = {img(p1.data(), 2 * W, H), img(p2.data(), 2 * W, H)};
    image2d_t clq[2] = {img(q1.data(), W, H), img(q2.data(), W, H)};
    image2d_t in = img(input, W, H), d = img(dt, W, H);
    const float4 lam(lambda[0], lambda[1], lambda[2], lambda[3]);
    auto step = [&](int s) {
        nd_range(pad16(W), pad16(H), 16, 16, true, [&]() {
            static thread_local float4 lbuf[18 * 18];
            static thread_local float8 lbuf2[18 * 18];
            hub::PDDHuberDiffTensor(climg[s], clp[s], clq[s], climg[1 - s], clp[1 - s], clq[1 - s], in, d, lam, eps,
                                    lbuf, lbuf2);
        });
    };
    int swap = 0;
    for (int i = 0; i < iters; i++) {
        swap = i & 1;
        step(swap);
    }
    if (!swap) step(1);   /* (:1211-1225): one more step back into `output` */
    memcpy(out, outu.data(), 4 * N * sizeof(float));
    return 0;
}

int ref_k_rof(float* out, const float* input, const float* dt, const float lambda[4], int iters, int W, int H)
{
    const size_t N = (size_t)W * H;
    /* output = input (:1119-1120); p/q images, fill(clp[1]) and fill(clq[1]) with 0 (:1131-1132) */
    std::vector<float> tmpu(4 * N, 0.0f), outu(input, input + 4 * N);
    std::vector<float> p1(8 * N, 0.0f), p2(8 * N, 0.0f), q1(4 * N, 0.0f), q2(4 * N, 0.0f);
    image2d_t climg[2] = {img(tmpu.data(), W, H), img(outu.data(), W, H)};
    image2d_t clp[2] = {img(p1.data(), 2 * W, H), img(p2.data(), 2 * W, H)};
    image2d_t clq[2] = {img(q1.data(), W, H), img(q2.data(), W, H)};
    image2d_t in = img(input, W, H), d = img(dt, W, H);
    const float4 lam(lambda[0], lambda[1], lambda[2], lambda[3]);
    int swap = 0;
    auto step = [&](int s) {
        nd_range(pad16(W), pad16(H), 16, 16, true, [&]() {
            static thread_local float4 lbuf[18 * 18];
            static thread_local float8 lbuf2[18 * 18];
            rof::PDDROFDiffTensor(climg[s], clp[s], clq[s], climg[1 - s], clp[1 - s], clq[1 - s], in, d, lam, lbuf, lbuf2);
        });
    };
    for (int i = 0; i < iters; i++) {
        swap = i & 1;
        step(swap);
    }
    if (!swap) {
        /* (:1152-1166): one more step back into `output` */
        nd_range(pad16(W), pad16(H), 16, 16, true, [&]() {
            static thread_local float4 lbuf[18 * 18];
            static thread_local float8 lbuf2[18 * 18];
            rof::PDDROFDiffTensor(climg[1], clp[1], clq[1], climg[0], clp[0], clq[0], in, d, lam, lbuf, lbuf2);
        });
    }
    memcpy(out, outu.data(), 4 * N * sizeof(float));
    return 0;
}

}  // extern "C"
