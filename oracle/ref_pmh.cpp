/*
 * ORACLE — test infrastructure only.
 *
 * Glue around cvt/cl/kernel/pmhstereo.cl compiled from its own source (after
 * oracle/translate.py): each ref_k_* function launches one reference kernel
 * over the NDRange PMHuberStereo uses, (pad(W,16), pad(H,16)) with 16x16
 * work-groups (PMHuberStereo.cpp:35-36, e.g. :360).
 */
#include <cstdint>
#include <cstring>
#include <vector>

#include "ref_exec.h"

namespace clk {
namespace pmh {
#include "_ref/pmhstereo.cl.cpp"
}  // namespace pmh
}  // namespace clk

using namespace clk;

namespace {
inline int pad16(int v) { return (v + 15) / 16 * 16; }
inline image2d_t img(const float* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_RGBA_FLOAT}; }
inline image2d_t img1(const float* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_INTENSITY_FLOAT}; }
inline image2d_t img8(const uint8_t* p, int W, int H) { return image2d_t{(void*)p, W, H, IMG_RGBA_UNORM8}; }
}

extern "C" {

/* rgba8 must be packed (stride 4W) */
int ref_k_prep(const uint8_t* rgba8, int W, int H, int r, float* bw, float* grad)
{
    image2d_t src = img8(rgba8, W, H);
    image2d_t obw = img(bw, W, H), og = img(grad, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { pmh::pmhstereo_bilateral_weight_to_alpha(obw, src, r); });
    nd_range(pad16(W), pad16(H), 16, 16, true, [&]() { pmh::pmhstereo_gradxy(og, src); });
    return 0;
}

int ref_k_init(float* out, const float* bw1, const float* bw2, const float* g1, const float* g2, int W, int H, int r,
               float dmax, int lr, const float* initdisp, const float* initnormal)
{
    image2d_t o = img(out, W, H), a = img(bw1, W, H), b = img(bw2, W, H), ga = img(g1, W, H), gb = img(g2, W, H);
    if (!initdisp) {
        nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { pmh::pmhstereo_init(o, a, b, ga, gb, r, dmax, lr); });
    } else {
        image2d_t d = img1(initdisp, W, H), n = img(initnormal, W, H);
        nd_range(pad16(W), pad16(H), 16, 16, false,
                 [&]() { pmh::pmhstereo_init_disparity_normal(o, a, b, ga, gb, r, dmax, lr, d, n); });
    }
    return 0;
}

int ref_k_propagate(float* out, const float* old, const float* bw1, const float* bw2, const float* g1, const float* g2,
                    const float* smooth, float theta, int W, int H, int r, float dmax, int lr, int iter,
                    const int32_t* vin_n, const float* vin_val, int32_t* vout_n, float* vout_val)
{
    const size_t N = (size_t)W * H;
    std::vector<pmh::VIEWPROP_t> vin(N), vout(N);
    for (size_t i = 0; i < N; i++) {
        vin[i].n = vin_n ? vin_n[i] : 0;
        for (int k = 0; k < 2; k++)
            vin[i].value[k] = vin_val ? float4(vin_val[8 * i + 4 * k], vin_val[8 * i + 4 * k + 1],
                                               vin_val[8 * i + 4 * k + 2], vin_val[8 * i + 4 * k + 3])
                                      : float4(0.0f);
        vout[i].n = vout_n ? vout_n[i] : 0;
        for (int k = 0; k < 2; k++)
            vout[i].value[k] = vout_val ? float4(vout_val[8 * i + 4 * k], vout_val[8 * i + 4 * k + 1],
                                                 vout_val[8 * i + 4 * k + 2], vout_val[8 * i + 4 * k + 3])
                                        : float4(0.0f);
    }
    image2d_t o = img(out, W, H), ol = img(old, W, H), a = img(bw1, W, H), b = img(bw2, W, H);
    image2d_t ga = img(g1, W, H), gb = img(g2, W, H), sm = img(smooth, W, H);
    pmh::VIEWPROP_t* pin = vin.data();
    pmh::VIEWPROP_t* pout = vout.data();
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() {
        pmh::pmhstereo_propagate_view(o, ol, a, b, ga, gb, sm, theta, r, dmax, lr, iter, pin, pout);
    });
    if (vout_n) {
        for (size_t i = 0; i < N; i++) {
            vout_n[i] = vout[i].n;
            for (int k = 0; k < 2; k++) {
                vout_val[8 * i + 4 * k] = vout[i].value[k].x; vout_val[8 * i + 4 * k + 1] = vout[i].value[k].y;
                vout_val[8 * i + 4 * k + 2] = vout[i].value[k].z; vout_val[8 * i + 4 * k + 3] = vout[i].value[k].w;
            }
        }
    }
    return 0;
}

/* patch_eval for each pixel: not a kernel of its own in the reference, so it is
 * called per work item exactly as pmhstereo_init calls it (pmhstereo.cl:770) */
int ref_k_cost(float* cost, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
               int W, int H, int r, float mincost)
{
    image2d_t a = img(bw1, W, H), b = img(bw2, W, H), ga = img(g1, W, H), gb = img(g2, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() {
        const int x = (int)get_global_id(0), y = (int)get_global_id(1);
        if (x >= W || y >= H) return;
        const size_t i = (size_t)y * W + x;
        const float4 s(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], planes[4 * i + 3]);
        cost[i] = pmh::patch_eval(a, ga, b, gb, float2((float)x, (float)y), s, r, mincost);
    });
    return 0;
}

int ref_k_klt(float* out, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
              int W, int H, int r)
{
    image2d_t a = img(bw1, W, H), b = img(bw2, W, H), ga = img(g1, W, H), gb = img(g2, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() {
        const int x = (int)get_global_id(0), y = (int)get_global_id(1);
        if (x >= W || y >= H) return;
        const size_t i = (size_t)y * W + x;
        const float4 s(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], planes[4 * i + 3]);
        const float4 o = pmh::patch_census_klt2(a, ga, b, gb, float2((float)x, (float)y), s, r);
        out[4 * i] = o.x; out[4 * i + 1] = o.y; out[4 * i + 2] = o.z; out[4 * i + 3] = o.w;
    });
    return 0;
}

int ref_k_normal_depth(float* out, const float* planes, int W, int H, float dispscale, int lr)
{
    image2d_t o = img(out, W, H), in = img(planes, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { pmh::pmhstereo_normal_depth(o, in, dispscale, lr); });
    return 0;
}

int ref_k_consistency(float* out, const float* left, const float* right, int W, int H, float maxdd, float maxad)
{
    image2d_t o = img(out, W, H), l = img(left, W, H), rr = img(right, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { pmh::pmhstereo_consistency(o, l, rr, maxdd, maxad, 1); });
    return 0;
}

int ref_k_to_disparity(float* out, const float* planes, int W, int H, float scale, int lr)
{
    image2d_t o = img1(out, W, H), in = img(planes, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { pmh::pmhstereo_to_disparity(o, in, scale, lr); });
    return 0;
}

int ref_k_fill_depthmap(float* out, const float* planes, int W, int H, float scale)
{
    image2d_t o = img1(out, W, H), in = img(planes, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { pmh::pmhstereo_fill_depthmap(o, in, scale); });
    return 0;
}

int ref_k_fill_normalmap(float* out, const float* planes, int W, int H, int lr)
{
    image2d_t o = img(out, W, H), in = img(planes, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false, [&]() { pmh::pmhstereo_fill_normalmap(o, in, lr); });
    return 0;
}

int ref_k_fill_state(float* out, const float* planes, int W, int H, float dispscale, int lr)
{
    /* the `otherimg` argument is read but unused by the kernel (pmhstereo.cl:1144) */
    image2d_t o = img(out, W, H), in = img(planes, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, false,
             [&]() { pmh::pmhstereo_fill_state(o, in, in, dispscale, lr); });
    return 0;
}

int ref_k_disparity_to_normal(float* out, const float* disp, int W, int H)
{
    image2d_t o = img(out, W, H), in = img1(disp, W, H);
    nd_range(pad16(W), pad16(H), 16, 16, true, [&]() { pmh::pmhstereo_disparity_to_normal(o, in); });
    return 0;
}

}  // extern "C"
