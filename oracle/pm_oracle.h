/*
 * ORACLE — test infrastructure only.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load liboracle.so; the product never does.
 *
 * CPU restatement of cvt::PMHuberStereo (cvt/vision/PMHuberStereo.cpp) and of
 * the OpenCL kernels it drives (cvt/cl/kernel/pmhstereo.cl, RNG.cl, MWC64X.cl,
 * Matrix3.cl, PDDiffTensor.cl, PDDROFDiffTensor.cl).  Each function names the
 * reference lines it follows.
 *
 * Layout: an RGBA8 image is W*H*4 bytes with a row stride in bytes; every
 * float4 field (planes (a,b,c,cost), gradients, diffusion tensor, smoothing
 * state, normals) is W*H*4 floats, row-major, channel fastest; a grey field is
 * W*H floats.  The ROF dual p is a (2W)*H float4 field as in the reference.
 *
 * Arithmetic modes (argument `fused`):
 *   0  strict: every operation rounds separately, in the reference's source
 *      order; this is the mode pinned against the reference kernels compiled
 *      from their own source (oracle/build_ref.py).
 *   1  fused: inside the per-window-sample loops (ASW cost, Gauss-Newton
 *      plane step, support-weight sum) the products named in
 *      pm_oracle.cpp (ORC_HOT) are contracted into fused multiply-adds, the
 *      contraction OpenCL's FP_CONTRACT permits.  Everything else is strict.
 *   The CUDA kernels implement both modes; fused is their default.
 *
 * View-propagation order: the reference appends cross-view candidates with
 * atomic_inc (pmhstereo.cl:1063-1067), so which two survive depends on work
 * item scheduling.  The oracle fixes the order of a sequential OpenCL
 * executor: within an image row, sources are appended in ascending x, so the
 * two kept candidates are those from the two smallest source columns.
 */
#ifndef PM_ORACLE_H
#define PM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* counters[0] = ASW cost window samples evaluated (passed the skip test)
 * counters[1] = Gauss-Newton window samples with the 3-point cost evaluated
 * counters[2] = patch_eval calls that entered the window loop
 * counters[3] = early exits taken
 * Evaluations of candidates whose plane equals the current plane and whose outcome is
 * known are not counted: the CUDA kernels skip them (try_candidate in pm_oracle.cpp). */
enum { ORC_NCOUNTERS = 4 };

int orc_version(void);

/* pmhstereo_bilateral_weight_to_alpha (pmhstereo.cl:1462-1498) + pmhstereo_gradxy
 * (:1549-1602) + PDDiffTensorColor (PDDiffTensor.cl:26-75, alpha 24, beta 1)   */
int orc_prep(const uint8_t* img, int W, int H, int stride, int r, int fused,
             float* bw, float* grad, float* dt);

/* pmhstereo_init / pmhstereo_init_disparity_normal (pmhstereo.cl:755-828) */
int orc_init(float* out, const float* bw1, const float* bw2, const float* g1, const float* g2,
             int W, int H, int r, float dmax, int lr, const float* initdisp, const float* initnormal,
             int fused);

/* pmhstereo_propagate_view (pmhstereo.cl:880-1071).  viewin/viewout use the
 * reference's VIEWPROP_t content split in three arrays: n[W*H] (int32),
 * val[W*H*8] (two float4), and, for viewout only, src[W*H*2] (source column of
 * each kept value, -1 if none; not part of the reference, used by tests).   */
int orc_propagate(float* out, const float* old, const float* bw1, const float* bw2,
                  const float* g1, const float* g2, const float* smooth, float theta,
                  int W, int H, int r, float dmax, int lr, int iter,
                  const int32_t* vin_n, const float* vin_val,
                  int32_t* vout_n, float* vout_val, int32_t* vout_src,
                  int fused, int64_t* counters);

/* patch_eval_census for every pixel with a given plane field and mincost (test hook) */
int orc_cost(float* cost, const float* planes, const float* bw1, const float* bw2,
             const float* g1, const float* g2, int W, int H, int r, float mincost, int fused);

/* patch_census_klt2 once per pixel (test hook); out = planes after one step */
int orc_klt(float* out, const float* planes, const float* bw1, const float* bw2,
            const float* g1, const float* g2, int W, int H, int r, int fused);

/* pmhstereo_normal_depth (pmhstereo.cl:1384-1402) */
int orc_normal_depth(float* out, const float* planes, int W, int H, float dispscale, int lr);

/* PDOptCL::denoiseDiffusionTensorROF_PDD (PDOptCL.cpp:1114-1168) over PDDROFDiffTensor
 * (PDDROFDiffTensor.cl:43-127): iters primal-dual steps from u=input, p=q=0  */
int orc_rof(float* out, const float* input, const float* dt, const float lambda[4], int iters, int W, int H);

/* pmhstereo_consistency (pmhstereo.cl:1095-1129) */
int orc_consistency(float* out, const float* left, const float* right, int W, int H,
                    float maxdispdiff, float maxanglediff);
/* pmhstereo_to_disparity (:1232-1257), pmhstereo_fill_depthmap (:1187-1230),
 * pmhstereo_fill_normalmap (:1259-1305), pmhstereo_disparity_to_normal (:1604-1637) */
int orc_to_disparity(float* out, const float* planes, int W, int H, float scale, int lr);
int orc_fill_depthmap(float* out, const float* planes, int W, int H, float scale);
int orc_fill_normalmap(float* out, const float* planes, int W, int H, int lr);
int orc_disparity_to_normal(float* out, const float* disp, int W, int H);

/* MWC64X seeded and skipped by linpos * nd, followed by `ndraws` RNG_float draws (RNG.cl:54-57, MWC64X.cl) */
int orc_rng_floats(int64_t linpos, int nd, int ndraws, float* out);
/* out[0]: candidates the CUDA kernels skip as known (plane equal to the current one, see
 * try_candidate in pm_oracle.cpp) since the library was loaded; out[1]: those of them that
 * changed the state when evaluated (must stay 0) */
void orc_known_counts(int64_t out[2]);
/* elementary functions, for tests */
float orc_exp(float x);
float orc_log(float x);
float orc_sin(float x);
float orc_cos(float x);
float orc_acospi(float x);

/* PMHuberStereo::disparityMap + disparityMapAll (PMHuberStereo.cpp:75-143, :406-581)
 * pp: 0 none, 1 LR check, 2 LR check + fill.  views: 2 (reference) or 1 (left only,
 * pp must be 0).  planesL/planesR/normal may be NULL.  counters may be NULL.  */
int orc_disparity_map(const uint8_t* left, const uint8_t* right, int W, int H, int stride,
                      int r, float dmax, int iterations, int pp, int views,
                      float* dmap, float* normal, const float* initdisp, const float* initnormal,
                      float* planesL, float* planesR, int fused, int64_t* counters);

/* depthMap's inputs (PMHuberStereo.cpp:184-190, :203-204): the image as floats (r, g, b, a),
 * pmhstereo_gradxy, and PDDiffTensorColor with edge weight alpha (beta 1) */
int orc_prep_raw(const uint8_t* img, int W, int H, int stride, float alpha, float* colour, float* grad, float* dt);
/* pmhstereo_fill_state (pmhstereo.cl:1131-1185) */
int orc_fill_state(float* out, const float* planes, int W, int H, float dispscale, int lr);
/* PDOptCL::denoiseDiffusionTensorHuber_PDD (PDOptCL.cpp:1170-1226) over PDDHuberDiffTensor
 * (PDDHuberDiffTensor.cl:38-107): iters primal-dual steps from u = input, p = q = 0 */
int orc_huber(float* out, const float* input, const float* dt, const float lambda[4], float eps, int iters, int W, int H);

/* pyrdown (cvt/cl/kernel/pyr/pyrdown.cl): RGBA8 Wi x Hi -> RGBA8 Wo x Ho, tight rows */
int orc_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, int Wi, int Hi);
/* pyrup_mul4f (cvt/cl/kernel/pyr/pyrupmul.cl): float images of 1 or 4 channels */
int orc_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, const float mul[4]);

/* as orc_disparity_map with `levels` pyramid levels (1: the reference's setting), calling
 * dump(stage, iter, W, H, field, user) after init, each propagate pair and each smoothing
 * pair with the W*H*4 float field of that stage (NULL: no dumps) */
int orc_disparity_map_dump(const uint8_t* left, const uint8_t* right, int W, int H, int stride,
                           int r, float dmax, int iterations, int pp, int views, int levels,
                           float* dmap, float* normal, const float* initdisp, const float* initnormal,
                           float* planesL, float* planesR, int fused, int64_t* counters,
                           void (*dump)(const char*, int, int, int, const float*, void*), void* user);

/* PMHuberStereo::depthMap (PMHuberStereo.cpp:145-347); dscale <= 0 means 1 / dmax */
int orc_depth_map_dump(const uint8_t* left, const uint8_t* right, int W, int H, int stride, int r, float dmax,
                       int iterations, float dscale, int pp, int views, float* dmap, float* normal,
                       const float* initdisp, const float* initnormal, float* planesL, float* planesR, int fused,
                       int64_t* counters, void (*dump)(const char*, int, int, int, const float*, void*), void* user);

/* VPMStereoCL (cvt/vision/VPMStereoCL.cpp, cvt/cl/kernel/VPMStereo.cl, gradxy.cl): colour
 * images RGBA8 with `stride` bytes per row, plane states W*H*4 floats (a, b, c, cost) */
int orc_vpm_grad(float* out, const uint8_t* img, int W, int H, int stride);
int orc_vpm_init(float* out, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2, int W, int H,
                 int stride, int r, float dmax, const float* initdisp);
int orc_vpm_iter(float* out, const float* in, const uint8_t* c1, const float* g1, const uint8_t* c2,
                 const float* g2, int W, int H, int stride, int r, float dmax, int iter);
int orc_vpm_disparity(float* out, const float* states, int W, int H, float scale);
/* VPMStereoCL::disparitySimple; states (NULL: not returned) gets the final plane states */
int orc_vpm_disparity_simple(float* disparity, float* states, const uint8_t* c1, const uint8_t* c2, int W, int H,
                             int stride, int r, int iterations, float dmax, const float* initdisp);

/* SVPMFlowCL (cvt/vision/SVPMFlowCL.cpp, cvt/cl/kernel/SVPMFlow.cl): RGBA8 frames with
 * `stride` bytes per row, states and duals W*H float4, flow W*H float2 */
int orc_svpm_init(float* out, const uint8_t* img1, const uint8_t* img2, int W, int H, int stride, int r, float flowmax);
int orc_svpm_prop(float* out, float* pout, const float* in, const float* pin, const uint8_t* img1,
                  const uint8_t* img2, int W, int H, int stride, int r, float flowmax, int iter);
int orc_svpm_to_flow(float* flow, const float* states, int W, int H);
int orc_svpm_flow(float* flow, float* states, float* duals, const uint8_t* img1, const uint8_t* img2, int W, int H,
                  int stride, int r, float flowmax, int iterations);

#ifdef __cplusplus
}
#endif
#endif
