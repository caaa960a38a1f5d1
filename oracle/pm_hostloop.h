/*
 * ORACLE — test infrastructure only.
 *
 * Restatement of the host side of cvt::PMHuberStereo::disparityMap and
 * disparityMapAll (cvt/vision/PMHuberStereo.cpp:75-143, :406-581) without the
 * PMDEBUG blocks (which block on getchar() and write PNG files, :495-529).  It
 * is shared by the oracle restatement (pm_oracle.cpp) and by the driver of the
 * reference kernels compiled from their own source (ref_driver.cpp); each
 * supplies the kernel entry points through PmKernels.
 */
#ifndef PM_ORACLE_HOSTLOOP_H
#define PM_ORACLE_HOSTLOOP_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

struct PmKernels {
    int (*prep)(const uint8_t*, int, int, int, int, int, float*, float*, float*);
    int (*init)(float*, const float*, const float*, const float*, const float*, int, int, int, float, int,
                const float*, const float*, int);
    int (*propagate)(float*, const float*, const float*, const float*, const float*, const float*, const float*,
                     float, int, int, int, float, int, int, const int32_t*, const float*, int32_t*, float*,
                     int32_t*, int, int64_t*);
    int (*normal_depth)(float*, const float*, int, int, float, int);
    int (*rof)(float*, const float*, const float*, const float*, int, int, int);
    int (*consistency)(float*, const float*, const float*, int, int, float, float);
    int (*to_disparity)(float*, const float*, int, int, float, int);
    int (*fill_depthmap)(float*, const float*, int, int, float);
    int (*fill_normalmap)(float*, const float*, int, int, int);
    int (*disparity_to_normal)(float*, const float*, int, int);
};

/* Optional per-stage dump: called with a stage name and a W*H*4 float field. */
typedef void (*PmDumpFn)(const char* stage, int iter, const float* field, void* user);

static inline int pm_host_disparity_map(const PmKernels& K, const uint8_t* left, const uint8_t* right, int W,
                                        int H, int stride, int r, float dmax, int iterations, int pp, int views,
                                        float* dmap, float* normal, const float* initdisp, const float* initnormal,
                                        float* planesL, float* planesR, int fused, int64_t* counters,
                                        PmDumpFn dump, void* user)
{
    if (W <= 0 || H <= 0 || r < 0 || iterations < 0) return -1;
    if (views != 1 && views != 2) return -1;
    if (views == 1 && pp != 0) return -1;
    const size_t N = (size_t)W * H;
    std::vector<float> Lbw(4 * N), Rbw(4 * N), Lg(4 * N), Rg(4 * N), LDT(4 * N), RDT(4 * N);
    std::vector<float> Ls(4 * N, 0.0f), Rs(4 * N, 0.0f), tmp(4 * N);   /* clear() (:457-458) */
    std::vector<float> mL[2] = {std::vector<float>(4 * N), std::vector<float>(4 * N)};
    std::vector<float> mR[2] = {std::vector<float>(4 * N), std::vector<float>(4 * N)};
    std::vector<int32_t> vb1n(N, 0), vb2n(N, 0);
    std::vector<float> vb1v(8 * N, 0.0f), vb2v(8 * N, 0.0f);
    const float thetamin = 1e-4f;                                              /* :92 */
    float theta = thetamin;
    K.prep(left, W, H, stride, r, fused, Lbw.data(), Lg.data(), LDT.data());     /* :445-454 */
    K.prep(right, W, H, stride, r, fused, Rbw.data(), Rg.data(), RDT.data());
    std::vector<float> nrm;
    const float* initn = initnormal;
    if (initdisp && !initnormal) {                                             /* :363-365 */
        nrm.resize(4 * N);
        K.disparity_to_normal(nrm.data(), initdisp, W, H);
        initn = nrm.data();
    }
    K.init(mL[0].data(), Lbw.data(), Rbw.data(), Lg.data(), Rg.data(), W, H, r, dmax, 1, initdisp, initn, fused);
    if (views == 2)
        K.init(mR[0].data(), Rbw.data(), Lbw.data(), Rg.data(), Lg.data(), W, H, r, dmax, 0, nullptr, nullptr, fused);
    if (dump) { dump("init_left", -1, mL[0].data(), user); if (views == 2) dump("init_right", -1, mR[0].data(), user); }
    if (initdisp) {                                                            /* :473-477 */
        const float lam[4] = {theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, 1.0f};
        K.normal_depth(tmp.data(), mL[0].data(), W, H, 1.0f / dmax, 1);
        K.rof(Ls.data(), tmp.data(), LDT.data(), lam, 40, W, H);
    }
    int swap = 0;
    iterations |= 1;                                                           /* :490 */
    for (int iter = 0; iter < iterations; iter++) {
        const float lam[4] = {theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, 1.0f};   /* :532 */
        std::fill(vb1n.begin(), vb1n.end(), 0);                                                            /* :534 */
        K.propagate(mL[1 - swap].data(), mL[swap].data(), Lbw.data(), Rbw.data(), Lg.data(), Rg.data(), Ls.data(),
                    theta * 50.0f, W, H, r, dmax, 1, iter, vb2n.data(), vb2v.data(),
                    views == 2 ? vb1n.data() : nullptr, vb1v.data(), nullptr, fused, counters);
        if (views == 2) {
            std::fill(vb2n.begin(), vb2n.end(), 0);                                                        /* :540 */
            K.propagate(mR[1 - swap].data(), mR[swap].data(), Rbw.data(), Lbw.data(), Rg.data(), Lg.data(), Rs.data(),
                        theta * 50.0f, W, H, r, dmax, 0, iter, vb1n.data(), vb1v.data(), vb2n.data(), vb2v.data(),
                        nullptr, fused, counters);
        }
        if (dump) { dump("prop_left", iter, mL[1 - swap].data(), user); if (views == 2) dump("prop_right", iter, mR[1 - swap].data(), user); }
        K.normal_depth(tmp.data(), mL[1 - swap].data(), W, H, 1.0f / dmax, 1);                             /* :552-553 */
        K.rof(Ls.data(), tmp.data(), LDT.data(), lam, 40, W, H);
        if (views == 2) {
            K.normal_depth(tmp.data(), mR[1 - swap].data(), W, H, 1.0f / dmax, 0);                         /* :566-567 */
            K.rof(Rs.data(), tmp.data(), RDT.data(), lam, 40, W, H);
        }
        if (dump) { dump("smooth_left", iter, Ls.data(), user); if (views == 2) dump("smooth_right", iter, Rs.data(), user); }
        theta = (float)iter / (float)iterations;                                                          /* :575-576 */
        theta = powf(theta, 4.0f) + thetamin;
        swap = 1 - swap;
    }
    const std::vector<float>& ml = mL[1];
    if (planesL) memcpy(planesL, ml.data(), 4 * N * sizeof(float));
    if (planesR && views == 2) memcpy(planesR, mR[1].data(), 4 * N * sizeof(float));
    if (pp == 0) {                                                             /* :123-129 */
        if (dmap) K.to_disparity(dmap, ml.data(), W, H, 1.0f, 1);
        if (normal) K.fill_normalmap(normal, ml.data(), W, H, 1);
    } else {                                                                   /* :130-141 */
        std::vector<float> chk(4 * N);
        K.consistency(chk.data(), ml.data(), mR[1].data(), W, H, 1.0f, 5.0f);
        if (dump) dump("consistency", -1, chk.data(), user);
        if (dmap) {
            if (pp == 1) K.to_disparity(dmap, chk.data(), W, H, 1.0f, 1);
            else K.fill_depthmap(dmap, chk.data(), W, H, 1.0f);
        }
        if (normal) K.fill_normalmap(normal, chk.data(), W, H, 1);
    }
    return 0;
}

#endif
