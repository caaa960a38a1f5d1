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
#include <stdio.h>
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
    int (*pyrdown)(uint8_t*, int, int, const uint8_t*, int, int);
    int (*pyrup_mul)(float*, int, int, const float*, int, int, int, const float*);
    int (*prep_raw)(const uint8_t*, int, int, int, float, float*, float*, float*);
    int (*fill_state)(float*, const float*, int, int, float, int);
    int (*huber)(float*, const float*, const float*, const float*, float, int, int, int);
};

/* Optional per-stage dump: called with a stage name and a W*H*4 float field.  Stages of a
 * pyramid level l > 0 carry the prefix "l<l>_". */
typedef void (*PmDumpFn)(const char* stage, int iter, int W, int H, const float* field, void* user);

/* PMHuberStereo::disparityMapAll (PMHuberStereo.cpp:406-581) on one pyramid level: the
 * final plane fields are left in mLout, mRout (W*H*4 floats each).  Left images are
 * RGBA8 with a row stride; the init images are W*H fields (NULL: none). */
static inline int pm_host_level(const PmKernels& K, const uint8_t* left, const uint8_t* right, int W, int H,
                                int stride, int r, float dmax, int iterations, int views, float thetamin,
                                const float* initdL, const float* initdR, const float* initnL,
                                const float* initnR, int fused, int64_t* counters, PmDumpFn dump, void* user,
                                const char* pfx, float* mLout, float* mRout)
{
    const size_t N = (size_t)W * H;
    std::vector<float> Lbw(4 * N), Rbw(4 * N), Lg(4 * N), Rg(4 * N), LDT(4 * N), RDT(4 * N);
    std::vector<float> Ls(4 * N, 0.0f), Rs(4 * N, 0.0f), tmp(4 * N);   /* clear() (:457-458) */
    std::vector<float> mL[2] = {std::vector<float>(4 * N), std::vector<float>(4 * N)};
    std::vector<float> mR[2] = {std::vector<float>(4 * N), std::vector<float>(4 * N)};
    std::vector<int32_t> vb1n(N, 0), vb2n(N, 0);
    std::vector<float> vb1v(8 * N, 0.0f), vb2v(8 * N, 0.0f);
    float theta = thetamin;
    char name[64];
    auto stage = [&](const char* s, int it, const float* f) {
        if (!dump) return;
        snprintf(name, sizeof name, "%s%s", pfx, s);
        dump(name, it, W, H, f, user);
    };
    K.prep(left, W, H, stride, r, fused, Lbw.data(), Lg.data(), LDT.data());     /* :445-454 */
    K.prep(right, W, H, stride, r, fused, Rbw.data(), Rg.data(), RDT.data());
    /* init (:469-470, :349-379): a given disparity without normals gets normals from it */
    std::vector<float> nrmL, nrmR;
    if (initdL && !initnL) {
        nrmL.resize(4 * N);
        K.disparity_to_normal(nrmL.data(), initdL, W, H);
        initnL = nrmL.data();
    }
    if (initdR && !initnR) {
        nrmR.resize(4 * N);
        K.disparity_to_normal(nrmR.data(), initdR, W, H);
        initnR = nrmR.data();
    }
    K.init(mL[0].data(), Lbw.data(), Rbw.data(), Lg.data(), Rg.data(), W, H, r, dmax, 1, initdL, initnL, fused);
    if (views == 2)
        K.init(mR[0].data(), Rbw.data(), Lbw.data(), Rg.data(), Lg.data(), W, H, r, dmax, 0, initdR, initnR, fused);
    stage("init_left", -1, mL[0].data());
    if (views == 2) stage("init_right", -1, mR[0].data());
    if (initdL) {                                                              /* :473-477 */
        const float lam[4] = {theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, 1.0f};
        K.normal_depth(tmp.data(), mL[0].data(), W, H, 1.0f / dmax, 1);
        K.rof(Ls.data(), tmp.data(), LDT.data(), lam, 40, W, H);
    }
    if (initdR && views == 2) {                                                /* :479-483 */
        const float lam[4] = {theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, 1.0f};
        K.normal_depth(tmp.data(), mR[0].data(), W, H, 1.0f / dmax, 0);
        K.rof(Rs.data(), tmp.data(), RDT.data(), lam, 40, W, H);
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
        stage("prop_left", iter, mL[1 - swap].data());
        if (views == 2) stage("prop_right", iter, mR[1 - swap].data());
        K.normal_depth(tmp.data(), mL[1 - swap].data(), W, H, 1.0f / dmax, 1);                             /* :552-553 */
        K.rof(Ls.data(), tmp.data(), LDT.data(), lam, 40, W, H);
        if (views == 2) {
            K.normal_depth(tmp.data(), mR[1 - swap].data(), W, H, 1.0f / dmax, 0);                         /* :566-567 */
            K.rof(Rs.data(), tmp.data(), RDT.data(), lam, 40, W, H);
        }
        stage("smooth_left", iter, Ls.data());
        if (views == 2) stage("smooth_right", iter, Rs.data());
        theta = (float)iter / (float)iterations;                                                          /* :575-576 */
        theta = powf(theta, 4.0f) + thetamin;
        swap = 1 - swap;
    }
    memcpy(mLout, mL[1].data(), 4 * N * sizeof(float));
    if (views == 2) memcpy(mRout, mR[1].data(), 4 * N * sizeof(float));
    return 0;
}

/* size of the next pyramid level: CLPyramid::update (cvt/cl/CLPyramid.cpp:51-57) multiplies
 * the size_t width by the float scale 0.35f and truncates */
static inline int pm_pyr_next(int n) { return (int)(size_t)((float)(size_t)n * 0.35f); }

/* PMHuberStereo::disparityMap (PMHuberStereo.cpp:75-143) with `levels` pyramid levels (the
 * reference fixes levels = 1, :78; levels > 1 runs its coarse-to-fine loop, :94-120). */
static inline int pm_host_disparity_map(const PmKernels& K, const uint8_t* left, const uint8_t* right, int W,
                                        int H, int stride, int r, float dmax, int iterations, int pp, int views,
                                        int levels, float* dmap, float* normal, const float* initdisp,
                                        const float* initnormal, float* planesL, float* planesR, int fused,
                                        int64_t* counters, PmDumpFn dump, void* user)
{
    if (W <= 0 || H <= 0 || r < 0 || iterations < 0 || levels < 1) return -1;
    if (views != 1 && views != 2) return -1;
    if (views == 1 && pp != 0) return -1;
    const size_t N = (size_t)W * H;
    std::vector<float> ml(4 * N), mr(4 * N);
    if (levels == 1) {
        pm_host_level(K, left, right, W, H, stride, r, dmax, iterations, views, 1e-4f, initdisp, nullptr, initnormal,
                      nullptr, fused, counters, dump, user, "", ml.data(), mr.data());   /* :92-93 */
    } else {
        /* CLPyramid(0.35f, levels) of both images (:83-87); level 0 is the input */
        std::vector<int> Wl(levels), Hl(levels);
        std::vector<std::vector<uint8_t>> pl(levels), pr(levels);
        Wl[0] = W;
        Hl[0] = H;
        pl[0].resize(4 * N);
        pr[0].resize(4 * N);
        for (int y = 0; y < H; y++) {
            memcpy(&pl[0][(size_t)y * W * 4], left + (size_t)y * stride, (size_t)W * 4);
            memcpy(&pr[0][(size_t)y * W * 4], right + (size_t)y * stride, (size_t)W * 4);
        }
        for (int l = 1; l < levels; l++) {
            Wl[l] = pm_pyr_next(Wl[l - 1]);
            Hl[l] = pm_pyr_next(Hl[l - 1]);
            if (Wl[l] < 1 || Hl[l] < 1) return -1;
            pl[l].resize((size_t)Wl[l] * Hl[l] * 4);
            pr[l].resize((size_t)Wl[l] * Hl[l] * 4);
            K.pyrdown(pl[l].data(), Wl[l], Hl[l], pl[l - 1].data(), Wl[l - 1], Hl[l - 1]);
            K.pyrdown(pr[l].data(), Wl[l], Hl[l], pr[l - 1].data(), Wl[l - 1], Hl[l - 1]);
        }
        /* coarsest level with the caller's init images, read at the level's integer
         * coordinates (SAMPLER_NN, pmhstereo.cl:815-816): their top-left corner */
        const int L = levels - 1;
        const size_t NL = (size_t)Wl[L] * Hl[L];
        std::vector<float> id, in, nfull;
        const float* initn = initnormal;
        if (initdisp && !initnormal) {                                         /* :363-365, at the image's size */
            nfull.resize(4 * N);
            K.disparity_to_normal(nfull.data(), initdisp, W, H);
            initn = nfull.data();
        }
        if (initdisp) {
            id.resize(NL);
            in.resize(4 * NL);
            for (int y = 0; y < Hl[L]; y++) {
                memcpy(&id[(size_t)y * Wl[L]], initdisp + (size_t)y * W, (size_t)Wl[L] * sizeof(float));
                memcpy(&in[4 * (size_t)y * Wl[L]], initn + 4 * (size_t)y * W, (size_t)Wl[L] * 4 * sizeof(float));
            }
        }
        std::vector<float> cl(4 * NL), cr(4 * NL);
        char pfx[16];
        snprintf(pfx, sizeof pfx, "l%d_", L);
        const float dmaxL = dmax * ((float)Wl[L] / (float)Wl[0]);             /* :91 */
        pm_host_level(K, pl[L].data(), pr[L].data(), Wl[L], Hl[L], 4 * Wl[L], r, dmaxL, iterations, views, 1e-4f,
                      initdisp ? id.data() : nullptr, nullptr, initdisp ? in.data() : nullptr, nullptr, fused,
                      counters, dump, user, pfx, cl.data(), cr.data());
        for (int l = L - 1; l >= 0; l--) {                                     /* :94-120 */
            const int Wc = Wl[l + 1], Hc = Hl[l + 1], Wf = Wl[l], Hf = Hl[l];
            const size_t Nc = (size_t)Wc * Hc, Nf = (size_t)Wf * Hf;
            std::vector<float> t1(Nc), t4(4 * Nc), dl(Nf), dr(Nf), nl(4 * Nf), nr(4 * Nf);
            const float up = (float)Wf / (float)Wc;
            const float mulD[4] = {up, up, up, up}, mulN[4] = {1.0f, 1.0f, 1.0f, 1.0f};
            K.to_disparity(t1.data(), cl.data(), Wc, Hc, 1.0f, 1);
            K.pyrup_mul(dl.data(), Wf, Hf, t1.data(), Wc, Hc, 1, mulD);
            K.to_disparity(t1.data(), cr.data(), Wc, Hc, 1.0f, 0);
            K.pyrup_mul(dr.data(), Wf, Hf, t1.data(), Wc, Hc, 1, mulD);
            K.fill_normalmap(t4.data(), cl.data(), Wc, Hc, 1);
            K.pyrup_mul(nl.data(), Wf, Hf, t4.data(), Wc, Hc, 4, mulN);
            K.fill_normalmap(t4.data(), cr.data(), Wc, Hc, 0);
            K.pyrup_mul(nr.data(), Wf, Hf, t4.data(), Wc, Hc, 4, mulN);
            const float mintheta = (float)(levels - l) / (float)levels;
            const float dmaxl = dmax * ((float)Wf / (float)Wl[0]);
            std::vector<float> fl(4 * Nf), fr(4 * Nf);
            snprintf(pfx, sizeof pfx, l ? "l%d_" : "", l);
            pm_host_level(K, pl[l].data(), pr[l].data(), Wf, Hf, 4 * Wf, r, dmaxl, iterations, views,
                          1e-1f * mintheta + 1e-4f, dl.data(), views == 2 ? dr.data() : nullptr, nl.data(),
                          views == 2 ? nr.data() : nullptr, fused, counters, dump, user, pfx, fl.data(), fr.data());
            cl.swap(fl);
            cr.swap(fr);
        }
        ml.swap(cl);
        mr.swap(cr);
    }
    if (planesL) memcpy(planesL, ml.data(), 4 * N * sizeof(float));
    if (planesR && views == 2) memcpy(planesR, mr.data(), 4 * N * sizeof(float));
    if (pp == 0) {                                                             /* :123-129 */
        if (dmap) K.to_disparity(dmap, ml.data(), W, H, 1.0f, 1);
        if (normal) K.fill_normalmap(normal, ml.data(), W, H, 1);
    } else {                                                                   /* :130-141 */
        std::vector<float> chk(4 * N);
        K.consistency(chk.data(), ml.data(), mr.data(), W, H, 1.0f, 5.0f);
        if (dump) dump("consistency", -1, W, H, chk.data(), user);
        if (dmap) {
            if (pp == 1) K.to_disparity(dmap, chk.data(), W, H, 1.0f, 1);
            else K.fill_depthmap(dmap, chk.data(), W, H, 1.0f);
        }
        if (normal) K.fill_normalmap(normal, chk.data(), W, H, 1);
    }
    return 0;
}

/* PMHuberStereo::depthMap (PMHuberStereo.cpp:145-347): the Huber-smoothed variant.  Its kernels
 * read the images themselves as colour (no window weight sum, :203-204), the diffusion tensors use
 * alpha = 12 (:152), the smoothing is denoiseDiffusionTensorHuber_PDD (eps 1e-4, 40 steps) of the
 * gap-filled planes (convertFillNormalDisparity, :273, :295), theta starts at 1e-3 and follows
 * :320-323, the iteration count is not made odd, and the disparity is scaled by dscale (1 / dmax
 * when dscale <= 0, :164-165).  The occlusion maps of :271 and :289 feed nothing and are left out. */
static inline int pm_host_depth_map(const PmKernels& K, const uint8_t* left, const uint8_t* right, int W, int H,
                                    int stride, int r, float dmax, int iterations, float dscale, int pp, int views,
                                    float* dmap, float* normal, const float* initdisp, const float* initnormal,
                                    float* planesL, float* planesR, int fused, int64_t* counters, PmDumpFn dump,
                                    void* user)
{
    if (W <= 0 || H <= 0 || r < 0 || iterations < 0) return -1;
    if (views != 1 && views != 2) return -1;
    if (views == 1 && pp != 0) return -1;
    const float HUBEREPS = 0.0001f, THETASCALE_D = 15.0f, THETABIAS_D = 2.0f, THETASCALE = 10.0f;   /* :154-161 */
    float theta = 1e-3f;                                                                           /* :163 */
    if (dscale <= 0.0f) dscale = 1.0f / dmax;
    const size_t N = (size_t)W * H;
    std::vector<float> Lc(4 * N), Rc(4 * N), Lg(4 * N), Rg(4 * N), LDT(4 * N), RDT(4 * N);
    std::vector<float> Ls(4 * N, 0.0f), Rs(4 * N, 0.0f), tmp(4 * N);
    std::vector<float> m1[2] = {std::vector<float>(4 * N), std::vector<float>(4 * N)};
    std::vector<float> m2[2] = {std::vector<float>(4 * N), std::vector<float>(4 * N)};
    std::vector<int32_t> vb1n(N, 0), vb2n(N, 0);
    std::vector<float> vb1v(8 * N, 0.0f), vb2v(8 * N, 0.0f);
    K.prep_raw(left, W, H, stride, 12.0f, Lc.data(), Lg.data(), LDT.data());    /* :184-190 */
    K.prep_raw(right, W, H, stride, 12.0f, Rc.data(), Rg.data(), RDT.data());
    std::vector<float> nrm;
    const float* initn = initnormal;
    if (initdisp && !initnormal) {                                             /* :363-365 */
        nrm.resize(4 * N);
        K.disparity_to_normal(nrm.data(), initdisp, W, H);
        initn = nrm.data();
    }
    K.init(m1[0].data(), Lc.data(), Rc.data(), Lg.data(), Rg.data(), W, H, r, dmax, 1, initdisp, initn, fused);
    if (views == 2)
        K.init(m2[0].data(), Rc.data(), Lc.data(), Rg.data(), Lg.data(), W, H, r, dmax, 0, nullptr, nullptr, fused);
    if (dump) { dump("init_left", -1, W, H, m1[0].data(), user); if (views == 2) dump("init_right", -1, W, H, m2[0].data(), user); }
    int swap = 0;
    for (int iter = 0; iter < iterations; iter++) {
        const float l = theta * THETASCALE_D + THETABIAS_D;                                               /* :259 */
        const float lam[4] = {l, l, l, l};
        std::fill(vb1n.begin(), vb1n.end(), 0);                                                           /* :261 */
        K.propagate(m1[1 - swap].data(), m1[swap].data(), Lc.data(), Rc.data(), Lg.data(), Rg.data(), Ls.data(),
                    theta * THETASCALE, W, H, r, dmax, 1, iter, vb2n.data(), vb2v.data(),
                    views == 2 ? vb1n.data() : nullptr, vb1v.data(), nullptr, fused, counters);
        if (views == 2) {
            std::fill(vb2n.begin(), vb2n.end(), 0);                                                       /* :266 */
            K.propagate(m2[1 - swap].data(), m2[swap].data(), Rc.data(), Lc.data(), Rg.data(), Lg.data(), Rs.data(),
                        theta * THETASCALE, W, H, r, dmax, 0, iter, vb1n.data(), vb1v.data(), vb2n.data(),
                        vb2v.data(), nullptr, fused, counters);
        }
        if (dump) { dump("prop_left", iter, W, H, m1[1 - swap].data(), user); if (views == 2) dump("prop_right", iter, W, H, m2[1 - swap].data(), user); }
        K.fill_state(tmp.data(), m1[1 - swap].data(), W, H, 1.0f / dmax, 1);                               /* :273-274 */
        K.huber(Ls.data(), tmp.data(), LDT.data(), lam, HUBEREPS, 40, W, H);
        if (views == 2) {
            K.fill_state(tmp.data(), m2[1 - swap].data(), W, H, 1.0f / dmax, 0);                           /* :295-296 */
            K.huber(Rs.data(), tmp.data(), RDT.data(), lam, HUBEREPS, 40, W, H);
        }
        if (dump) { dump("smooth_left", iter, W, H, Ls.data(), user); if (views == 2) dump("smooth_right", iter, W, H, Rs.data(), user); }
        if (iter >= 3) {                                                                                 /* :320-323 */
            theta = ((float)iter - 3.0f) / ((float)iterations - 4.0f);
            theta = theta * theta * theta + 1e-3f;
        }
        swap = 1 - swap;
    }
    const std::vector<float>& ml = m1[swap];
    const std::vector<float>& mr = m2[swap];
    if (planesL) memcpy(planesL, ml.data(), 4 * N * sizeof(float));
    if (planesR && views == 2) memcpy(planesR, mr.data(), 4 * N * sizeof(float));
    if (pp == 0) {                                                             /* :331-337 */
        if (dmap) K.to_disparity(dmap, ml.data(), W, H, dscale, 1);
        if (normal) K.fill_normalmap(normal, ml.data(), W, H, 1);
    } else {                                                                   /* :338-345 */
        std::vector<float> chk(4 * N);
        K.consistency(chk.data(), ml.data(), mr.data(), W, H, 1.0f, 5.0f);
        if (dmap) {
            if (pp == 1) K.to_disparity(dmap, chk.data(), W, H, dscale, 1);
            else K.fill_depthmap(dmap, chk.data(), W, H, dscale);
        }
        if (normal) K.fill_normalmap(normal, chk.data(), W, H, 1);
    }
    return 0;
}

#endif
