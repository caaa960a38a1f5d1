/*
 * ORACLE — test infrastructure only.
 *
 * Runtime for the reference kernels compiled from their own source: the
 * NDRange executor (work items, fibers for barrier()), and ref_* entry points
 * with the same signatures as the orc_* restatement, so that tests can run the
 * two side by side.  The host loop is the shared restatement of
 * PMHuberStereo::disparityMapAll (pm_hostloop.h).
 */
#include <ucontext.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pm_hostloop.h"
#include "ref_exec.h"

namespace clk {

thread_local WorkItem g_wi;

namespace {
struct FiberPool {
    std::vector<ucontext_t> ctx;
    std::vector<std::vector<char>> stacks;
    std::vector<char> done;
    ucontext_t main;
    int cur = -1;
};
thread_local FiberPool* t_pool = nullptr;
thread_local const std::function<void()>* t_fn = nullptr;

void fiber_entry()
{
    (*t_fn)();
    t_pool->done[t_pool->cur] = 1;
}

void set_item(int gx, int gy, int lx, int ly, int lw, int lh, int gw, int gh)
{
    g_wi.gid[0] = (size_t)(gx * lw + lx); g_wi.gid[1] = (size_t)(gy * lh + ly);
    g_wi.lid[0] = (size_t)lx; g_wi.lid[1] = (size_t)ly;
    g_wi.grp[0] = (size_t)gx; g_wi.grp[1] = (size_t)gy;
    g_wi.lsz[0] = (size_t)lw; g_wi.lsz[1] = (size_t)lh;
    g_wi.gsz[0] = (size_t)gw; g_wi.gsz[1] = (size_t)gh;
}
}  // namespace

void barrier(int)
{
    if (!t_pool) { fprintf(stderr, "barrier() outside a fiber group\n"); abort(); }
    swapcontext(&t_pool->ctx[t_pool->cur], &t_pool->main);
}

void nd_range(int gw, int gh, int lw, int lh, bool barriers, const std::function<void()>& fn)
{
    const int ngx = gw / lw, ngy = gh / lh;
#pragma omp parallel for schedule(dynamic, 1)
    for (int gy = 0; gy < ngy; gy++) {
        FiberPool pool;
        if (barriers) {
            pool.ctx.resize(lw * lh);
            pool.stacks.resize(lw * lh, std::vector<char>(128 * 1024));
            pool.done.resize(lw * lh);
        }
        t_fn = &fn;
        for (int gx = 0; gx < ngx; gx++) {
            if (!barriers) {
                for (int ly = 0; ly < lh; ly++)
                    for (int lx = 0; lx < lw; lx++) {
                        set_item(gx, gy, lx, ly, lw, lh, gw, gh);
                        fn();
                    }
                continue;
            }
            t_pool = &pool;
            const int n = lw * lh;
            for (int i = 0; i < n; i++) {
                getcontext(&pool.ctx[i]);
                pool.ctx[i].uc_stack.ss_sp = pool.stacks[i].data();
                pool.ctx[i].uc_stack.ss_size = pool.stacks[i].size();
                pool.ctx[i].uc_link = &pool.main;
                makecontext(&pool.ctx[i], fiber_entry, 0);
                pool.done[i] = 0;
            }
            int alive = n;
            while (alive > 0) {
                alive = 0;
                for (int i = 0; i < n; i++) {
                    if (pool.done[i]) continue;
                    set_item(gx, gy, i % lw, i / lw, lw, lh, gw, gh);
                    pool.cur = i;
                    swapcontext(&pool.main, &pool.ctx[i]);
                    if (!pool.done[i]) alive++;
                }
            }
            t_pool = nullptr;
        }
    }
}

}  // namespace clk

extern "C" {
int ref_k_prep(const uint8_t* rgba8, int W, int H, int r, float* bw, float* grad);
int ref_k_difftensor(const uint8_t* rgba8, int W, int H, float alpha, float beta, float* dt);
int ref_k_init(float* out, const float* bw1, const float* bw2, const float* g1, const float* g2, int W, int H, int r,
               float dmax, int lr, const float* initdisp, const float* initnormal);
int ref_k_propagate(float* out, const float* old, const float* bw1, const float* bw2, const float* g1, const float* g2,
                    const float* smooth, float theta, int W, int H, int r, float dmax, int lr, int iter,
                    const int32_t* vin_n, const float* vin_val, int32_t* vout_n, float* vout_val);
int ref_k_normal_depth(float* out, const float* planes, int W, int H, float dispscale, int lr);
int ref_k_rof(float* out, const float* input, const float* dt, const float lambda[4], int iters, int W, int H);
int ref_k_consistency(float* out, const float* left, const float* right, int W, int H, float maxdd, float maxad);
int ref_k_to_disparity(float* out, const float* planes, int W, int H, float scale, int lr);
int ref_k_fill_depthmap(float* out, const float* planes, int W, int H, float scale);
int ref_k_fill_normalmap(float* out, const float* planes, int W, int H, int lr);
int ref_k_disparity_to_normal(float* out, const float* disp, int W, int H);
int ref_k_fill_state(float* out, const float* planes, int W, int H, float dispscale, int lr);
int ref_k_huber(float* out, const float* input, const float* dt, const float lambda[4], float eps, int iters, int W,
                int H);

int ref_version(void) { return 1; }

/* orc_prep_raw signature: the image as floats (what the kernels read from it), its gradients
 * (pmhstereo_gradxy) and its diffusion tensor with edge weight alpha (PDDiffTensorColor, beta 1) */
int ref_prep_raw(const uint8_t* img, int W, int H, int stride, float alpha, float* colour, float* grad, float* dt)
{
    std::vector<uint8_t> packed((size_t)W * H * 4);
    for (int y = 0; y < H; y++) memcpy(&packed[(size_t)y * W * 4], img + (size_t)y * stride, (size_t)W * 4);
    std::vector<float> b((size_t)W * H * 4), g((size_t)W * H * 4), d((size_t)W * H * 4);
    ref_k_prep(packed.data(), W, H, 0, b.data(), g.data());
    ref_k_difftensor(packed.data(), W, H, alpha, 1.0f, d.data());
    if (colour)
        for (size_t i = 0; i < packed.size(); i++) colour[i] = (float)packed[i] / 255.0f;
    if (grad) memcpy(grad, g.data(), g.size() * 4);
    if (dt) memcpy(dt, d.data(), d.size() * 4);
    return 0;
}
int ref_fill_state(float* out, const float* planes, int W, int H, float dispscale, int lr)
{ return ref_k_fill_state(out, planes, W, H, dispscale, lr); }
int ref_huber(float* out, const float* input, const float* dt, const float lambda[4], float eps, int iters, int W, int H)
{ return ref_k_huber(out, input, dt, lambda, eps, iters, W, H); }

/* orc_prep signature; `fused` must be 0 (the reference source has one arithmetic) */
int ref_prep(const uint8_t* img, int W, int H, int stride, int r, int fused, float* bw, float* grad, float* dt)
{
    if (fused) return -2;
    std::vector<uint8_t> packed((size_t)W * H * 4);
    for (int y = 0; y < H; y++) memcpy(&packed[(size_t)y * W * 4], img + (size_t)y * stride, (size_t)W * 4);
    std::vector<float> b((size_t)W * H * 4), g((size_t)W * H * 4), d((size_t)W * H * 4);
    ref_k_prep(packed.data(), W, H, r, b.data(), g.data());
    ref_k_difftensor(packed.data(), W, H, 24.0f, 1.0f, d.data());   /* PMHuberStereo.cpp:416-417 */
    if (bw) memcpy(bw, b.data(), b.size() * 4);
    if (grad) memcpy(grad, g.data(), g.size() * 4);
    if (dt) memcpy(dt, d.data(), d.size() * 4);
    return 0;
}

int ref_init(float* out, const float* bw1, const float* bw2, const float* g1, const float* g2, int W, int H, int r,
             float dmax, int lr, const float* initdisp, const float* initnormal, int fused)
{
    if (fused) return -2;
    return ref_k_init(out, bw1, bw2, g1, g2, W, H, r, dmax, lr, initdisp, initnormal);
}

int ref_propagate(float* out, const float* old, const float* bw1, const float* bw2, const float* g1, const float* g2,
                  const float* smooth, float theta, int W, int H, int r, float dmax, int lr, int iter,
                  const int32_t* vin_n, const float* vin_val, int32_t* vout_n, float* vout_val, int32_t* vout_src,
                  int fused, int64_t* counters)
{
    (void)vout_src; (void)counters;
    if (fused) return -2;
    return ref_k_propagate(out, old, bw1, bw2, g1, g2, smooth, theta, W, H, r, dmax, lr, iter, vin_n, vin_val, vout_n,
                           vout_val);
}

int ref_k_cost(float* cost, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
               int W, int H, int r, float mincost);
int ref_k_klt(float* out, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
              int W, int H, int r);

int ref_cost(float* cost, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
             int W, int H, int r, float mincost, int fused)
{
    if (fused) return -2;
    return ref_k_cost(cost, planes, bw1, bw2, g1, g2, W, H, r, mincost);
}
int ref_klt(float* out, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
            int W, int H, int r, int fused)
{
    if (fused) return -2;
    return ref_k_klt(out, planes, bw1, bw2, g1, g2, W, H, r);
}

int ref_normal_depth(float* out, const float* planes, int W, int H, float dispscale, int lr)
{ return ref_k_normal_depth(out, planes, W, H, dispscale, lr); }
int ref_rof(float* out, const float* input, const float* dt, const float lambda[4], int iters, int W, int H)
{ return ref_k_rof(out, input, dt, lambda, iters, W, H); }
int ref_consistency(float* out, const float* left, const float* right, int W, int H, float maxdd, float maxad)
{ return ref_k_consistency(out, left, right, W, H, maxdd, maxad); }
int ref_to_disparity(float* out, const float* planes, int W, int H, float scale, int lr)
{ return ref_k_to_disparity(out, planes, W, H, scale, lr); }
int ref_fill_depthmap(float* out, const float* planes, int W, int H, float scale)
{ return ref_k_fill_depthmap(out, planes, W, H, scale); }
int ref_fill_normalmap(float* out, const float* planes, int W, int H, int lr)
{ return ref_k_fill_normalmap(out, planes, W, H, lr); }
int ref_disparity_to_normal(float* out, const float* disp, int W, int H)
{ return ref_k_disparity_to_normal(out, disp, W, H); }

int ref_k_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, int Wi, int Hi);
int ref_k_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, const float* mul);
int ref_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, int Wi, int Hi)
{ return ref_k_pyrdown(out, Wo, Ho, in, Wi, Hi); }
int ref_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, const float* mul)
{ return ref_k_pyrup_mul(out, Wo, Ho, in, Wi, Hi, channels, mul); }

static const PmKernels REF_KERNELS = {ref_prep, ref_init, ref_propagate, ref_normal_depth, ref_rof, ref_consistency,
                                      ref_to_disparity, ref_fill_depthmap, ref_fill_normalmap, ref_disparity_to_normal,
                                      ref_pyrdown, ref_pyrup_mul, ref_prep_raw, ref_fill_state, ref_huber};

int ref_disparity_map_dump(const uint8_t* left, const uint8_t* right, int W, int H, int stride, int r, float dmax,
                           int iterations, int pp, int views, int levels, float* dmap, float* normal,
                           const float* initdisp, const float* initnormal, float* planesL, float* planesR,
                           PmDumpFn dump, void* user)
{
    return pm_host_disparity_map(REF_KERNELS, left, right, W, H, stride, r, dmax, iterations, pp, views, levels, dmap,
                                 normal, initdisp, initnormal, planesL, planesR, 0, nullptr, dump, user);
}

int ref_disparity_map(const uint8_t* left, const uint8_t* right, int W, int H, int stride, int r, float dmax,
                      int iterations, int pp, int views, float* dmap, float* normal, const float* initdisp,
                      const float* initnormal, float* planesL, float* planesR)
{
    return ref_disparity_map_dump(left, right, W, H, stride, r, dmax, iterations, pp, views, 1, dmap, normal, initdisp,
                                  initnormal, planesL, planesR, nullptr, nullptr);
}

int ref_depth_map_dump(const uint8_t* left, const uint8_t* right, int W, int H, int stride, int r, float dmax,
                       int iterations, float dscale, int pp, int views, float* dmap, float* normal,
                       const float* initdisp, const float* initnormal, float* planesL, float* planesR, PmDumpFn dump,
                       void* user)
{
    return pm_host_depth_map(REF_KERNELS, left, right, W, H, stride, r, dmax, iterations, dscale, pp, views, dmap,
                             normal, initdisp, initnormal, planesL, planesR, 0, nullptr, dump, user);
}

}  // extern "C"
