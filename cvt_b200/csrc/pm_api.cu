// C ABI of the library (include/cvtpm.h): handles, device workspaces and the
// host orchestration of PMHuberStereo::disparityMap / disparityMapAll
// (cvt/vision/PMHuberStereo.cpp:75-143, :406-581) on one CUDA stream.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cvtpm.h"
#include "pm_kernels.h"

using namespace pm;

struct pm_handle {
    pm_options opt;
    std::string err;
    int counting = 0;
    uint64_t counters[4] = {0, 0, 0, 0};
    // phase timing: events recorded at phase boundaries, summed per phase after the call
    int profiling = 0;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_phase, ev_launches;
    int ev_used = 0;
    float phase_ms[PM_NPHASES] = {0, 0, 0, 0, 0, 0};
    int phase_launches[PM_NPHASES] = {0, 0, 0, 0, 0, 0};
    // device workspace for one image size
    int W = 0, H = 0;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    cudaStream_t own = nullptr;   // blocking stream for calls made on the legacy default stream
    // CUDA graphs of the last single-pair and batched calls, replayed while the call's
    // arguments (buffers, sizes, parameters) are unchanged
    int capturing = 0;
    std::vector<uint64_t> key1, keyb;
    cudaGraphExec_t exec1 = nullptr, execb = nullptr;
    // batched calls: one workspace per pair, branch streams and their fork/join events
    std::vector<void*> bws;
    std::vector<size_t> bws_bytes;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> bev;
    // pyramid levels 1.. of single-pair calls: one workspace each
    std::vector<void*> lws;
    std::vector<size_t> lws_bytes;
    // the right view's initial disparity of the call in progress (pm_disparity_map_init2_device)
    const float* init_right = nullptr;
    const float* init_normal_right = nullptr;   // with init_right: the right view's initial normals
    // concurrent branches of batched calls (pm_set_batch_branches; 0: PM_BATCH_BRANCHES)
    int batch_branches = 0;
    // schedule of batched calls (pm_set_batch_schedule)
    int batch_schedule = PM_BATCH_BRANCHED, batch_ctas = 0, batch_order = 0, batch_tile_w = 32;
    // lockstep batched calls: per-pair argument tables, job lists and work counters in one
    // device allocation, and the host bytes last uploaded into it
    void* btab = nullptr;
    size_t btab_bytes = 0;
    std::vector<unsigned char> btab_host;
};

namespace {

thread_local std::string t_err;

int fail(pm_handle* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    t_err = msg;
    return code;
}

int cuda_fail(pm_handle* h, cudaError_t e, const char* what)
{
    return fail(h, PM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PM_CUDA(h, call)                                         \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, #call); \
    } while (0)

// Scratch of pm_k_rof_static: a file-scope device array, so that the entry point
// allocates nothing.  It holds the ROF intermediates of launch_rof (7 float4 per
// pixel: u, two dual images p of 2 float4, two q) for up to
// PM_ROF_STATIC_MAX_PIXELS pixels = 28 MiB of every context that loads this
// library.  Its device address belongs to the CUDA context it was looked up in, so
// it is cached per context, keyed on the driver's unique context id
// (cuCtxGetId: never reused within a process, unlike a context handle or a
// device ordinal after cudaDeviceReset).  The driver functions are taken through
// cudaGetDriverEntryPointByVersion, so the library does not link the driver.
constexpr size_t kRofStaticBytes = (size_t)PM_ROF_STATIC_MAX_PIXELS * 7 * sizeof(float4);
__device__ __align__(256) unsigned char g_rof_static[kRofStaticBytes];
constexpr int kRofCacheSlots = 64;
std::mutex g_rof_static_mu;
struct RofStaticSlot {
    unsigned long long ctx_id;
    void* ptr;
};
RofStaticSlot g_rof_static_cache[kRofCacheSlots] = {};
int g_rof_static_used = 0;
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// id of the calling thread's current context (0 when none is current yet)
int current_ctx_id(unsigned long long* id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa = cudaDriverEntryPointSymbolNotFound, qb = qa;
        PM_CUDA(nullptr, cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &a, 12000, cudaEnableDefault, &qa));
        PM_CUDA(nullptr, cudaGetDriverEntryPointByVersion("cuCtxGetId", &b, 12000, cudaEnableDefault, &qb));
        if (qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
            return fail(nullptr, PM_ECUDA, "pm_k_rof_static: the driver lacks cuCtxGetCurrent or cuCtxGetId");
        get_current = reinterpret_cast<CtxGetCurrentFn>(a);
        get_id = reinterpret_cast<CtxGetIdFn>(b);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return fail(nullptr, PM_ECUDA, "pm_k_rof_static: cuCtxGetCurrent failed");
    *id = 0;
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return fail(nullptr, PM_ECUDA, "pm_k_rof_static: cuCtxGetId failed");
    return PM_OK;
}

// device address of g_rof_static in the current context; the first call in a context looks
// it up, which must not happen while `st` is being captured into a graph
int rof_static_scratch(cudaStream_t st, void** out)
{
    std::lock_guard<std::mutex> lock(g_rof_static_mu);
    unsigned long long id = 0;
    int rc = current_ctx_id(&id);
    if (rc) return rc;
    for (int i = 0; id && i < g_rof_static_used; i++)
        if (g_rof_static_cache[i].ctx_id == id) {
            *out = g_rof_static_cache[i].ptr;
            return PM_OK;
        }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PM_CUDA(nullptr, cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(nullptr, PM_EINVAL_ARG,
                    "pm_k_rof_static: the first call in a CUDA context looks up the static scratch and must come "
                    "before stream capture; call it once outside the capture first");
    void* p = nullptr;
    PM_CUDA(nullptr, cudaGetSymbolAddress(&p, g_rof_static));   // makes the primary context current if none was
    if (!id) {
        rc = current_ctx_id(&id);
        if (rc) return rc;
    }
    if (id && g_rof_static_used < kRofCacheSlots) g_rof_static_cache[g_rof_static_used++] = RofStaticSlot{id, p};
    *out = p;
    return PM_OK;
}

int check_shape(pm_handle* h, int W, int H, int r)
{
    if (W <= 0 || H <= 0 || W > PM_MAX_WIDTH || H > PM_MAX_HEIGHT)
        return fail(h, PM_EINVAL_SHAPE, "image size out of range");
    if (r < 0 || r > PM_MAX_RADIUS) return fail(h, PM_EINVAL_SHAPE, "patch size out of range");
    return PM_OK;
}

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

// record a phase boundary: the interval since the previous mark belongs to `phase`
// and contained `launches` kernel launches
void prof_mark(pm_handle* h, cudaStream_t st, int phase, int launches)
{
    if (!h->profiling || h->capturing) return;
    if (h->ev_used == (int)h->ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return; }
        h->ev.push_back(e);
        h->ev_phase.push_back(0);
        h->ev_launches.push_back(0);
    }
    cudaEventRecord(h->ev[h->ev_used], st);
    h->ev_phase[h->ev_used] = phase;
    h->ev_launches[h->ev_used] = launches;
    h->ev_used++;
}

int prof_collect(pm_handle* h, cudaStream_t st)
{
    if (!h->profiling || h->capturing) return PM_OK;
    PM_CUDA(h, cudaStreamSynchronize(st));
    for (int k = 0; k < PM_NPHASES; k++) { h->phase_ms[k] = 0.0f; h->phase_launches[k] = 0; }
    for (int i = 1; i < h->ev_used; i++) {
        float ms = 0.0f;
        PM_CUDA(h, cudaEventElapsedTime(&ms, h->ev[i - 1], h->ev[i]));
        h->phase_ms[h->ev_phase[i]] += ms;
        h->phase_launches[h->ev_phase[i]] += h->ev_launches[i];
        h->phase_ms[PM_PHASE_TOTAL] += ms;
        h->phase_launches[PM_PHASE_TOTAL] += h->ev_launches[i];
    }
    h->ev_used = 0;
    return PM_OK;
}

// workspace layout for a W x H pair (float4 fields unless noted)
struct Layout {
    enum {
        Lbw, Rbw, Lg, Rg, LDT, RDT, Ls, Rs, tmp, mL0, mL1, mR0, mR1, chk, nrm,   // float4 x N
        pself, pnb,                                                             // float4 x N
        vb1c, vb2c,                                                             // int x N
        vb1s, vb2s,                                                             // u64 x N
        texL, texR,                                                             // texel rows
        rof,                                                                    // rof scratch
        ctr, errf,                                                              // counters (4 u64), error int
        img0, img1, disp, dmap, nmap, initd, initn,                             // staging for host entry
        initdR, initnR,                                                         // right-view init (pyramid)
        outpL, outpR,                                                           // plane outputs for host entry
        COUNT
    };
    size_t N;
    size_t off[COUNT];
    size_t total;
};

Layout layout(int W, int H, size_t stride)
{
    Layout L;
    L.N = (size_t)W * H;
    size_t o = 0;
    auto put = [&](int k, size_t bytes) { L.off[k] = o; o += (bytes + 255) / 256 * 256; };
    for (int k = Layout::Lbw; k <= Layout::nrm; k++) put(k, L.N * 16);
    put(Layout::vb1c, L.N * 4);
    put(Layout::vb2c, L.N * 4);
    put(Layout::vb1s, L.N * 8);
    put(Layout::vb2s, L.N * 8);
    put(Layout::pself, L.N * 16);
    put(Layout::pnb, L.N * 16);
    put(Layout::texL, tex_bytes(W, H));
    put(Layout::texR, tex_bytes(W, H));
    put(Layout::rof, rof_scratch_bytes(W, H));
    put(Layout::ctr, 64);
    put(Layout::errf, 64);
    put(Layout::img0, stride * H);
    put(Layout::img1, stride * H);
    put(Layout::disp, L.N * 4);
    put(Layout::dmap, L.N * 4);
    put(Layout::nmap, L.N * 16);
    put(Layout::initd, L.N * 4);
    put(Layout::initn, L.N * 16);
    put(Layout::initdR, L.N * 4);
    put(Layout::initnR, L.N * 16);
    put(Layout::outpL, L.N * 16);
    put(Layout::outpR, L.N * 16);
    L.total = o;
    return L;
}

template <class T> T* at(void* base, const Layout& L, int k) { return reinterpret_cast<T*>(static_cast<char*>(base) + L.off[k]); }

// grow a workspace to `bytes` (contents are not kept); a replayable graph that holds the
// old address is dropped by the caller through the argument key
int grow(pm_handle* h, void*& ws, size_t& have, size_t bytes)
{
    if (ws && have >= bytes) return PM_OK;
    if (ws) { cudaFree(ws); ws = nullptr; have = 0; }
    cudaError_t e = cudaMalloc(&ws, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(h, PM_ENOMEM, "device workspace allocation failed"); }
    have = bytes;
    return PM_OK;
}

int ensure_ws(pm_handle* h, int W, int H, size_t stride)
{
    return grow(h, h->ws, h->ws_bytes, layout(W, H, stride).total);
}

// the fields of one pair's workspace that disparityMapAll works on
struct LevelBufs {
    float4 *Lbw, *Rbw, *Lg, *Rg, *LDT, *RDT, *Ls, *Rs, *tmp;
    float4* mL[2];
    float4* mR[2];
    int *vb1c, *vb2c;
    unsigned long long *vb1s, *vb2s;
    void* rofs;
    float4 *texL, *texR, *pself, *pnb;
    ViewData VL, VR;
    int W, H;
};

LevelBufs level_bufs(void* ws, const Layout& L, int W, int H, int r)
{
    LevelBufs B;
    B.Lbw = at<float4>(ws, L, Layout::Lbw);
    B.Rbw = at<float4>(ws, L, Layout::Rbw);
    B.Lg = at<float4>(ws, L, Layout::Lg);
    B.Rg = at<float4>(ws, L, Layout::Rg);
    B.LDT = at<float4>(ws, L, Layout::LDT);
    B.RDT = at<float4>(ws, L, Layout::RDT);
    B.Ls = at<float4>(ws, L, Layout::Ls);
    B.Rs = at<float4>(ws, L, Layout::Rs);
    B.tmp = at<float4>(ws, L, Layout::tmp);
    B.mL[0] = at<float4>(ws, L, Layout::mL0);
    B.mL[1] = at<float4>(ws, L, Layout::mL1);
    B.mR[0] = at<float4>(ws, L, Layout::mR0);
    B.mR[1] = at<float4>(ws, L, Layout::mR1);
    B.vb1c = at<int>(ws, L, Layout::vb1c);
    B.vb2c = at<int>(ws, L, Layout::vb2c);
    B.vb1s = at<unsigned long long>(ws, L, Layout::vb1s);
    B.vb2s = at<unsigned long long>(ws, L, Layout::vb2s);
    B.rofs = at<void>(ws, L, Layout::rof);
    B.texL = at<float4>(ws, L, Layout::texL);
    B.texR = at<float4>(ws, L, Layout::texR);
    B.pself = at<float4>(ws, L, Layout::pself);
    B.pnb = at<float4>(ws, L, Layout::pnb);
    B.VL = make_view(B.texL, B.texR, W, H, r);
    B.VR = make_view(B.texR, B.texL, W, H, r);
    B.W = W;
    B.H = H;
    return B;
}

// theta of iteration k of `iterations` (already made odd): thetamin, then
// (k - 1) / iterations to the fourth plus thetamin (PMHuberStereo.cpp:575-576)
float theta_at(int k, int iterations, float thetamin)
{
    if (k == 0) return thetamin;
    float theta = (float)(k - 1) / (float)iterations;
    return powf(theta, 4.0f) + thetamin;
}

// the arguments of the propagate pass of view `view` (0 left, 1 right) in iteration `iter`
// (:536-537, :542-543), `swap` the parity of the plane fields
PropParams prop_params(const pm_handle* h, const LevelBufs& B, int view, int iter, int swap, float theta, float dmax,
                       unsigned long long* ctr, int* errf)
{
    const int views = h->opt.views;
    PropParams P;
    P.V = view ? B.VR : B.VL;
    P.out = view ? B.mR[1 - swap] : B.mL[1 - swap];
    P.old = view ? B.mR[swap] : B.mL[swap];
    P.smooth = view ? B.Rs : B.Ls;
    P.theta = theta * 50.0f;
    P.dmax = dmax;
    P.lr = view ? 0 : 1;
    P.iter = iter;
    if (view == 0) {
        P.vin_count = views == 2 ? B.vb2c : nullptr;
        P.vin_src = B.vb2s;
        P.vin_planes = B.mR[swap];
        P.vout_count = views == 2 ? B.vb1c : nullptr;
        P.vout_src = B.vb1s;
    } else {
        P.vin_count = B.vb1c;
        P.vin_src = B.vb1s;
        P.vin_planes = B.mL[1 - swap];
        P.vout_count = B.vb2c;
        P.vout_src = B.vb2s;
    }
    P.counters = h->counting ? ctr : nullptr;
    P.error = errf;
    P.tmp_self = B.pself;
    P.tmp_nb = B.pnb;
    P.dual = 0;
    return P;
}

// the part of disparityMapAll before its iterations (:445-483): prep, clears, texel planes,
// init (random or from given fields) and, with given fields, the first smoothing
int level_begin(pm_handle* h, const LevelBufs& B, const uint8_t* left, const uint8_t* right, size_t stride, int r,
                float dmax, float thetamin, const float* initdL, const float* initdR, const float4* initnL,
                const float4* initnR, float4* nrmL, float4* nrmR, cudaStream_t st)
{
    const pm_options& o = h->opt;
    const int views = o.views;
    const int F = o.fused;
    const int W = B.W, H = B.H;
    const size_t N = (size_t)W * H;

    // prep (PMHuberStereo.cpp:445-454)
    launch_prep(left, stride, W, H, r, F, B.Lbw, B.Lg, B.LDT, st);
    if (views == 2) launch_prep(right, stride, W, H, r, F, B.Rbw, B.Rg, B.RDT, st);
    else launch_prep(right, stride, W, H, r, F, B.Rbw, B.Rg, nullptr, st);
    // clear the smoothing images (:457-458) and both view buffers (:487)
    PM_CUDA(h, cudaMemsetAsync(B.Ls, 0, N * 16, st));
    PM_CUDA(h, cudaMemsetAsync(B.Rs, 0, N * 16, st));
    launch_view_clear(B.vb1c, B.vb1s, N, st);
    launch_view_clear(B.vb2c, B.vb2s, N, st);
    launch_pack_tex(B.texL, B.Lbw, B.Lg, W, H, st);
    launch_pack_tex(B.texR, B.Rbw, B.Rg, W, H, st);
    prof_mark(h, st, PM_PHASE_PREP, 6);
    // init (:469-470, :349-379): a given disparity without normals gets normals from it
    int nl = 0;
    if (initdL && !initnL) {
        launch_disparity_to_normal(nrmL, initdL, W, H, st);   // :363-365
        initnL = nrmL;
        nl++;
    }
    if (initdR && !initnR && views == 2) {
        launch_disparity_to_normal(nrmR, initdR, W, H, st);
        initnR = nrmR;
        nl++;
    }
    launch_init(B.mL[0], B.VL, dmax, 1, initdL, initnL, F, st);
    nl += window_kernel_launches(F, false);
    if (views == 2) {
        launch_init(B.mR[0], B.VR, dmax, 0, initdR, initnR, F, st);
        nl += window_kernel_launches(F, false);
    }
    const int rof_launches = pd_launch_count(o.rof_iters);
    const float theta = thetamin;
    const float4 lam0 = make_float4(theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, 1.0f);
    if (initdL) {   // :473-477
        launch_normal_depth(B.tmp, B.mL[0], W, H, 1.0f / dmax, 1, st);
        launch_rof(B.Ls, B.tmp, B.LDT, lam0, o.rof_iters, W, H, B.rofs, st);
        nl += 1 + rof_launches;
    }
    if (initdR && views == 2) {   // :479-483
        launch_normal_depth(B.tmp, B.mR[0], W, H, 1.0f / dmax, 0, st);
        launch_rof(B.Rs, B.tmp, B.RDT, lam0, o.rof_iters, W, H, B.rofs, st);
        nl += 1 + rof_launches;
    }
    prof_mark(h, st, PM_PHASE_INIT, nl);
    return PM_OK;
}

// the smoothing weight of an iteration at theta (:532)
float4 smooth_lambda(float theta)
{
    return make_float4(theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, theta * 10.0f + 1.0f, 1.0f);
}

// PMHuberStereo::disparityMapAll (PMHuberStereo.cpp:406-581) on one pyramid level, in the
// workspace `ws` (layout L): the final plane fields end in mL1 and mR1.  initdL/initnL and
// initdR/initnR are W x H init fields of the views (NULL: random init); counters and the
// view-buffer error flag are the caller's.
int run_level(pm_handle* h, void* ws, const Layout& L, const uint8_t* left, const uint8_t* right, int W, int H,
              size_t stride, int r, float dmax, int iterations, float thetamin, const float* initdL,
              const float* initdR, const float4* initnL, const float4* initnR, unsigned long long* ctr, int* errf,
              cudaStream_t st)
{
    const pm_options& o = h->opt;
    const int views = o.views;
    const int F = o.fused;
    const LevelBufs B = level_bufs(ws, L, W, H, r);
    int rc = level_begin(h, B, left, right, stride, r, dmax, thetamin, initdL, initdR, initnL, initnR,
                         at<float4>(ws, L, Layout::nrm), at<float4>(ws, L, Layout::initnR), st);
    if (rc) return rc;
    const int rof_launches = pd_launch_count(o.rof_iters);
    int swap = 0;
    iterations |= 1;   // :490
    for (int iter = 0; iter < iterations; iter++) {
        const float theta = theta_at(iter, iterations, thetamin);
        const float4 lam = smooth_lambda(theta);
        launch_propagate(prop_params(h, B, 0, iter, swap, theta, dmax, ctr, errf), F, st);   // :536-537
        if (views == 2) launch_propagate(prop_params(h, B, 1, iter, swap, theta, dmax, ctr, errf), F, st);   // :542-543
        prof_mark(h, st, PM_PHASE_PROPAGATE, 3 * window_kernel_launches(F, h->counting) * views);
        // the smoothing feeds the next iteration's propagation only: after the last one it is
        // left out (every output is formed from the planes, :105-142)
        if (iter + 1 < iterations) {
            launch_normal_depth(B.tmp, B.mL[1 - swap], W, H, 1.0f / dmax, 1, st);   // :552-553
            launch_rof(B.Ls, B.tmp, B.LDT, lam, o.rof_iters, W, H, B.rofs, st);
            if (views == 2) {
                launch_normal_depth(B.tmp, B.mR[1 - swap], W, H, 1.0f / dmax, 0, st);   // :566-567
                launch_rof(B.Rs, B.tmp, B.RDT, lam, o.rof_iters, W, H, B.rofs, st);
            }
            prof_mark(h, st, PM_PHASE_SMOOTH, views * (1 + rof_launches));
        }
        swap = 1 - swap;
    }
    return PM_OK;
}

// PMHuberStereo::depthMap (PMHuberStereo.cpp:145-347) on device buffers in `ws`: the kernels read
// the images themselves as colour (:203-204), the diffusion tensors use alpha 12 (:152), each
// iteration smooths the gap-filled planes (pmhstereo_fill_state) with the tensor-weighted Huber
// model (eps 1e-4, 40 steps, :273-296), theta starts at 1e-3 and follows :320-323, the iteration
// count is not made odd, and outputs are scaled by dscale (1 / dmax when dscale <= 0, :164-165).
// The occlusion maps of :271 and :289 feed nothing and are not computed.
int run_depth(pm_handle* h, void* ws, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride, int r,
              float dmax, int iterations, float dscale, int pp, float* dmap, float4* normal, const float* initdisp,
              const float4* initnormal, float4* planesL, float4* planesR, cudaStream_t st)
{
    const pm_options& o = h->opt;
    const int views = o.views;
    const int F = o.fused;
    const Layout L = layout(W, H, stride);
    const size_t N = L.N;
    const float HUBEREPS = 0.0001f, THETASCALE_D = 15.0f, THETABIAS_D = 2.0f, THETASCALE = 10.0f;   // :154-161
    if (dscale <= 0.0f) dscale = 1.0f / dmax;
    float4 *Lc = at<float4>(ws, L, Layout::Lbw), *Rc = at<float4>(ws, L, Layout::Rbw);
    float4 *Lg = at<float4>(ws, L, Layout::Lg), *Rg = at<float4>(ws, L, Layout::Rg);
    float4 *LDT = at<float4>(ws, L, Layout::LDT), *RDT = at<float4>(ws, L, Layout::RDT);
    float4 *Ls = at<float4>(ws, L, Layout::Ls), *Rs = at<float4>(ws, L, Layout::Rs), *tmp = at<float4>(ws, L, Layout::tmp);
    float4* mL[2] = {at<float4>(ws, L, Layout::mL0), at<float4>(ws, L, Layout::mL1)};
    float4* mR[2] = {at<float4>(ws, L, Layout::mR0), at<float4>(ws, L, Layout::mR1)};
    float4* chk = at<float4>(ws, L, Layout::chk);
    int *vb1c = at<int>(ws, L, Layout::vb1c), *vb2c = at<int>(ws, L, Layout::vb2c);
    unsigned long long *vb1s = at<unsigned long long>(ws, L, Layout::vb1s), *vb2s = at<unsigned long long>(ws, L, Layout::vb2s);
    void* pds = at<void>(ws, L, Layout::rof);
    unsigned long long* ctr = at<unsigned long long>(ws, L, Layout::ctr);
    int* errf = at<int>(ws, L, Layout::errf);

    PM_CUDA(h, cudaMemsetAsync(ctr, 0, 64, st));
    PM_CUDA(h, cudaMemsetAsync(errf, 0, 64, st));
    h->ev_used = 0;
    prof_mark(h, st, PM_PHASE_PREP, 0);
    launch_prep(left, stride, W, H, r, F, Lc, Lg, LDT, st, 12.0f, 1);   // :184-190
    launch_prep(right, stride, W, H, r, F, Rc, Rg, views == 2 ? RDT : nullptr, st, 12.0f, 1);
    PM_CUDA(h, cudaMemsetAsync(Ls, 0, N * 16, st));   // :193-194
    PM_CUDA(h, cudaMemsetAsync(Rs, 0, N * 16, st));
    launch_view_clear(vb1c, vb1s, N, st);
    launch_view_clear(vb2c, vb2s, N, st);   // :212
    float4* texL = at<float4>(ws, L, Layout::texL);
    float4* texR = at<float4>(ws, L, Layout::texR);
    launch_pack_tex(texL, Lc, Lg, W, H, st);
    launch_pack_tex(texR, Rc, Rg, W, H, st);
    prof_mark(h, st, PM_PHASE_PREP, 6);
    int nl = 0;
    const float4* initn = initnormal;
    if (initdisp && !initnormal) {
        float4* nrm = at<float4>(ws, L, Layout::nrm);
        launch_disparity_to_normal(nrm, initdisp, W, H, st);   // :363-365
        initn = nrm;
        nl++;
    }
    const ViewData VL = make_view(texL, texR, W, H, r);
    const ViewData VR = make_view(texR, texL, W, H, r);
    launch_init(mL[0], VL, dmax, 1, initdisp, initn, F, st);   // :206-207
    nl += window_kernel_launches(F, false);
    if (views == 2) {
        launch_init(mR[0], VR, dmax, 0, nullptr, nullptr, F, st);
        nl += window_kernel_launches(F, false);
    }
    prof_mark(h, st, PM_PHASE_INIT, nl);
    const int pd_launches = pd_launch_count(o.rof_iters);
    float theta = 1e-3f;   // :163
    int swap = 0;
    for (int iter = 0; iter < iterations; iter++) {
        const float l = theta * THETASCALE_D + THETABIAS_D;   // :259
        const float4 lam = make_float4(l, l, l, l);
        PropParams P;
        P.V = VL;
        P.out = mL[1 - swap];
        P.old = mL[swap];
        P.smooth = Ls;
        P.theta = theta * THETASCALE;
        P.dmax = dmax;
        P.lr = 1;
        P.iter = iter;
        P.vin_count = views == 2 ? vb2c : nullptr;
        P.vin_src = vb2s;
        P.vin_planes = mR[swap];
        P.vout_count = views == 2 ? vb1c : nullptr;
        P.vout_src = vb1s;
        P.counters = h->counting ? ctr : nullptr;
        P.error = errf;
        P.tmp_self = at<float4>(ws, L, Layout::pself);
        P.tmp_nb = at<float4>(ws, L, Layout::pnb);
        P.dual = 0;
        launch_propagate(P, F, st);   // :263-264
        if (views == 2) {
            P.V = VR;
            P.out = mR[1 - swap];
            P.old = mR[swap];
            P.smooth = Rs;
            P.lr = 0;
            P.vin_count = vb1c;
            P.vin_src = vb1s;
            P.vin_planes = mL[1 - swap];
            P.vout_count = vb2c;
            P.vout_src = vb2s;
            launch_propagate(P, F, st);   // :268-269
        }
        prof_mark(h, st, PM_PHASE_PROPAGATE, 3 * window_kernel_launches(F, h->counting) * views);
        // as in run_level, the smoothing after the last iteration feeds nothing (:326-345)
        if (iter + 1 < iterations) {
            launch_fill_state(tmp, mL[1 - swap], W, H, 1.0f / dmax, 1, st);   // :273-274
            launch_huber(Ls, tmp, LDT, lam, HUBEREPS, o.rof_iters, W, H, pds, st);
            if (views == 2) {
                launch_fill_state(tmp, mR[1 - swap], W, H, 1.0f / dmax, 0, st);   // :295-296
                launch_huber(Rs, tmp, RDT, lam, HUBEREPS, o.rof_iters, W, H, pds, st);
            }
            prof_mark(h, st, PM_PHASE_SMOOTH, views * (1 + pd_launches));
        }
        if (iter >= 3) {   // :320-323
            theta = ((float)iter - 3.0f) / ((float)iterations - 4.0f);
            theta = theta * theta * theta + 1e-3f;
        }
        swap = 1 - swap;
    }
    float4* ml = mL[swap];
    float4* mr = mR[swap];
    if (planesL) PM_CUDA(h, cudaMemcpyAsync(planesL, ml, N * 16, cudaMemcpyDeviceToDevice, st));
    if (planesR && views == 2) PM_CUDA(h, cudaMemcpyAsync(planesR, mr, N * 16, cudaMemcpyDeviceToDevice, st));
    nl = 0;
    if (pp == PM_PP_NONE) {   // :331-337
        if (dmap) { launch_to_disparity(dmap, ml, W, H, dscale, 1, st); nl++; }
        if (normal) { launch_fill_normalmap(normal, ml, W, H, st); nl++; }
    } else {   // :338-345
        launch_consistency(chk, ml, mr, W, H, o.maxdispdiff, o.maxanglediff, st);
        nl++;
        if (dmap) {
            if (pp == PM_PP_LRCHECK) launch_to_disparity(dmap, chk, W, H, dscale, 1, st);
            else launch_fill_depthmap(dmap, chk, W, H, dscale, st);
            nl++;
        }
        if (normal) { launch_fill_normalmap(normal, chk, W, H, st); nl++; }
    }
    prof_mark(h, st, PM_PHASE_POST, nl);
    PM_CUDA(h, cudaGetLastError());
    return prof_collect(h, st);
}

// pyramid level sizes of a W x H pair (level 0 first); PM_EINVAL_SHAPE when a level would
// be empty
int level_sizes(pm_handle* h, int W, int H, std::vector<int>& Wl, std::vector<int>& Hl)
{
    const int levels = h->opt.levels;
    Wl.assign(levels, W);
    Hl.assign(levels, H);
    for (int l = 1; l < levels; l++) {
        Wl[l] = pyr_next(Wl[l - 1]);
        Hl[l] = pyr_next(Hl[l - 1]);
        if (Wl[l] < 1 || Hl[l] < 1) return fail(h, PM_EINVAL_SHAPE, "image too small for the pyramid levels");
    }
    return PM_OK;
}

// workspaces of pyramid levels 1.. (level 0 uses the caller's)
int ensure_level_ws(pm_handle* h, int W, int H)
{
    std::vector<int> Wl, Hl;
    int rc = level_sizes(h, W, H, Wl, Hl);
    if (rc) return rc;
    const int levels = h->opt.levels;
    if ((int)h->lws.size() < levels) { h->lws.resize(levels, nullptr); h->lws_bytes.resize(levels, 0); }
    for (int l = 1; l < levels; l++) {
        rc = grow(h, h->lws[l], h->lws_bytes[l], layout(Wl[l], Hl[l], (size_t)Wl[l] * 4).total);
        if (rc) return rc;
    }
    return PM_OK;
}

// PMHuberStereo::disparityMap (PMHuberStereo.cpp:75-143) on device buffers: with
// h->opt.levels = 1 (the reference's setting, :78) one disparityMapAll on the pair; with more
// levels the coarse-to-fine loop of :83-120 (CLPyramid with scale 0.35, each finer level
// initialised from the upsampled coarser result).  Level 0 runs in `ws`, levels 1.. in the
// handle's level workspaces (ensure_level_ws first).
// the end of disparityMap (PMHuberStereo.cpp:123-141) on the final plane fields mL1 / mR1 of
// `ws`: plane outputs, LR check, disparity and normal maps
int pair_post(pm_handle* h, void* ws, const Layout& L, int W, int H, int pp, float* dmap, float4* normal,
              float4* planesL, float4* planesR, cudaStream_t st)
{
    const pm_options& o = h->opt;
    const size_t N = L.N;
    float4* chk = at<float4>(ws, L, Layout::chk);
    float4* ml = at<float4>(ws, L, Layout::mL1);
    float4* mr = at<float4>(ws, L, Layout::mR1);
    if (planesL) PM_CUDA(h, cudaMemcpyAsync(planesL, ml, N * 16, cudaMemcpyDeviceToDevice, st));
    if (planesR && o.views == 2) PM_CUDA(h, cudaMemcpyAsync(planesR, mr, N * 16, cudaMemcpyDeviceToDevice, st));
    int nl = 0;
    if (pp == PM_PP_NONE) {   // :123-129
        if (dmap) { launch_to_disparity(dmap, ml, W, H, 1.0f, 1, st); nl++; }
        if (normal) { launch_fill_normalmap(normal, ml, W, H, st); nl++; }
    } else {   // :130-141
        launch_consistency(chk, ml, mr, W, H, o.maxdispdiff, o.maxanglediff, st);
        nl++;
        if (dmap) {
            if (pp == PM_PP_LRCHECK) launch_to_disparity(dmap, chk, W, H, 1.0f, 1, st);
            else launch_fill_depthmap(dmap, chk, W, H, 1.0f, st);
            nl++;
        }
        if (normal) { launch_fill_normalmap(normal, chk, W, H, st); nl++; }
    }
    prof_mark(h, st, PM_PHASE_POST, nl);
    return PM_OK;
}

int run_pipeline(pm_handle* h, void* ws, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride,
                 int r, float dmax, int iterations, int pp, float* dmap, float4* normal, const float* initdisp,
                 const float4* initnormal, float4* planesL, float4* planesR, cudaStream_t st)
{
    const pm_options& o = h->opt;
    const int views = o.views;
    const int levels = o.levels;
    const Layout L = layout(W, H, stride);
    unsigned long long* ctr = at<unsigned long long>(ws, L, Layout::ctr);
    int* errf = at<int>(ws, L, Layout::errf);

    PM_CUDA(h, cudaMemsetAsync(ctr, 0, 64, st));
    PM_CUDA(h, cudaMemsetAsync(errf, 0, 64, st));
    h->ev_used = 0;
    prof_mark(h, st, PM_PHASE_PREP, 0);
    int rc;
    if (levels == 1) {
        rc = run_level(h, ws, L, left, right, W, H, stride, r, dmax, iterations, o.thetamin, initdisp, h->init_right,
                       initnormal, reinterpret_cast<const float4*>(h->init_normal_right), ctr, errf, st);   // :92-93 (the right view's init: disparityMapAll's)
        if (rc) return rc;
    } else {
        std::vector<int> Wl, Hl;
        rc = level_sizes(h, W, H, Wl, Hl);
        if (rc) return rc;
        std::vector<void*> lw(levels);
        std::vector<Layout> ll(levels);
        lw[0] = ws;
        ll[0] = L;
        for (int l = 1; l < levels; l++) {
            lw[l] = h->lws[l];
            ll[l] = layout(Wl[l], Hl[l], (size_t)Wl[l] * 4);
        }
        // CLPyramid(0.35f, levels) of both images (:83-87): level l in its workspace's staging
        std::vector<const uint8_t*> il(levels), ir(levels);
        std::vector<size_t> is(levels);
        il[0] = left;
        ir[0] = right;
        is[0] = stride;
        int nl = 0;
        for (int l = 1; l < levels; l++) {
            uint8_t* a = at<uint8_t>(lw[l], ll[l], Layout::img0);
            uint8_t* b = at<uint8_t>(lw[l], ll[l], Layout::img1);
            launch_pyrdown(a, Wl[l], Hl[l], il[l - 1], is[l - 1], Wl[l - 1], Hl[l - 1], st);
            launch_pyrdown(b, Wl[l], Hl[l], ir[l - 1], is[l - 1], Wl[l - 1], Hl[l - 1], st);
            il[l] = a;
            ir[l] = b;
            is[l] = (size_t)Wl[l] * 4;
            nl += 2;
        }
        // the coarsest level reads the caller's init fields at its integer coordinates
        // (SAMPLER_NN, pmhstereo.cl:815-816): their top-left corner; normals missing from
        // them come from the full-size disparity (:363-365)
        const int T = levels - 1;
        const float* id = nullptr;
        const float4* in = nullptr;
        if (initdisp) {
            const float4* nfull = initnormal;
            if (!nfull) {
                float4* nrm = at<float4>(ws, L, Layout::nrm);
                launch_disparity_to_normal(nrm, initdisp, W, H, st);
                nfull = nrm;
                nl++;
            }
            float* cd = at<float>(lw[T], ll[T], Layout::initd);
            float4* cn = at<float4>(lw[T], ll[T], Layout::initn);
            launch_crop(cd, Wl[T], Hl[T], initdisp, W, 1, st);
            launch_crop((float*)cn, Wl[T], Hl[T], (const float*)nfull, W, 4, st);
            nl += 2;
            id = cd;
            in = cn;
        }
        prof_mark(h, st, PM_PHASE_PREP, nl);
        rc = run_level(h, lw[T], ll[T], il[T], ir[T], Wl[T], Hl[T], is[T], r, dmax * ((float)Wl[T] / (float)Wl[0]),
                       iterations, o.thetamin, id, nullptr, in, nullptr, ctr, errf, st);   // :91-93
        if (rc) return rc;
        for (int l = T - 1; l >= 0; l--) {   // :94-120
            const int Wc = Wl[l + 1], Hc = Hl[l + 1], Wf = Wl[l], Hf = Hl[l];
            void* wc = lw[l + 1];
            const Layout& lc = ll[l + 1];
            float* t1 = at<float>(wc, lc, Layout::disp);
            float4* t4 = at<float4>(wc, lc, Layout::nmap);
            float* dl = at<float>(lw[l], ll[l], Layout::initd);
            float* dr = at<float>(lw[l], ll[l], Layout::initdR);
            float4* nlf = at<float4>(lw[l], ll[l], Layout::initn);
            float4* nrf = at<float4>(lw[l], ll[l], Layout::initnR);
            const float4* cl = at<float4>(wc, lc, Layout::mL1);
            const float4* cr = at<float4>(wc, lc, Layout::mR1);
            const float up = (float)Wf / (float)Wc;
            const float4 mulD = make_float4(up, up, up, up), mulN = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
            launch_to_disparity(t1, cl, Wc, Hc, 1.0f, 1, st);
            launch_pyrup_mul(dl, Wf, Hf, t1, Wc, Hc, 1, mulD, st);
            launch_fill_normalmap(t4, cl, Wc, Hc, st);
            launch_pyrup_mul((float*)nlf, Wf, Hf, (const float*)t4, Wc, Hc, 4, mulN, st);
            nl = 4;
            if (views == 2) {
                launch_to_disparity(t1, cr, Wc, Hc, 1.0f, 0, st);
                launch_pyrup_mul(dr, Wf, Hf, t1, Wc, Hc, 1, mulD, st);
                launch_fill_normalmap(t4, cr, Wc, Hc, st);
                launch_pyrup_mul((float*)nrf, Wf, Hf, (const float*)t4, Wc, Hc, 4, mulN, st);
                nl += 4;
            }
            prof_mark(h, st, PM_PHASE_INIT, nl);
            const float mintheta = (float)(levels - l) / (float)levels;
            rc = run_level(h, lw[l], ll[l], il[l], ir[l], Wf, Hf, is[l], r, dmax * ((float)Wf / (float)Wl[0]),
                           iterations, 1e-1f * mintheta + o.thetamin, dl, views == 2 ? dr : nullptr, nlf,
                           views == 2 ? nrf : nullptr, ctr, errf, st);
            if (rc) return rc;
        }
    }
    rc = pair_post(h, ws, L, W, H, pp, dmap, normal, planesL, planesR, st);
    if (rc) return rc;
    PM_CUDA(h, cudaGetLastError());
    return prof_collect(h, st);
}

// texel rows (pm_window.cuh) of both views for the per-kernel entry points, in
// stream-ordered scratch released once the stream has used it
struct TexPair {
    float4* t1 = nullptr;
    float4* t2 = nullptr;
    cudaStream_t st = nullptr;
    int make(const float* bw1, const float* g1, const float* bw2, const float* g2, int W, int H, cudaStream_t s)
    {
        st = s;
        PM_CUDA(nullptr, cudaMallocAsync((void**)&t1, tex_bytes(W, H), s));
        PM_CUDA(nullptr, cudaMallocAsync((void**)&t2, tex_bytes(W, H), s));
        launch_pack_tex(t1, (const float4*)bw1, (const float4*)g1, W, H, s);
        launch_pack_tex(t2, (const float4*)bw2, (const float4*)g2, W, H, s);
        return PM_OK;
    }
    ViewData view(int W, int H, int r) const { return make_view(t1, t2, W, H, r); }
    ~TexPair()
    {
        if (t1) cudaFreeAsync(t1, st);
        if (t2) cudaFreeAsync(t2, st);
    }
};

inline bool aligned(const void* p, size_t n) { return ((uintptr_t)p % n) == 0; }

int check_args(pm_handle* h, const void* left, const void* right, int W, int H, size_t stride, int r, float dmax,
               int iterations, int pp)
{
    if (!h) return fail(h, PM_EINVAL_ARG, "null handle");
    if (!left || !right) return fail(h, PM_EINVAL_ARG, "null image");
    if (!aligned(left, 4) || !aligned(right, 4)) return fail(h, PM_EINVAL_ARG, "images must be 4-byte aligned");
    int rc = check_shape(h, W, H, r);
    if (rc) return rc;
    if (stride < (size_t)W * 4 || stride % 4) return fail(h, PM_EINVAL_SHAPE, "row stride must be >= 4*width and a multiple of 4");
    if (!(dmax > 0.0f) || !isfinite(dmax)) return fail(h, PM_EINVAL_ARG, "disparity range must be positive");
    if (iterations < 0) return fail(h, PM_EINVAL_ARG, "negative iteration count");
    if (pp < PM_PP_NONE || pp > PM_PP_LRCHECK_FILL) return fail(h, PM_EINVAL_ARG, "unknown post-processing mode");
    if (h->opt.views == 1 && pp != PM_PP_NONE) return fail(h, PM_EINVAL_ARG, "the left-right check needs both views");
    return PM_OK;
}

// the handle's own blocking stream: graphs are captured on it (capture is not possible on
// the legacy default stream) and launched on the caller's stream
int own_stream(pm_handle* h, cudaStream_t* out)
{
    if (!h->own) PM_CUDA(h, cudaStreamCreate(&h->own));
    *out = h->own;
    return PM_OK;
}

uint64_t fbits(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

// Run `body(cs)` as a CUDA graph on `st`: captured on the handle's own stream `cs` the first
// time, replayed while `key` (every argument the captured work depends on) is unchanged.
template <class Fn>
int run_graph(pm_handle* h, std::vector<uint64_t>& cached, cudaGraphExec_t& exec, const std::vector<uint64_t>& key,
              cudaStream_t st, Fn body)
{
    if (!(exec && cached == key)) {
        if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
        cached.clear();
        cudaStream_t cs;
        int rc = own_stream(h, &cs);
        if (rc) return rc;
        PM_CUDA(h, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        h->capturing = 1;
        rc = body(cs);
        h->capturing = 0;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cs, &g);
        if (rc) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return rc; }
        if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) { exec = nullptr; return cuda_fail(h, ei, "cudaGraphInstantiate"); }
        cached = key;
    }
    PM_CUDA(h, cudaGraphLaunch(exec, st));
    return PM_OK;
}

// graphs are used unless disabled, while profiling (per-phase events need eager launches),
// or when the caller is itself capturing `st` (the launches then go into the caller's graph)
int use_graph(pm_handle* h, cudaStream_t st, bool* yes)
{
    *yes = false;
    if (!h->opt.use_graph || h->profiling) return PM_OK;
    if (st) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        PM_CUDA(h, cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) return PM_OK;
    }
    *yes = true;
    return PM_OK;
}

// the single-pair pipeline on `st`, through the handle's graph when graphs are in use
int pipeline_on(pm_handle* h, void* ws, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride, int r,
                float dmax, int iterations, int pp, float* dmap, float4* normal, const float* initdisp,
                const float4* initnormal, float4* planesL, float4* planesR, cudaStream_t st, int depth = 0,
                float dscale = 0.0f)
{
    auto run = [&](cudaStream_t s) {
        if (depth)
            return run_depth(h, ws, left, right, W, H, stride, r, dmax, iterations, dscale, pp, dmap, normal, initdisp,
                             initnormal, planesL, planesR, s);
        return run_pipeline(h, ws, left, right, W, H, stride, r, dmax, iterations, pp, dmap, normal, initdisp,
                            initnormal, planesL, planesR, s);
    };
    bool graph = false;
    int rc = use_graph(h, st, &graph);
    if (rc) return rc;
    if (!graph) return run(st);
    const pm_options& o = h->opt;
    std::vector<uint64_t> key = {
        (uint64_t)(uintptr_t)ws, (uint64_t)(uintptr_t)left, (uint64_t)(uintptr_t)right, (uint64_t)W, (uint64_t)H,
        (uint64_t)stride, (uint64_t)r, fbits(dmax), (uint64_t)iterations, (uint64_t)pp, (uint64_t)(uintptr_t)dmap,
        (uint64_t)(uintptr_t)normal, (uint64_t)(uintptr_t)initdisp, (uint64_t)(uintptr_t)initnormal,
        (uint64_t)(uintptr_t)planesL, (uint64_t)(uintptr_t)planesR, (uint64_t)o.views, (uint64_t)o.fused,
        fbits(o.thetamin), fbits(o.maxdispdiff), fbits(o.maxanglediff), (uint64_t)o.rof_iters, (uint64_t)h->counting,
        (uint64_t)o.levels, (uint64_t)depth, fbits(dscale), (uint64_t)(uintptr_t)h->init_right,
        (uint64_t)(uintptr_t)h->init_normal_right};
    for (void* p : h->lws) key.push_back((uint64_t)(uintptr_t)p);
    return run_graph(h, h->key1, h->exec1, key, st, run);
}

}  // namespace

extern "C" {

const char* pm_status_string(int s)
{
    switch (s) {
        case PM_OK: return "ok";
        case PM_EINVAL_SHAPE: return "invalid shape";
        case PM_EINVAL_ARG: return "invalid argument";
        case PM_ENOMEM: return "out of memory";
        case PM_ECUDA: return "CUDA error";
        case PM_ETIMEOUT: return "device wait timed out";
        case PM_ENOTIMPL: return "not implemented";
        case PM_ENODEV: return "no CUDA device";
        default: return "unknown status";
    }
}

int pm_options_default(pm_options* o)
{
    if (!o) return PM_EINVAL_ARG;
    o->views = 2;
    o->fused = 0;
    o->thetamin = 1e-4f;
    o->maxdispdiff = 1.0f;
    o->maxanglediff = 5.0f;
    o->rof_iters = 40;
    o->device = 0;
    o->use_graph = 1;
    o->levels = 1;
    return PM_OK;
}

int pm_create(pm_handle** out, const pm_options* opt)
{
    if (!out) return fail(nullptr, PM_EINVAL_ARG, "null handle pointer");
    *out = nullptr;
    pm_options o;
    pm_options_default(&o);
    if (opt) o = *opt;
    if (o.views != 1 && o.views != 2) return fail(nullptr, PM_EINVAL_ARG, "views must be 1 or 2");
    if (o.rof_iters < 0) return fail(nullptr, PM_EINVAL_ARG, "negative smoothing iteration count");
    if (o.levels < 1 || o.levels > PM_MAX_LEVELS) return fail(nullptr, PM_EINVAL_ARG, "pyramid levels out of range");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return fail(nullptr, PM_ENODEV, "no CUDA device"); }
    if (o.device < 0 || o.device >= n) return fail(nullptr, PM_EINVAL_ARG, "device ordinal out of range");
    pm_handle* h = new pm_handle();
    h->opt = o;
    *out = h;
    return PM_OK;
}

int pm_destroy(pm_handle* h)
{
    if (!h) return PM_OK;
    if (h->ws) cudaFree(h->ws);
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    if (h->exec1) cudaGraphExecDestroy(h->exec1);
    if (h->execb) cudaGraphExecDestroy(h->execb);
    for (void* p : h->bws)
        if (p) cudaFree(p);
    for (void* p : h->lws)
        if (p) cudaFree(p);
    if (h->btab) cudaFree(h->btab);
    for (cudaStream_t b : h->branch) cudaStreamDestroy(b);
    for (cudaEvent_t e : h->bev) cudaEventDestroy(e);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
    return PM_OK;
}

int pm_set_profiling(pm_handle* h, int on)
{
    if (!h) return PM_EINVAL_ARG;
    h->profiling = on ? 1 : 0;
    return PM_OK;
}

int pm_get_phase_times(pm_handle* h, float ms[PM_NPHASES], int launches[PM_NPHASES])
{
    if (!h) return PM_EINVAL_ARG;
    for (int k = 0; k < PM_NPHASES; k++) {
        if (ms) ms[k] = h->phase_ms[k];
        if (launches) launches[k] = h->phase_launches[k];
    }
    return PM_OK;
}

int pm_measure_fp32_peak(int device, float ms, float* tflops)
{
    if (!tflops || !(ms > 0.0f)) return fail(nullptr, PM_EINVAL_ARG, "bad argument");
    PM_CUDA(nullptr, cudaSetDevice(device));
    float* buf = nullptr;
    int sms = 0;
    PM_CUDA(nullptr, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * 8, threads = 256;
    PM_CUDA(nullptr, cudaMalloc(&buf, (size_t)blocks * threads * sizeof(float)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 0.0f;
    int iters = 4096;
    for (int rep = 0; rep < 6; rep++) {
        cudaEventRecord(a);
        launch_fma_peak(buf, iters, blocks, threads, 0);
        cudaEventRecord(b);
        cudaError_t e = cudaEventSynchronize(b);
        if (e != cudaSuccess) { cudaFree(buf); return cuda_fail(nullptr, e, "fp32 peak kernel"); }
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, b);
        const double flops = (double)blocks * threads * iters * fma_peak_flops_per_iter();
        best = fmaxf(best, (float)(flops / (t * 1e-3) / 1e12));
        if (t < ms && iters < (1 << 24)) iters = (int)(iters * fminf(8.0f, ms / fmaxf(t, 1e-3f)));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(buf);
    *tflops = best;
    return PM_OK;
}

const char* pm_last_error(const pm_handle* h) { return h ? h->err.c_str() : t_err.c_str(); }

int pm_set_batch_branches(pm_handle* h, int n)
{
    if (!h) return fail(nullptr, PM_EINVAL_ARG, "null handle");
    if (n < 0 || n > PM_BATCH_BRANCHES) return fail(h, PM_EINVAL_ARG, "branch count out of range");
    h->batch_branches = n;
    return PM_OK;
}

int pm_set_counting(pm_handle* h, int on)
{
    if (!h) return PM_EINVAL_ARG;
    h->counting = on ? 1 : 0;
    return PM_OK;
}

int pm_get_counters(pm_handle* h, uint64_t c[4])
{
    if (!h || !c) return PM_EINVAL_ARG;
    if (!h->ws) { memset(c, 0, 32); return PM_OK; }
    const Layout L = layout(h->W, h->H, (size_t)h->W * 4);
    (void)L;
    memcpy(c, h->counters, 32);
    return PM_OK;
}

}  // extern "C"

namespace {

// single-pair entry with device buffers: disparityMap (depth = 0) or depthMap (depth = 1)
int entry_device(pm_handle* h, int depth, float dscale, const uint8_t* left, const uint8_t* right, int W, int H,
                 size_t stride, int patchsize, float dispmax, int iterations, int pp, float* dmap, float* normalmap,
                 const float* initdisp, const float* initnormal, float* planes_left, float* planes_right,
                 cudaStream_t st)
{
    int rc = check_args(h, left, right, W, H, stride, patchsize, dispmax, iterations, pp);
    if (rc) return rc;
    if (!aligned(dmap, 4) || !aligned(initdisp, 4) || !aligned(normalmap, 16) || !aligned(initnormal, 16) ||
        !aligned(planes_left, 16) || !aligned(planes_right, 16))
        return fail(h, PM_EINVAL_ARG, "float fields must be 4-byte aligned, float4 fields 16-byte aligned");
    PM_CUDA(h, cudaSetDevice(h->opt.device));
    h->W = W;
    h->H = H;
    rc = ensure_ws(h, W, H, stride);
    if (rc) return rc;
    if (!depth) {
        rc = ensure_level_ws(h, W, H);
        if (rc) return rc;
    }
    rc = pipeline_on(h, h->ws, left, right, W, H, stride, patchsize, dispmax, iterations, pp, dmap,
                     reinterpret_cast<float4*>(normalmap), initdisp, reinterpret_cast<const float4*>(initnormal),
                     reinterpret_cast<float4*>(planes_left), reinterpret_cast<float4*>(planes_right), st, depth, dscale);
    if (rc) return rc;
    if (h->counting) {
        const Layout L = layout(W, H, stride);
        unsigned long long c[4];
        PM_CUDA(h, cudaMemcpyAsync(c, at<unsigned long long>(h->ws, L, Layout::ctr), 32, cudaMemcpyDeviceToHost, st));
        PM_CUDA(h, cudaStreamSynchronize(st));
        for (int k = 0; k < 4; k++) h->counters[k] = c[k];
    }
    return PM_OK;
}

// single-pair entry with host buffers: inputs staged into the workspace, outputs copied back,
// on the legacy default stream; returns once the outputs are written
int entry_host(pm_handle* h, int depth, float dscale, const uint8_t* left, const uint8_t* right, int W, int H,
               size_t stride, int patchsize, float dispmax, int iterations, int pp, float* dmap, float* normalmap,
               const float* initdisp, const float* initnormal, float* planes_left, float* planes_right)
{
    int rc = check_args(h, left, right, W, H, stride, patchsize, dispmax, iterations, pp);
    if (rc) return rc;
    PM_CUDA(h, cudaSetDevice(h->opt.device));
    rc = ensure_ws(h, W, H, stride);
    if (rc) return rc;
    if (!depth) {
        rc = ensure_level_ws(h, W, H);
        if (rc) return rc;
    }
    h->W = W;
    h->H = H;
    const Layout L = layout(W, H, stride);
    const size_t N = L.N;
    cudaStream_t st = 0;
    uint8_t* dl = at<uint8_t>(h->ws, L, Layout::img0);
    uint8_t* dr = at<uint8_t>(h->ws, L, Layout::img1);
    float* dd = at<float>(h->ws, L, Layout::dmap);
    float4* dn = at<float4>(h->ws, L, Layout::nmap);
    float* di = at<float>(h->ws, L, Layout::initd);
    float4* dni = at<float4>(h->ws, L, Layout::initn);
    float4* dpl = at<float4>(h->ws, L, Layout::outpL);
    float4* dpr = at<float4>(h->ws, L, Layout::outpR);
    PM_CUDA(h, cudaMemcpyAsync(dl, left, stride * H, cudaMemcpyHostToDevice, st));
    PM_CUDA(h, cudaMemcpyAsync(dr, right, stride * H, cudaMemcpyHostToDevice, st));
    if (initdisp) PM_CUDA(h, cudaMemcpyAsync(di, initdisp, N * 4, cudaMemcpyHostToDevice, st));
    if (initnormal) PM_CUDA(h, cudaMemcpyAsync(dni, initnormal, N * 16, cudaMemcpyHostToDevice, st));
    rc = pipeline_on(h, h->ws, dl, dr, W, H, stride, patchsize, dispmax, iterations, pp, dmap ? dd : nullptr,
                     normalmap ? dn : nullptr, initdisp ? di : nullptr, initnormal ? dni : nullptr,
                     planes_left ? dpl : nullptr, planes_right ? dpr : nullptr, st, depth, dscale);
    if (rc) return rc;
    if (dmap) PM_CUDA(h, cudaMemcpyAsync(dmap, dd, N * 4, cudaMemcpyDeviceToHost, st));
    if (normalmap) PM_CUDA(h, cudaMemcpyAsync(normalmap, dn, N * 16, cudaMemcpyDeviceToHost, st));
    if (planes_left) PM_CUDA(h, cudaMemcpyAsync(planes_left, dpl, N * 16, cudaMemcpyDeviceToHost, st));
    if (planes_right && h->opt.views == 2) PM_CUDA(h, cudaMemcpyAsync(planes_right, dpr, N * 16, cudaMemcpyDeviceToHost, st));
    if (h->counting) {
        unsigned long long c[4];
        PM_CUDA(h, cudaMemcpyAsync(c, at<unsigned long long>(h->ws, L, Layout::ctr), 32, cudaMemcpyDeviceToHost, st));
        PM_CUDA(h, cudaStreamSynchronize(st));
        for (int k = 0; k < 4; k++) h->counters[k] = c[k];
    }
    int errv = 0;
    PM_CUDA(h, cudaMemcpyAsync(&errv, at<int>(h->ws, L, Layout::errf), 4, cudaMemcpyDeviceToHost, st));
    PM_CUDA(h, cudaStreamSynchronize(st));
    if (errv) return fail(h, PM_ETIMEOUT, "view-buffer insertion retried too often");
    return PM_OK;
}

}  // namespace

extern "C" {

int pm_disparity_map_device(pm_handle* h, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride,
                            int patchsize, float dispmax, int iterations, int pp, float* dmap, float* normalmap,
                            const float* initdisp, const float* initnormal, float* planes_left, float* planes_right,
                            void* stream)
{
    return entry_device(h, 0, 0.0f, left, right, W, H, stride, patchsize, dispmax, iterations, pp, dmap, normalmap,
                        initdisp, initnormal, planes_left, planes_right, S(stream));
}

int pm_disparity_map_init2_device(pm_handle* h, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride,
                                  int patchsize, float dispmax, int iterations, int pp, float* dmap, float* normalmap,
                                  const float* initdisp_left, const float* initdisp_right, const float* initnormal_left,
                                  const float* initnormal_right, float* planes_left, float* planes_right, void* stream)
{
    if (!h) return fail(nullptr, PM_EINVAL_ARG, "null handle");
    if (initdisp_right && (h->opt.levels != 1 || h->opt.views != 2))
        return fail(h, PM_EINVAL_ARG, "a right-view initial disparity needs one pyramid level and both views");
    if (initnormal_right && !initdisp_right)
        return fail(h, PM_EINVAL_ARG, "a right-view initial normal map needs a right-view initial disparity");
    if (!aligned(initdisp_right, 4) || !aligned(initnormal_right, 16))
        return fail(h, PM_EINVAL_ARG, "float fields must be 4-byte aligned, normal maps 16-byte aligned");
    h->init_right = initdisp_right;
    h->init_normal_right = initnormal_right;
    const int rc = entry_device(h, 0, 0.0f, left, right, W, H, stride, patchsize, dispmax, iterations, pp, dmap, normalmap,
                                initdisp_left, initnormal_left, planes_left, planes_right, S(stream));
    h->init_right = nullptr;
    h->init_normal_right = nullptr;
    return rc;
}

int pm_disparity_map(pm_handle* h, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride,
                     int patchsize, float dispmax, int iterations, int pp, float* dmap, float* normalmap,
                     const float* initdisp, const float* initnormal, float* planes_left, float* planes_right)
{
    return entry_host(h, 0, 0.0f, left, right, W, H, stride, patchsize, dispmax, iterations, pp, dmap, normalmap,
                      initdisp, initnormal, planes_left, planes_right);
}

int pm_depth_map_device(pm_handle* h, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride,
                        int patchsize, float dispmax, int iterations, float dscale, int pp, float* dmap,
                        float* normalmap, const float* initdisp, const float* initnormal, float* planes_left,
                        float* planes_right, void* stream)
{
    return entry_device(h, 1, dscale, left, right, W, H, stride, patchsize, dispmax, iterations, pp, dmap, normalmap,
                        initdisp, initnormal, planes_left, planes_right, S(stream));
}

int pm_depth_map(pm_handle* h, const uint8_t* left, const uint8_t* right, int W, int H, size_t stride, int patchsize,
                 float dispmax, int iterations, float dscale, int pp, float* dmap, float* normalmap,
                 const float* initdisp, const float* initnormal, float* planes_left, float* planes_right)
{
    return entry_host(h, 1, dscale, left, right, W, H, stride, patchsize, dispmax, iterations, pp, dmap, normalmap,
                      initdisp, initnormal, planes_left, planes_right);
}

// longest processing time first: pairs in decreasing window work W*H*(2r+1)^2 (stable), each
// to the least loaded of nb branches (the lowest index among equals)
static void batch_schedule(int n, int nb, const int* width, const int* height, const int* patchsize, int* order,
                           int* owner)
{
    std::vector<double> work(n), load(nb, 0.0);
    for (int i = 0; i < n; i++) {
        order[i] = i;
        work[i] = (double)width[i] * height[i] * (2.0 * patchsize[i] + 1.0) * (2.0 * patchsize[i] + 1.0);
    }
    std::stable_sort(order, order + n, [&](int a, int b) { return work[a] > work[b]; });
    for (int k = 0; k < n; k++) {
        const int i = order[k];
        int best = 0;
        for (int b = 1; b < nb; b++)
            if (load[b] < load[best]) best = b;
        owner[i] = best;
        load[best] += work[i];
    }
}

int pm_batch_schedule(int n, int branches, const int* width, const int* height, const int* patchsize, int* order,
                      int* owner)
{
    if (n < 0 || n > PM_MAX_BATCH) return fail(nullptr, PM_EINVAL_ARG, "batch size out of range");
    if (branches < 1 || branches > PM_BATCH_BRANCHES) return fail(nullptr, PM_EINVAL_ARG, "branch count out of range");
    if (n == 0) return PM_OK;
    if (!width || !height || !patchsize || !order || !owner) return fail(nullptr, PM_EINVAL_ARG, "null array");
    batch_schedule(n, n < branches ? n : branches, width, height, patchsize, order, owner);
    return PM_OK;
}

// Split of a batch over `ranks` processes (one GPU each), balanced by each pair's work
// W*H*(2r+1)^2*dispmax: the pairs in decreasing work (stable), each to the least loaded rank
// (the lowest index among equals).  Host only; no collective is involved, every rank computes
// the same split from the same arrays.
int pm_batch_partition(int n, int ranks, const int* width, const int* height, const int* patchsize,
                       const float* dispmax, int* rank_of, double* load)
{
    if (n < 0 || n > PM_MAX_BATCH) return fail(nullptr, PM_EINVAL_ARG, "batch size out of range");
    if (ranks < 1 || ranks > PM_MAX_RANKS) return fail(nullptr, PM_EINVAL_ARG, "rank count out of range");
    if (n > 0 && (!width || !height || !patchsize || !dispmax || !rank_of))
        return fail(nullptr, PM_EINVAL_ARG, "null array");
    std::vector<double> work(n), ld(ranks, 0.0);
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) {
        if (width[i] < 1 || height[i] < 1 || patchsize[i] < 0 || !(dispmax[i] > 0.0f))
            return fail(nullptr, PM_EINVAL_ARG, "pair " + std::to_string(i) + " has no work");
        order[i] = i;
        const double win = (2.0 * patchsize[i] + 1.0) * (2.0 * patchsize[i] + 1.0);
        work[i] = (double)width[i] * height[i] * win * dispmax[i];
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
    for (int k = 0; k < n; k++) {
        const int i = order[k];
        int best = 0;
        for (int r = 1; r < ranks; r++)
            if (ld[r] < ld[best]) best = r;
        rank_of[i] = best;
        ld[best] += work[i];
    }
    if (load)
        for (int r = 0; r < ranks; r++) load[r] = ld[r];
    return PM_OK;
}

// the tile jobs of a lockstep batch (pm_batch_jobs): `order` lists the pairs in decreasing work
static void batch_jobs(int n, const int* width, const int* height, const int* order, int tw, int th, int tile_order,
                       std::vector<uint32_t>& jobs)
{
    jobs.clear();
    int rows_max = 0;
    for (int k = 0; k < n; k++) rows_max = std::max(rows_max, (height[order[k]] + th - 1) / th);
    auto row = [&](int i, int by) {
        const int gx = (width[i] + tw - 1) / tw;
        for (int bx = 0; bx < gx; bx++) {
            jobs.push_back((uint32_t)i);
            jobs.push_back(((uint32_t)by << 16) | (uint32_t)bx);
        }
    };
    if (tile_order == 0) {
        for (int k = 0; k < n; k++)
            for (int by = 0; by < (height[order[k]] + th - 1) / th; by++) row(order[k], by);
    } else {
        for (int by = 0; by < rows_max; by++)
            for (int k = 0; k < n; k++)
                if (by < (height[order[k]] + th - 1) / th) row(order[k], by);
    }
}

int pm_set_batch_schedule(pm_handle* h, int schedule, int ctas_per_sm, int tile_order, int tile_w)
{
    if (!h) return fail(nullptr, PM_EINVAL_ARG, "null handle");
    if (schedule != PM_BATCH_LOCKSTEP && schedule != PM_BATCH_BRANCHED) return fail(h, PM_EINVAL_ARG, "unknown batch schedule");
    if (ctas_per_sm < 0 || ctas_per_sm > 64) return fail(h, PM_EINVAL_ARG, "CTAs per SM out of range");
    if (tile_order != 0 && tile_order != 1) return fail(h, PM_EINVAL_ARG, "unknown tile order");
    if (tile_w != 0 && tile_w != 16 && tile_w != 32) return fail(h, PM_EINVAL_ARG, "tile width must be 16 or 32");
    h->batch_tile_w = tile_w ? tile_w : 32;
    h->batch_schedule = schedule;
    h->batch_ctas = ctas_per_sm;
    h->batch_order = tile_order;
    return PM_OK;
}

int pm_batch_jobs(int n, const int* width, const int* height, const int* patchsize, int tile_w, int tile_h,
                  int tile_order, uint32_t* jobs, int njobs_cap, int* njobs)
{
    if (n < 0 || n > PM_MAX_BATCH) return fail(nullptr, PM_EINVAL_ARG, "batch size out of range");
    if (!njobs) return fail(nullptr, PM_EINVAL_ARG, "null job count");
    if (tile_w < 1 || tile_h < 1) return fail(nullptr, PM_EINVAL_ARG, "tile size out of range");
    if (tile_order != 0 && tile_order != 1) return fail(nullptr, PM_EINVAL_ARG, "unknown tile order");
    *njobs = 0;
    if (n == 0) return PM_OK;
    if (!width || !height || !patchsize) return fail(nullptr, PM_EINVAL_ARG, "null array");
    for (int i = 0; i < n; i++)
        if (width[i] < 1 || height[i] < 1 || width[i] > PM_MAX_WIDTH || height[i] > PM_MAX_HEIGHT)
            return fail(nullptr, PM_EINVAL_SHAPE, "pair " + std::to_string(i) + " has an unsupported size");
    std::vector<int> order(n), owner(n);
    batch_schedule(n, 1, width, height, patchsize, order.data(), owner.data());
    std::vector<uint32_t> v;
    batch_jobs(n, width, height, order.data(), tile_w, tile_h, tile_order, v);
    const int cnt = (int)(v.size() / 2);
    *njobs = cnt;
    if (jobs) {
        if (njobs_cap < cnt) return fail(nullptr, PM_EINVAL_ARG, "job array too small");
        memcpy(jobs, v.data(), v.size() * sizeof(uint32_t));
    }
    return PM_OK;
}

// Lockstep batched call (PM_BATCH_LOCKSTEP): the pairs' prep / init and post-processing as
// branches of `cs`, every iteration's propagate passes and smoothing stages as persistent
// launches over the tiles of all pairs.  Each pair sees the same operations in the same order
// as in run_pipeline (levels 1), so the results are the same.
static int batch_lockstep(pm_handle* h, int n, const uint8_t* const* left, const uint8_t* const* right,
                          const int* width, const int* height, const size_t* stride, const int* patchsize,
                          const float* dispmax, int iterations, int pp, float* const* dmap,
                          float* const* planes_left, float* const* planes_right, int nb, const int* order,
                          const int* owner, cudaStream_t st, bool graph)
{
    const pm_options& o = h->opt;
    const int views = o.views, F = o.fused;
    const int itx = iterations | 1;   // PMHuberStereo.cpp:490
    std::vector<Layout> L(n);
    std::vector<LevelBufs> B(n);
    for (int i = 0; i < n; i++) {
        L[i] = layout(width[i], height[i], stride[i]);
        B[i] = level_bufs(h->bws[i], L[i], width[i], height[i], patchsize[i]);
    }
    // host tables: propagate arguments per (iteration, view, pair) (launch parameters),
    // smoothing arguments per (view, pair), the job lists and the work counters (device
    // memory, the counters zeroed in the stream)
    std::vector<PropParams> ptab((size_t)itx * views * n);
    for (int it = 0; it < itx; it++) {
        const float theta = theta_at(it, itx, o.thetamin);
        for (int v = 0; v < views; v++)
            for (int i = 0; i < n; i++) {
                PropParams P = prop_params(h, B[i], v, it, it & 1, theta, dispmax[i],
                                           at<unsigned long long>(h->bws[i], L[i], Layout::ctr),
                                           at<int>(h->bws[i], L[i], Layout::errf));
                P.dual = h->counting ? 0 : 1;
                ptab[((size_t)it * views + v) * n + i] = P;
            }
    }
    std::vector<SmoothArgs> stab((size_t)views * n);
    for (int v = 0; v < views; v++)
        for (int i = 0; i < n; i++) {
            SmoothArgs A;
            A.out = v ? B[i].Rs : B[i].Ls;
            A.tmp = B[i].tmp;
            A.dt = v ? B[i].RDT : B[i].LDT;
            A.scratch = static_cast<float4*>(B[i].rofs);
            A.planes[0] = v ? B[i].mR[0] : B[i].mL[0];
            A.planes[1] = v ? B[i].mR[1] : B[i].mL[1];
            A.dispscale = 1.0f / dispmax[i];
            A.lr = v ? 0 : 1;
            A.W = width[i];
            A.H = height[i];
            stab[(size_t)v * n + i] = A;
        }
    // the propagate passes run per group of up to PROP_GROUP pairs (consecutive in `order`),
    // whose arguments are the launch's parameters: group g's table lists its pairs' arguments
    // in order and its job list indexes that table
    int ptw, pth;
    if (!prop_batch_tile_shape(h->batch_tile_w, &ptw, &pth)) return fail(h, PM_EINVAL_ARG, "unsupported tile width");
    const int ngroups = (n + PROP_GROUP - 1) / PROP_GROUP;
    std::vector<std::vector<PropParams>> gtab((size_t)ngroups * itx * views);
    std::vector<std::vector<uint32_t>> jpg(ngroups);
    for (int g = 0; g < ngroups; g++) {
        const int k0 = g * PROP_GROUP, m = std::min(n - k0, PROP_GROUP);
        std::vector<int> gw(m), gh(m), gorder(m);
        for (int k = 0; k < m; k++) {
            gw[k] = width[order[k0 + k]];
            gh[k] = height[order[k0 + k]];
            gorder[k] = k;
        }
        batch_jobs(m, gw.data(), gh.data(), gorder.data(), ptw, pth, h->batch_order, jpg[g]);
        for (int it = 0; it < itx; it++)
            for (int v = 0; v < views; v++) {
                std::vector<PropParams>& t = gtab[((size_t)g * itx + it) * views + v];
                for (int k = 0; k < m; k++) t.push_back(ptab[((size_t)it * views + v) * n + order[k0 + k]]);
            }
    }
    std::vector<uint32_t> jp, j8, j16;
    for (int g = 0; g < ngroups; g++) jp.insert(jp.end(), jpg[g].begin(), jpg[g].end());
    batch_jobs(n, width, height, order, SMOOTH_TW, SMOOTH_TH8, h->batch_order, j8);
    batch_jobs(n, width, height, order, SMOOTH_TW, SMOOTH_TH16, h->batch_order, j16);
    const int per_iter = views * (ngroups * propagate_batch_launches(h->counting) + smooth_batch_launches(o.rof_iters));
    const size_t nslots = (size_t)itx * per_iter;
    auto pad = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t o_s = 0;
    const size_t o_jp = o_s + pad(stab.size() * sizeof(SmoothArgs));
    const size_t o_j8 = o_jp + pad(jp.size() * 4), o_j16 = o_j8 + pad(j8.size() * 4);
    const size_t o_ctr = o_j16 + pad(j16.size() * 4), total = o_ctr + pad(nslots * 4);
    std::vector<unsigned char> hb(o_ctr, 0);
    memcpy(hb.data() + o_s, stab.data(), stab.size() * sizeof(SmoothArgs));
    memcpy(hb.data() + o_jp, jp.data(), jp.size() * 4);
    memcpy(hb.data() + o_j8, j8.data(), j8.size() * 4);
    memcpy(hb.data() + o_j16, j16.data(), j16.size() * 4);
    if (!(h->btab && h->btab_bytes >= total && h->btab_host == hb)) {
        // earlier calls on this stream may still read the tables: let them finish first
        PM_CUDA(h, cudaStreamSynchronize(st));
        if (h->btab_bytes < total) {
            if (h->btab) cudaFree(h->btab);
            h->btab = nullptr;
            h->btab_bytes = 0;
            h->btab_host.clear();
            int rc = grow(h, h->btab, h->btab_bytes, total);
            if (rc) return rc;
        }
        PM_CUDA(h, cudaMemcpy(h->btab, hb.data(), hb.size(), cudaMemcpyHostToDevice));
        h->btab_host.swap(hb);
    }
    char* base = static_cast<char*>(h->btab);
    const SmoothArgs* dS = reinterpret_cast<const SmoothArgs*>(base + o_s);
    std::vector<JobList> Jp(ngroups);
    for (int g = 0, off = 0; g < ngroups; off += (int)(jpg[g].size() / 2), g++)
        Jp[g] = JobList{reinterpret_cast<const uint2*>(base + o_jp) + off, (int)(jpg[g].size() / 2)};
    const JobList J8{reinterpret_cast<const uint2*>(base + o_j8), (int)(j8.size() / 2)};
    const JobList J16{reinterpret_cast<const uint2*>(base + o_j16), (int)(j16.size() / 2)};
    int* slots = reinterpret_cast<int*>(base + o_ctr);

    auto fork = [&](cudaStream_t cs) -> int {
        PM_CUDA(h, cudaEventRecord(h->bev[nb], cs));
        for (int b = 0; b < nb; b++) PM_CUDA(h, cudaStreamWaitEvent(h->branch[b], h->bev[nb], 0));
        return PM_OK;
    };
    auto join = [&](cudaStream_t cs) -> int {
        for (int b = 0; b < nb; b++) {
            PM_CUDA(h, cudaEventRecord(h->bev[b], h->branch[b]));
            PM_CUDA(h, cudaStreamWaitEvent(cs, h->bev[b], 0));
        }
        return PM_OK;
    };
    auto body = [&](cudaStream_t cs) -> int {
        PM_CUDA(h, cudaMemsetAsync(slots, 0, nslots * 4, cs));
        int rc = fork(cs);
        if (rc) return rc;
        for (int k = 0; k < n; k++) {
            const int i = order[k];
            const cudaStream_t bs = h->branch[owner[i]];
            PM_CUDA(h, cudaMemsetAsync(at<void>(h->bws[i], L[i], Layout::ctr), 0, 64, bs));
            PM_CUDA(h, cudaMemsetAsync(at<void>(h->bws[i], L[i], Layout::errf), 0, 64, bs));
            rc = level_begin(h, B[i], left[i], right[i], stride[i], patchsize[i], dispmax[i], o.thetamin, nullptr,
                             nullptr, nullptr, nullptr, at<float4>(h->bws[i], L[i], Layout::nrm),
                             at<float4>(h->bws[i], L[i], Layout::initnR), bs);
            if (rc) return rc;
        }
        if ((rc = join(cs))) return rc;
        int* next = slots;
        for (int it = 0; it < itx; it++) {
            for (int v = 0; v < views; v++)
                for (int g = 0; g < ngroups; g++) {
                    const std::vector<PropParams>& t = gtab[((size_t)g * itx + it) * views + v];
                    launch_propagate_batch(t.data(), (int)t.size(), Jp[g], ptw, h->batch_ctas, F, h->counting, next,
                                           cs);
                    next += propagate_batch_launches(h->counting);
                }
            if (it + 1 < itx) {   // as in run_level: no smoothing after the last iteration
                const float4 lam = smooth_lambda(theta_at(it, itx, o.thetamin));
                for (int v = 0; v < views; v++) {
                    launch_smooth_batch(dS + (size_t)v * n, J8, J16, 1 - (it & 1), lam, o.rof_iters, next, cs);
                    next += smooth_batch_launches(o.rof_iters);
                }
            }
        }
        if ((rc = fork(cs))) return rc;
        for (int k = 0; k < n; k++) {
            const int i = order[k];
            rc = pair_post(h, h->bws[i], L[i], width[i], height[i], pp, dmap ? dmap[i] : nullptr, nullptr,
                           planes_left ? reinterpret_cast<float4*>(planes_left[i]) : nullptr,
                           planes_right ? reinterpret_cast<float4*>(planes_right[i]) : nullptr,
                           h->branch[owner[i]]);
            if (rc) return rc;
        }
        if ((rc = join(cs))) return rc;
        PM_CUDA(h, cudaGetLastError());
        return PM_OK;
    };
    if (!graph) return body(st);
    std::vector<uint64_t> key = {(uint64_t)n, (uint64_t)nb, (uint64_t)iterations, (uint64_t)pp, (uint64_t)o.views,
                                 (uint64_t)o.fused, fbits(o.thetamin), fbits(o.maxdispdiff), fbits(o.maxanglediff),
                                 (uint64_t)o.rof_iters, (uint64_t)h->counting, (uint64_t)PM_BATCH_LOCKSTEP,
                                 (uint64_t)h->batch_ctas, (uint64_t)h->batch_order, (uint64_t)h->batch_tile_w,
                                 (uint64_t)(uintptr_t)h->btab};
    for (int i = 0; i < n; i++) {
        const uint64_t v[] = {(uint64_t)(uintptr_t)h->bws[i], (uint64_t)(uintptr_t)left[i], (uint64_t)(uintptr_t)right[i],
                              (uint64_t)width[i], (uint64_t)height[i], (uint64_t)stride[i], (uint64_t)patchsize[i],
                              fbits(dispmax[i]), (uint64_t)(uintptr_t)(dmap ? dmap[i] : nullptr),
                              (uint64_t)(uintptr_t)(planes_left ? planes_left[i] : nullptr),
                              (uint64_t)(uintptr_t)(planes_right ? planes_right[i] : nullptr)};
        key.insert(key.end(), v, v + 11);
    }
    return run_graph(h, h->keyb, h->execb, key, st, body);
}

int pm_disparity_map_batch_device(pm_handle* h, int n, const uint8_t* const* left, const uint8_t* const* right,
                                  const int* width, const int* height, const size_t* stride, const int* patchsize,
                                  const float* dispmax, int iterations, int pp, float* const* dmap,
                                  float* const* planes_left, float* const* planes_right, void* stream)
{
    if (!h) return fail(h, PM_EINVAL_ARG, "null handle");
    if (n < 0 || n > PM_MAX_BATCH) return fail(h, PM_EINVAL_ARG, "batch size out of range");
    if (h->opt.levels != 1) return fail(h, PM_EINVAL_ARG, "pyramid levels apply to single-pair calls only");
    if (n == 0) return PM_OK;
    if (!left || !right || !width || !height || !stride || !patchsize || !dispmax)
        return fail(h, PM_EINVAL_ARG, "null per-pair array");
    for (int i = 0; i < n; i++) {
        const int rc = check_args(h, left[i], right[i], width[i], height[i], stride[i], patchsize[i], dispmax[i],
                                  iterations, pp);
        if (rc) return rc;
    }
    PM_CUDA(h, cudaSetDevice(h->opt.device));
    // one workspace per pair
    if ((int)h->bws.size() < n) { h->bws.resize(n, nullptr); h->bws_bytes.resize(n, 0); }
    for (int i = 0; i < n; i++) {
        const int rc = grow(h, h->bws[i], h->bws_bytes[i], layout(width[i], height[i], stride[i]).total);
        if (rc) return rc;
    }
    // pairs in decreasing window work, each to the least loaded branch (longest processing
    // time first); the branches run concurrently inside one graph
    const int cap = h->batch_branches > 0 ? h->batch_branches : PM_BATCH_BRANCHES;
    const int nb = n < cap ? n : cap;
    while ((int)h->branch.size() < nb) {
        cudaStream_t b;
        PM_CUDA(h, cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
        h->branch.push_back(b);
    }
    while ((int)h->bev.size() < nb + 1) {
        cudaEvent_t e;
        PM_CUDA(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->bev.push_back(e);
    }
    std::vector<int> order(n), owner(n);
    batch_schedule(n, nb, width, height, patchsize, order.data(), owner.data());
    const cudaStream_t st = S(stream);
    if (h->batch_schedule == PM_BATCH_LOCKSTEP) {
        // lockstep needs its tables uploaded before the launch: not inside a caller's capture
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (st) PM_CUDA(h, cudaStreamIsCapturing(st, &cap));
        if (cap == cudaStreamCaptureStatusNone) {
            bool graph = false;
            int rc = use_graph(h, st, &graph);
            if (rc) return rc;
            const int saved = h->profiling;
            h->profiling = 0;   // per-phase timing covers single-pair calls only
            rc = batch_lockstep(h, n, left, right, width, height, stride, patchsize, dispmax, iterations, pp, dmap,
                                planes_left, planes_right, nb, order.data(), owner.data(), st, graph);
            h->profiling = saved;
            return rc;
        }
    }
    auto body = [&](cudaStream_t cs) -> int {
        PM_CUDA(h, cudaEventRecord(h->bev[nb], cs));
        for (int b = 0; b < nb; b++) PM_CUDA(h, cudaStreamWaitEvent(h->branch[b], h->bev[nb], 0));
        for (int i : order) {
            const int rc = run_pipeline(h, h->bws[i], left[i], right[i], width[i], height[i], stride[i], patchsize[i],
                                        dispmax[i], iterations, pp, dmap ? dmap[i] : nullptr, nullptr, nullptr,
                                        nullptr, planes_left ? reinterpret_cast<float4*>(planes_left[i]) : nullptr,
                                        planes_right ? reinterpret_cast<float4*>(planes_right[i]) : nullptr,
                                        h->branch[owner[i]]);
            if (rc) return rc;
        }
        for (int b = 0; b < nb; b++) {
            PM_CUDA(h, cudaEventRecord(h->bev[b], h->branch[b]));
            PM_CUDA(h, cudaStreamWaitEvent(cs, h->bev[b], 0));
        }
        return PM_OK;
    };
    bool graph = false;
    int rc = use_graph(h, st, &graph);
    if (rc) return rc;
    const int saved = h->profiling;
    h->profiling = 0;   // per-phase timing covers single-pair calls only
    if (!graph) {
        // eager: the same fork / join on the caller's stream
        rc = body(st);
        h->profiling = saved;
        return rc;
    }
    const pm_options& o = h->opt;
    std::vector<uint64_t> key = {(uint64_t)n, (uint64_t)nb, (uint64_t)iterations, (uint64_t)pp, (uint64_t)o.views,
                                 (uint64_t)o.fused,
                                 fbits(o.thetamin), fbits(o.maxdispdiff), fbits(o.maxanglediff), (uint64_t)o.rof_iters,
                                 (uint64_t)h->counting, (uint64_t)PM_BATCH_BRANCHED};
    for (int i = 0; i < n; i++) {
        const uint64_t v[] = {(uint64_t)(uintptr_t)h->bws[i], (uint64_t)(uintptr_t)left[i], (uint64_t)(uintptr_t)right[i],
                              (uint64_t)width[i], (uint64_t)height[i], (uint64_t)stride[i], (uint64_t)patchsize[i],
                              fbits(dispmax[i]), (uint64_t)(uintptr_t)(dmap ? dmap[i] : nullptr),
                              (uint64_t)(uintptr_t)(planes_left ? planes_left[i] : nullptr),
                              (uint64_t)(uintptr_t)(planes_right ? planes_right[i] : nullptr)};
        key.insert(key.end(), v, v + 11);
    }
    rc = run_graph(h, h->keyb, h->execb, key, st, body);
    h->profiling = saved;
    return rc;
}

// ---- per-kernel entry points ------------------------------------------------------------

int pm_k_prep(const uint8_t* img, int W, int H, size_t stride, int r, int fused, float* bw, float* grad, float* dt,
              void* stream)
{
    int rc = check_shape(nullptr, W, H, r);
    if (rc) return rc;
    if (!img || stride < (size_t)W * 4 || stride % 4) return fail(nullptr, PM_EINVAL_ARG, "bad image");
    launch_prep(img, stride, W, H, r, fused, (float4*)bw, (float4*)grad, (float4*)dt, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_init(float* out, const float* bw1, const float* bw2, const float* g1, const float* g2, int W, int H, int r,
              float dmax, int lr, const float* initdisp, const float* initnormal, int fused, void* stream)
{
    int rc = check_shape(nullptr, W, H, r);
    if (rc) return rc;
    if (!out || !bw1 || !bw2 || !g1 || !g2 || (initdisp && !initnormal)) return fail(nullptr, PM_EINVAL_ARG, "null argument");
    TexPair tp;
    if ((rc = tp.make(bw1, g1, bw2, g2, W, H, S(stream)))) return rc;
    const ViewData V = tp.view(W, H, r);
    launch_init((float4*)out, V, dmax, lr, initdisp, (const float4*)initnormal, fused, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_cost(float* cost, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
              int W, int H, int r, float mincost, int fused, void* stream)
{
    int rc = check_shape(nullptr, W, H, r);
    if (rc) return rc;
    if (!cost || !planes || !bw1 || !bw2 || !g1 || !g2) return fail(nullptr, PM_EINVAL_ARG, "null argument");
    TexPair tp;
    if ((rc = tp.make(bw1, g1, bw2, g2, W, H, S(stream)))) return rc;
    const ViewData V = tp.view(W, H, r);
    launch_cost(cost, (const float4*)planes, V, mincost, fused, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_klt(float* out, const float* planes, const float* bw1, const float* bw2, const float* g1, const float* g2,
             int W, int H, int r, int fused, void* stream)
{
    int rc = check_shape(nullptr, W, H, r);
    if (rc) return rc;
    if (!out || !planes || !bw1 || !bw2 || !g1 || !g2) return fail(nullptr, PM_EINVAL_ARG, "null argument");
    TexPair tp;
    if ((rc = tp.make(bw1, g1, bw2, g2, W, H, S(stream)))) return rc;
    const ViewData V = tp.view(W, H, r);
    launch_klt((float4*)out, (const float4*)planes, V, fused, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_propagate(float* out, const float* old, const float* bw1, const float* bw2, const float* g1, const float* g2,
                   const float* smooth, float theta, int W, int H, int r, float dmax, int lr, int iter,
                   int32_t* vin_count, uint64_t* vin_src, const float* vin_planes, int32_t* vout_count,
                   uint64_t* vout_src, int fused, uint64_t* counters, void* stream)
{
    int rc = check_shape(nullptr, W, H, r);
    if (rc) return rc;
    if (!out || !old || !bw1 || !bw2 || !g1 || !g2 || !smooth) return fail(nullptr, PM_EINVAL_ARG, "null argument");
    if (vin_count && (!vin_src || !vin_planes)) return fail(nullptr, PM_EINVAL_ARG, "incomplete input view buffer");
    if (vout_count && !vout_src) return fail(nullptr, PM_EINVAL_ARG, "incomplete output view buffer");
    static int* d_err = nullptr;
    if (!d_err) PM_CUDA(nullptr, cudaMalloc(&d_err, sizeof(int)));
    PropParams P;
    TexPair tp;
    if ((rc = tp.make(bw1, g1, bw2, g2, W, H, S(stream)))) return rc;
    P.V = tp.view(W, H, r);
    P.out = (float4*)out;
    P.old = (const float4*)old;
    P.smooth = (const float4*)smooth;
    P.theta = theta;
    P.dmax = dmax;
    P.lr = lr;
    P.iter = iter;
    P.vin_count = vin_count;
    P.vin_src = (unsigned long long*)vin_src;
    P.vin_planes = (const float4*)vin_planes;
    P.vout_count = vout_count;
    P.vout_src = (unsigned long long*)vout_src;
    P.counters = (unsigned long long*)counters;
    P.error = d_err;
    float4* tmp = nullptr;
    PM_CUDA(nullptr, cudaMallocAsync((void**)&tmp, (size_t)W * H * 2 * sizeof(float4), S(stream)));
    P.tmp_self = tmp;
    P.tmp_nb = tmp + (size_t)W * H;
    launch_propagate(P, fused, S(stream));
    PM_CUDA(nullptr, cudaFreeAsync(tmp, S(stream)));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_normal_depth(float* out, const float* planes, int W, int H, float dispscale, int lr, void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    launch_normal_depth((float4*)out, (const float4*)planes, W, H, dispscale, lr, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

size_t pm_rof_scratch_bytes(int W, int H) { return rof_scratch_bytes(W, H); }

int pm_k_rof(float* out, const float* input, const float* dt, const float lambda[4], int iters, int W, int H,
             void* scratch, void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    if (!out || !input || !dt || !lambda || !scratch || out == input) return fail(nullptr, PM_EINVAL_ARG, "bad argument");
    if (iters < 0) return fail(nullptr, PM_EINVAL_ARG, "pm_k_rof: negative step count");
    launch_rof((float4*)out, (const float4*)input, (const float4*)dt,
               make_float4(lambda[0], lambda[1], lambda[2], lambda[3]), iters, W, H, scratch, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

// Same steps as pm_k_rof on the library's static scratch.  Nothing in the scratch has
// to start at zero: the first step takes p = q = 0 and u = input without reading it,
// and every later step reads only what the step before wrote, so the contents left by
// the previous call never reach the result.  Two calls in flight at once (two streams,
// two host threads, two handles) share the scratch and race.
int pm_k_rof_static(float* out, const float* input, const float* dt, const float lambda[4], int iters, int W, int H,
                    void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    if ((int64_t)W * H > PM_ROF_STATIC_MAX_PIXELS)
        return fail(nullptr, PM_EINVAL_SHAPE,
                    "pm_k_rof_static: " + std::to_string(W) + " x " + std::to_string(H) +
                        " pixels exceed the static scratch of PM_ROF_STATIC_MAX_PIXELS = " +
                        std::to_string(PM_ROF_STATIC_MAX_PIXELS) + "; use pm_k_rof with a caller buffer");
    if (!out || !input || !dt || !lambda || out == input) return fail(nullptr, PM_EINVAL_ARG, "bad argument");
    if (iters < 0) return fail(nullptr, PM_EINVAL_ARG, "pm_k_rof_static: negative step count");
    void* scratch = nullptr;
    rc = rof_static_scratch(S(stream), &scratch);
    if (rc) return rc;
    launch_rof((float4*)out, (const float4*)input, (const float4*)dt,
               make_float4(lambda[0], lambda[1], lambda[2], lambda[3]), iters, W, H, scratch, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_consistency(float* out, const float* left, const float* right, int W, int H, float maxdd, float maxad,
                     void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    launch_consistency((float4*)out, (const float4*)left, (const float4*)right, W, H, maxdd, maxad, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_to_disparity(float* out, const float* planes, int W, int H, float scale, int lr, void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    launch_to_disparity(out, (const float4*)planes, W, H, scale, lr, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_fill_depthmap(float* out, const float* planes, int W, int H, float scale, void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    launch_fill_depthmap(out, (const float4*)planes, W, H, scale, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_fill_normalmap(float* out, const float* planes, int W, int H, int lr, void* stream)
{
    (void)lr;
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    launch_fill_normalmap((float4*)out, (const float4*)planes, W, H, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_disparity_to_normal(float* out, const float* disp, int W, int H, void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    launch_disparity_to_normal((float4*)out, disp, W, H, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_fill_state(float* out, const float* planes, int W, int H, float dispscale, int lr, void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    if (!out || !planes || !aligned(out, 16) || !aligned(planes, 16)) return fail(nullptr, PM_EINVAL_ARG, "bad argument");
    launch_fill_state((float4*)out, (const float4*)planes, W, H, dispscale, lr, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_huber(float* out, const float* input, const float* dt, const float lambda[4], float eps, int iters, int W,
               int H, void* scratch, void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    if (!out || !input || !dt || !lambda || !scratch || out == input || iters < 0)
        return fail(nullptr, PM_EINVAL_ARG, "bad argument");
    launch_huber((float4*)out, (const float4*)input, (const float4*)dt,
                 make_float4(lambda[0], lambda[1], lambda[2], lambda[3]), eps, iters, W, H, scratch, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_prep_raw(const uint8_t* img, int W, int H, size_t stride, float alpha, float* colour, float* grad, float* dt,
                  void* stream)
{
    int rc = check_shape(nullptr, W, H, 0);
    if (rc) return rc;
    if (!img || stride < (size_t)W * 4 || stride % 4 || !aligned(img, 4)) return fail(nullptr, PM_EINVAL_ARG, "bad image");
    launch_prep(img, stride, W, H, 0, 0, (float4*)colour, (float4*)grad, (float4*)dt, S(stream), alpha, 1);
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, size_t stride, int Wi, int Hi, void* stream)
{
    int rc = check_shape(nullptr, Wi, Hi, 0);
    if (rc) return rc;
    rc = check_shape(nullptr, Wo, Ho, 0);
    if (rc) return rc;
    if (!out || !in || stride < (size_t)Wi * 4 || stride % 4 || !aligned(in, 4) || !aligned(out, 4))
        return fail(nullptr, PM_EINVAL_ARG, "bad argument");
    launch_pyrdown(out, Wo, Ho, in, stride, Wi, Hi, S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_k_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, const float mul[4],
                   void* stream)
{
    int rc = check_shape(nullptr, Wi, Hi, 0);
    if (rc) return rc;
    rc = check_shape(nullptr, Wo, Ho, 0);
    if (rc) return rc;
    const size_t al = channels == 4 ? 16 : 4;
    if (!out || !in || !mul || (channels != 1 && channels != 4) || !aligned(in, al) || !aligned(out, al))
        return fail(nullptr, PM_EINVAL_ARG, "bad argument");
    launch_pyrup_mul(out, Wo, Ho, in, Wi, Hi, channels, make_float4(mul[0], mul[1], mul[2], mul[3]), S(stream));
    PM_CUDA(nullptr, cudaGetLastError());
    return PM_OK;
}

int pm_pyramid_size(int n, int levels)
{
    for (int l = 1; l < levels; l++) n = pyr_next(n);
    return n;
}

// ---- host evaluation of the shared arithmetic -----------------------------------------

int pm_rng_floats(int64_t linpos, int nd, int n, float* out)
{
    if (!out || n < 0) return PM_EINVAL_ARG;
    Rng r;
    r.init_skip((int)linpos * nd);
    for (int i = 0; i < n; i++) out[i] = r.next();
    return PM_OK;
}
float pm_expf_host(float x) { return expf_(x); }
float pm_sinf_host(float x) { float s, c; sincosf_(x, &s, &c); return s; }
float pm_cosf_host(float x) { float s, c; sincosf_(x, &s, &c); return c; }
float pm_acospif_host(float x) { return acospif_(x); }
float pm_logf_host(float x) { return logf_(x); }
float pm_exit_threshold_host(float m, float b) { return exit_threshold(m, b); }

}  // extern "C"
