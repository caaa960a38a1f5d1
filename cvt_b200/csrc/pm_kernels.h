// Launchers of the PatchMatch-Huber kernels (pm_kernels.cu).  All pointers are
// device pointers; every launcher only enqueues work on the given stream.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "pm_window.cuh"

namespace pm {

// Arguments of one pmhstereo_propagate_view launch (pmhstereo.cl:880-884).
// View buffer (VIEWPROP_t, :830-833): per pixel a count of appended candidates and
// the two smallest source columns appended so far (low / high 32 bits, 0xffffffff
// when absent).  Keeping the two smallest columns reproduces the sequential
// executor's append order (sources of one target share its row, and a sequential
// executor appends them in ascending column order); the candidate plane itself is
// read back from the source view's output field, which holds the same `self` the
// reference stores (:1066).
struct PropParams {
    float4* out;
    const float4* old;
    ViewData V;
    const float4* smooth;
    float theta;
    float dmax;
    int lr;
    int iter;
    int* vin_count;                 // may be null: no cross-view candidates
    unsigned long long* vin_src;
    const float4* vin_planes;       // the other view's plane field that vin refers to
    int* vout_count;                // may be null: no scatter
    unsigned long long* vout_src;
    unsigned long long* counters;   // null: not counted
    int* error;                     // incremented if a view-buffer insert gave up
    float4* tmp_self;               // per-pixel state between the three propagate kernels
    float4* tmp_nb;
    int dual;                       // the window-loop kernels run as two variants (pm_window.cuh)
};

// Batched launches over many pairs (pm_disparity_map_batch_device run in lockstep): a job is
// one tile of one pair, jobs[k] = (pair, (tile row << 16) | tile column), in schedule order.
// The kernels are persistent: a grid of a few CTAs per SM takes jobs in list order from a work
// counter (zero before the launch) until the list is exhausted.
struct JobList {
    const uint2* jobs;
    int njobs;
};

// next job of the calling CTA: one atomic per CTA, broadcast through shared memory.  The
// first barrier also orders the previous job's shared-memory reads before the next job's writes.
__device__ __forceinline__ int grab_job(int* next)
{
    __shared__ int s_job;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) s_job = atomicAdd(next, 1);
    __syncthreads();
    return s_job;
}

// propagate tile of the single-pair kernels (threads per CTA = width x height pixels)
void prop_tile_shape(int* w, int* h);
// propagate tile of the batched kernels for tile width 32 or 16 (the same threads per CTA);
// false for any other width
bool prop_batch_tile_shape(int tile_w, int* w, int* h);
// pairs per batched propagate launch: their arguments are one kernel parameter block
// (128 x 184 bytes, within the 32,764 bytes a launch may pass)
constexpr int PROP_GROUP = 128;
struct PropGroup {
    PropParams p[PROP_GROUP];
};
static_assert(sizeof(PropGroup) + 64 <= 32764, "a batched propagate launch's parameters exceed the launch limit");
// the propagate pass of a group of n <= PROP_GROUP pairs of a batch: group[k] (host memory)
// holds pair k's arguments, J the group's tiles (prop_batch_tile_shape(tile_w)) with job.x = k;
// at most ctas_per_sm CTAs per SM (0: as many as fit); next: propagate_batch_launches(counting)
// work counters, zero
void launch_propagate_batch(const PropParams* group, int n, const JobList& J, int tile_w, int ctas_per_sm, int fused,
                            int counting, int* next, cudaStream_t st);
int propagate_batch_launches(int counting);

// Per pair and view, the smoothing stage of one iteration of a batch: the normal/depth image
// of the plane field planes[sel] (k_normal_depth) and the tensor-weighted ROF steps on it
// (launch_rof), which leave the smoothing image in `out`.
struct SmoothArgs {
    float4* out;
    float4* tmp;               // normal/depth image: the ROF input
    const float4* dt;
    float4* scratch;           // rof_scratch_bytes(W, H)
    const float4* planes[2];
    float dispscale;
    int lr, W, H;
};
// tile shapes of the smoothing jobs: j8 lists 32x8 tiles (normal/depth, single ROF steps),
// j16 32x16 tiles (double ROF steps)
constexpr int SMOOTH_TW = 32, SMOOTH_TH8 = 8, SMOOTH_TH16 = 16;
// every pair's smoothing stage of one iteration; next: smooth_batch_launches(iters) counters, zero
void launch_smooth_batch(const SmoothArgs* tab, const JobList& j8, const JobList& j16, int sel, float4 lam, int iters,
                         int* next, cudaStream_t st);
int smooth_batch_launches(int iters);

// prep of disparityMapAll (bw = colour + window weight sum, tensor edge weight alpha = 24) or,
// with raw, of depthMap (bw = the image as floats, alpha = 12)
void launch_prep(const uint8_t* img, size_t stride, int W, int H, int r, int fused, float4* bw, float4* grad,
                 float4* dt, cudaStream_t st, float alpha = 24.0f, int raw = 0);
void launch_init(float4* out, const ViewData& V, float dmax, int lr, const float* initdisp, const float4* initnormal,
                 int fused, cudaStream_t st);
void launch_cost(float* cost, const float4* planes, const ViewData& V, float mincost, int fused, cudaStream_t st);
void launch_klt(float4* out, const float4* planes, const ViewData& V, int fused, cudaStream_t st);
void launch_propagate(const PropParams& P, int fused, cudaStream_t st);
// launches per window-loop kernel (init, cost, klt, each of the three propagate kernels):
// uncounted runs launch both variants (pm_window.cuh)
inline int window_kernel_launches(int fused, bool counting)
{
    (void)fused;
    return counting ? 1 : 2;
}
void launch_normal_depth(float4* out, const float4* planes, int W, int H, float dispscale, int lr, cudaStream_t st);
size_t rof_scratch_bytes(int W, int H);
// kernel launches of launch_rof / launch_huber for `iters` steps (two steps per launch)
int pd_launch_count(int iters);
void launch_huber(float4* out, const float4* input, const float4* dt, float4 lam, float eps, int iters, int W, int H,
                  void* scratch, cudaStream_t st);
void launch_fill_state(float4* out, const float4* planes, int W, int H, float dispscale, int lr, cudaStream_t st);
void launch_rof(float4* out, const float4* input, const float4* dt, float4 lam, int iters, int W, int H, void* scratch,
                cudaStream_t st);
void launch_consistency(float4* out, const float4* L, const float4* R, int W, int H, float maxdd, float maxad,
                        cudaStream_t st);
void launch_to_disparity(float* out, const float4* planes, int W, int H, float scale, int lr, cudaStream_t st);
void launch_fill_depthmap(float* out, const float4* planes, int W, int H, float scale, cudaStream_t st);
void launch_fill_normalmap(float4* out, const float4* planes, int W, int H, cudaStream_t st);
void launch_disparity_to_normal(float4* out, const float* d, int W, int H, cudaStream_t st);
// pyramid steps: RGBA8 downscale (input rows of `stride` bytes, output tight) and the
// upscale-and-multiply of a float image of 1 or 4 channels (tight rows)
void launch_pyrdown(uint8_t* out, int Wo, int Ho, const uint8_t* in, size_t stride, int Wi, int Hi, cudaStream_t st);
void launch_pyrup_mul(float* out, int Wo, int Ho, const float* in, int Wi, int Hi, int channels, float4 mul,
                      cudaStream_t st);
// the top-left Wd x Hd corner of a field of Ws columns, 1 or 4 floats per texel
void launch_crop(float* dst, int Wd, int Hd, const float* src, int Ws, int channels, cudaStream_t st);
// size of the next pyramid level: CLPyramid::update (cvt/cl/CLPyramid.cpp:51-57) multiplies
// the size_t width by the float scale 0.35f and truncates
inline int pyr_next(int n) { return (int)(size_t)((float)(size_t)n * 0.35f); }
void launch_view_clear(int* count, unsigned long long* src, size_t n, cudaStream_t st);
// texel planes of a view (pm_window.cuh) from its bw and grad fields
int tex_pitch(int W);
size_t tex_bytes(int W, int H);
inline ViewData make_view(const float4* t1, const float4* t2, int W, int H, int r)
{
    const int plane = tex_pitch(W) * H;
    return ViewData{t1, t2, W, H, r, tex_pitch(W), plane, reinterpret_cast<const int*>(t1 + (size_t)3 * plane),
                    reinterpret_cast<const int*>(t2 + (size_t)3 * plane)};
}
void launch_pack_tex(float4* tex, const float4* bw, const float4* grad, int W, int H, cudaStream_t st);
// FP32 peak probe: `iters` rounds of independent fma chains per thread
void launch_fma_peak(float* out, int iters, int blocks, int threads, cudaStream_t st);
double fma_peak_flops_per_iter();

}  // namespace pm
