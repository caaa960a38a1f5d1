/*
 * cvtpm — B200 (sm_100a) PatchMatch-Huber stereo, C ABI.
 *
 * Drop-in boundary for cvt::PMHuberStereo (cvt/vision/PMHuberStereo.h:42-110
 * in phheise/cvt).  The reference exposes a C++ class whose methods run OpenCL
 * kernels and throw cvt::Exception on error; this library exposes the same
 * operations as plain C functions over host or device pointers that return a
 * status code (the C++ header include/cvt/vision/PMHuberStereo.h turns the
 * codes back into exceptions).
 *
 * Data layout (all row-major, channel fastest):
 *   image     RGBA8, `stride` bytes per row (>= 4*width)
 *   planes    float4 per pixel (a, b, c, cost): the matched column of pixel
 *             (x, y) is a*x + b*y + c (pmhstereo.cl:183-186)
 *   dmap      float per pixel; normalmap float4 per pixel (nx, ny, nz, 0)
 *   fields    bw (r, g, b, support-weight sum), grad (4 grey differences),
 *             dt (2x2 diffusion tensor), smooth (nx, ny, nz, d/dmax): float4
 *   view buffer (cross-view candidates, VIEWPROP_t of pmhstereo.cl:830-833)
 *             count int32 per pixel + source columns uint64 per pixel
 *             (lowest kept column in the low 32 bits, next in the high 32 bits,
 *             0xffffffff = empty); the candidate planes are read from the other
 *             view's plane field.  An empty buffer is count 0, columns all ones.
 *
 * Threading: one handle per host thread (or per stream); handles are
 * independent.  Every entry point is synchronous unless it takes a stream.
 */
#ifndef CVTPM_H
#define CVTPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    PM_OK = 0,
    PM_EINVAL_SHAPE = 1,   /* width/height/stride/patch size out of range; image sizes differ */
    PM_EINVAL_ARG = 2,     /* null or inconsistent argument */
    PM_ENOMEM = 3,         /* device or host allocation failed */
    PM_ECUDA = 4,          /* a CUDA call failed; pm_last_error has the text */
    PM_ETIMEOUT = 5,       /* a bounded device wait ran out */
    PM_ENOTIMPL = 6,
    PM_ENODEV = 7          /* no CUDA device */
};

/* cvt::DisparityPostProcessing (PMHuberStereo.h:36-40) */
enum { PM_PP_NONE = 0, PM_PP_LRCHECK = 1, PM_PP_LRCHECK_FILL = 2 };

/* limits: images up to 4096 columns (window coordinates stay exact in FP32
 * products), window half-width 0..32 */
enum { PM_MAX_WIDTH = 4096, PM_MAX_HEIGHT = 4096, PM_MAX_RADIUS = 32 };

typedef struct pm_options {
    int views;           /* 2: both views, as the reference (default); 1: left view only (pp must be NONE) */
    int fused;           /* 0 (default): every operation rounds separately, in the reference kernels' order
                            (bit-exact with them); 1: the window loops contract a*b+c into fma (faster,
                            results differ from the reference in the last bits and then diverge) */
    float thetamin;      /* 1e-4 (PMHuberStereo.cpp:92) */
    float maxdispdiff;   /* 1.0 px (PMHuberStereo.cpp:79) */
    float maxanglediff;  /* 5.0 degrees (PMHuberStereo.cpp:80) */
    int rof_iters;       /* 40 (PMHuberStereo.cpp:427) */
    int device;          /* CUDA device ordinal, default 0 */
    int use_graph;       /* 1 (default): run each call as a CUDA graph, captured once and replayed while the
                            call's arguments are unchanged; 0: launch eagerly */
    int levels;          /* pyramid levels, 1 (default; the reference fixes levels = 1,
                            PMHuberStereo.cpp:78) .. PM_MAX_LEVELS: with more, disparityMap's
                            coarse-to-fine loop (:83-120) over a CLPyramid of scale 0.35, each
                            level initialised from the upsampled result of the coarser one.
                            Single-pair calls only. */
} pm_options;

enum { PM_MAX_LEVELS = 8 };

typedef struct pm_handle pm_handle;

int pm_options_default(pm_options* opt);
int pm_create(pm_handle** h, const pm_options* opt);
int pm_destroy(pm_handle* h);
const char* pm_last_error(const pm_handle* h);
const char* pm_status_string(int status);

/* PMHuberStereo::disparityMap (PMHuberStereo.cpp:75-143) with host buffers.
 * patchsize is the window half-width r (the window is (2r+1)^2, pmhstereo.cl:685-687);
 * iterations is rounded up to odd as in the reference (:490).  normalmap,
 * initdisp (left-view disparity, > 0 where valid), initnormal (float4),
 * planes_left and planes_right may be NULL. */
int pm_disparity_map(pm_handle* h, const uint8_t* left, const uint8_t* right, int width, int height,
                     size_t stride, int patchsize, float dispmax, int iterations, int pp, float* dmap,
                     float* normalmap, const float* initdisp, const float* initnormal, float* planes_left,
                     float* planes_right);

/* The same with device pointers, enqueued on `stream` (cudaStream_t; NULL = legacy default stream).
 * Returns once the work is enqueued; synchronise the stream before reading the outputs. */
int pm_disparity_map_device(pm_handle* h, const uint8_t* left, const uint8_t* right, int width, int height,
                            size_t stride, int patchsize, float dispmax, int iterations, int pp, float* dmap,
                            float* normalmap, const float* initdisp, const float* initnormal, float* planes_left,
                            float* planes_right, void* stream);

/* As pm_disparity_map_device with an initial disparity for each view, as disparityMapAll takes
 * them (PMHuberStereo.cpp:406-581, :469-483; disparityMap passes the right one as NULL): the
 * right view's disparity is positive, its match in the left image at x + d.  Either may be NULL.
 * initnormal_left / initnormal_right (float4 per pixel, nullable): the views' initial normals,
 * as disparityMapAll's initnormalleft / initnormalright; where NULL they come from the
 * disparities (pmhstereo_disparity_to_normal).  For the right view, nx / nz and ny / nz are the
 * x- and y-slopes of its disparity (pmhstereo_init_disparity_normal, pmhstereo.cl:816-819).  One
 * pyramid level and both views. */
int pm_disparity_map_init2_device(pm_handle* h, const uint8_t* left, const uint8_t* right, int width, int height,
                                  size_t stride, int patchsize, float dispmax, int iterations, int pp, float* dmap,
                                  float* normalmap, const float* initdisp_left, const float* initdisp_right,
                                  const float* initnormal_left, const float* initnormal_right, float* planes_left,
                                  float* planes_right, void* stream);

/* PMHuberStereo::depthMap (PMHuberStereo.cpp:145-347), the Huber-smoothed variant: its kernels
 * read the images themselves as colour, the diffusion tensors use alpha 12, each iteration
 * smooths the gap-filled planes (pmhstereo_fill_state) with the tensor-weighted Huber model
 * (PDDHuberDiffTensor, eps 1e-4), theta follows :320-323, the iteration count is used as given
 * (not made odd), and dmap is the disparity times dscale (dscale <= 0: 1 / dispmax, :164-165).
 * Arguments otherwise as pm_disparity_map / pm_disparity_map_device; pyramid levels do not
 * apply. */
int pm_depth_map(pm_handle* h, const uint8_t* left, const uint8_t* right, int width, int height, size_t stride,
                 int patchsize, float dispmax, int iterations, float dscale, int pp, float* dmap, float* normalmap,
                 const float* initdisp, const float* initnormal, float* planes_left, float* planes_right);
int pm_depth_map_device(pm_handle* h, const uint8_t* left, const uint8_t* right, int width, int height,
                        size_t stride, int patchsize, float dispmax, int iterations, float dscale, int pp, float* dmap,
                        float* normalmap, const float* initdisp, const float* initnormal, float* planes_left,
                        float* planes_right, void* stream);

/* Window-sample counters of the last pm_disparity_map* call on this handle when
 * counting was requested with pm_set_counting(h, 1): [0] cost-window samples,
 * [1] Gauss-Newton window samples, [2] cost evaluations that entered the window,
 * [3] early exits.  Counting adds atomics; it is off by default. */
int pm_set_counting(pm_handle* h, int on);
int pm_get_counters(pm_handle* h, uint64_t counters[4]);

/* Phase timing of the last pm_disparity_map* call (CUDA events on its stream) when
 * enabled with pm_set_profiling(h, 1); the call then synchronises its stream before
 * returning.  ms[PM_PHASE_*] in milliseconds; launches[PM_PHASE_*] kernel launches. */
enum { PM_PHASE_PREP = 0, PM_PHASE_INIT = 1, PM_PHASE_PROPAGATE = 2, PM_PHASE_SMOOTH = 3, PM_PHASE_POST = 4,
       PM_PHASE_TOTAL = 5, PM_NPHASES = 6 };
int pm_set_profiling(pm_handle* h, int on);
int pm_get_phase_times(pm_handle* h, float ms[6], int launches[6]);

/* FP32 FMA throughput of `device` in TFLOP/s (2 flop per FMA), measured with a
 * kernel of independent fma chains over every SM for about `ms` milliseconds. */
int pm_measure_fp32_peak(int device, float ms, float* tflops);

/* Batched form: n independent pairs, each with its own size, patch size and
 * disparity range, enqueued on `stream` as one CUDA graph launch.  Each pair's pipeline
 * is a branch of the graph; pairs go longest-first (by W*H*window) to the least loaded of
 * up to PM_BATCH_BRANCHES concurrent branches, so small pairs fill the GPU beside large
 * ones.  The graph is captured on the first call and replayed while every argument is the
 * same.  Arrays are indexed by pair; device pointers; outputs as in
 * pm_disparity_map_device (dmap, planes_left, planes_right may be NULL, or hold NULL
 * entries).  Results equal n calls of pm_disparity_map_device.  Every pair has its own
 * workspace, kept by the handle for the next call.  Counting and phase timing apply
 * to single-pair calls only. */
enum { PM_MAX_BATCH = 4096, PM_BATCH_BRANCHES = 16 };
int pm_disparity_map_batch_device(pm_handle* h, int n, const uint8_t* const* left, const uint8_t* const* right,
                                  const int* width, const int* height, const size_t* stride,
                                  const int* patchsize, const float* dispmax, int iterations, int pp,
                                  float* const* dmap, float* const* planes_left, float* const* planes_right,
                                  void* stream);
/* the number of concurrent branches of later batched calls on this handle, 1..PM_BATCH_BRANCHES
 * (0: PM_BATCH_BRANCHES); cvt_b200.autotune picks it by timing the caller's batch */
int pm_set_batch_branches(pm_handle* h, int n);
/* How later batched calls on this handle run.  PM_BATCH_BRANCHED (the default): every pair's
 * whole pipeline is one branch, as above.  PM_BATCH_LOCKSTEP: the pairs' prep, init and
 * post-processing are graph branches, and every iteration's propagate passes and smoothing
 * stages run for ALL pairs at once as persistent launches:
 * a few CTAs per SM take tiles of any pair from one job list until it is exhausted
 * (pm_batch_jobs; tile_order 0: pairs in decreasing window work, each pair's tiles row-major;
 * 1: the pairs' tile rows interleaved, row 0 of every pair first), so one launch spans the
 * whole batch and no pair waits on a launch tail.  ctas_per_sm caps the propagate launches'
 * CTAs per SM (0: as many as fit); tile_w is the width of their tiles of 128 pixels, 32 (32 x 4,
 * the single-pair kernels' shape) or 16 (16 x 8); 0 means 32.  Results are the same bit for bit
 * under every schedule and tile shape;
 * cvt_b200.autotune picks one by timing the caller's batch.  A lockstep call uploads
 * per-pair argument tables before its launch, waiting for the handle's earlier work on
 * `stream` when they change; when the caller is capturing `stream` itself, the call runs
 * branched.  The reference runs one pair per call (PMHuberStereo.cpp:75) and has no
 * counterpart. */
enum { PM_BATCH_LOCKSTEP = 0, PM_BATCH_BRANCHED = 1 };
int pm_set_batch_schedule(pm_handle* h, int schedule, int ctas_per_sm, int tile_order, int tile_w);
/* host only: the tile job list of a lockstep batch for tiles of tile_w x tile_h pixels, as the
 * batched call builds it: jobs[2k] = the pair, jobs[2k + 1] = (tile row << 16) | tile column.
 * *njobs receives the job count; jobs may be NULL to query it, else it has room for njobs_cap
 * jobs (2 * njobs_cap entries).  Pairs in decreasing W*H*(2r+1)^2 (stable). */
int pm_batch_jobs(int n, const int* width, const int* height, const int* patchsize, int tile_w, int tile_h,
                  int tile_order, uint32_t* jobs, int njobs_cap, int* njobs);
/* the schedule a batched call uses, host only: order[] = the pairs in decreasing window work
 * W*H*(2r+1)^2 (stable), owner[i] = the branch of pair i (least loaded when the pair is
 * placed, lowest index among equals) over min(n, branches) branches */
int pm_batch_schedule(int n, int branches, const int* width, const int* height, const int* patchsize, int* order,
                      int* owner);
/* the split of a batch over `ranks` processes, one GPU each (pairs are independent: no
 * collective on the data path), host only: rank_of[i] = the rank of pair i, chosen longest
 * processing time first by the work W*H*(2r+1)^2*dispmax (pairs in decreasing work, stable,
 * each to the least loaded rank, the lowest index among equals); load[r] (nullable) = the
 * work given to rank r.  The reference runs one pair per call on one device and has no
 * counterpart (cvt/cl/OpenCL.cpp:30-45, a single global queue). */
enum { PM_MAX_RANKS = 1024 };
int pm_batch_partition(int n, int ranks, const int* width, const int* height, const int* patchsize,
                       const float* dispmax, int* rank_of, double* load);

/* ---- per-kernel entry points (device pointers, enqueued on `stream`) ----------------
 * These expose each reference kernel on injected state for parity testing. */

/* pmhstereo_bilateral_weight_to_alpha + pmhstereo_gradxy + PDDiffTensorColor(alpha 24, beta 1)
 * (pmhstereo.cl:1462-1498, :1549-1602; PDDiffTensor.cl:26-75); any output may be NULL */
int pm_k_prep(const uint8_t* img, int width, int height, size_t stride, int patchsize, int fused, float* bw,
              float* grad, float* dt, void* stream);
/* pmhstereo_init / pmhstereo_init_disparity_normal (pmhstereo.cl:755-828) */
int pm_k_init(float* out, const float* bw1, const float* bw2, const float* g1, const float* g2, int width,
              int height, int patchsize, float dispmax, int lr, const float* initdisp, const float* initnormal,
              int fused, void* stream);
/* patch_eval_census (pmhstereo.cl:661-736) at every pixel for the given planes */
int pm_k_cost(float* cost, const float* planes, const float* bw1, const float* bw2, const float* g1,
              const float* g2, int width, int height, int patchsize, float mincost, int fused, void* stream);
/* patch_census_klt2 (pmhstereo.cl:326-410), one Gauss-Newton step at every pixel */
int pm_k_klt(float* out, const float* planes, const float* bw1, const float* bw2, const float* g1,
             const float* g2, int width, int height, int patchsize, int fused, void* stream);
/* pmhstereo_propagate_view (pmhstereo.cl:880-1071).  Reads and then empties the
 * input view buffer (vin_*; candidate planes from vin_planes, the other view's
 * field); appends to the output view buffer (vout_*; must start empty).  vin
 * and vout may be NULL (no candidates / no scatter).  counters (4 x uint64) may be NULL. */
int pm_k_propagate(float* out, const float* old, const float* bw1, const float* bw2, const float* g1,
                   const float* g2, const float* smooth, float theta, int width, int height, int patchsize,
                   float dispmax, int lr, int iter, int32_t* vin_count, uint64_t* vin_src,
                   const float* vin_planes, int32_t* vout_count, uint64_t* vout_src, int fused,
                   uint64_t* counters, void* stream);
/* pmhstereo_normal_depth (pmhstereo.cl:1384-1402) */
int pm_k_normal_depth(float* out, const float* planes, int width, int height, float dispscale, int lr,
                      void* stream);
/* PDOptCL::denoiseDiffusionTensorROF_PDD (PDOptCL.cpp:1114-1168): `iters` steps of
 * PDDROFDiffTensor (PDDROFDiffTensor.cl:43-127) from u = input, p = q = 0.
 * scratch: device buffer of pm_rof_scratch_bytes(width, height) bytes; iters < 0 returns
 * PM_EINVAL_ARG. */
size_t pm_rof_scratch_bytes(int width, int height);
int pm_k_rof(float* out, const float* input, const float* dt, const float lambda[4], int iters, int width,
             int height, void* scratch, void* stream);
/* No counterpart in the reference (whose PDOptCL::denoiseDiffusionTensorROF_PDD,
 * PDOptCL.cpp:1114-1168, allocates its temporaries on every call).  pm_k_rof without
 * a scratch argument and without any allocation: the intermediates live in a
 * library-owned static device array of PM_ROF_STATIC_MAX_PIXELS pixels (28 MiB per
 * context).  For callers that cannot allocate device memory on this path: a binding
 * that only passes image pointers and has no device allocator to make a scratch
 * buffer, or a loop under a fixed device-memory budget that must not stall other
 * streams behind cudaMalloc/cudaFree.  Results equal pm_k_rof's.
 * - The first call in each CUDA context (the context current at the call) looks up
 *   the array's address in that context; make that first call before any stream
 *   capture begins.  A first call while `stream` is being captured returns
 *   PM_EINVAL_ARG with a message.  After cudaDeviceReset the next call looks it up
 *   again in the new context.
 * - width*height > PM_ROF_STATIC_MAX_PIXELS returns PM_EINVAL_SHAPE with a message;
 *   iters < 0 returns PM_EINVAL_ARG.
 * - All calls share one array: calls in flight at the same time (two streams, two
 *   host threads) race; serialise them. */
#define PM_ROF_STATIC_MAX_PIXELS 262144
int pm_k_rof_static(float* out, const float* input, const float* dt, const float lambda[4], int iters,
                    int width, int height, void* stream);
/* pmhstereo_consistency (pmhstereo.cl:1095-1129) */
int pm_k_consistency(float* out, const float* left, const float* right, int width, int height,
                     float maxdispdiff, float maxanglediff, void* stream);
/* pmhstereo_to_disparity (:1232-1257), pmhstereo_fill_depthmap (:1187-1230),
 * pmhstereo_fill_normalmap (:1259-1305), pmhstereo_disparity_to_normal (:1604-1637) */
int pm_k_to_disparity(float* out, const float* planes, int width, int height, float scale, int lr, void* stream);
int pm_k_fill_depthmap(float* out, const float* planes, int width, int height, float scale, void* stream);
int pm_k_fill_normalmap(float* out, const float* planes, int width, int height, int lr, void* stream);
int pm_k_disparity_to_normal(float* out, const float* disp, int width, int height, void* stream);
/* pmhstereo_fill_state (pmhstereo.cl:1131-1185, run by PMHuberStereo::convertFillNormalDisparity,
 * PMHuberStereo.cpp:606-614): planes -> (normal, depth * dispscale) with gaps filled from the row */
int pm_k_fill_state(float* out, const float* planes, int width, int height, float dispscale, int lr, void* stream);
/* PDOptCL::denoiseDiffusionTensorHuber_PDD (PDOptCL.cpp:1170-1226): `iters` steps of
 * PDDHuberDiffTensor (PDDHuberDiffTensor.cl:38-107) from u = input, p = q = 0.
 * scratch: device buffer of pm_rof_scratch_bytes(width, height) bytes. */
int pm_k_huber(float* out, const float* input, const float* dt, const float lambda[4], float eps, int iters,
               int width, int height, void* scratch, void* stream);
/* prep of depthMap (PMHuberStereo.cpp:184-190, :203-204): colour = the image as floats
 * (r, g, b, a), gradients, diffusion tensor with edge weight alpha (beta 1); any output may be NULL */
int pm_k_prep_raw(const uint8_t* img, int width, int height, size_t stride, float alpha, float* colour, float* grad,
                  float* dt, void* stream);
/* pyrdown (cvt/cl/kernel/pyr/pyrdown.cl, run by CLPyramid::pyrDown, cvt/cl/CLPyramid.cpp:73-78):
 * RGBA8 in_width x in_height (rows of `stride` bytes) -> RGBA8 out_width x out_height (tight
 * rows), each output texel the linear sample at (Wi/Wo (x + 0.5), Hi/Ho (y + 0.5)) */
int pm_k_pyrdown(uint8_t* out, int out_width, int out_height, const uint8_t* in, size_t stride, int in_width,
                 int in_height, void* stream);
/* pyrup_mul4f (cvt/cl/kernel/pyr/pyrupmul.cl, run by PMHuberStereo::pyrUpMul,
 * PMHuberStereo.cpp:709-721): a float image of `channels` (1 or 4) per texel, tight rows,
 * resampled the same way and multiplied by mul per component */
int pm_k_pyrup_mul(float* out, int out_width, int out_height, const float* in, int in_width, int in_height,
                   int channels, const float mul[4], void* stream);
/* width (or height) of pyramid level `levels` - 1 of an image of n columns (rows):
 * CLPyramid::update (cvt/cl/CLPyramid.cpp:51-57), each level (size_t)(n * 0.35f) */
int pm_pyramid_size(int n, int levels);

/* ---- host-side helpers ------------------------------------------------------------- */

/* MWC64X stream of RNG_init(linpos, nd) (RNG.cl:54-57): `n` RNG_float draws, computed
 * by the same code the kernels run, on the host */
int pm_rng_floats(int64_t linpos, int nd, int n, float* out);
/* the elementary functions the kernels use, evaluated on the host by the same code */
float pm_expf_host(float x);
float pm_sinf_host(float x);
float pm_cosf_host(float x);
float pm_acospif_host(float x);
float pm_logf_host(float x);
/* smallest c >= 0 with RN(c / b) >= m (the early-exit threshold of the cost loop) */
float pm_exit_threshold_host(float m, float b);

/* Procedural stereo pair: `nplanes` slanted planar patches (disparity in [dlo, dhi],
 * |nx|, |ny| <= nmax) with 4-octave value-noise texture; right = left warped by the
 * ground-truth disparity + noise of standard deviation sigma.  gt_disp (float per
 * pixel) and gt_normal (float4 per pixel) may be NULL. */
int pm_scene_generate(uint64_t seed, int width, int height, int nplanes, float dlo, float dhi, float nmax,
                      float sigma, uint8_t* left, uint8_t* right, int stride, float* gt_disp, float* gt_normal);

/* ---- images on disk (host buffers), in the formats cvt saves them in ---------------
 * PFM (plugins/isaver/PFM/PFMSaver.cpp, plugins/iloader/PFM/PFMLoader.cpp): "Pf" grey or
 * "PF" RGB, "<width> <height>", scale (negative: little endian), float rows bottom to top.
 * Saving a 4-channel image drops its alpha (as PFMSaver does); loading "PF" gives 4
 * channels with alpha 1 (as PFMLoader does).  stride in bytes.  pm_pfm_load with out NULL
 * only reads the size; capacity counts floats.
 * CVTRaw (plugins/isaver/CVTRaw/, plugins/iloader/CVTRaw/): uint32 width, height, stride
 * (bytes), IFormat id (PM_IFORMAT_*), then height rows of stride bytes.  pm_cvtraw_load with
 * out NULL only reads the header; out_stride 0 keeps the saved stride; capacity in bytes.
 * Errors: a status code, the message in pm_io_last_error(). */
enum { PM_IFORMAT_GRAY_FLOAT = 4, PM_IFORMAT_GRAYALPHA_FLOAT = 8, PM_IFORMAT_RGBA_UINT8 = 9, PM_IFORMAT_RGBA_FLOAT = 12 };
int pm_pfm_save(const char* path, const float* data, int width, int height, int channels, size_t stride);
int pm_pfm_load(const char* path, float* out, size_t capacity, int* width, int* height, int* channels);
int pm_cvtraw_save(const char* path, const void* data, int width, int height, size_t stride, int format_id);
int pm_cvtraw_load(const char* path, void* out, size_t capacity, size_t out_stride, int* width, int* height,
                   size_t* stride, int* format_id);
const char* pm_io_last_error(void);

/* ---- VPMStereoCL (cvt/vision/VPMStereoCL.h:33-65, VPMStereoCL.cpp, cvt/cl/kernel/VPMStereo.cl)
 * The one-view slanted-plane PatchMatch: states (a, b, c) with x' = a x + b y + c, van der
 * Corput candidates, eight neighbour states, three Gauss-Newton steps per iteration.
 * Images RGBA8 with `stride` bytes per row; disparities and initial disparities W*H floats;
 * states (optional) W*H float4 (a, b, c, cost).  Errors: a status code, the message in
 * pm_vpm_last_error(handle) (NULL handle: the calling thread's last handle-free error). */
typedef struct pm_vpm pm_vpm;

/* VPMStereoCL::VPMStereoCL(patchsize, iterations, disparitymax) (VPMStereoCL.cpp:36-48) on a
 * CUDA device; PM_ENODEV without one */
int pm_vpm_create(pm_vpm** out, int patchsize, int iterations, float disparitymax, int device);
/* VPMStereoCL::~VPMStereoCL (:50-52) */
int pm_vpm_destroy(pm_vpm* h);
const char* pm_vpm_last_error(const pm_vpm* h);
/* VPMStereoCL::disparitySimple(output, image0, image1, initdisparity) (:54-85), host buffers,
 * synchronous.  The reference's debugging block (:74-81: a PNG of every iterate and a wait
 * for a key press) is not reproduced; it changes no result.  initdisparity and states may be
 * NULL. */
int pm_vpm_disparity_simple(pm_vpm* h, const uint8_t* image0, const uint8_t* image1, int W, int H, size_t stride,
                            float* disparity, const float* initdisparity, float* states);
/* the same on device buffers, enqueued on `stream` (a cudaStream_t; NULL: legacy default) */
int pm_vpm_disparity_simple_device(pm_vpm* h, const uint8_t* image0, const uint8_t* image1, int W, int H,
                                   size_t stride, float* disparity, const float* initdisparity, float* states,
                                   void* stream);
/* window-tap counters of the calls made while counting is on: c[0] cost-window taps,
 * c[1] Gauss-Newton taps (for the FLOP count of the iteration kernel) */
int pm_vpm_set_counting(pm_vpm* h, int on);
int pm_vpm_get_counters(pm_vpm* h, uint64_t c[2]);

/* One reference kernel per call, device buffers, enqueued on `stream`.  c1 / c2 RGBA8 images
 * with `stride` bytes per row, g1 / g2 their gradient images (W*H float4), states W*H float4.
 *   pm_k_vpm_grad       grad_gray_xydiag (cvt/cl/kernel/gradxy.cl:60-97)
 *   pm_k_vpm_init       vpmstereo_init, or vpmstereo_init_disparity when initdisp is given
 *                       (VPMStereo.cl:260-309)
 *   pm_k_vpm_iter       vpmstereo_iter_simple (:311-361)
 *   pm_k_vpm_disparity  vpmstereo_disparity (:363-377) */
int pm_k_vpm_grad(float* out, const uint8_t* img, int W, int H, size_t stride, void* stream);
int pm_k_vpm_init(float* out, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2, int W, int H,
                  size_t stride, int r, float dmax, const float* initdisp, void* stream);
int pm_k_vpm_iter(float* out, const float* in, const uint8_t* c1, const float* g1, const uint8_t* c2, const float* g2,
                  int W, int H, size_t stride, int r, float dmax, int iter, void* stream);
int pm_k_vpm_disparity(float* out, const float* states, int W, int H, float scale, void* stream);

/* ---- SVPMFlowCL (cvt/vision/SVPMFlowCL.h, SVPMFlowCL.cpp, cvt/cl/kernel/SVPMFlow.cl) ----
 * PatchMatch optical flow with a TV pull: states (u, v, cost, 0) (pixel (x, y) of the first
 * frame moves to (x + u, y + v)), duals W*H float4 (the dual field p of the flow's TV), flow
 * W*H float2 (u, v).  Frames RGBA8 with `stride` bytes per row.  Errors: a status code, the
 * message in pm_svpm_last_error(handle) (NULL handle: the calling thread's last handle-free
 * error).
 * The reference's propagation kernel reads and writes the group buffer in one barrier
 * interval in its jump steps (SVPMFlow.cl:673-690), which OpenCL leaves undefined; here every
 * jump step reads the states of the previous step.  Its svpmflow_state_refine reads an
 * unwritten vector (:60-61), taken as zero. */
typedef struct pm_svpm pm_svpm;
enum { PM_SVPM_MAXITER = 200 };   /* MAXITER, the passes SVPMFlowCL::flow runs (SVPMFlowCL.cpp:40) */

/* SVPMFlowCL::SVPMFlowCL / ~SVPMFlowCL (SVPMFlowCL.cpp:41-56) on a CUDA device; PM_ENODEV without one */
int pm_svpm_create(pm_svpm** out, int device);
int pm_svpm_destroy(pm_svpm* h);
const char* pm_svpm_last_error(const pm_svpm* h);
/* SVPMFlowCL::flow(flow, first, second, patchsize, flowmax) (:58-89), host buffers, synchronous,
 * with `iterations` passes (PM_SVPM_MAXITER in the reference).  Its debugging block (:74-84: an
 * AEE print, a colour-coded PNG and a wait for a key press after every pass) is not reproduced;
 * it changes no result.  states and duals may be NULL. */
int pm_svpm_flow(pm_svpm* h, const uint8_t* first, const uint8_t* second, int W, int H, size_t stride, int patchsize,
                 float flowmax, int iterations, float* flow, float* states, float* duals);
/* the same on device buffers, enqueued on `stream` */
int pm_svpm_flow_device(pm_svpm* h, const uint8_t* first, const uint8_t* second, int W, int H, size_t stride,
                        int patchsize, float flowmax, int iterations, float* flow, float* states, float* duals,
                        void* stream);
/* cost-window taps of the propagation passes of the calls made while counting is on */
int pm_svpm_set_counting(pm_svpm* h, int on);
int pm_svpm_get_counters(pm_svpm* h, uint64_t c[1]);
/* One reference kernel per call, device buffers, enqueued on `stream`:
 *   pm_k_svpm_init     svpmflow_init (SVPMFlow.cl:213-233)
 *   pm_k_svpm_prop     svpmflow_prop_local_tv_admm (:574-731), pass index `iter` (1-based in flow)
 *   pm_k_svpm_to_flow  svpmflow_flow (:733-744) */
int pm_k_svpm_init(float* out, const uint8_t* first, const uint8_t* second, int W, int H, size_t stride, int r,
                   float flowmax, void* stream);
int pm_k_svpm_prop(float* out, float* pout, const float* in, const float* pin, const uint8_t* first,
                   const uint8_t* second, int W, int H, size_t stride, int r, float flowmax, int iter, void* stream);
int pm_k_svpm_to_flow(float* flow, const float* states, int W, int H, void* stream);

/* ---- learned plane proposal (cvt_b200/csrc/pm_learn.cu) -----------------------------
 * A BF16 CNN at 1 / scale of the image resolution (W4 = W / scale, H4 = H / scale, "feature
 * pixels") whose per-pixel (disparity, nx, ny) replaces the random initialisation of
 * disparityMap through its initdisparity and initnormalmap arguments
 * (pmhstereo_init_disparity_normal, pmhstereo.cl:802-828).  Input: the left and right RGB as
 * 16 BF16 channels (6 used); 8 layers of 3x3 convolutions, channels 16 -> 32 -> 32 -> 64 ->
 * 64 -> 64 -> 64 -> 32 -> 16 (3 used), dilations 1, 1, 2, 4, 8, 16, 1, 1, ReLU after the first
 * seven (pm_lpp_layer_shape).  Activations are NHWC BF16 (batch, rows, columns, channels);
 * layer l's parameters are COUT * 9 * CIN weights w[co][t][ci] (tap t = (dy + 1) * 3 + (dx + 1)
 * in units of the dilation) then COUT biases, FP32 masters with BF16 copies.  Convolutions
 * and weight gradients run on the tensor cores (tcgen05, FP32 accumulation) or, for checking,
 * on the CUDA cores (tensor_cores = 0).  `err` (device int) is set when a bounded wait inside
 * a tensor-core kernel runs out.  Errors: a status code, the message in pm_lpp_last_error().
 * All entry points enqueue on `stream`.  The reference has no learned component; this is the
 * initdisparity / initnormalmap producer north of its init kernel. */
const char* pm_lpp_last_error(void);
int pm_lpp_layers(void);
int pm_lpp_layer_shape(int layer, int* cin, int* cout, int* dilation);
/* total FP32 parameters of all layers (weights then biases per layer, layer after layer) */
size_t pm_lpp_param_count(void);
/* the network's input for a pair (RGBA8 rows of `stride` bytes): W4 * H4 * 16 BF16, channels
 * 0-5 = the first and second view's RGB block means of k / 255 minus 0.5.  right_view 0: left
 * then right; 1: the mirrored pair (right image flipped left-right first), whose output is the
 * right view's proposal */
int pm_lpp_input(const uint8_t* left, const uint8_t* right, int W, int H, size_t stride, int scale, int right_view,
                 void* out, void* stream);
/* one convolution of layer `layer` over a batch of B maps.  mode 0 (forward): + bias, ReLU, BF16
 * out (the last layer: + bias, FP32 out); mode 1 (data gradient, layer >= 1): in = the gradient
 * of the layer's output, w = the transposed, tap-mirrored weights wt[ci][8 - t][co], mask = the
 * layer's input (the previous ReLU's output), out = the gradient of the layer's input, zero
 * where mask <= 0 */
int pm_lpp_conv(int layer, int mode, int tensor_cores, const void* in, const void* w, const float* bias,
                const void* mask, void* out, int B, int H4, int W4, int* err, void* stream);
/* weight and bias gradients of layer `layer` (COUT * 9 * CIN then COUT floats) from its input x
 * and the gradient dy of its output; the tensor-core path writes one partial sum per CTA (each
 * CTA sums a fixed set of 16 x 4-pixel units) into `scratch` (pm_lpp_wgrad_scratch_floats
 * floats) and then reduces them in a fixed order (deterministic) */
size_t pm_lpp_wgrad_scratch_floats(int layer, int B, int H4, int W4);
int pm_lpp_wgrad(int layer, int tensor_cores, const void* x, const void* dy, float* scratch, float* grad, int B, int H4,
                 int W4, int* err, void* stream);
/* training target at 1 / scale resolution from plain PatchMatch's final planes of one view
 * (W * H float4 a b c cost) and of the other view: out = W4 * H4 float4 (d / scale, nx, ny,
 * valid), the means over each block's valid pixels (finite plane, 0 < d <= dmax, the other
 * view's disparity at the matched column within 1 px) of the disparity and of the normal
 * (a - 1, b, 1) / |..|, valid = 1 when at least half of the block is.  right_view: the right
 * view's planes, as seen in the mirrored pair (blocks mirrored, normal (a - 1, -b, 1) / |..|) */
int pm_lpp_target(const float* planes, const float* other, int W, int H, int scale, int right_view, float dmax,
                  float* out, void* stream);
/* L1 loss of M outputs (16 FP32 channels, d nx ny used) against M targets (float4 d nx ny valid):
 * |d - d*| + wn (|nx - nx*| + |ny - ny*|) over valid pixels; dout (M * 16 BF16) = its gradient
 * times `scale`; parts (nullable) = per-256-pixel loss sums */
int pm_lpp_loss(const float* out, const float* target, float wn, float scale, int M, void* dout, float* parts,
                void* stream);
/* full-resolution initial disparity (pixels, clamped to [0, dmax]) and, when normal is not NULL,
 * normal map (float4 nx ny nz 0) from the last layer's W4 x H4 output, bilinear; right_view: the
 * output of the mirrored pair (read mirrored, ny negated) */
int pm_lpp_upsample(const float* out4, int W4, int H4, int W, int H, int scale, int right_view, float dmax,
                    float* disp, float* normal, void* stream);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected for `step` >= 1) on n FP32 values */
int pm_lpp_adam(float* p, const float* g, float* m1, float* m2, int n, float lr, int step, void* stream);
/* BF16 copies of layer `layer`'s FP32 weights p: wmat (forward) and wt (data gradient, nullable) */
int pm_lpp_weights_bf16(int layer, const float* p, void* wmat, void* wt, void* stream);
/* the whole proposal for one view of a pair: weights = every layer's BF16 wmat back to back,
 * biases = every layer's biases back to back; disp W * H floats, normal W * H float4 (nullable);
 * workspace 256-byte aligned, pm_lpp_propose_workspace_bytes(W, H, scale) bytes */
size_t pm_lpp_propose_workspace_bytes(int W, int H, int scale);
int pm_lpp_propose_device(const void* weights, const float* biases, int scale, const uint8_t* left, const uint8_t* right,
                          int W, int H, size_t stride, int right_view, float dmax, float* disp, float* normal,
                          void* workspace, size_t ws_bytes, int* err, void* stream);

#ifdef __cplusplus
}
#endif
#endif
