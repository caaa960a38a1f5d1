// pmhstereo_propagate_view (cvt/cl/kernel/pmhstereo.cl:880-1071) on sm_100a, as three
// kernels over the same pixels:
//   k_prop_chain  the candidate chain up to the randomized refinement (:927-1028)
//   k_prop_klt    the six Gauss-Newton steps (:1034-1038)
//   k_prop_final  the evaluation of their result, the view scatter and the output (:1039-1070)
// The state between them is `self` and the Gauss-Newton result (two float4 fields).
//
// The candidate chain keeps the source's structure: the lanes of a warp evaluate their
// pixels' k-th candidates together, so that neighbouring lanes read neighbouring texels of
// both views (a per-lane schedule, where each lane moves on to its next candidate as soon as
// its window ends, measured slower: the lanes' windows then diverge in rows and planes and
// the L1 hit rate halves).
#include <cuda_runtime.h>
#include <stdint.h>

#include "pm_kernels.h"

namespace pm {

namespace {

// block shape: PM_PROP_BX consecutive pixels of a row (a warp is 32 of them, or two rows of 16
// when PM_PROP_BX = 16), PM_PROP_BY rows per block
#ifndef PM_PROP_BX
#define PM_PROP_BX 32
#endif
#ifndef PM_PROP_BY
#define PM_PROP_BY 4
#endif
constexpr int PROP_BX = PM_PROP_BX, PROP_BY = PM_PROP_BY, PROP_THREADS = PROP_BX * PROP_BY;
// resident threads per SM asked of the register allocator for each kernel (768 threads =
// 80 registers, 640 = 96; measured best at 768 for both)
#ifndef PM_CHAIN_THREADS
#define PM_CHAIN_THREADS 768
#endif
#ifndef PM_KLT_THREADS
#define PM_KLT_THREADS 768
#endif
constexpr int PM_CHAIN_BLOCKS = PM_CHAIN_THREADS / PROP_THREADS, PM_KLT_BLOCKS = PM_KLT_THREADS / PROP_THREADS;
// the batched (persistent) forms read each pair's arguments from global memory instead of the
// parameter bank, which takes registers: at 768 threads per SM they spill in the window loops,
// so they are compiled for 640 (96 registers)
#ifndef PM_BATCH_THREADS
#define PM_BATCH_THREADS 640
#endif
constexpr int PM_BATCH_BLOCKS = PM_BATCH_THREADS / PROP_THREADS;

inline dim3 grid2d(int W, int H, dim3 b) { return dim3((W + b.x - 1) / b.x, (H + b.y - 1) / b.y); }

template <bool COUNT>
__device__ __forceinline__ void flush_counters(const Counters& cnt, unsigned long long* out)
{
    if (!COUNT) return;
    unsigned long long v[4] = {cnt.eval, cnt.klt, cnt.calls, cnt.exits};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        unsigned long long s = v[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && s) atomicAdd(out + k, s);
    }
}

// keep the two smallest source columns of a view-buffer entry (see pm_kernels.h)
__device__ __forceinline__ bool view_insert(unsigned long long* slot, unsigned int x)
{
    unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(slot);
    for (int guard = 0; guard < 4096; guard++) {
        const unsigned int lo = (unsigned int)cur, hi = (unsigned int)(cur >> 32);
        unsigned long long nv;
        if (x < lo) nv = ((unsigned long long)lo << 32) | x;
        else if (x < hi) nv = ((unsigned long long)x << 32) | lo;
        else return true;
        const unsigned long long prev = atomicCAS(slot, cur, nv);
        if (prev == cur) return true;
        cur = prev;
    }
    return false;
}

// A candidate whose plane (a, b, c) equals the current one bit for bit has the current
// plane's smoothing distance d (smoothDistance reads no cost).  Evaluated without an early
// exit it returns the current cost and is taken, which changes nothing; with an exit it
// returns 1 and is taken only if 1 + theta d <= cost + theta d.  When that comparison fails,
// the candidate leaves the state as it is whatever its window gives, and is not evaluated.
__device__ __forceinline__ bool known_outcome(float4 nb, float4 self, float theta, float sd_self)
{
    return __float_as_uint(nb.x) == __float_as_uint(self.x) && __float_as_uint(nb.y) == __float_as_uint(self.y) &&
           __float_as_uint(nb.z) == __float_as_uint(self.z) && !(1.0f + theta * sd_self <= self.w + theta * sd_self);
}

// pmhstereo_propagate_view (:927-1028): candidates k = 0 (the current plane, re-evaluated,
// :939-940), 1 smooth (:968-976), 2-5 random neighbours with offsets drawn x first, in
// [-4, 5] (:982-991), 6 a random plane (:996-1002), 7-8 cross-view planes (:1007-1016),
// 9 the randomized refinement (:1021-1028).  One loop, so that the window evaluation has a
// single call site.
template <bool F, bool COUNT, bool CHK, int BX = PROP_BX, int BY = PROP_BY>
__device__ __forceinline__ void chain_tile(const PropParams& P, int bx, int by, Counters& cnt)
{
    const ViewData& V = P.V;
    const int px = bx * BX + threadIdx.x, py = by * BY + threadIdx.y;
    if (px < V.W && py < V.H) {
        const int W = V.W;
        const size_t idx = (size_t)py * W + px;
        const float cx = (float)px, cy = (float)py;
        const int lr = P.lr;
        const float theta = P.theta, dmax = P.dmax;
        float4 smooth = P.smooth[idx];
        smooth.w = clampf(smooth.w, 0.0f, 1.0f) * dmax;   // :927-928
        float4 self = P.old[idx];

        // cross-view candidates of this pixel; the entry is emptied for the next writer
        int nview = 0;
        unsigned long long vsrc = ~0ULL;
        if (P.vin_count) {
            nview = min(P.vin_count[idx], 2);
            vsrc = P.vin_src[idx];
            P.vin_count[idx] = 0;
            P.vin_src[idx] = ~0ULL;
        }

        Rng rng;
        // RNG_init(&rng, lin, ((1*1 - 1) + NUMRNDTRIES) * 3 + 2 * NUMRNDSAMPLE) (:942) expands to
        // (lin) * ((1*1 - 1) + 2) * 3 + 2 * 4 = 6 * lin + 8
        rng.init_skip((py * W + px + P.iter) * 6 + 8);

        float sd_self = 0.0f;   // smoothing distance of `self` (smoothDistance does not read the cost)
        for (int k = 0; k < 10; k++) {
            float4 nb;
            if (k == 0) {
                nb = self;
            } else if (k == 1) {
                nb = from_disparity_normal(cx, cy, smooth.w * (lr ? -1.0f : 1.0f),
                                           normalize3(make_float3(smooth.x, smooth.y, smooth.z)));
                if (!lr) nb = viewprop(nb);
            } else if (k <= 5) {
                const int ox = (int)((rng.next() - 0.5f) * 2.0f * 5.0f + 0.5f);
                const int oy = (int)((rng.next() - 0.5f) * 2.0f * 5.0f + 0.5f);
                nb = P.old[(size_t)min(max(py + oy, 0), V.H - 1) * W + min(max(px + ox, 0), W - 1)];
            } else if (k == 6) {
                nb = nd_state_init(rng, cx, cy, lr, dmax);
            } else if (k <= 8) {
                if (k - 7 >= nview) continue;
                nb = viewprop(P.vin_planes[(size_t)py * W + (k == 7 ? (unsigned int)vsrc : (unsigned int)(vsrc >> 32))]);
            } else {
                nb = nd_state_refine(rng, self, cx, cy, dmax, lr);
            }
            if (k == 0) {
                self.w = patch_eval<F, COUNT, CHK>(V, px, py, nb, 1e10f, cnt);
                sd_self = smooth_dist1(self, smooth, cx, cy, dmax, lr);
            } else {
                if (known_outcome(nb, self, theta, sd_self)) continue;
                const float sd = smooth_dist1(nb, smooth, cx, cy, dmax, lr);
                // minimalCost (:873-877)
                const float mincost = self.w + theta * sd_self - theta * sd;
                nb.w = patch_eval<F, COUNT, CHK>(V, px, py, nb, mincost, cnt);
                if (nb.w + theta * sd <= self.w + theta * sd_self) {   // :976 etc.
                    self = nb;
                    sd_self = sd;
                }
            }
        }
        P.tmp_self[idx] = self;
    }
}

template <bool F, bool COUNT, bool CHK>
__global__ void __launch_bounds__(PROP_THREADS, PM_CHAIN_BLOCKS) k_prop_chain(PropParams P)
{
    if (variant_skips<CHK>(P.V, P.dual)) return;
    Counters cnt = {0, 0, 0, 0};
    chain_tile<F, COUNT, CHK>(P, blockIdx.x, blockIdx.y, cnt);
    flush_counters<COUNT>(cnt, P.counters);
}

// Gauss-Newton plane steps (:1034-1038)
template <bool F, bool COUNT, bool CHK, int BX = PROP_BX, int BY = PROP_BY>
__device__ __forceinline__ void klt_tile(const PropParams& P, int bx, int by, Counters& cnt)
{
    const ViewData& V = P.V;
    const int px = bx * BX + threadIdx.x, py = by * BY + threadIdx.y;
    if (px < V.W && py < V.H) {
        const size_t idx = (size_t)py * V.W + px;
        float4 nb = P.tmp_self[idx];
        for (int k = 0; k < 6; k++) nb = klt2<F, COUNT, CHK>(V, px, py, nb, cnt);
        P.tmp_nb[idx] = nb;
    }
}

template <bool F, bool COUNT, bool CHK>
__global__ void __launch_bounds__(PROP_THREADS, PM_KLT_BLOCKS) k_prop_klt(PropParams P)
{
    if (variant_skips<CHK>(P.V, P.dual)) return;
    Counters cnt = {0, 0, 0, 0};
    klt_tile<F, COUNT, CHK>(P, blockIdx.x, blockIdx.y, cnt);
    flush_counters<COUNT>(cnt, P.counters);
}

// evaluation of the Gauss-Newton result (:1039-1052), view scatter (:1060-1067), output (:1070)
template <bool F, bool COUNT, bool CHK, int BX = PROP_BX, int BY = PROP_BY>
__device__ __forceinline__ void final_tile(const PropParams& P, int bx, int by, Counters& cnt)
{
    const ViewData& V = P.V;
    const int px = bx * BX + threadIdx.x, py = by * BY + threadIdx.y;
    if (px < V.W && py < V.H) {
        const int W = V.W;
        const size_t idx = (size_t)py * W + px;
        const float cx = (float)px, cy = (float)py;
        const int lr = P.lr;
        const float dmax = P.dmax, theta = P.theta;
        float4 smooth = P.smooth[idx];
        smooth.w = clampf(smooth.w, 0.0f, 1.0f) * dmax;
        float4 self = P.tmp_self[idx];
        float4 nb = P.tmp_nb[idx];
        const float2 sd = smooth_distance(nb, self, smooth, cx, cy, dmax, lr);
        if (!known_outcome(nb, self, theta, sd.y)) {
            const float mincost = self.w + theta * sd.y - theta * sd.x;
            nb.w = patch_eval<F, COUNT, CHK>(V, px, py, nb, mincost, cnt);
            if (nb.w + theta * sd.x <= self.w + theta * sd.y) self = nb;
        }

        if (P.vout_count) {
            const float sidesign = lr ? -1.0f : 1.0f;
            const float tx = transform_x(self, cx, cy);
            const int xpv = __float2int_rn(tx);           // convert_int_rte
            const int disp = (int)((tx - cx) * sidesign);  // convert_int
            if (xpv >= 0 && xpv < W && disp > 0) {
                const size_t t = (size_t)py * W + xpv;
                atomicAdd(P.vout_count + t, 1);
                if (!view_insert(P.vout_src + t, (unsigned int)px)) atomicAdd(P.error, 1);
            }
        }
        P.out[idx] = self;
    }
}

template <bool F, bool COUNT, bool CHK>
__global__ void __launch_bounds__(PROP_THREADS) k_prop_final(PropParams P)
{
    if (variant_skips<CHK>(P.V, P.dual)) return;
    Counters cnt = {0, 0, 0, 0};
    final_tile<F, COUNT, CHK>(P, blockIdx.x, blockIdx.y, cnt);
    flush_counters<COUNT>(cnt, P.counters);
}

// Batched propagate passes (a batch of pairs in lockstep): persistent CTAs take tiles of
// any pair of a group from the job list (grab_job) and run the single-pair kernels' tile
// functions on them with that pair's arguments.  The group's arguments travel as one kernel
// parameter block (read through the constant cache, as a single-pair launch reads its own),
// job.x indexing it.  Every pixel runs the same operations on the same fields as in a
// single-pair launch, so the results are the same bit for bit.
template <bool F, bool COUNT, bool CHK, int BX>
__global__ void __launch_bounds__(PROP_THREADS, PM_BATCH_BLOCKS)
    k_prop_chain_b(const __grid_constant__ PropGroup G, const uint2* __restrict__ jobs, int njobs, int* next)
{
    for (;;) {
        const int j = grab_job(next);
        if (j >= njobs) return;
        const uint2 job = jobs[j];
        const PropParams& P = G.p[job.x];
        if (variant_skips<CHK>(P.V, P.dual)) continue;
        Counters cnt = {0, 0, 0, 0};
        chain_tile<F, COUNT, CHK, BX, PROP_THREADS / BX>(P, (int)(job.y & 0xffffu), (int)(job.y >> 16), cnt);
        flush_counters<COUNT>(cnt, P.counters);
    }
}

template <bool F, bool COUNT, bool CHK, int BX>
__global__ void __launch_bounds__(PROP_THREADS, PM_BATCH_BLOCKS)
    k_prop_klt_b(const __grid_constant__ PropGroup G, const uint2* __restrict__ jobs, int njobs, int* next)
{
    for (;;) {
        const int j = grab_job(next);
        if (j >= njobs) return;
        const uint2 job = jobs[j];
        const PropParams& P = G.p[job.x];
        if (variant_skips<CHK>(P.V, P.dual)) continue;
        Counters cnt = {0, 0, 0, 0};
        klt_tile<F, COUNT, CHK, BX, PROP_THREADS / BX>(P, (int)(job.y & 0xffffu), (int)(job.y >> 16), cnt);
        flush_counters<COUNT>(cnt, P.counters);
    }
}

template <bool F, bool COUNT, bool CHK, int BX>
__global__ void __launch_bounds__(PROP_THREADS, PM_BATCH_BLOCKS)
    k_prop_final_b(const __grid_constant__ PropGroup G, const uint2* __restrict__ jobs, int njobs, int* next)
{
    for (;;) {
        const int j = grab_job(next);
        if (j >= njobs) return;
        const uint2 job = jobs[j];
        const PropParams& P = G.p[job.x];
        if (variant_skips<CHK>(P.V, P.dual)) continue;
        Counters cnt = {0, 0, 0, 0};
        final_tile<F, COUNT, CHK, BX, PROP_THREADS / BX>(P, (int)(job.y & 0xffffu), (int)(job.y >> 16), cnt);
        flush_counters<COUNT>(cnt, P.counters);
    }
}

// resident CTAs per SM of a kernel with PROP_THREADS threads (at least 1)
template <class K>
int resident_ctas(K kernel)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, PROP_THREADS, 0) != cudaSuccess) {
        cudaGetLastError();
        n = 1;
    }
    return n < 1 ? 1 : n;
}

template <bool F, bool COUNT, bool CHK, int BX>
void launch_batch_shape(const PropGroup& tab, const JobList& J, int ctas_per_sm, int sms, int* next, cudaStream_t st)
{
    const dim3 b(BX, PROP_THREADS / BX);
    auto grid = [&](int resident) {
        const int per_sm = ctas_per_sm > 0 && ctas_per_sm < resident ? ctas_per_sm : resident;
        const long long g = (long long)per_sm * sms;
        return (unsigned)(g < J.njobs ? g : J.njobs);
    };
    k_prop_chain_b<F, COUNT, CHK, BX><<<grid(resident_ctas(k_prop_chain_b<F, COUNT, CHK, BX>)), b, 0, st>>>(
        tab, J.jobs, J.njobs, next);
    k_prop_klt_b<F, COUNT, CHK, BX><<<grid(resident_ctas(k_prop_klt_b<F, COUNT, CHK, BX>)), b, 0, st>>>(
        tab, J.jobs, J.njobs, next + 1);
    k_prop_final_b<F, COUNT, CHK, BX><<<grid(resident_ctas(k_prop_final_b<F, COUNT, CHK, BX>)), b, 0, st>>>(
        tab, J.jobs, J.njobs, next + 2);
}

// the tile shapes of the batched kernels: 32 x 4 pixels (a warp = 32 pixels of a row) or
// 16 x 8 (a warp = two rows of 16)
template <bool F, bool COUNT, bool CHK>
void launch_batch_variant(const PropGroup& tab, const JobList& J, int tile_w, int ctas_per_sm, int sms, int* next,
                          cudaStream_t st)
{
    if (tile_w == 16) launch_batch_shape<F, COUNT, CHK, 16>(tab, J, ctas_per_sm, sms, next, st);
    else launch_batch_shape<F, COUNT, CHK, 32>(tab, J, ctas_per_sm, sms, next, st);
}

}  // namespace

void prop_tile_shape(int* w, int* h)
{
    *w = PROP_BX;
    *h = PROP_BY;
}

bool prop_batch_tile_shape(int tile_w, int* w, int* h)
{
    if (tile_w != 16 && tile_w != 32) return false;
    *w = tile_w;
    *h = PROP_THREADS / tile_w;
    return true;
}

int propagate_batch_launches(int counting) { return counting ? 3 : 6; }

void launch_propagate_batch(const PropParams* group, int n, const JobList& J, int tile_w, int ctas_per_sm, int fused,
                            int counting, int* next, cudaStream_t st)
{
    if (J.njobs <= 0 || n < 1 || n > PROP_GROUP) return;
    static thread_local PropGroup tab;   // 23 KB: off the stack; copied into the launch
    for (int i = 0; i < n; i++) tab.p[i] = group[i];
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
        cudaGetLastError();
        sms = 1;
    }
    // as launch_propagate: uncounted passes run both variants (each table entry has dual = 1),
    // counted ones the checked variant alone (dual = 0)
    if (counting) {
        if (fused) launch_batch_variant<true, true, true>(tab, J, tile_w, ctas_per_sm, sms, next, st);
        else launch_batch_variant<false, true, true>(tab, J, tile_w, ctas_per_sm, sms, next, st);
    } else if (fused) {
        launch_batch_variant<true, false, false>(tab, J, tile_w, ctas_per_sm, sms, next, st);
        launch_batch_variant<true, false, true>(tab, J, tile_w, ctas_per_sm, sms, next + 3, st);
    } else {
        launch_batch_variant<false, false, false>(tab, J, tile_w, ctas_per_sm, sms, next, st);
        launch_batch_variant<false, false, true>(tab, J, tile_w, ctas_per_sm, sms, next + 3, st);
    }
}

void launch_propagate(const PropParams& P, int fused, cudaStream_t st)
{
    const dim3 b(PROP_BX, PROP_BY);
    const dim3 g = grid2d(P.V.W, P.V.H, b);
    const bool count = P.counters != nullptr;
#define PM_PROP_LAUNCH(FF, CC, KK, PP)                  \
    do {                                                \
        k_prop_chain<FF, CC, KK><<<g, b, 0, st>>>(PP);  \
        k_prop_klt<FF, CC, KK><<<g, b, 0, st>>>(PP);    \
        k_prop_final<FF, CC, KK><<<g, b, 0, st>>>(PP);  \
    } while (0)
    PropParams Q = P;
    if (!count) {
        // both variants; the one that does not apply returns at once (pm_window.cuh).  Each
        // kernel of the pass finishes before the next starts, for either variant.
        Q.dual = 1;
        if (fused) {
            k_prop_chain<true, false, false><<<g, b, 0, st>>>(Q);
            k_prop_chain<true, false, true><<<g, b, 0, st>>>(Q);
            k_prop_klt<true, false, false><<<g, b, 0, st>>>(Q);
            k_prop_klt<true, false, true><<<g, b, 0, st>>>(Q);
            k_prop_final<true, false, false><<<g, b, 0, st>>>(Q);
            k_prop_final<true, false, true><<<g, b, 0, st>>>(Q);
        } else {
            k_prop_chain<false, false, false><<<g, b, 0, st>>>(Q);
            k_prop_chain<false, false, true><<<g, b, 0, st>>>(Q);
            k_prop_klt<false, false, false><<<g, b, 0, st>>>(Q);
            k_prop_klt<false, false, true><<<g, b, 0, st>>>(Q);
            k_prop_final<false, false, false><<<g, b, 0, st>>>(Q);
            k_prop_final<false, false, true><<<g, b, 0, st>>>(Q);
        }
    } else {
        Q.dual = 0;
        if (fused) PM_PROP_LAUNCH(true, true, true, Q);
        else PM_PROP_LAUNCH(false, true, true, Q);
    }
#undef PM_PROP_LAUNCH
}

}  // namespace pm
