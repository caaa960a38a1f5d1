// Procedural stereo scenes: slanted planar patches textured with value noise.
//
// The left image is a Voronoi partition of the frame into `nplanes` cells;
// cell k carries the disparity plane d_k(x, y) = d0_k + gx_k (x - cx_k) +
// gy_k (y - cy_k) and its own 4-octave value-noise texture (values 0..255).
// The plane normal (nx, ny, nz) of the PatchMatch parametrisation has
// gx = -nx/nz, gy = -ny/nz; |nx|, |ny| <= nmax, and the slopes are scaled
// down where needed so that d stays inside [dlo, dhi] over the cell.  The
// right image is the left one warped by the ground-truth disparity: right
// pixel (x, y) shows the closest surface k whose left pixel
// xl = x + d_k(xl, y) lies in cell k; texture is evaluated at the continuous
// xl, so no resampling blur is introduced.  Occluded right pixels take the
// texture of the cell under them.  Noise of standard deviation `sigma`
// (Irwin-Hall sum of 12 uniforms, close to Gaussian) is added to the right
// image.  Everything derives from integer hashes of (seed, ...), and the
// floating-point work is plain IEEE double arithmetic, so a seed gives the same
// bytes on every x86-64 host.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/cvtpm.h"

namespace {

inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
inline uint64_t hash4(uint64_t a, uint64_t b, uint64_t c, uint64_t d)
{
    return mix64(a * 0x9e3779b97f4a7c15ULL + mix64(b + 0x632be59bd9b4e019ULL * mix64(c + 0x85157af5ULL * mix64(d))));
}
inline double unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

struct Plane {
    double cx, cy, d0, gx, gy, nx, ny, nz;
    uint64_t tex;
};

/* value noise: lattice values at integer points, smoothstep interpolation */
double value_noise(uint64_t key, double u, double v)
{
    const double fu = floor(u), fv = floor(v);
    const int64_t iu = (int64_t)fu, iv = (int64_t)fv;
    double a = u - fu, b = v - fv;
    a = a * a * (3.0 - 2.0 * a);
    b = b * b * (3.0 - 2.0 * b);
    const double v00 = unit(hash4(key, (uint64_t)iu, (uint64_t)iv, 1));
    const double v10 = unit(hash4(key, (uint64_t)(iu + 1), (uint64_t)iv, 1));
    const double v01 = unit(hash4(key, (uint64_t)iu, (uint64_t)(iv + 1), 1));
    const double v11 = unit(hash4(key, (uint64_t)(iu + 1), (uint64_t)(iv + 1), 1));
    return (v00 * (1 - a) + v10 * a) * (1 - b) + (v01 * (1 - a) + v11 * a) * b;
}

/* 4 octaves, base period 24 px, amplitudes 1, 1/2, 1/4, 1/8; result in [0, 255] */
double texture(uint64_t key, int ch, double x, double y)
{
    double s = 0.0, amp = 1.0, norm = 0.0, f = 1.0 / 24.0;
    for (int o = 0; o < 4; o++) {
        s += amp * value_noise(hash4(key, (uint64_t)ch, (uint64_t)o, 7), x * f, y * f);
        norm += amp;
        amp *= 0.5;
        f *= 2.0;
    }
    return 255.0 * s / norm;
}

inline uint8_t to_u8(double v)
{
    v = floor(v + 0.5);
    return (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
}

}  // namespace

extern "C" int pm_scene_generate(uint64_t seed, int W, int H, int nplanes, float dlo, float dhi, float nmax,
                                 float sigma, uint8_t* left, uint8_t* right, int stride, float* gt_disp,
                                 float* gt_normal)
{
    if (W <= 0 || H <= 0 || nplanes <= 0 || !left || !right || stride < 4 * W || !(dhi >= dlo)) return PM_EINVAL_ARG;
    std::vector<Plane> P(nplanes);
    for (int k = 0; k < nplanes; k++) {
        Plane& p = P[k];
        p.cx = unit(hash4(seed, 11, (uint64_t)k, 0)) * W;
        p.cy = unit(hash4(seed, 12, (uint64_t)k, 0)) * H;
        p.d0 = dlo + (dhi - dlo) * unit(hash4(seed, 13, (uint64_t)k, 0));
        p.nx = nmax * (2.0 * unit(hash4(seed, 14, (uint64_t)k, 0)) - 1.0);
        p.ny = nmax * (2.0 * unit(hash4(seed, 15, (uint64_t)k, 0)) - 1.0);
        p.nz = sqrt(1.0 - p.nx * p.nx - p.ny * p.ny);
        p.tex = hash4(seed, 16, (uint64_t)k, 0);
    }
    std::vector<int> cell((size_t)W * H);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            int best = 0;
            double bd = 1e300;
            for (int k = 0; k < nplanes; k++) {
                const double dx = x - P[k].cx, dy = y - P[k].cy, d = dx * dx + dy * dy;
                if (d < bd) { bd = d; best = k; }
            }
            cell[(size_t)y * W + x] = best;
        }
    /* slopes from the normals, scaled so that the plane stays in [dlo, dhi] on its cell */
    std::vector<double> x0(nplanes, 1e300), x1(nplanes, -1e300), y0(nplanes, 1e300), y1(nplanes, -1e300);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const int k = cell[(size_t)y * W + x];
            x0[k] = std::min(x0[k], (double)x); x1[k] = std::max(x1[k], (double)x);
            y0[k] = std::min(y0[k], (double)y); y1[k] = std::max(y1[k], (double)y);
        }
    for (int k = 0; k < nplanes; k++) {
        Plane& p = P[k];
        p.gx = -p.nx / p.nz;
        p.gy = -p.ny / p.nz;
        if (x0[k] > x1[k]) continue;
        double lo = p.d0, hi = p.d0;
        const double cxs[2] = {x0[k], x1[k]}, cys[2] = {y0[k], y1[k]};
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) {
                const double d = p.d0 + p.gx * (cxs[i] - p.cx) + p.gy * (cys[j] - p.cy);
                lo = std::min(lo, d); hi = std::max(hi, d);
            }
        double s = 1.0;
        if (hi > dhi) s = std::min(s, (dhi - p.d0) / (hi - p.d0));
        if (lo < dlo) s = std::min(s, (p.d0 - dlo) / (p.d0 - lo));
        if (s < 1.0) {
            p.gx *= s; p.gy *= s;
            /* recover the normal of the flattened plane */
            const double n = sqrt(1.0 + p.gx * p.gx + p.gy * p.gy);
            p.nx = -p.gx / n; p.ny = -p.gy / n; p.nz = 1.0 / n;
        }
    }
    auto disp = [&](int k, double x, double y) { return P[k].d0 + P[k].gx * (x - P[k].cx) + P[k].gy * (y - P[k].cy); };
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            const int k = cell[(size_t)y * W + x];
            uint8_t* px = left + (size_t)y * stride + 4 * x;
            for (int c = 0; c < 3; c++) px[c] = to_u8(texture(P[k].tex, c, x, y));
            px[3] = 255;
            if (gt_disp) gt_disp[(size_t)y * W + x] = (float)disp(k, x, y);
            if (gt_normal) {
                float* n = gt_normal + 4 * ((size_t)y * W + x);
                n[0] = (float)P[k].nx; n[1] = (float)P[k].ny; n[2] = (float)P[k].nz; n[3] = 0.0f;
            }
        }
        for (int x = 0; x < W; x++) {
            int best = -1;
            double bestd = -1e300, bestxl = 0.0;
            for (int k = 0; k < nplanes; k++) {
                const Plane& p = P[k];
                if (fabs(1.0 - p.gx) < 1e-9) continue;
                const double xl = (x + p.d0 - p.gx * p.cx + p.gy * (y - p.cy)) / (1.0 - p.gx);
                const int xi = (int)floor(xl + 0.5);
                if (xi < 0 || xi >= W || cell[(size_t)y * W + xi] != k) continue;
                const double d = disp(k, xl, y);
                if (d > bestd) { bestd = d; best = k; bestxl = xl; }
            }
            if (best < 0) {
                best = cell[(size_t)y * W + x];
                bestxl = x + disp(best, x, y);
            }
            uint8_t* px = right + (size_t)y * stride + 4 * x;
            for (int c = 0; c < 3; c++) {
                double n = 0.0;
                for (int i = 0; i < 12; i++) n += unit(hash4(seed, 0x5eed0000ULL + (uint64_t)c, (uint64_t)((size_t)y * W + x), (uint64_t)i));
                px[c] = to_u8(texture(P[best].tex, c, bestxl, y) + sigma * (n - 6.0));
            }
            px[3] = 255;
        }
    }
    return PM_OK;
}
