// A user of cvt::PMHuberStereo switching to this library: the reference's calls,
// unchanged, on a procedural pair.  Writes the disparity map of disparityMap (float32, W*H)
// to argv[1] and, given argv[2], the map of depthMap (default dscale 1 / depthmax) there;
// given argv[3], round-trips the disparity map through a .pfm file of that name; given
// argv[4], writes the map of cvt::VPMStereoCL::disparitySimple (patch 3, 4 iterations,
// range 24) there; given argv[5], writes the flow of cvt::SVPMFlowCL::flow (patch 2, range 16,
// 8 passes) there and checks that flowInit throws, as it does in the reference.
#include <cstdio>
#include <cstring>

#include "cvt/vision/PMHuberStereo.h"
#include "cvt/vision/SVPMFlowCL.h"
#include "cvt/vision/VPMStereoCL.h"

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const int W = 96, H = 64;
    cvt::Image left(W, H, cvt::IFormat::RGBA_UINT8), right(W, H, cvt::IFormat::RGBA_UINT8);
    size_t sl, sr;
    uint8_t* pl = left.map(&sl);
    uint8_t* pr = right.map(&sr);
    if (pm_scene_generate(7, W, H, 6, 2.0f, 20.0f, 0.3f, 2.0f, pl, pr, (int)sl, NULL, NULL) != PM_OK) return 3;
    try {
        cvt::PMHuberStereo pmh;
        cvt::Image dmap, normals;
        pmh.disparityMap(dmap, left, right, 4, 24.0f, 3, cvt::DISPARITY_PP_LRCHECK, &normals);
        size_t sd;
        const uint8_t* pd = dmap.map(&sd);
        FILE* f = fopen(argv[1], "wb");
        for (int y = 0; y < H; y++) fwrite(pd + y * sd, 4, W, f);
        fclose(f);
        if (argc > 3) {   // the disparity map through Image::save / Image::load (.pfm)
            dmap.save(argv[3]);
            cvt::Image back;
            back.load(argv[3]);
            size_t sb;
            const uint8_t* pb = back.map(&sb);
            for (int y = 0; y < H; y++)
                if (memcmp(pb + y * sb, pd + y * sd, 4 * W) != 0) return 5;
        }
        if (argc > 2) {
            pmh.depthMap(dmap, left, right, 4, 24.0f, 5);
            pd = dmap.map(&sd);
            f = fopen(argv[2], "wb");
            for (int y = 0; y < H; y++) fwrite(pd + y * sd, 4, W, f);
            fclose(f);
        }
        if (argc > 4) {
            cvt::VPMStereoCL vpm(3, 4, 24.0f);
            cvt::Image vd;
            vpm.disparitySimple(vd, left, right);
            pd = vd.map(&sd);
            f = fopen(argv[4], "wb");
            for (int y = 0; y < H; y++) fwrite(pd + y * sd, 4, W, f);
            fclose(f);
        }
        if (argc > 5) {
            cvt::SVPMFlowCL svpm;
            cvt::Image fl;
            svpm.flow(fl, left, right, 2, 16.0f, NULL, 8);
            pd = fl.map(&sd);
            f = fopen(argv[5], "wb");
            for (int y = 0; y < H; y++) fwrite(pd + y * sd, 8, W, f);
            fclose(f);
            try {
                svpm.flowInit(fl, left, right, fl, 2, 16.0f);
                return 6;
            } catch (const cvt::Exception&) {
            }
        }
        // inconsistent inputs throw, as in the reference (PMHuberStereo.cpp:412-414)
        cvt::Image small(W / 2, H, cvt::IFormat::RGBA_UINT8);
        try {
            pmh.disparityMap(dmap, left, small, 4, 24.0f, 3);
            return 4;
        } catch (const cvt::Exception&) {
        }
    } catch (const cvt::Exception& e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
