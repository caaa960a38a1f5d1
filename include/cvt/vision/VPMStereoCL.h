/*
 * Drop-in replacement for cvt::VPMStereoCL (cvt/vision/VPMStereoCL.h:33-65 in phheise/cvt),
 * header-only, over the C ABI of cvtpm.h (libcvtpm.so).  cvt::Image and cvt::Exception
 * come from PMHuberStereo.h.
 *
 * The class keeps the reference's constructor and method:
 *   VPMStereoCL(int patchsize, int iterations, float disparitymax);
 *   void disparitySimple(Image& output, const Image& image0, const Image& image1,
 *                        const Image* initdisparity = NULL);
 * image0 / image1 RGBA_UINT8 of one size, initdisparity GRAY_FLOAT of that size; output
 * receives the GRAY_FLOAT disparity map |x' - x| (reallocated when its size or format
 * differs; the reference writes into the caller's image).
 *
 * Differences from the reference, by design: no OpenCL context is needed; the debugging
 * block of disparitySimple (VPMStereoCL.cpp:74-81, a PNG of every iterate and a wait for a
 * key press) is absent; it changes no result.
 */
#ifndef CVT_B200_VPMSTEREOCL_H
#define CVT_B200_VPMSTEREOCL_H

#include "PMHuberStereo.h"

namespace cvt {

class VPMStereoCL {
  public:
    VPMStereoCL(int patchsize, int iterations, float disparitymax, int device = 0) : _h(nullptr)
    {
        if (pm_vpm_create(&_h, patchsize, iterations, disparitymax, device) != PM_OK)
            throw Exception(std::string("VPMStereoCL: ") + pm_vpm_last_error(NULL));
    }
    ~VPMStereoCL() { pm_vpm_destroy(_h); }
    VPMStereoCL(const VPMStereoCL&) = delete;
    VPMStereoCL& operator=(const VPMStereoCL&) = delete;

    void disparitySimple(Image& output, const Image& image0, const Image& image1, const Image* initdisparity = NULL)
    {
        if (image0.width() != image1.width() || image0.height() != image1.height() ||
            image0.format() != IFormat::RGBA_UINT8 || image1.format() != IFormat::RGBA_UINT8)
            throw Exception("VPMStereoCL: images inconsistent or incompatible format");
        const size_t w = image0.width(), h = image0.height();
        size_t s0, s1, so;
        const uint8_t* p0 = image0.map(&s0);
        const uint8_t* p1 = image1.map(&s1);
        if (s0 != s1) throw Exception("VPMStereoCL: images have different strides");
        if (output.width() != w || output.height() != h || output.format() != IFormat::GRAY_FLOAT)
            output.reallocate(w, h, IFormat::GRAY_FLOAT);
        float* po = reinterpret_cast<float*>(output.map(&so));
        std::vector<float> init;
        if (initdisparity) {
            if (initdisparity->format() != IFormat::GRAY_FLOAT || initdisparity->width() != w ||
                initdisparity->height() != h)
                throw Exception("VPMStereoCL: initial disparity has the wrong size or format");
            size_t si;
            const uint8_t* pi = initdisparity->map(&si);
            init.resize(w * h);
            for (size_t y = 0; y < h; y++)
                for (size_t x = 0; x < w; x++) init[y * w + x] = reinterpret_cast<const float*>(pi + y * si)[x];
        }
        if (pm_vpm_disparity_simple(_h, p0, p1, (int)w, (int)h, s0, po, initdisparity ? init.data() : NULL, NULL) !=
            PM_OK)
            throw Exception(std::string("VPMStereoCL: ") + pm_vpm_last_error(_h));
    }

  private:
    pm_vpm* _h;
};

}  // namespace cvt

#endif
