/*
 * Drop-in replacement for cvt::SVPMFlowCL (cvt/vision/SVPMFlowCL.h in phheise/cvt),
 * header-only, over the C ABI of cvtpm.h (libcvtpm.so).  cvt::Image and cvt::Exception come
 * from PMHuberStereo.h.
 *
 *   SVPMFlowCL();
 *   void flow(Image& flow, const Image& first, const Image& second, int patchsize, float flowmax,
 *             Image* gtflow = NULL);
 * first / second RGBA_UINT8 of one size; flow is reallocated to GRAYALPHA_FLOAT (u, v), as in
 * the reference (SVPMFlowCL.cpp:215).  The reference runs MAXITER = 200 passes; `iterations` (an extra,
 * defaulted argument) makes that a parameter.  gtflow only fed the reference's debugging
 * print and is ignored.
 *
 * flowInit and flowPyramid are not offered: in the reference they bind 7 arguments to the
 * 9-argument propagation kernel (SVPMFlowCL.cpp:187-197 against SVPMFlow.cl:574-577), so
 * CLKernel::setArg throws on their first pass; here they throw at once with that reason.
 */
#ifndef CVT_B200_SVPMFLOWCL_H
#define CVT_B200_SVPMFLOWCL_H

#include "PMHuberStereo.h"

namespace cvt {

class SVPMFlowCL {
  public:
    explicit SVPMFlowCL(int device = 0) : _h(nullptr)
    {
        if (pm_svpm_create(&_h, device) != PM_OK) throw Exception(std::string("SVPMFlowCL: ") + pm_svpm_last_error(NULL));
    }
    ~SVPMFlowCL() { pm_svpm_destroy(_h); }
    SVPMFlowCL(const SVPMFlowCL&) = delete;
    SVPMFlowCL& operator=(const SVPMFlowCL&) = delete;

    void flow(Image& flow, const Image& first, const Image& second, int patchsize, float flowmax, Image* gtflow = NULL,
              int iterations = PM_SVPM_MAXITER)
    {
        (void)gtflow;
        if (first.width() != second.width() || first.height() != second.height() ||
            first.format() != IFormat::RGBA_UINT8 || second.format() != IFormat::RGBA_UINT8)
            throw Exception("SVPMFlowCL: frames inconsistent or incompatible format");
        const size_t w = first.width(), h = first.height();
        size_t s0, s1, sf;
        const uint8_t* p0 = first.map(&s0);
        const uint8_t* p1 = second.map(&s1);
        if (s0 != s1) throw Exception("SVPMFlowCL: frames have different strides");
        flow.reallocate(w, h, IFormat::GRAYALPHA_FLOAT);
        float* pf = reinterpret_cast<float*>(flow.map(&sf));
        if (pm_svpm_flow(_h, p0, p1, (int)w, (int)h, s0, patchsize, flowmax, iterations, pf, NULL, NULL) != PM_OK)
            throw Exception(std::string("SVPMFlowCL: ") + pm_svpm_last_error(_h));
    }

    void flowInit(Image&, const Image&, const Image&, const Image&, int, float)
    {
        throw Exception("SVPMFlowCL::flowInit: the reference binds 7 arguments to the 9-argument propagation kernel "
                        "(SVPMFlowCL.cpp:187-197) and fails in CLKernel::setArg");
    }
    void flowPyramid(Image&, const Image&, const Image&, int, float, Image* = NULL)
    {
        throw Exception("SVPMFlowCL::flowPyramid: runs flowInit on its finer levels, which fails in the reference "
                        "(SVPMFlowCL.cpp:149, :187-197)");
    }

  private:
    pm_svpm* _h;
};

}  // namespace cvt

#endif
