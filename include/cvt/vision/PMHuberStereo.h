/*
 * Drop-in replacement for cvt::PMHuberStereo (cvt/vision/PMHuberStereo.h:36-110 in
 * phheise/cvt), header-only, over the C ABI of cvtpm.h (libcvtpm.so).
 *
 * The class keeps the reference's names and signatures (disparityMap below, and
 * depthMap(dmap, left, right, patchsize, depthmax, iterations, dscale = -1, pp, normalmap,
 * initdisparity, initnormalmap), PMHuberStereo.h:50-51):
 *   void disparityMap(Image& dmap, const Image& left, const Image& right, size_t patchsize,
 *                     float disparitymax, size_t iterations,
 *                     DisparityPostProcessing pp = DISPARITY_PP_LRCHECK, Image* normalmap = NULL,
 *                     const Image* initdisparity = NULL, const Image* initnormalmap = NULL);
 * and its error behaviour (a cvt::Exception on inconsistent inputs or a device error).
 * cvt::Image here is a minimal host image with the formats the path uses:
 * RGBA_UINT8 (inputs), GRAY_FLOAT (disparity), RGBA_FLOAT (normals), GRAYALPHA_FLOAT (flow).  As in the
 * reference, dmap and *normalmap are reallocated by the callee.
 *
 * Differences from the reference, by design: no OpenCL context (CL::init) is needed;
 * the object owns a CUDA workspace instead of 20 compiled OpenCL programs; the
 * interactive debug output of the reference (PMHuberStereo.cpp:495-529) is absent.
 */
#ifndef CVT_B200_PMHUBERSTEREO_H
#define CVT_B200_PMHUBERSTEREO_H

#include <stddef.h>
#include <stdint.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../cvtpm.h"

namespace cvt {

class Exception : public std::runtime_error {
  public:
    explicit Exception(const std::string& msg) : std::runtime_error(msg) {}
};

struct IFormat {
    enum Id { GRAY_FLOAT_ID, RGBA_UINT8_ID, RGBA_FLOAT_ID, GRAYALPHA_FLOAT_ID };
    Id id;
    size_t channels, bpc;
    static const IFormat GRAY_FLOAT;
    static const IFormat RGBA_UINT8;
    static const IFormat RGBA_FLOAT;
    static const IFormat GRAYALPHA_FLOAT;
    bool operator==(const IFormat& o) const { return id == o.id; }
    bool operator!=(const IFormat& o) const { return id != o.id; }
};
inline const IFormat IFormat::GRAY_FLOAT = {IFormat::GRAY_FLOAT_ID, 1, 4};
inline const IFormat IFormat::RGBA_UINT8 = {IFormat::RGBA_UINT8_ID, 4, 1};
inline const IFormat IFormat::RGBA_FLOAT = {IFormat::RGBA_FLOAT_ID, 4, 4};
inline const IFormat IFormat::GRAYALPHA_FLOAT = {IFormat::GRAYALPHA_FLOAT_ID, 2, 4};

/* host image, rows of `stride` bytes */
class Image {
  public:
    Image() : _w(0), _h(0), _fmt(IFormat::RGBA_UINT8), _stride(0) {}
    Image(size_t w, size_t h, const IFormat& f) : _fmt(f) { reallocate(w, h, f); }
    void reallocate(size_t w, size_t h, const IFormat& f)
    {
        _w = w;
        _h = h;
        _fmt = f;
        _stride = w * f.channels * f.bpc;
        _data.assign(_stride * h, 0);
    }
    size_t width() const { return _w; }
    size_t height() const { return _h; }
    const IFormat& format() const { return _fmt; }
    /* reference-style access: pointer to the first row and its stride in bytes */
    uint8_t* map(size_t* stride) { *stride = _stride; return _data.data(); }
    const uint8_t* map(size_t* stride) const { *stride = _stride; return _data.data(); }
    void unmap(const uint8_t*) const {}

    /* Image::save / Image::load for the formats disparity, normal and plane images are kept in,
     * chosen by extension as cvt's plugins do: ".pfm" (PFMSaver / PFMLoader: float images; an
     * RGBA image is saved without alpha and loaded with alpha 1) and ".cvtraw" (CVTRawSaver /
     * CVTRawLoader: any of the three formats, raw rows). */
    void save(const std::string& path) const
    {
        const int w = (int)_w, h = (int)_h;
        int rc;
        if (ends_with(path, ".pfm") || ends_with(path, ".PFM")) {
            if (_fmt == IFormat::RGBA_UINT8 || _fmt == IFormat::GRAYALPHA_FLOAT)
                throw Exception("PFM holds grey or RGB float images");
            rc = pm_pfm_save(path.c_str(), reinterpret_cast<const float*>(_data.data()), w, h, (int)_fmt.channels,
                             _stride);
        } else if (ends_with(path, ".cvtraw")) {
            rc = pm_cvtraw_save(path.c_str(), _data.data(), w, h, _stride, format_id(_fmt));
        } else {
            throw Exception("no saver for " + path);
        }
        if (rc != PM_OK) throw Exception(pm_io_last_error());
    }
    void load(const std::string& path)
    {
        int w = 0, h = 0, c = 0, fid = 0;
        size_t st = 0;
        if (ends_with(path, ".pfm") || ends_with(path, ".PFM")) {
            if (pm_pfm_load(path.c_str(), NULL, 0, &w, &h, &c) != PM_OK) throw Exception(pm_io_last_error());
            reallocate(w, h, c == 1 ? IFormat::GRAY_FLOAT : IFormat::RGBA_FLOAT);
            if (pm_pfm_load(path.c_str(), reinterpret_cast<float*>(_data.data()), _data.size() / 4, &w, &h, &c) != PM_OK)
                throw Exception(pm_io_last_error());
        } else if (ends_with(path, ".cvtraw")) {
            if (pm_cvtraw_load(path.c_str(), NULL, 0, 0, &w, &h, &st, &fid) != PM_OK) throw Exception(pm_io_last_error());
            if (fid == PM_IFORMAT_GRAY_FLOAT) reallocate(w, h, IFormat::GRAY_FLOAT);
            else if (fid == PM_IFORMAT_RGBA_UINT8) reallocate(w, h, IFormat::RGBA_UINT8);
            else if (fid == PM_IFORMAT_RGBA_FLOAT) reallocate(w, h, IFormat::RGBA_FLOAT);
            else if (fid == PM_IFORMAT_GRAYALPHA_FLOAT) reallocate(w, h, IFormat::GRAYALPHA_FLOAT);
            else throw Exception("CVTRaw: format not supported here");
            if (pm_cvtraw_load(path.c_str(), _data.data(), _data.size(), _stride, &w, &h, &st, &fid) != PM_OK)
                throw Exception(pm_io_last_error());
        } else {
            throw Exception("no loader for " + path);
        }
    }

  private:
    static bool ends_with(const std::string& s, const char* e)
    {
        const size_t n = strlen(e);
        return s.size() >= n && s.compare(s.size() - n, n, e) == 0;
    }
    static int format_id(const IFormat& f)
    {
        if (f == IFormat::GRAY_FLOAT) return PM_IFORMAT_GRAY_FLOAT;
        if (f == IFormat::RGBA_UINT8) return PM_IFORMAT_RGBA_UINT8;
        if (f == IFormat::GRAYALPHA_FLOAT) return PM_IFORMAT_GRAYALPHA_FLOAT;
        return PM_IFORMAT_RGBA_FLOAT;
    }
    size_t _w, _h;
    IFormat _fmt;
    size_t _stride;
    std::vector<uint8_t> _data;
};

enum DisparityPostProcessing { DISPARITY_PP_NONE, DISPARITY_PP_LRCHECK, DISPARITY_PP_LRCHECK_FILL };

class PMHuberStereo {
  public:
    // levels: pyramid levels of disparityMap's coarse-to-fine loop; the reference fixes 1
    // (PMHuberStereo.cpp:78)
    explicit PMHuberStereo(int device = 0, int levels = 1) : _h(nullptr)
    {
        pm_options o;
        pm_options_default(&o);
        o.device = device;
        o.levels = levels;
        check(pm_create(&_h, &o));
    }
    ~PMHuberStereo() { pm_destroy(_h); }
    PMHuberStereo(const PMHuberStereo&) = delete;
    PMHuberStereo& operator=(const PMHuberStereo&) = delete;

    void disparityMap(Image& dmap, const Image& left, const Image& right, size_t patchsize, float disparitymax,
                      size_t iterations, DisparityPostProcessing pp = DISPARITY_PP_LRCHECK, Image* normalmap = NULL,
                      const Image* initdisparity = NULL, const Image* initnormalmap = NULL)
    {
        if (left.width() != right.width() || left.height() != right.height() ||
            left.format() != IFormat::RGBA_UINT8 || right.format() != IFormat::RGBA_UINT8)
            throw Exception("Left/Right stereo images inconsistent or incompatible format");
        const size_t w = left.width(), h = left.height();
        size_t sl, sr, sd, sn = 0;
        const uint8_t* pl = left.map(&sl);
        const uint8_t* pr = right.map(&sr);
        if (sl != sr) throw Exception("Left/Right stereo images have different strides");
        dmap.reallocate(w, h, IFormat::GRAY_FLOAT);
        float* pd = reinterpret_cast<float*>(dmap.map(&sd));
        float* pn = NULL;
        if (normalmap) {
            normalmap->reallocate(w, h, IFormat::RGBA_FLOAT);
            pn = reinterpret_cast<float*>(normalmap->map(&sn));
        }
        std::vector<float> idisp, inorm;
        if (initdisparity) idisp = dense(*initdisparity, IFormat::GRAY_FLOAT, w, h);
        if (initnormalmap) inorm = dense(*initnormalmap, IFormat::RGBA_FLOAT, w, h);
        check(pm_disparity_map(_h, pl, pr, (int)w, (int)h, sl, (int)patchsize, disparitymax, (int)iterations, (int)pp,
                               pd, pn, initdisparity ? idisp.data() : NULL, initnormalmap ? inorm.data() : NULL, NULL,
                               NULL));
    }

    // PMHuberStereo::depthMap (PMHuberStereo.h:50-51, PMHuberStereo.cpp:145-347): dmap holds the
    // disparity times dscale (dscale <= 0: 1 / depthmax)
    void depthMap(Image& dmap, const Image& left, const Image& right, size_t patchsize, float depthmax,
                  size_t iterations, float dscale = -1.0f, DisparityPostProcessing pp = DISPARITY_PP_LRCHECK,
                  Image* normalmap = NULL, const Image* initdisparity = NULL, const Image* initnormalmap = NULL)
    {
        if (left.width() != right.width() || left.height() != right.height() ||
            left.format() != IFormat::RGBA_UINT8 || right.format() != IFormat::RGBA_UINT8)
            throw Exception("Left/Right stereo images inconsistent or incompatible memory type");
        const size_t w = left.width(), h = left.height();
        size_t sl, sr, sd, sn = 0;
        const uint8_t* pl = left.map(&sl);
        const uint8_t* pr = right.map(&sr);
        if (sl != sr) throw Exception("Left/Right stereo images have different strides");
        dmap.reallocate(w, h, IFormat::GRAY_FLOAT);
        float* pd = reinterpret_cast<float*>(dmap.map(&sd));
        float* pn = NULL;
        if (normalmap) {
            normalmap->reallocate(w, h, IFormat::RGBA_FLOAT);
            pn = reinterpret_cast<float*>(normalmap->map(&sn));
        }
        std::vector<float> idisp, inorm;
        if (initdisparity) idisp = dense(*initdisparity, IFormat::GRAY_FLOAT, w, h);
        if (initnormalmap) inorm = dense(*initnormalmap, IFormat::RGBA_FLOAT, w, h);
        check(pm_depth_map(_h, pl, pr, (int)w, (int)h, sl, (int)patchsize, depthmax, (int)iterations, dscale, (int)pp,
                           pd, pn, initdisparity ? idisp.data() : NULL, initnormalmap ? inorm.data() : NULL, NULL,
                           NULL));
    }

  private:
    void check(int status) const
    {
        if (status != PM_OK) throw Exception(std::string("PMHuberStereo: ") + pm_last_error(_h));
    }
    static std::vector<float> dense(const Image& im, const IFormat& f, size_t w, size_t h)
    {
        if (im.format() != f || im.width() != w || im.height() != h) throw Exception("initial image has the wrong size or format");
        size_t s;
        const uint8_t* p = im.map(&s);
        std::vector<float> v(w * h * f.channels);
        for (size_t y = 0; y < h; y++)
            for (size_t x = 0; x < w * f.channels; x++) v[y * w * f.channels + x] = reinterpret_cast<const float*>(p + y * s)[x];
        return v;
    }
    pm_handle* _h;
};

}  // namespace cvt

#endif
