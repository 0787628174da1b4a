// Test infrastructure (oracle): MonkeyGL's host library (core/*.cpp, built
// unmodified by oracle/Makefile) linked against these stand-ins for its CUDA
// launchers instead of core/kernel.cu.  Each stand-in records the arguments
// MonkeyGL's host code computed for the kernel and returns a zero image, so
// the camera matrices, label windows, plane frames and CPR frames produced by
// MonkeyGL's own HelloMonkey API can be read back on a machine without a GPU.
// tests/golden/make_host_golden.py drives this through the mkrh_* functions.
#include <malloc.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "AnnotationUtils.h"
#include "CuDataManager.h"
#include "DataManager.h"
#include "Defines.h"
#include "HelloMonkey.h"
#include "Methods.h"
#include "TransferFunction.h"

using namespace MonkeyGL;

namespace {

struct Capture {
    std::vector<double> vr;      // cu_render arguments, flattened
    std::vector<double> plane;   // cu_renderPlane_* arguments
    std::vector<double> cpr;     // cu_renderCPR: w, h, invertZ, then points and dirs
    int plane_type = -1;         // 0 Average, 1 MIP, 2 MinIP
};

Capture cap;

void push3(std::vector<double> &v, float3 f) {
    v.push_back(f.x);
    v.push_back(f.y);
    v.push_back(f.z);
}

}  // namespace

// Built with -DMKREF_FULL (oracle/Makefile target ref-full) the stand-ins
// below are left out and MonkeyGL's own core/kernel.cu and
// core/CuDataManager.cu provide the launchers: the same driver then runs
// MonkeyGL's complete HelloMonkey path on the GPU.
#ifndef MKREF_FULL
extern "C" void cu_copyVolumeData(short *, cudaExtent, cudaArray *&, cudaTextureObject_t &) {}
extern "C" void cu_copyMaskData(unsigned char *, cudaExtent, cudaArray *&, cudaTextureObject_t &) {}
extern "C" void cu_setTransferFunc(float *, int, cudaArray *&, cudaTextureObject_t &) {}

extern "C" void cu_render(unsigned char *pVR, int width, int height, cudaTextureObject_t, cudaExtent volumeSize,
                          cudaTextureObject_t, cudaTextureObjects, AlphaAndWWWLInfo info, float3 mls,
                          float3 sp, float3 sv, float xT, float yT, float scale, float3x3 M, bool invertZ,
                          VOI voi, RGBA bg, RenderType type) {
    std::vector<double> &v = cap.vr;
    v.clear();
    v.push_back(width);
    v.push_back(height);
    v.push_back((double)volumeSize.width);
    v.push_back((double)volumeSize.height);
    v.push_back((double)volumeSize.depth);
    push3(v, mls);
    push3(v, sp);
    push3(v, sv);
    v.push_back(xT);
    v.push_back(yT);
    v.push_back(scale);
    for (int r = 0; r < 3; ++r) push3(v, M.m[r]);
    v.push_back(invertZ ? 1 : 0);
    v.push_back(voi.left);
    v.push_back(voi.right);
    v.push_back(voi.posterior);
    v.push_back(voi.anterior);
    v.push_back(voi.head);
    v.push_back(voi.foot);
    v.push_back(bg.red);
    v.push_back(bg.green);
    v.push_back(bg.blue);
    v.push_back(bg.alpha);
    v.push_back((int)type);
    for (int l = 0; l <= MAXOBJECTCOUNT; ++l) {
        v.push_back(info.m[l].alpha);
        v.push_back(info.m[l].ww);
        v.push_back(info.m[l].wl);
    }
    memset(pVR, 0, (size_t)width * height * 3);
}

static void plane_capture(int kind, short *pData, int width, int height, cudaExtent ext, float3 sp, float3 dh,
                          float3 dv, float3 dn, float3 lt, float ps, bool inv, float half) {
    std::vector<double> &v = cap.plane;
    v.clear();
    v.push_back(width);
    v.push_back(height);
    v.push_back((double)ext.width);
    v.push_back((double)ext.height);
    v.push_back((double)ext.depth);
    push3(v, sp);
    push3(v, dh);
    push3(v, dv);
    push3(v, dn);
    push3(v, lt);
    v.push_back(ps);
    v.push_back(inv ? 1 : 0);
    v.push_back(half);
    cap.plane_type = kind;
    memset(pData, 0, (size_t)width * height * sizeof(short));
}

extern "C" void cu_renderPlane_Average(short *d, int w, int h, cudaTextureObject_t, cudaExtent e, float3 sp,
                                       float3 dh, float3 dv, float3 dn, float3 lt, float ps, bool inv,
                                       float half) {
    plane_capture(0, d, w, h, e, sp, dh, dv, dn, lt, ps, inv, half);
}
extern "C" void cu_renderPlane_MIP(short *d, int w, int h, cudaTextureObject_t, cudaExtent e, float3 sp,
                                   float3 dh, float3 dv, float3 dn, float3 lt, float ps, bool inv, float half) {
    plane_capture(1, d, w, h, e, sp, dh, dv, dn, lt, ps, inv, half);
}
extern "C" void cu_renderPlane_MinIP(short *d, int w, int h, cudaTextureObject_t, cudaExtent e, float3 sp,
                                     float3 dh, float3 dv, float3 dn, float3 lt, float ps, bool inv,
                                     float half) {
    plane_capture(2, d, w, h, e, sp, dh, dv, dn, lt, ps, inv, half);
}

extern "C" void cu_renderCPR(short *pData, int width, int height, cudaTextureObject_t, cudaExtent,
                             double *pts, double *dirs, bool invertZ) {
    std::vector<double> &v = cap.cpr;
    v.clear();
    if (!pts) return;
    v.push_back(width);
    v.push_back(height);
    v.push_back(invertZ ? 1 : 0);
    for (int i = 0; i < 3 * height; ++i) v.push_back(pts[i]);
    for (int i = 0; i < 3 * height; ++i) v.push_back(dirs[i]);
    memset(pData, 0, (size_t)width * height * sizeof(short));
}

#endif  // MKREF_FULL

// ------------------------------------------------------------------------
// Driver ABI.  HelloMonkey's constructor loads ./resources/human.stl
// (core/MarchingCube.cpp:298), so mkrh_create takes the directory that holds
// resources/ and constructs the object from there.

// Array allocations of MonkeyGL's host code in this library come zero-filled:
// the library is linked with -Bsymbolic-functions, so MonkeyGL's new[] binds
// to this definition.  MonkeyGL allocates its label volume with new[] and
// never clears it (core/VolumeInfo.cpp:96-104); recycled heap memory there
// leaves labels above 64 outside every mask, which its kernel then uses to
// index 65-entry tables.  Zero-filled, the label volume starts at zero, as
// MonkeyGL evidently assumes, whatever the process allocated before.
void *operator new[](size_t n) {
    void *p = calloc(1, n ? n : 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void operator delete[](void *p) noexcept { free(p); }
void operator delete[](void *p, size_t) noexcept { free(p); }

// mkrh_zero_heap(1) also makes allocations of 64 KiB or more come from fresh
// pages (a second line of defence for allocations not made with new[]).
extern "C" int mkrh_zero_heap(int on) {
    return on ? mallopt(M_MMAP_THRESHOLD, 64 * 1024) : 1;
}

// Largest label in MonkeyGL's stored label volume (-1 if there is none).
extern "C" int mkrh_mask_max_label(void *h);

extern "C" void *mkrh_create(const char *asset_dir) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return nullptr;
    if (asset_dir && chdir(asset_dir) != 0) return nullptr;
    HelloMonkey *h = new HelloMonkey();
    if (chdir(cwd) != 0) return h;
    return h;
}
extern "C" void mkrh_destroy(void *h) { delete static_cast<HelloMonkey *>(h); }

#define HM static_cast<HelloMonkey *>(h)

extern "C" int mkrh_set_volume(void *h, const short *vox, int w, int hh, int d) {
    std::shared_ptr<short> p(new short[(size_t)w * hh * d], std::default_delete<short[]>());
    memcpy(p.get(), vox, (size_t)w * hh * d * sizeof(short));
    return HM->SetVolumeData(p, w, hh, d) ? 1 : 0;
}
extern "C" int mkrh_add_mask(void *h, const unsigned char *m, int w, int hh, int d) {
    std::shared_ptr<unsigned char> p(new unsigned char[(size_t)w * hh * d], std::default_delete<unsigned char[]>());
    memcpy(p.get(), m, (size_t)w * hh * d);
    return HM->AddNewObjectMask(p, w, hh, d);
}
extern "C" void mkrh_set_spacing(void *h, double x, double y, double z) { HM->SetSpacing(x, y, z); }
extern "C" void mkrh_set_direction(void *h, const double *d) {
    HM->SetDirection(Direction3d(d[0], d[1], d[2]), Direction3d(d[3], d[4], d[5]), Direction3d(d[6], d[7], d[8]));
}
extern "C" void mkrh_set_background(void *h, float r, float g, float b, float a) {
    HM->SetColorBackground(RGBA(r, g, b, a));
}
extern "C" int mkrh_set_wwwl(void *h, float ww, float wl, int label) {
    return (label < 0 ? HM->SetVRWWWL(ww, wl) : HM->SetVRWWWL(ww, wl, (unsigned char)label)) ? 1 : 0;
}
extern "C" int mkrh_set_alpha(void *h, float a, int label) {
    return (label < 0 ? HM->SetObjectAlpha(a) : HM->SetObjectAlpha(a, (unsigned char)label)) ? 1 : 0;
}
extern "C" void mkrh_set_render_type(void *h, int t) { HM->SetRenderType((RenderType)t); }
extern "C" void mkrh_orientation(void *h, int which) {
    switch (which) {
        case 0: HM->Anterior(); break;
        case 1: HM->Posterior(); break;
        case 2: HM->Left(); break;
        case 3: HM->Right(); break;
        case 4: HM->Head(); break;
        default: HM->Foot(); break;
    }
}
extern "C" void mkrh_rotate(void *h, float fx, float fy) { HM->Rotate(fx, fy); }
extern "C" float mkrh_zoom(void *h, float r) { return HM->Zoom(r); }
extern "C" void mkrh_pan(void *h, float x, float y) { HM->Pan(x, y); }
extern "C" int mkrh_set_vr_size(void *h, int w, int hh) { return HM->SetVRSize(w, hh) ? 1 : 0; }
extern "C" void mkrh_set_mpr_type(void *h, int t) { HM->SetMPRType((MPRType)t); }
extern "C" void mkrh_set_thickness(void *h, double v, int plane) { HM->SetThickness(v, (PlaneType)plane); }
extern "C" void mkrh_update_thickness(void *h, double v) { HM->UpdateThickness(v); }
extern "C" void mkrh_browse(void *h, float d, int plane) { HM->Browse(d, (PlaneType)plane); }
extern "C" void mkrh_pan_crosshair(void *h, float x, float y, int plane) { HM->PanCrossHair(x, y, (PlaneType)plane); }
extern "C" void mkrh_rotate_crosshair(void *h, float a, int plane) { HM->RotateCrossHair(a, (PlaneType)plane); }
extern "C" void mkrh_set_plane_index(void *h, int i, int plane) { HM->SetPlaneIndex(i, (PlaneType)plane); }
extern "C" int mkrh_get_plane_index(void *h, int plane) { return HM->GetPlaneIndex((PlaneType)plane); }
extern "C" int mkrh_get_plane_number(void *h, int plane) { return HM->GetPlaneNumber((PlaneType)plane); }
extern "C" void mkrh_reset(void *h) { HM->Reset(); }
extern "C" int mkrh_set_cpr_line_voxel(void *h, const double *pts, int n) {
    std::vector<Point3d> v;
    for (int i = 0; i < n; ++i) v.push_back(Point3d(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
    return HM->SetCPRLineVoxel(v) ? 1 : 0;
}
extern "C" int mkrh_rotate_cpr(void *h, float a, int plane) { return HM->RotateCPR(a, (PlaneType)plane) ? 1 : 0; }
extern "C" int mkrh_crosshair(void *h, int plane, double *xy) {
    double x = 0, y = 0;
    bool ok = HM->GetCrossHairPoint(x, y, (PlaneType)plane);
    xy[0] = x;
    xy[1] = y;
    return ok ? 1 : 0;
}
extern "C" int mkrh_direction3d(void *h, int plane, double *hv) {
    Direction3d a, b;
    bool ok = HM->GetDirection3D(a, b, (PlaneType)plane);
    hv[0] = a.x(); hv[1] = a.y(); hv[2] = a.z();
    hv[3] = b.x(); hv[4] = b.y(); hv[5] = b.z();
    return ok ? 1 : 0;
}
extern "C" double mkrh_pixel_spacing(void *h, int plane) { return HM->GetPixelSpacing((PlaneType)plane); }
extern "C" int mkrh_vr_size(void *h, int *wh) {
    std::shared_ptr<unsigned char> p;
    (void)p;
    int w = 0, hh = 0;
    HM->GetPlaneMaxSize(w, hh, PlaneVR);
    wh[0] = w;
    wh[1] = hh;
    return 1;
}

// Runs GetVRData and returns the number of doubles captured from cu_render.
extern "C" int mkrh_get_vr(void *h, int w, int hh) {
    std::shared_ptr<unsigned char> p;
    cap.vr.clear();
    HM->GetVRData(p, w, hh);
    return (int)cap.vr.size();
}
// Runs GetPlaneData and returns the number of doubles captured (planes or CPR).
extern "C" int mkrh_get_plane(void *h, int plane, int *wh) {
    std::shared_ptr<short> p;
    int w = 0, hh = 0;
    cap.plane.clear();
    cap.cpr.clear();
    bool ok = HM->GetPlaneData(p, w, hh, (PlaneType)plane);
    wh[0] = w;
    wh[1] = hh;
    if (!ok) return 0;
    return (int)(plane >= (int)PlaneStretchedCPR ? cap.cpr.size() : cap.plane.size());
}
// SetTransferFunc(rgb points[, alpha points], label); label < 0 = active label.
extern "C" int mkrh_set_tf(void *h, const int *rgb_pos, const float *rgba, int n_rgb, const int *a_pos,
                           const float *alpha, int n_alpha, int label) {
    std::map<int, RGBA> rgb;
    for (int i = 0; i < n_rgb; ++i)
        rgb[rgb_pos[i]] = RGBA(rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]);
    std::map<int, float> al;
    for (int i = 0; i < n_alpha; ++i) al[a_pos[i]] = alpha[i];
    bool ok;
    if (n_alpha > 0)
        ok = label < 0 ? HM->SetTransferFunc(rgb, al) : HM->SetTransferFunc(rgb, al, (unsigned char)label);
    else
        ok = label < 0 ? HM->SetTransferFunc(rgb) : HM->SetTransferFunc(rgb, (unsigned char)label);
    return ok ? 1 : 0;
}

// GetVRData into `out` (capacity `cap_bytes`); wh receives the image size.
extern "C" int mkrh_vr_image(void *h, unsigned char *out, long long cap_bytes, int *wh) {
    std::shared_ptr<unsigned char> p;
    int w = 0, hh = 0;
    HM->GetPlaneMaxSize(w, hh, PlaneVR);
    wh[0] = w;
    wh[1] = hh;
    if (!HM->GetVRData(p, w, hh) || !p || (long long)w * hh * 3 > cap_bytes) return 0;
    memcpy(out, p.get(), (size_t)w * hh * 3);
    return 1;
}

// GetPlaneData into `out` (capacity in values); wh receives the plane size.
extern "C" int mkrh_plane_image(void *h, int plane, short *out, long long cap_values, int *wh) {
    std::shared_ptr<short> p;
    int w = 0, hh = 0;
    bool ok = HM->GetPlaneData(p, w, hh, (PlaneType)plane);
    wh[0] = w;
    wh[1] = hh;
    if (!ok || !p || (long long)w * hh > cap_values) return 0;
    memcpy(out, p.get(), (size_t)w * hh * sizeof(short));
    return 1;
}

extern "C" int mkrh_mask_max_label(void *h) {
    int w = 0, hh = 0, d = 0;
    HM->GetVolumeData(w, hh, d);
    // HelloMonkey exposes no mask accessor; IRender's GetMaskData is reached
    // through the DataManager that every instance shares
    std::shared_ptr<unsigned char> m = DataManager::Instance()->GetMaskData();
    if (!m) return -1;
    int mx = 0;
    for (size_t i = 0; i < (size_t)w * hh * d; ++i) mx = m.get()[i] > mx ? m.get()[i] : mx;
    return mx;
}

extern "C" int mkrh_plane_kind(void) { return cap.plane_type; }
extern "C" void mkrh_copy_vr(double *out) { memcpy(out, cap.vr.data(), cap.vr.size() * sizeof(double)); }
extern "C" void mkrh_copy_plane(double *out) { memcpy(out, cap.plane.data(), cap.plane.size() * sizeof(double)); }
extern "C" void mkrh_copy_cpr(double *out) { memcpy(out, cap.cpr.data(), cap.cpr.size() * sizeof(double)); }

// TransferFunction::GetTransferFunction (core/TransferFunction.cpp:38-140) on
// explicit control points; returns the LUT length (0 on failure).
extern "C" int mkrh_tf_lut(const int *rgb_pos, const float *rgba, int n_rgb, const int *a_pos,
                           const float *alpha, int n_alpha, float *out_rgba, int max_len) {
    std::map<int, RGBA> rgb;
    for (int i = 0; i < n_rgb; ++i)
        rgb[rgb_pos[i]] = RGBA(rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]);
    std::map<int, float> al;
    for (int i = 0; i < n_alpha; ++i) al[a_pos[i]] = alpha[i];
    TransferFunction tf;
    tf.SetControlPoints(rgb, al);
    std::shared_ptr<RGBA> buf;
    int n = 0;
    if (!tf.GetTransferFunction(buf, n)) return 0;
    if (n > max_len) return -n;
    memcpy(out_rgba, buf.get(), (size_t)n * sizeof(RGBA));
    return n;
}

// RenderInfo's rotate matrix (the one VRImageLayer::GetMeshPoints turns the
// orientation mesh with), row-major.
extern "C" void mkrh_rotate_matrix(float *out) {
    memcpy(out, DataManager::Instance()->GetRenderInfo().GetRotateMatrix(), 9 * sizeof(float));
}

// Methods::DrawLineInImage24Bit on an RGB image.
extern "C" void mkrh_draw_line(unsigned char *img, int w, int h, float x0, float y0, float x1, float y1, int lw,
                               float r, float g, float b) {
    Methods::DrawLineInImage24Bit(img, w, h, x0, y0, x1, y1, lw, RGBA(r, g, b));
}

// HelloMonkey::AddAnnotation / RemoveAllAnnotations (core/HelloMonkey.h:121-123).
extern "C" int mkrh_add_annotation(void *h, const char *txt, int x, int y, int font_size, int format, float r,
                                   float g, float b, float a) {
    return HM->AddAnnotation(PlaneVR, std::string(txt), x, y, (FontSize)font_size, (AnnotationFormat)format,
                             RGBA(r, g, b, a)) ? 1 : 0;
}
extern "C" int mkrh_remove_annotations(void *h) { return HM->RemoveAllAnnotations() ? 1 : 0; }

// MonkeyGL's text rendering (core/AnnotationUtils.cpp:419-458) on an RGB image.
extern "C" int mkrh_textout(const char *txt, int x, int y, int font_size, int format, float r, float g, float b,
                            unsigned char *img, int w, int hh) {
    static bool init = AnnotationUtils::Init();
    (void)init;
    AnnotationUtils::SetFontSize((FontSize)font_size);
    return AnnotationUtils::Textout2Image(std::string(txt), x, y, (AnnotationFormat)format, RGBA(r, g, b), img, w,
                                          hh) ? 1 : 0;
}

// The glyph mask MonkeyGL draws character `c` with at `font_size`: its size
// from AnnotationUtils::GetSize and its mask values read back from a
// Textout2Image call in white on black (pixel = mask * 1.0 where mask > 0).
// Returns 1 with wh = (width, height) and the mask in out (row-major), 0 for
// a character MonkeyGL has no glyph for.
extern "C" int mkrh_glyph(const char *c, int font_size, unsigned char *out, int cap, int *wh) {
    static bool init = AnnotationUtils::Init();
    (void)init;
    AnnotationUtils::SetFontSize((FontSize)font_size);
    int w = -1, hh = -1;
    AnnotationUtils::GetSize(std::string(c), w, hh);
    wh[0] = w;
    wh[1] = hh;
    if (w <= 0 || hh <= 0 || w * hh > cap) return 0;
    const int cw = w < 16 ? 16 : w, ch = hh < 16 ? 16 : hh;
    std::vector<unsigned char> img((size_t)cw * ch * 3, 0);
    if (!AnnotationUtils::Textout2Image(std::string(c), 0, 0, AnnotationFormatLeft, RGBA(1.0f, 1.0f, 1.0f),
                                        img.data(), cw, ch))
        return 0;
    for (int yy = 0; yy < hh; ++yy)
        for (int xx = 0; xx < w; ++xx) out[yy * w + xx] = img[((size_t)yy * cw + xx) * 3];
    return 1;
}
