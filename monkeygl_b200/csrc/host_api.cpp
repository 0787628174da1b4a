// host_api.cpp -- MonkeyGL's public C++ API (HelloMonkey, IRender, Render)
// over the per-instance engine and the C ABI.  Method by method this follows
// core/HelloMonkey.cpp, core/IRender.cpp and core/Render.cpp; the outputs of
// GetVRData / GetPlaneData come from the sm_100a kernels.  PNG output is
// written by host_encode.cpp (zlib in parallel bands; MonkeyGL uses fpng):
// the decoded pixels are the same, the compressed bytes are not.
#include <zlib.h>

#include <cstdio>
#include <cstring>

#include "../../include/monkeygl/HelloMonkey.h"
#include "../../include/monkeygl/IRender.h"
#include "host_encode.h"
#include "host_engine.h"

namespace MonkeyGL {

namespace {

LogLevel g_log_level = LogLevelWarn;

}  // namespace

// ---------------------------------------------------------------------------
// IRender: forwards to this instance's engine (core/IRender.cpp)

IRender::IRender() : m_engine(std::make_shared<detail::Engine>()) {}
IRender::~IRender() {}

bool IRender::SetVolumeData(std::shared_ptr<short> p, int w, int h, int d) { return m_engine->SetVolumeData(p, w, h, d); }
unsigned char IRender::AddNewObjectMask(std::shared_ptr<unsigned char> p, int w, int h, int d) {
    return m_engine->AddNewObjectMask(p, w, h, d);
}
// File ingest needs a volume reader (MonkeyGL uses ITK); like MonkeyGL's
// failed read this returns (unsigned char)-1.
unsigned char IRender::AddObjectMaskFile(const char *) { return (unsigned char)-1; }
bool IRender::UpdateObjectMask(std::shared_ptr<unsigned char> p, int w, int h, int d, const unsigned char &l) {
    return m_engine->UpdateObjectMask(p, w, h, d, l);
}
void IRender::LoadVolumeFile(const char *szFile) {
    if (g_log_level <= LogLevelError)
        std::fprintf(stderr, "[MonkeyGL] LoadVolumeFile(%s): file ingest is not available; use SetVolumeData\n",
                     szFile ? szFile : "");
}
void IRender::SetDirection(Direction3d x, Direction3d y, Direction3d z) { m_engine->SetDirection(x, y, z); }
void IRender::SetSpacing(double x, double y, double z) { m_engine->SetSpacing(x, y, z); }
void IRender::SetOrigin(Point3d pt) { m_engine->SetOrigin(pt); }
void IRender::Reset() { m_engine->Reset(); }
void IRender::SetColorBackground(RGBA c) { m_engine->SetColorBackground(c); }
void IRender::Browse(float d, PlaneType t) { m_engine->Browse(d, t); }
void IRender::SetPlaneIndex(int i, PlaneType t) { m_engine->SetPlaneIndex(i, t); }
void IRender::PanCrossHair(float x, float y, PlaneType t) { m_engine->PanCrossHair(x, y, t); }
void IRender::RotateCrossHair(float a, PlaneType t) { m_engine->RotateCrossHair(a, t); }
void IRender::UpdateThickness(double v) { m_engine->UpdateThickness(v); }
void IRender::SetThickness(double v, PlaneType t) { m_engine->SetThickness(v, t); }
double IRender::GetThickness(PlaneType t) { return m_engine->Thickness(t); }
void IRender::SetMPRType(MPRType t) { m_engine->SetMPRType(t); }
bool IRender::TransferVoxel2ImageInVR(float &fx, float &fy, int w, int h, Point3d v) {
    return m_engine->TransferVoxel2ImageInVR(fx, fy, w, h, v);
}
std::shared_ptr<short> IRender::GetVolumeData(int &w, int &h, int &d) { return m_engine->GetVolumeData(w, h, d); }
std::shared_ptr<unsigned char> IRender::GetMaskData() { return m_engine->GetMaskData(); }
bool IRender::GetPlaneMaxSize(int &w, int &h, const PlaneType &t) { return m_engine->PlaneMaxSize(w, h, t); }
bool IRender::GetPlaneData(std::shared_ptr<short> &, int &, int &, const PlaneType &) { return false; }
bool IRender::TransferImage2Voxel(double &x, double &y, double &z, double xi, double yi, PlaneType t) {
    Point3d v;
    if (!m_engine->TransferImage2Voxel(v, xi, yi, t)) return false;
    x = v[0];
    y = v[1];
    z = v[2];
    return true;
}
bool IRender::GetCrossHairPoint3D(Point3d &pt) {
    pt = m_engine->CrossHair();
    return true;
}
bool IRender::GetDirection(Direction2d &h, Direction2d &v, const PlaneType &t) { return m_engine->Direction2D(h, v, t); }
bool IRender::GetDirection3D(Direction3d &h, Direction3d &v, const PlaneType &t) { return m_engine->Direction3D(h, v, t); }
bool IRender::GetBatchDirection3D(Direction3d &h, Direction3d &v, double a, const PlaneType &t) {
    return m_engine->BatchDirection3D(h, v, a, t);
}
double IRender::GetPixelSpacing(PlaneType t) { return m_engine->PixelSpacing(t); }
bool IRender::SetVRSize(int w, int h) { return m_engine->SetVRSize(w, h); }
void IRender::GetVRSize(int &w, int &h) { m_engine->GetVRSize(w, h); }
bool IRender::GetPlaneIndex(int &i, PlaneType t) { return m_engine->PlaneIndex(i, t); }
bool IRender::GetPlaneNumber(int &n, PlaneType t) { return m_engine->PlaneNumber(n, t); }
bool IRender::GetPlaneRotateMatrix(float *m, PlaneType t) { return m_engine->PlaneRotateMatrix(m, t); }
void IRender::Anterior() { m_engine->Orientation(0); }
void IRender::Posterior() { m_engine->Orientation(1); }
void IRender::Left() { m_engine->Orientation(2); }
void IRender::Right() { m_engine->Orientation(3); }
void IRender::Head() { m_engine->Orientation(4); }
void IRender::Foot() { m_engine->Orientation(5); }
void IRender::SetRenderType(RenderType t) { m_engine->SetRenderType(t); }
void IRender::Rotate(float fx, float fy) { m_engine->Rotate(fx, fy); }
float IRender::Zoom(float r) { return m_engine->Zoom(r); }
float IRender::GetZoomRatio() { return m_engine->ZoomRatio(); }
void IRender::Pan(float x, float y) { m_engine->Pan(x, y); }
bool IRender::SetVRWWWL(float ww, float wl) { return m_engine->SetVRWWWL(ww, wl, m_engine->ActiveLabel()); }
bool IRender::SetVRWWWL(float ww, float wl, unsigned char l) { return m_engine->SetVRWWWL(ww, wl, l); }
bool IRender::SetObjectAlpha(float a) { return m_engine->SetObjectAlpha(a, m_engine->ActiveLabel()); }
bool IRender::SetObjectAlpha(float a, unsigned char l) { return m_engine->SetObjectAlpha(a, l); }
bool IRender::SetTransferFunc(std::map<int, RGBA> c) { return m_engine->SetControlPoints(c, m_engine->ActiveLabel()); }
bool IRender::SetTransferFunc(std::map<int, RGBA> c, unsigned char l) { return m_engine->SetControlPoints(c, l); }
bool IRender::SetTransferFunc(std::map<int, RGBA> c, std::map<int, float> a) {
    return m_engine->SetControlPoints(c, a, m_engine->ActiveLabel());
}
bool IRender::SetTransferFunc(std::map<int, RGBA> c, std::map<int, float> a, unsigned char l) {
    return m_engine->SetControlPoints(c, a, l);
}
bool IRender::LoadTransferFunction(const char *f) { return m_engine->LoadTransferFunction(f); }
bool IRender::SaveTransferFunction(const char *f) { return m_engine->SaveTransferFunction(f); }
bool IRender::AddAnnotation(PlaneType t, std::string txt, int x, int y, FontSize s, AnnotationFormat f, RGBA c) {
    return m_engine->AddAnnotation(t, txt, x, y, s, f, c);
}
bool IRender::RemovePlaneAnnotations(PlaneType t) { return m_engine->RemovePlaneAnnotations(t); }
bool IRender::RemoveAllAnnotations() { return m_engine->RemoveAllAnnotations(); }
bool IRender::EnableLayer(LayerType t, bool on) { return m_engine->EnableLayer(t, on); }
bool IRender::SetCPRLinePatient(std::vector<Point3d> l) { return m_engine->SetCPRLinePatient(l); }
bool IRender::SetCPRLineVoxel(std::vector<Point3d> l) { return m_engine->SetCPRLineVoxel(l); }
std::vector<Point3d> IRender::GetCPRLineVoxel() { return m_engine->CPRLineVoxel(); }
bool IRender::RotateCPR(float a, PlaneType t) { return m_engine->RotateCPR(a, t); }
void IRender::SetCPRLineColor(RGBA c) { m_engine->SetCPRLineColor(c); }
void IRender::ShowPlaneInVR(bool b) { m_engine->ShowPlaneInVR(b); }

// ---------------------------------------------------------------------------
// Render: the concrete IRender (core/Render.cpp)

class Render : public IRender {
public:
    bool GetPlaneData(std::shared_ptr<short> &p, int &w, int &h, const PlaneType &t) override {
        return m_engine->RenderPlane(p, w, h, t);
    }
    bool GetCrossHairPoint(double &x, double &y, const PlaneType &t) override {
        if (t == PlaneVR) return true;   // MonkeyGL leaves (x, y) untouched for VR (core/Render.cpp:71-99)
        return m_engine->CrossHairPoint(x, y, t);
    }
    void PanCrossHair(float fx, float fy, PlaneType t) override {
        if (t != PlaneVR) m_engine->PanCrossHair(fx, fy, t);
    }
    bool GetVRData(std::shared_ptr<unsigned char> &p, int, int) override {
        int w = 0, h = 0;
        m_engine->RenderVR(p, w, h);
        return true;   // MonkeyGL reports success whatever its layers did (core/BaseDataProvider.cpp:37-45)
    }
    bool GetBatchData(std::vector<short *> &out, BatchInfo info) override { return m_engine->RenderBatch(out, info); }
};

// ---------------------------------------------------------------------------
// HelloMonkey (core/HelloMonkey.cpp)

HelloMonkey::HelloMonkey() : m_pRender(std::make_shared<Render>()) {}
HelloMonkey::~HelloMonkey() {}

void HelloMonkey::SetLogLevel(LogLevel level) { g_log_level = level; }
void HelloMonkey::LoadVolumeFile(const char *f) { m_pRender->LoadVolumeFile(f); }
void HelloMonkey::SetDirection(Direction3d x, Direction3d y, Direction3d z) { m_pRender->SetDirection(x, y, z); }
void HelloMonkey::SetSpacing(double x, double y, double z) { m_pRender->SetSpacing(x, y, z); }
void HelloMonkey::SetOrigin(Point3d pt) { m_pRender->SetOrigin(pt); }
void HelloMonkey::Reset() { m_pRender->Reset(); }
void HelloMonkey::SetColorBackground(RGBA c) { m_pRender->SetColorBackground(c); }
bool HelloMonkey::SetVolumeData(std::shared_ptr<short> p, int w, int h, int d) { return m_pRender->SetVolumeData(p, w, h, d); }
unsigned char HelloMonkey::AddNewObjectMask(std::shared_ptr<unsigned char> p, int w, int h, int d) {
    return m_pRender->AddNewObjectMask(p, w, h, d);
}
unsigned char HelloMonkey::AddObjectMaskFile(const char *f) { return m_pRender->AddObjectMaskFile(f); }
bool HelloMonkey::UpdateObjectMask(std::shared_ptr<unsigned char> p, int w, int h, int d, const unsigned char &l) {
    return m_pRender->UpdateObjectMask(p, w, h, d, l);
}
std::shared_ptr<short> HelloMonkey::GetVolumeData(int &w, int &h, int &d) { return m_pRender->GetVolumeData(w, h, d); }
bool HelloMonkey::GetPlaneMaxSize(int &w, int &h, const PlaneType &t) { return m_pRender->GetPlaneMaxSize(w, h, t); }
bool HelloMonkey::GetPlaneData(std::shared_ptr<short> &p, int &w, int &h, const PlaneType &t) {
    return m_pRender->GetPlaneData(p, w, h, t);
}

// int16 plane as an RGBA8 PNG of half the width (two values per pixel),
// Base64 encoded (core/HelloMonkey.cpp:212-259)
std::string HelloMonkey::GetPlaneData_pngString(const PlaneType &t) {
    int w = 0, h = 0;
    std::shared_ptr<short> p;
    if (!m_pRender->GetPlaneData(p, w, h, t) || !p) return "";
    std::vector<uint8_t> png = mk::encode_png(reinterpret_cast<uint8_t *>(p.get()), w / 2, h, 4);
    return mk::base64_string(png.data(), png.size());
}

// Axial slice of the stored volume, voxels outside every object set to
// -2048 when a label volume exists (core/HelloMonkey.cpp:261-320)
std::string HelloMonkey::GetOriginData_pngString(int slice) {
    int w = 0, h = 0, d = 0;
    std::shared_ptr<short> vol = GetVolumeData(w, h, d);
    if (!vol) return "";
    std::shared_ptr<unsigned char> mask = m_pRender->GetMaskData();
    slice = slice < 0 ? 0 : (slice >= d ? d - 1 : slice);
    std::vector<short> s((size_t)w * h);
    std::memcpy(s.data(), vol.get() + (size_t)w * h * slice, s.size() * sizeof(short));
    if (mask) {
        const unsigned char *m = mask.get() + (size_t)w * h * slice;
        for (size_t i = 0; i < s.size(); ++i)
            if (m[i] == 0) s[i] = -2048;
    }
    std::vector<uint8_t> png = mk::encode_png(reinterpret_cast<uint8_t *>(s.data()), w / 2, h, 4);
    return mk::base64_string(png.data(), png.size());
}

bool HelloMonkey::GetCrossHairPoint(double &x, double &y, const PlaneType &t) { return m_pRender->GetCrossHairPoint(x, y, t); }
Point2d HelloMonkey::GetCrossHairPoint(const PlaneType &t) {
    double x = 0, y = 0;
    m_pRender->GetCrossHairPoint(x, y, t);
    return Point2d(x, y);
}
bool HelloMonkey::TransferImage2Voxel(double &x, double &y, double &z, double xi, double yi, PlaneType t) {
    return m_pRender->TransferImage2Voxel(x, y, z, xi, yi, t);
}
bool HelloMonkey::GetCrossHairPoint3D(Point3d &pt) { return m_pRender->GetCrossHairPoint3D(pt); }
bool HelloMonkey::GetDirection(Direction2d &h, Direction2d &v, const PlaneType &t) { return m_pRender->GetDirection(h, v, t); }
bool HelloMonkey::GetDirection3D(Direction3d &h, Direction3d &v, const PlaneType &t) {
    return m_pRender->GetDirection3D(h, v, t);
}
bool HelloMonkey::GetBatchDirection3D(Direction3d &h, Direction3d &v, double a, const PlaneType &t) {
    return m_pRender->GetBatchDirection3D(h, v, a, t);
}
double HelloMonkey::GetPixelSpacing(PlaneType t) { return m_pRender->GetPixelSpacing(t); }
bool HelloMonkey::SetVRSize(int w, int h) { return m_pRender->SetVRSize(w, h); }
bool HelloMonkey::GetVRData(std::shared_ptr<unsigned char> &p, int w, int h) { return m_pRender->GetVRData(p, w, h); }

// RGB PNG of the VR image at the stored VR size (core/HelloMonkey.cpp:333-413)
std::vector<uint8_t> HelloMonkey::GetVRData_png(int, int) {
    int w = 0, h = 0;
    m_pRender->GetVRSize(w, h);
    std::shared_ptr<unsigned char> p;
    if (!m_pRender->GetVRData(p, w, h) || !p) return std::vector<uint8_t>();
    return mk::encode_png(p.get(), w, h, 3);
}
std::string HelloMonkey::GetVRData_pngString() {
    std::vector<uint8_t> png = GetVRData_png(0, 0);
    return mk::base64_string(png.data(), png.size());
}
void HelloMonkey::SaveVR2Png(const char *file, int w, int h) {
    std::vector<uint8_t> png = GetVRData_png(w, h);
    FILE *fp = std::fopen(file, "wb");
    if (!fp) {
        if (g_log_level <= LogLevelError) std::fprintf(stderr, "[MonkeyGL] failed to save png file [%s]\n", file);
        return;
    }
    std::fwrite(png.data(), 1, png.size(), fp);
    std::fclose(fp);
}
bool HelloMonkey::GetBatchData(std::vector<short *> &out, const BatchInfo &b) { return m_pRender->GetBatchData(out, b); }
bool HelloMonkey::GetPlaneIndex(int &i, const PlaneType &t) { return m_pRender->GetPlaneIndex(i, t); }
int HelloMonkey::GetPlaneIndex(const PlaneType &t) {
    int i = -1;
    m_pRender->GetPlaneIndex(i, t);
    return i;
}
bool HelloMonkey::GetPlaneNumber(int &n, const PlaneType &t) { return m_pRender->GetPlaneNumber(n, t); }
int HelloMonkey::GetPlaneNumber(const PlaneType &t) {
    int n = 0;
    m_pRender->GetPlaneNumber(n, t);
    return n;
}
bool HelloMonkey::GetPlaneRotateMatrix(float *m, PlaneType t) { return m_pRender->GetPlaneRotateMatrix(m, t); }
void HelloMonkey::Anterior() { m_pRender->Anterior(); }
void HelloMonkey::Posterior() { m_pRender->Posterior(); }
void HelloMonkey::Left() { m_pRender->Left(); }
void HelloMonkey::Right() { m_pRender->Right(); }
void HelloMonkey::Head() { m_pRender->Head(); }
void HelloMonkey::Foot() { m_pRender->Foot(); }
void HelloMonkey::SetRenderType(RenderType t) { m_pRender->SetRenderType(t); }
void HelloMonkey::Rotate(float fx, float fy) { m_pRender->Rotate(fx, fy); }
float HelloMonkey::Zoom(float r) { return m_pRender->Zoom(r); }
float HelloMonkey::GetZoomRatio() { return m_pRender->GetZoomRatio(); }
void HelloMonkey::Pan(float x, float y) { m_pRender->Pan(x, y); }
bool HelloMonkey::SetVRWWWL(float ww, float wl) { return m_pRender->SetVRWWWL(ww, wl); }
bool HelloMonkey::SetVRWWWL(float ww, float wl, unsigned char l) { return m_pRender->SetVRWWWL(ww, wl, l); }
bool HelloMonkey::SetObjectAlpha(float a) { return m_pRender->SetObjectAlpha(a); }
bool HelloMonkey::SetObjectAlpha(float a, unsigned char l) { return m_pRender->SetObjectAlpha(a, l); }
bool HelloMonkey::SetTransferFunc(std::map<int, RGBA> c) { return m_pRender->SetTransferFunc(c); }
bool HelloMonkey::SetTransferFunc(std::map<int, RGBA> c, unsigned char l) { return m_pRender->SetTransferFunc(c, l); }
bool HelloMonkey::SetTransferFunc(std::map<int, RGBA> c, std::map<int, float> a) { return m_pRender->SetTransferFunc(c, a); }
bool HelloMonkey::SetTransferFunc(std::map<int, RGBA> c, std::map<int, float> a, unsigned char l) {
    return m_pRender->SetTransferFunc(c, a, l);
}
bool HelloMonkey::LoadTransferFunction(const char *f) { return m_pRender->LoadTransferFunction(f); }
bool HelloMonkey::SaveTransferFunction(const char *f) { return m_pRender->SaveTransferFunction(f); }
void HelloMonkey::Browse(float d, PlaneType t) { m_pRender->Browse(d, t); }
void HelloMonkey::PanCrossHair(float x, float y, PlaneType t) { m_pRender->PanCrossHair(x, y, t); }
void HelloMonkey::RotateCrossHair(float a, PlaneType t) { m_pRender->RotateCrossHair(a, t); }
void HelloMonkey::SetPlaneIndex(int i, PlaneType t) { m_pRender->SetPlaneIndex(i, t); }
void HelloMonkey::UpdateThickness(double v) { m_pRender->UpdateThickness(v); }
void HelloMonkey::SetThickness(double v, PlaneType t) { m_pRender->SetThickness(v, t); }
double HelloMonkey::GetThickness(PlaneType t) { return m_pRender->GetThickness(t); }
void HelloMonkey::SetMPRType(MPRType t) { m_pRender->SetMPRType(t); }
bool HelloMonkey::AddAnnotation(PlaneType t, std::string txt, int x, int y, FontSize s, AnnotationFormat f, RGBA c) {
    return m_pRender->AddAnnotation(t, txt, x, y, s, f, c);
}
bool HelloMonkey::RemovePlaneAnnotations(PlaneType t) { return m_pRender->RemovePlaneAnnotations(t); }
bool HelloMonkey::RemoveAllAnnotations() { return m_pRender->RemoveAllAnnotations(); }
bool HelloMonkey::EnableLayer(LayerType t, bool on) { return m_pRender->EnableLayer(t, on); }
bool HelloMonkey::SetCPRLinePatient(std::vector<Point3d> l) { return m_pRender->SetCPRLinePatient(l); }
bool HelloMonkey::SetCPRLineVoxel(std::vector<Point3d> l) { return m_pRender->SetCPRLineVoxel(l); }
bool HelloMonkey::RotateCPR(float a, PlaneType t) { return m_pRender->RotateCPR(a, t); }
void HelloMonkey::SetCPRLineColor(RGBA c) { m_pRender->SetCPRLineColor(c); }
void HelloMonkey::ShowPlaneInVR(bool b) { m_pRender->ShowPlaneInVR(b); }

// Base64 of the first w*h bytes, printed as a quoted line (core/HelloMonkey.cpp:53-61)
void HelloMonkey::Transfer2Base64(unsigned char *p, int w, int h) {
    std::string s = mk::base64_string(p, (size_t)w * h);
    std::printf("\"%s\",\n", s.c_str());
}

// ---- introspection -----------------------------------------------------------

void HelloMonkey::GetVRSize(int &w, int &h) { m_pRender->GetVRSize(w, h); }
bool HelloMonkey::GetVRParams(mk_vr_params &p) { return m_pRender->engine().VRParams(p); }
std::vector<float> HelloMonkey::GetLabelTable() { return m_pRender->engine().LabelTable(); }
bool HelloMonkey::GetPlaneParams(mk_plane_params &p, PlaneType t) { return m_pRender->engine().PlaneParams(p, t); }
bool HelloMonkey::GetCPRRows(std::vector<double> &pts, std::vector<double> &dirs, int &w, int &h, PlaneType t) {
    return m_pRender->engine().CPRRows(pts, dirs, w, h, t);
}
bool HelloMonkey::GetTransferFunctionLUT(std::vector<float> &rgba, unsigned char l) {
    std::vector<RGBA> lut;
    if (!m_pRender->engine().TransferFunctionLUT(l, lut)) return false;
    rgba.resize(4 * lut.size());
    for (size_t i = 0; i < lut.size(); ++i) {
        rgba[4 * i] = lut[i].red;
        rgba[4 * i + 1] = lut[i].green;
        rgba[4 * i + 2] = lut[i].blue;
        rgba[4 * i + 3] = lut[i].alpha;
    }
    return true;
}
mk_volume HelloMonkey::GetDeviceVolume() { return m_pRender->engine().DeviceVolume(); }

}  // namespace MonkeyGL
