// host_engine.cpp -- per-instance host state of the MonkeyGL API (see
// host_engine.h).  Each function names the MonkeyGL source it restates.  The
// file is compiled with -ffp-contract=off so float and double expressions
// round exactly as MonkeyGL's host build (x86-64, SSE, no FMA) does.
#include "host_engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>

namespace MonkeyGL {

std::string PlaneTypeName(PlaneType t) {
    switch (t) {
        case PlaneNotDefined: return "PlaneNotDefined";
        case PlaneAxial: return "PlaneAxial";
        case PlaneSagittal: return "PlaneSagittal";
        case PlaneCoronal: return "PlaneCoronal";
        case PlaneAxialOblique: return "PlaneAxialOblique";
        case PlaneSagittalOblique: return "PlaneSagittalOblique";
        case PlaneCoronalOblique: return "PlaneCoronalOblique";
        case PlaneVR: return "PlaneVR";
        case PlaneStretchedCPR: return "PlaneStretchedCPR";
        case PlaneStraightenedCPR: return "PlaneStraightenedCPR";
        default: return "";
    }
}

namespace detail {

namespace {

// --- small geometry helpers (core/Methods.cpp:134-160, 563-616) ---------

void identity(float *m) {
    for (int i = 0; i < 9; ++i) m[i] = (i % 4 == 0) ? 1.0f : 0.0f;
}

// dst = a * b for row-major 3x3 float matrices, each entry accumulated left
// to right in float.
void matmul(float *dst, const float *a, const float *b) {
    float t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float s = a[i * 3] * b[j];
            for (int k = 1; k < 3; ++k) s += a[i * 3 + k] * b[k * 3 + j];
            t[i * 3 + j] = s;
        }
    std::memcpy(dst, t, sizeof(t));
}

// float matrix times double point, double accumulation.
Point3d matvec(const float *m, const Point3d &p) {
    double x = m[0] * p.x() + m[1] * p.y() + m[2] * p.z();
    double y = m[3] * p.x() + m[4] * p.y() + m[5] * p.z();
    double z = m[6] * p.x() + m[7] * p.y() + m[8] * p.z();
    return Point3d(x, y, z);
}

Point3d transfer_point(const double m[3][3], const Point3d &p) {
    double r[3];
    for (int i = 0; i < 3; ++i) {
        r[i] = 0;
        for (int j = 0; j < 3; ++j) r[i] += m[i][j] * p[j];
    }
    return Point3d(r[0], r[1], r[2]);
}

double length_in_line(const Point3d &pt, const Direction3d &dir, const Point3d &on) {
    Point3d v = pt - on;
    return v.x() * dir.x() + v.y() * dir.y() + v.z() * dir.z();
}

double distance_to_plane(const Point3d &pt, const Direction3d &n, const Point3d &on) {
    Point3d v = pt - on;
    return v.x() * n.x() + v.y() * n.y() + v.z() * n.z();
}

Point3d project_to_plane(const Point3d &pt, const Direction3d &n, const Point3d &on) {
    double d = distance_to_plane(pt, n, on);
    return Point3d(pt.x() - d * n.x(), pt.y() - d * n.y(), pt.z() - d * n.z());
}

double distance_to_line(const Point3d &pt, const Direction3d &dir, const Point3d &on) {
    double lv = pt.DistanceTo(on);
    double lp = length_in_line(pt, dir, on);
    return std::sqrt(lv * lv - lp * lp);
}

// Rodrigues rotation with float sine and cosine (core/Methods.cpp RotatePoint3D).
Point3d rotate_point(const Point3d &pt, const Direction3d &n, const Point3d &c, float theta) {
    double dx = n.x(), dy = n.y(), dz = n.z();
    double x0 = pt.x() - c.x(), y0 = pt.y() - c.y(), z0 = pt.z() - c.z();
    const float ct = std::cos(theta), st = std::sin(theta);
    Point3d o;
    o.SetX(x0 * (dx * dx * (1 - ct) + ct) + y0 * (dx * dy * (1 - ct) - dz * st) + z0 * (dx * dz * (1 - ct) + dy * st));
    o.SetY(x0 * (dy * dx * (1 - ct) + dz * st) + y0 * (dy * dy * (1 - ct) + ct) + z0 * (dy * dz * (1 - ct) - dx * st));
    o.SetZ(x0 * (dz * dx * (1 - ct) - dy * st) + y0 * (dy * dz * (1 - ct) + dx * st) + z0 * (dz * dz * (1 - ct) + ct));
    return o + c;
}

// Rotation about axis `a` given the angle's sine and cosine, as a double 3x3
// matrix (core/MPRInfo.cpp RotateCrossHair, DataManager.cpp
// GetBatchDirection3D).  The callers take the sine in the precision MonkeyGL
// does: float for RotateCrossHair's float angle, double for the batch angle.
void axis_rotation(const Direction3d &a, double s, double c, double m[3][3]) {
    double x = a.x(), y = a.y(), z = a.z();
    double xx = x * x, yy = y * y, zz = z * z;
    double t = 1.0 - c;
    m[0][0] = xx + (1 - xx) * c;
    m[1][1] = yy + (1 - yy) * c;
    m[2][2] = zz + (1 - zz) * c;
    m[0][1] = x * y * t - z * s;
    m[0][2] = x * z * t + y * s;
    m[1][0] = x * y * t + z * s;
    m[1][2] = y * z * t - x * s;
    m[2][0] = x * z * t - y * s;
    m[2][1] = y * z * t + x * s;
}

int plane_init_size(int &w, int &h, int &n, const int dim[3], const double sp[3], PlaneType t) {
    if (dim[0] <= 0 || dim[1] <= 0 || dim[2] <= 0) return 0;
    if (sp[0] <= 0 || sp[1] <= 0 || sp[2] <= 0) return 0;
    double ms = sp[0] < sp[1] ? sp[0] : sp[1];
    ms = ms < sp[2] ? ms : sp[2];
    switch (t) {
        case PlaneAxial:
        case PlaneAxialOblique:
            w = dim[0] * sp[0] / ms;
            h = dim[1] * sp[1] / ms;
            n = dim[2] * sp[2] / ms;
            return 1;
        case PlaneSagittal:
        case PlaneSagittalOblique:
            w = dim[1] * sp[1] / ms;
            h = dim[2] * sp[2] / ms;
            n = dim[0] * sp[0] / ms;
            return 1;
        case PlaneCoronal:
        case PlaneCoronalOblique:
            w = dim[0] * sp[0] / ms;
            h = dim[2] * sp[2] / ms;
            n = dim[1] * sp[1] / ms;
            return 1;
        default:
            w = h = n = -1;
            return 0;
    }
}

}  // namespace

// --------------------------------------------------------------------------
// transfer functions (core/TransferFunction.cpp:38-140)

bool BuildTransferFunction(std::map<int, RGBA> rgb, std::map<int, float> alpha, std::vector<RGBA> &lut) {
    const int lo = 0, hi = 99;
    for (auto it = rgb.begin(); it != rgb.end();) {
        if (it->first < lo || it->first > hi) it = rgb.erase(it);
        else ++it;
    }
    if (rgb.size() < 2) return false;
    if (rgb.begin()->first != lo) rgb[lo] = rgb.begin()->second;
    if (rgb.rbegin()->first != hi) rgb[hi] = rgb.rbegin()->second;
    lut.assign(hi - lo + 1, RGBA());
    auto it = rgb.begin();
    int posPrev = it->first;
    RGBA prev = it->second;
    for (++it; it != rgb.end(); ++it) {
        const int posCur = it->first;
        const RGBA cur = it->second;
        const int n = posCur - posPrev + 1;
        for (int j = posPrev; j <= posCur; ++j) {
            RGBA &o = lut[j - lo];
            o.red = prev.red + (cur.red - prev.red) * (j - posPrev) / n;
            o.green = prev.green + (cur.green - prev.green) * (j - posPrev) / n;
            o.blue = prev.blue + (cur.blue - prev.blue) * (j - posPrev) / n;
            o.alpha = prev.alpha + (cur.alpha - prev.alpha) * (j - posPrev) / n;
        }
        posPrev = posCur;
        prev = cur;
    }
    if (alpha.size() > 1) {
        for (auto a = alpha.begin(); a != alpha.end();) {
            if (a->first < lo || a->first > hi) a = alpha.erase(a);
            else ++a;
        }
        if (alpha.empty()) return true;
        if (alpha.begin()->first != lo) alpha[lo] = 0;
        if (alpha.rbegin()->first != hi) {
            const float last = alpha.rbegin()->second;
            alpha[hi] = last;
        }
        auto a = alpha.begin();
        int pPrev = a->first;
        float aPrev = a->second;
        for (++a; a != alpha.end(); ++a) {
            const int pCur = a->first;
            const float aCur = a->second;
            const int n = pCur - pPrev + 1;
            for (int j = pPrev; j <= pCur; ++j) lut[j - lo].alpha = aPrev + (aCur - aPrev) * (j - pPrev) / n;
            pPrev = pCur;
            aPrev = aCur;
        }
    }
    return true;
}

bool WriteObjectInfo(const char *file, const ObjectInfo &info) {
    std::ofstream os(file);
    if (!os.is_open()) return false;
    os << "ww: " << info.ww << std::endl;
    os << "wl: " << info.wl << std::endl;
    os << "idx2rgba: " << info.idx2rgba.size() << std::endl;
    for (const auto &kv : info.idx2rgba)
        os << kv.first << " " << kv.second.red << " " << kv.second.green << " " << kv.second.blue << " "
           << kv.second.alpha << " " << std::endl;
    os << "idx2alpha: " << info.idx2alpha.size() << std::endl;
    for (const auto &kv : info.idx2alpha) os << kv.first << " " << kv.second << " " << std::endl;
    return true;
}

bool ReadObjectInfo(const char *file, ObjectInfo &info) {
    std::ifstream is(file);
    if (!is.is_open()) return false;
    std::string title;
    is >> title >> info.ww;
    is >> title >> info.wl;
    int n = 0;
    is >> title >> n;
    for (int i = 0; i < n && is; ++i) {
        int idx;
        float r, g, b, a;
        is >> idx >> r >> g >> b >> a;
        info.idx2rgba[idx] = RGBA(r, g, b, a);
    }
    is >> title >> n;
    for (int i = 0; i < n && is; ++i) {
        int idx;
        float a;
        is >> idx >> a;
        info.idx2alpha[idx] = a;
    }
    return true;
}

// --------------------------------------------------------------------------

Engine::Engine() {
    identity(rot_);
    identity(rotT_);
    identity(xf_);
    identity(xfT_);
    identity(kernelMatrix_);
    // MarchingCube's constructor reads the orientation mesh relative to the
    // working directory (core/MarchingCube.cpp:298)
    if (mk_mesh_load_stl("./resources/human.stl", &mesh_) != MK_OK) mesh_ = nullptr;
    // the annotation glyphs, from the same resource directory (no glyph
    // file: annotations are kept but not drawn)
    if (mk_font_load("./resources/annotation_glyphs.bin", &font_) != MK_OK) font_ = nullptr;
}

Engine::~Engine() {
    if (dev_) mk_volume_destroy(dev_);
    if (mesh_) mk_mesh_destroy(mesh_);
    if (font_) mk_font_destroy(font_);
}

// ---- volume (DataManager.cpp:144-175, VolumeInfo.cpp:78-148) -------------

bool Engine::SetVolumeData(std::shared_ptr<short> data, int w, int h, int d) {
    activeLabel_ = -1;
    objects_.clear();
    vol_.reset();
    mask_.reset();
    if (!data || w <= 0 || h <= 0 || d <= 0) return false;
    dims_[0] = w;
    dims_[1] = h;
    dims_[2] = d;
    vol_ = data;
    ResetPlaneInfos();
    activeLabel_ = 0;
    objects_[0] = ObjectInfo();
    std::memcpy(kernelMatrix_, xf_, sizeof(xf_));
    volumeDirty_ = true;
    maskDirty_ = true;
    tfDirty_ = true;
    return true;
}

std::shared_ptr<short> Engine::GetVolumeData(int &w, int &h, int &d) {
    w = dims_[0];
    h = dims_[1];
    d = dims_[2];
    return vol_;
}

void Engine::SetDirection(Direction3d x, Direction3d y, Direction3d z) {
    dirX_ = x;
    dirY_ = y;
    dirZ_ = z;
}

bool Engine::Need2InvertZ() const { return dirX_.cross(dirY_).dot(dirZ_) > 0; }

double Engine::MinSpacing() const {
    double m = spacing_[0] < spacing_[1] ? spacing_[0] : spacing_[1];
    return m < spacing_[2] ? m : spacing_[2];
}

Point3d Engine::Patient2Voxel(Point3d p) const {
    return Point3d(length_in_line(p, dirX_, origin_) / spacing_[0], length_in_line(p, dirY_, origin_) / spacing_[1],
                   length_in_line(p, dirZ_, origin_) / spacing_[2]);
}

// DataManager.cpp:435-442 and the float InitCommon of DataManager.h:201-216
void Engine::SetSpacing(double x, double y, double z) {
    spacing_[0] = x;
    spacing_[1] = y;
    spacing_[2] = z;
    cprSpacing_ = Point3d(x, y, z);
    cprMinSpacing_ = x < y ? x : y;
    cprMinSpacing_ = cprMinSpacing_ < z ? cprMinSpacing_ : z;
    ResetPlaneInfos();
    InitCommon();
}

void Engine::InitCommon() {
    const float fx = (float)spacing_[0], fy = (float)spacing_[1], fz = (float)spacing_[2];
    const float w = (float)(size_t)dims_[0], h = (float)(size_t)dims_[1], d = (float)(size_t)dims_[2];
    f3Spacing_[0] = fx;
    f3Spacing_[1] = fy;
    f3Spacing_[2] = fz;
    f3SpacingVoxel_[0] = 1.0f / w;
    f3SpacingVoxel_[1] = 1.0f / h;
    f3SpacingVoxel_[2] = 1.0f / d;
    const float maxLen = std::max(w * fx, std::max(h * fy, d * fz));
    f3MaxLenSpacing_[0] = 1.0f * maxLen / (w * fx);
    f3MaxLenSpacing_[1] = 1.0f * maxLen / (h * fy);
    f3MaxLenSpacing_[2] = 1.0f * maxLen / (d * fz);
}

// ---- labels (DataManager.cpp:280-335, VolumeInfo.cpp:94-134) --------------

unsigned char Engine::AddNewObjectMask(std::shared_ptr<unsigned char> data, int w, int h, int d) {
    unsigned char label = 0;
    if (objects_.empty()) {
        objects_[0] = ObjectInfo();
        label = 1;
    } else if (objects_.size() >= (size_t)MAXOBJECTCOUNT + 1) {
        return 0;
    } else {
        int idx = 1;
        for (auto it = std::next(objects_.begin()); it != objects_.end(); ++it) {
            if (idx != it->first) break;
            ++idx;
        }
        label = (unsigned char)idx;
    }
    if (!data || !vol_ || w != dims_[0] || h != dims_[1] || d != dims_[2]) return 0;
    const size_t n = (size_t)w * h * d;
    if (!mask_) {
        mask_.reset(new unsigned char[n], std::default_delete<unsigned char[]>());
        std::memset(mask_.get(), 0, n);
    }
    unsigned char *m = mask_.get();
    const unsigned char *p = data.get();
    size_t i = 0;
    for (int z = 0; z < d; ++z)
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x, ++i)
                if (p[i] > 0 && m[i] != label) {
                    m[i] = label;
                    GrowMaskBox(x, y, z);
                }
    objects_[label] = objects_[(unsigned char)activeLabel_];
    activeLabel_ = label;
    maskDirty_ = true;
    tfDirty_ = true;
    return label;
}

bool Engine::UpdateObjectMask(std::shared_ptr<unsigned char> data, int w, int h, int d, unsigned char label) {
    if (objects_.find(label) == objects_.end()) return false;
    if (!data || !mask_ || w != dims_[0] || h != dims_[1] || d != dims_[2]) return false;
    const size_t n = (size_t)w * h * d;
    unsigned char *m = mask_.get();
    const unsigned char *p = data.get();
    size_t i = 0;
    for (int z = 0; z < d; ++z)
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x, ++i) {
                const unsigned char nv = p[i] > 0 ? label : (m[i] == label ? 0 : m[i]);
                if (nv != m[i]) {
                    m[i] = nv;
                    GrowMaskBox(x, y, z);
                }
            }
    (void)n;
    maskDirty_ = true;
    return true;
}

void Engine::GrowMaskBox(int x, int y, int z) {
    int *b = maskBox_;
    if (b[0] >= b[3]) {   // empty
        b[0] = x, b[1] = y, b[2] = z, b[3] = x + 1, b[4] = y + 1, b[5] = z + 1;
        return;
    }
    b[0] = std::min(b[0], x), b[1] = std::min(b[1], y), b[2] = std::min(b[2], z);
    b[3] = std::max(b[3], x + 1), b[4] = std::max(b[4], y + 1), b[5] = std::max(b[5], z + 1);
}

// ---- transfer functions and windows (DataManager.cpp:337-611) -------------

bool Engine::SetControlPoints(std::map<int, RGBA> rgb, int label) {
    const unsigned char l = (unsigned char)label;
    if (l > MAXOBJECTCOUNT || objects_.find(l) == objects_.end()) return false;
    objects_[l].idx2rgba = rgb;
    tfDirty_ = true;
    return true;
}

bool Engine::SetControlPoints(std::map<int, RGBA> rgb, std::map<int, float> alpha, int label) {
    const unsigned char l = (unsigned char)label;
    if (l > MAXOBJECTCOUNT || objects_.find(l) == objects_.end()) return false;
    objects_[l].idx2rgba = rgb;
    objects_[l].idx2alpha = alpha;
    tfDirty_ = true;
    return true;
}

bool Engine::SetVRWWWL(float ww, float wl, int label) {
    const unsigned char l = (unsigned char)label;
    if (l > MAXOBJECTCOUNT) return false;
    if (ww <= 0) ww = 1.0;
    objects_[l].ww = ww;
    objects_[l].wl = wl;
    UpdateAlphaWWWL();
    return true;
}

bool Engine::SetObjectAlpha(float alpha, int label) {
    const unsigned char l = (unsigned char)label;
    if (l > MAXOBJECTCOUNT) return false;
    objects_[l].alpha = alpha;
    UpdateAlphaWWWL();
    return true;
}

// The kernel's per-label table is refreshed only here, i.e. by SetVRWWWL and
// SetObjectAlpha (core/DataManager.cpp:602-611); until the first such call
// every label reaches the kernel as (0, 0, 0).
void Engine::UpdateAlphaWWWL() {
    for (const auto &kv : objects_) {
        table_[kv.first][0] = kv.second.alpha;
        table_[kv.first][1] = kv.second.ww;
        table_[kv.first][2] = kv.second.wl;
    }
    tableDirty_ = true;
}

std::vector<float> Engine::LabelTable() const {
    std::vector<float> t(3 * MK_MAX_LABELS);
    for (int l = 0; l < MK_MAX_LABELS; ++l)
        for (int k = 0; k < 3; ++k) t[3 * l + k] = table_[l][k];
    return t;
}

bool Engine::TransferFunctionLUT(unsigned char label, std::vector<RGBA> &lut) {
    auto it = objects_.find(label);
    if (it == objects_.end()) return false;
    return BuildTransferFunction(it->second.idx2rgba, it->second.idx2alpha, lut);
}

// DataManager.cpp:390-416
bool Engine::LoadTransferFunction(const char *file) {
    ObjectInfo info;
    ReadObjectInfo(file, info);
    return SetVRWWWL(info.ww, info.wl, activeLabel_) &&
           SetControlPoints(info.idx2rgba, info.idx2alpha, activeLabel_);
}

bool Engine::SaveTransferFunction(const char *file) {
    if (activeLabel_ < 0 || objects_.empty()) return false;
    WriteObjectInfo(file, objects_[(unsigned char)activeLabel_]);
    return true;
}

// ---- VR camera (RenderInfo.cpp:28-134, Methods.cpp:52-132) ----------------

bool Engine::SetVRSize(int w, int h) {
    const float delta = (w * h) / (768 * 768);
    if (delta > 1) {
        vrWidth_ = w / delta;
        vrHeight_ = h / delta;
    } else {
        vrWidth_ = w;
        vrHeight_ = h;
    }
    if (vrWidth_ % 2) vrWidth_ += 1;
    return true;
}

void Engine::ComputeTransform(float fx, float fz, float fscale) {
    float Rx[9], Rz[9], S[9], T[9], RxT[9], RzT[9], ST[9];
    identity(Rx);
    identity(Rz);
    identity(T);
    identity(RxT);
    identity(RzT);
    identity(ST);
    identity(S);
    S[0] = S[4] = S[8] = 1.0f / fscale;
    const double ax = (fx) / 180.0f * PI, az = (fz) / 180.0f * PI;
    Rx[4] = std::cos(ax);
    Rx[5] = -std::sin(ax);
    Rx[7] = std::sin(ax);
    Rx[8] = std::cos(ax);
    Rz[0] = std::cos(az);
    Rz[1] = std::sin(az);
    Rz[3] = -std::sin(az);
    Rz[4] = std::cos(az);
    matmul(xf_, xf_, S);
    matmul(xf_, xf_, Rz);
    matmul(xf_, xf_, Rx);
    matmul(T, Rx, Rz);
    matmul(rot_, T, rot_);
    RxT[4] = std::cos(ax);
    RxT[5] = std::sin(ax);
    RxT[7] = -std::sin(ax);
    RxT[8] = std::cos(ax);
    RzT[0] = std::cos(az);
    RzT[1] = -std::sin(az);
    RzT[3] = std::sin(az);
    RzT[4] = std::cos(az);
    ST[0] = ST[4] = ST[8] = fscale;
    matmul(T, RxT, RzT);
    matmul(T, T, ST);
    matmul(xfT_, T, xfT_);
    matmul(rotT_, rotT_, RzT);
    matmul(rotT_, rotT_, RxT);
    std::memcpy(kernelMatrix_, xf_, sizeof(xf_));
}

void Engine::ResetCamera() {
    xT_ = yT_ = 0.0f;
    scale_ = 1.0f;
    identity(rot_);
    identity(rotT_);
    identity(xf_);
    identity(xfT_);
}

// RenderInfo::Rotate passes (fyRotate, fxRotate) as (x-angle, z-angle)
void Engine::Rotate(float fx, float fy) { ComputeTransform(fy, fx, 1.0f); }

float Engine::Zoom(float ratio) {
    scale_ *= ratio;
    ComputeTransform(0.0f, 0.0f, ratio);
    return scale_;
}

void Engine::Pan(float dx, float dy) {
    xT_ += dx;
    yT_ += dy;
}

void Engine::Orientation(int which) {
    static const float presets[6][2] = {{0, 0}, {0, 180}, {0, -90}, {0, 90}, {90, 180}, {-90, 0}};
    if (which < 0 || which > 5) return;
    ResetCamera();
    ComputeTransform(presets[which][0], presets[which][1], scale_);
}

// DataManager.cpp:211-234
bool Engine::TransferVoxel2ImageInVR(float &fx, float &fy, int w, int h, Point3d v) const {
    const double sx = spacing_[0], sy = spacing_[1], sz = spacing_[2];
    const float maxLen = std::max(dims_[0] * sx, std::max(dims_[1] * sy, dims_[2] * sz));
    Point3d per(maxLen / (dims_[0] * sx), maxLen / (dims_[1] * sy), maxLen / (dims_[2] * sz));
    Point3d p(v.x() / dims_[0], v.y() / dims_[1], v.z() / dims_[2]);
    if (Need2InvertZ()) p.SetZ(1.0 - p.z());
    p -= Point3d(0.5, 0.5, 0.5);
    p /= per;
    p = matvec(xfT_, p);
    fx = (p.x() + 0.5) * w + xT_;
    fy = (p.z() + 0.5) * h + yT_;
    return true;
}

// The cu_render arguments of VRImageLayer::GetRGBData (core/VRImageLayer.cpp:64-102)
bool Engine::VRParams(mk_vr_params &p) const {
    std::memset(&p, 0, sizeof(p));
    p.width = vrWidth_;
    p.height = vrHeight_;
    p.render_type = renderType_ == RenderTypeNotDefined ? 0 : (int)renderType_;
    for (int k = 0; k < 3; ++k) {
        p.max_len_spacing[k] = f3MaxLenSpacing_[k];
        p.spacing[k] = f3Spacing_[k];
        p.spacing_voxel[k] = f3SpacingVoxel_[k];
    }
    p.x_translate = xT_;
    p.y_translate = yT_;
    p.scale = scale_;
    std::memcpy(p.transform, kernelMatrix_, sizeof(kernelMatrix_));
    p.invert_z = Need2InvertZ() ? 1 : 0;
    p.voi[0] = 0;
    p.voi[1] = dims_[0] - 1;
    p.voi[2] = 0;
    p.voi[3] = dims_[1] - 1;
    p.voi[4] = 0;
    p.voi[5] = dims_[2] - 1;
    p.background[0] = background_.red;
    p.background[1] = background_.green;
    p.background[2] = background_.blue;
    p.background[3] = background_.alpha;
    p.pixel_format = MK_PIXEL_RGB8;
    p.flags = 0;
    return vol_ != nullptr;
}

// ---- MPR (MPRInfo.cpp, MPRImageLayer.cpp) ---------------------------------

// MPRInfo::ResetPlaneInfos (core/MPRInfo.cpp:96-156)
void Engine::ResetPlaneInfos() {
    const int *dim = dims_;
    const double *sp = spacing_;
    crossHair_ = Point3d(0.5 * dim[0] * sp[0], 0.5 * dim[1] * sp[1], 0.5 * dim[2] * sp[2]);
    planes_.clear();
    for (int i = (int)PlaneAxial; i <= (int)PlaneCoronalOblique; ++i) {
        PlaneType t = (PlaneType)i;
        PlaneInfo info;
        info.type = t;
        plane_init_size(info.width, info.height, info.number, dim, sp, t);
        switch (t) {
            case PlaneAxial:
            case PlaneAxialOblique:
                info.dirH = Direction3d(1, 0, 0);
                info.dirV = Direction3d(0, 1, 0);
                break;
            case PlaneSagittal:
            case PlaneSagittalOblique:
                info.dirH = Direction3d(0, 1, 0);
                info.dirV = Direction3d(0, 0, -1);
                break;
            default:
                info.dirH = Direction3d(1, 0, 0);
                info.dirV = Direction3d(0, 0, -1);
                break;
        }
        info.pixelSpacing = MinSpacing();
        info.sliceThickness = MinSpacing();
        planes_[t] = info;
        center_ = crossHair_;
    }
}

bool Engine::PlaneSize(int &w, int &h, PlaneType t) const {
    if (t < PlaneAxial || t > PlaneCoronalOblique) return false;
    auto it = planes_.find(t);
    if (it == planes_.end()) return false;
    w = it->second.width;
    h = it->second.height;
    return true;
}

// DataManager::GetPlaneMaxSize (core/DataManager.cpp:495-523)
bool Engine::PlaneMaxSize(int &w, int &h, PlaneType t) const {
    if (t == PlaneVR) {
        w = vrWidth_;
        h = vrHeight_;
        return true;
    }
    if (t == PlaneStretchedCPR || t == PlaneStraightenedCPR) return false;
    if (planes_.find(t) == planes_.end()) return false;
    const double xl = dims_[0] * spacing_[0], yl = dims_[1] * spacing_[1], zl = dims_[2] * spacing_[2];
    w = int(sqrtf(xl * xl + yl * yl + zl * zl) / MinSpacing()) + 1;
    h = w;
    return true;
}

Point3d Engine::CenterPointPlane(Direction3d n) const { return project_to_plane(center_, n, crossHair_); }

// MPRImageLayer::GetGrayscaleData (core/MPRImageLayer.cpp:84-139)
bool Engine::PlaneParams(mk_plane_params &p, PlaneType t) const {
    if (!LayerEnabled(LayerTypeImage)) return false;
    if (t < PlaneAxial || t > PlaneCoronalOblique) return false;
    int w = 0, h = 0;
    if (!PlaneSize(w, h, t)) return false;
    if (w % 2) w += 1;
    const PlaneInfo &info = planes_.at(t);
    const Direction3d &dirH = info.dirH, &dirV = info.dirV;
    const Direction3d dirN = info.Normal();
    const double ps = info.pixelSpacing;
    Point3d center = CenterPointPlane(dirN);
    Point3d lt = center - dirH * (0.5 * w * ps);
    lt = lt - dirV * (0.5 * h * ps);
    int nSlice = info.sliceThickness / ps;
    nSlice = nSlice < 1 ? 1 : nSlice;
    std::memset(&p, 0, sizeof(p));
    p.width = w;
    p.height = h;
    p.mpr_type = info.mprType == MPRTypeNotDefined ? 0 : (int)info.mprType;
    p.sampling = MK_SAMPLE_LINEAR;
    for (int k = 0; k < 3; ++k) p.spacing[k] = f3Spacing_[k];
    p.dir_h[0] = dirH.x();
    p.dir_h[1] = dirH.y();
    p.dir_h[2] = dirH.z();
    p.dir_v[0] = dirV.x();
    p.dir_v[1] = dirV.y();
    p.dir_v[2] = dirV.z();
    p.dir_n[0] = dirN.x();
    p.dir_n[1] = dirN.y();
    p.dir_n[2] = dirN.z();
    p.left_top[0] = lt[0];
    p.left_top[1] = lt[1];
    p.left_top[2] = lt[2];
    p.pixel_spacing = info.pixelSpacing;
    p.invert_z = Need2InvertZ() ? 1 : 0;
    p.half_num = 1.0f * (nSlice - 1) / 2;
    return true;
}

void Engine::SetMPRType(MPRType t) {
    for (auto &kv : planes_) kv.second.mprType = t;
}

void Engine::UpdateThickness(double v) {
    for (auto &kv : planes_) kv.second.sliceThickness = v;
}

void Engine::SetThickness(double v, PlaneType t) {
    auto it = planes_.find(t);
    if (it != planes_.end()) it->second.sliceThickness = v;
}

double Engine::Thickness(PlaneType t) const {
    auto it = planes_.find(t);
    return it == planes_.end() ? -1.0 : it->second.sliceThickness;
}

double Engine::PixelSpacing(PlaneType t) const {
    auto it = planes_.find(t);
    return it == planes_.end() ? 1.0 : it->second.pixelSpacing;
}

void Engine::Browse(float delta, PlaneType t) {
    auto it = planes_.find(t);
    if (it == planes_.end()) return;
    crossHair_ = crossHair_ + it->second.Normal() * delta;
}

bool Engine::TransferImage2Voxel(Point3d &v, double x, double y, PlaneType t) const {
    auto it = planes_.find(t);
    if (it == planes_.end()) return false;
    const PlaneInfo &info = it->second;
    Point3d center = CenterPointPlane(info.Normal());
    Point3d lt = info.LeftTop(center);
    v = lt + info.dirH * (x * info.pixelSpacing);
    v = v + info.dirV * (y * info.pixelSpacing);
    return true;
}

void Engine::PanCrossHair(float x, float y, PlaneType t) {
    Point3d v;
    if (!TransferImage2Voxel(v, x, y, t)) return;
    crossHair_ = v;
}

std::vector<PlaneType> Engine::CrossPlaneTypes(PlaneType t) const {
    switch (t) {
        case PlaneAxial: return {PlaneSagittal, PlaneCoronal};
        case PlaneSagittal: return {PlaneAxial, PlaneCoronal};
        case PlaneCoronal: return {PlaneAxial, PlaneSagittal};
        case PlaneAxialOblique: return {PlaneSagittalOblique, PlaneCoronalOblique};
        case PlaneSagittalOblique: return {PlaneAxialOblique, PlaneCoronalOblique};
        case PlaneCoronalOblique: return {PlaneAxialOblique, PlaneSagittalOblique};
        default: return {};
    }
}

// MPRInfo::RotateCrossHair (core/MPRInfo.cpp:353-404)
void Engine::RotateCrossHair(float crossAngle, PlaneType t) {
    PlaneInfo &self = planes_[t];
    const Direction3d dirA = self.Normal();
    float angle = crossAngle - self.crossHairAngle;
    self.crossHairAngle = crossAngle;
    angle = angle / 180 * PI;
    double m[3][3];
    axis_rotation(dirA, std::sin(angle), std::cos(angle), m);   // float overloads
    for (PlaneType ct : CrossPlaneTypes(t)) {
        PlaneInfo &info = planes_[ct];
        Direction3d &dirH = info.dirH;
        Direction3d &dirV = info.dirV;
        const Direction3d dirN = info.Normal();
        Point3d c = CenterPointPlane(dirN);
        const double fW = info.pixelSpacing * info.width;
        const double fH = info.pixelSpacing * info.height;
        Point3d lt = c - dirH * (fW / 2) - dirV * (fH / 2);
        Point3d rt = c + dirH * (fW / 2) - dirV * (fH / 2);
        Point3d lb = c - dirH * (fW / 2) + dirV * (fH / 2);
        lt -= crossHair_;
        lt = transfer_point(m, lt);
        lt += crossHair_;
        rt -= crossHair_;
        rt = transfer_point(m, rt);
        rt += crossHair_;
        lb -= crossHair_;
        lb = transfer_point(m, lb);
        lb += crossHair_;
        dirH = Direction3d(rt[0] - lt[0], rt[1] - lt[1], rt[2] - lt[2]);
        dirV = Direction3d(lb[0] - lt[0], lb[1] - lt[1], lb[2] - lt[2]);
        UpdatePlaneSize(ct);
    }
}

// MPRInfo::UpdatePlaneSize (core/MPRInfo.cpp:406-473)
void Engine::UpdatePlaneSize(PlaneType t) {
    auto it = planes_.find(t);
    if (it == planes_.end()) return;
    const PlaneInfo info = it->second;
    const double xl = dims_[0] * spacing_[0], yl = dims_[1] * spacing_[1], zl = dims_[2] * spacing_[2];
    const double sp = MinSpacing();
    const Point3d verts[8] = {Point3d(0, 0, 0),   Point3d(xl, 0, 0),   Point3d(0, yl, 0),   Point3d(xl, yl, 0),
                              Point3d(0, 0, zl),  Point3d(xl, 0, zl),  Point3d(0, yl, zl),  Point3d(xl, yl, zl)};
    double xn = 0, xp = 0, yn = 0, yp = 0, zn = 0, zp = 0;
    const Direction3d n = info.dirH.cross(info.dirV);
    for (const Point3d &v : verts) {
        Point3d proj = project_to_plane(v, n, crossHair_);
        double x = length_in_line(proj, info.dirH, crossHair_);
        if (x >= 0) xp = xp > x ? xp : x;
        else xn = xn < x ? xn : x;
        double y = length_in_line(proj, info.dirV, crossHair_);
        if (y >= 0) yp = yp > y ? yp : y;
        else yn = yn < y ? yn : y;
        double z = distance_to_plane(v, n, crossHair_);
        if (z >= 0) zp = zp > z ? zp : z;
        else zn = zn < z ? zn : z;
    }
    it->second.width = (xp - xn) / sp;
    it->second.height = (yp - yn) / sp;
    it->second.number = (zp - zn) / sp;
}

bool Engine::CrossHairPoint(double &x, double &y, PlaneType t) const {
    auto it = planes_.find(t);
    if (it == planes_.end()) return false;
    const PlaneInfo &info = it->second;
    Point3d v = crossHair_ - CenterPointPlane(info.Normal());
    const double lh = v.x() * info.dirH.x() + v.y() * info.dirH.y() + v.z() * info.dirH.z();
    const double lv = v.x() * info.dirV.x() + v.y() * info.dirV.y() + v.z() * info.dirV.z();
    x = (info.width - 1) / 2.0 + lh / info.pixelSpacing;
    y = (info.height - 1) / 2.0 + lv / info.pixelSpacing;
    return true;
}

bool Engine::PlaneIndex(int &index, PlaneType t) const {
    auto it = planes_.find(t);
    if (it == planes_.end()) return false;
    const int total = it->second.number;
    const double d = distance_to_plane(crossHair_, it->second.dirH.cross(it->second.dirV), center_);
    const int delta = d / MinSpacing();
    index = delta + (total - 1) / 2;
    return true;
}

void Engine::SetPlaneIndex(int index, PlaneType t) {
    auto it = planes_.find(t);
    if (it == planes_.end()) return;
    const PlaneInfo &info = it->second;
    const Direction3d n = info.Normal();
    const double dist = (index - (info.number - 1) / 2) * MinSpacing();
    Point3d proj = project_to_plane(crossHair_, info.dirH.cross(info.dirV), center_);
    crossHair_ = proj + n * dist;
}

bool Engine::PlaneNumber(int &n, PlaneType t) const {
    auto it = planes_.find(t);
    if (it == planes_.end()) return false;
    n = it->second.number;
    return true;
}

bool Engine::PlaneRotateMatrix(float *m, PlaneType t) const {
    if (t == PlaneVR) {
        std::memcpy(m, rot_, sizeof(rot_));
        return true;
    }
    auto it = planes_.find(t);
    if (it == planes_.end()) return false;
    const PlaneInfo &info = it->second;
    const Direction3d z = info.dirH.cross(info.dirV);
    m[0] = info.dirH.x();
    m[1] = info.dirH.y();
    m[2] = info.dirH.z();
    m[3] = info.dirV.x();
    m[4] = info.dirV.y();
    m[5] = info.dirV.z();
    m[6] = z.x();
    m[7] = z.y();
    m[8] = z.z();
    return true;
}

bool Engine::GroupPlanesExist(PlaneType t) const {
    auto has = [&](PlaneType p) { return planes_.find(p) != planes_.end(); };
    switch (t) {
        case PlaneAxial:
        case PlaneSagittal:
        case PlaneCoronal: return has(PlaneAxial) && has(PlaneSagittal) && has(PlaneCoronal);
        case PlaneAxialOblique:
        case PlaneSagittalOblique:
        case PlaneCoronalOblique:
            return has(PlaneAxialOblique) && has(PlaneSagittalOblique) && has(PlaneCoronalOblique);
        default: return false;
    }
}

// MPRInfo::GetDirection (core/MPRInfo.cpp:539-611)
bool Engine::Direction2D(Direction2d &h, Direction2d &v, PlaneType t) const {
    if (!GroupPlanesExist(t)) return false;
    auto proj = [](const Direction3d &axis, const PlaneInfo &self) {
        const double lh = axis.x() * self.dirH.x() + axis.y() * self.dirH.y() + axis.z() * self.dirH.z();
        const double lv = axis.x() * self.dirV.x() + axis.y() * self.dirV.y() + axis.z() * self.dirV.z();
        return Direction2d(lh, lv);
    };
    switch (t) {
        case PlaneAxial:
        case PlaneSagittal:
        case PlaneCoronal:
            h = Direction2d(1, 0);
            v = Direction2d(0, 1);
            break;
        case PlaneAxialOblique:
            h = proj(planes_.at(PlaneSagittalOblique).Normal(), planes_.at(t));
            v = proj(planes_.at(PlaneCoronalOblique).Normal(), planes_.at(t));
            break;
        case PlaneSagittalOblique:
            h = proj(planes_.at(PlaneCoronalOblique).Normal(), planes_.at(t));
            v = proj(planes_.at(PlaneAxialOblique).Normal(), planes_.at(t));
            break;
        case PlaneCoronalOblique:
            h = proj(planes_.at(PlaneSagittalOblique).Normal(), planes_.at(t));
            v = proj(planes_.at(PlaneAxialOblique).Normal(), planes_.at(t));
            break;
        default: break;
    }
    return true;
}

bool Engine::Direction3D(Direction3d &h, Direction3d &v, PlaneType t) const {
    auto it = planes_.find(t);
    if (it == planes_.end()) return false;
    h = it->second.dirH;
    v = it->second.dirV;
    return true;
}

// DataManager::GetBatchDirection3D (core/DataManager.cpp:613-646)
bool Engine::BatchDirection3D(Direction3d &h, Direction3d &v, double angle, PlaneType t) const {
    Direction3d ph, pv;
    Direction3D(ph, pv, t);
    const Direction3d a = ph.cross(pv);
    angle = angle / 180 * PI;
    double m[3][3];
    axis_rotation(a, std::sin(angle), std::cos(angle), m);   // double overloads
    Point3d p = transfer_point(m, Point3d(ph.x(), ph.y(), ph.z()));
    h = Direction3d(p.x(), p.y(), p.z());
    v = a;
    return true;
}

// ---- CPR (core/CPRInfo.cpp) ------------------------------------------------

bool Engine::RotateCPR(float angle, PlaneType t) {
    if (t == PlaneStretchedCPR) {
        cprAngleStretched_ += angle;
        return true;
    }
    if (t == PlaneStraightenedCPR) {
        cprAngleStraightened_ += angle;
        return true;
    }
    return false;
}

// CPRInfo::FirstDirectionProjection + UpdateCPRInfo (core/CPRInfo.cpp:185-238)
void Engine::UpdateCPRInfo() {
    const Point3d start = cprLine_.front(), end = cprLine_.back();
    cprDirStretched_ = Direction3d(start, end);
    cprStretchedRadius_ = 0;
    for (size_t i = 1; i < cprLine_.size(); ++i) {
        const double r = distance_to_line(cprLine_[i], cprDirStretched_, start);
        if (r > cprStretchedRadius_) cprStretchedRadius_ = r;
    }
    cprStretchedRadius_ += 100.0;
    const Direction3d n = cprDirStretched_;
    double x, y, z;
    if (std::abs(n.y()) > 0.3) {
        x = start.x();
        y = start.y() - n.z() / n.y();
        z = start.z() + 1;
    } else if (std::abs(n.x()) > 0.3) {
        x = start.x() - n.z() / n.x();
        y = start.y();
        z = start.z() + 1;
    } else {
        x = start.x() + 1;
        y = start.y();
        z = start.z() - n.x() / n.z();
    }
    const Direction3d first(start, Point3d(x, y, z));
    // MonkeyGL reads both radii through float getters (core/CPRInfo.h)
    cprOriginStretched_ = start + first * (double)(float)cprStretchedRadius_;
    cprOriginStraightened_ = start + first * (double)(float)cprStraightenedRadius_;
    cprAngleStretched_ = 0;
    cprAngleStraightened_ = 0;
}

bool Engine::SetCPRLineVoxel(const std::vector<Point3d> &line) {
    cprLine_ = line;
    if (cprLine_.size() < 2) return false;
    UpdateCPRInfo();
    return true;
}

bool Engine::SetCPRLinePatient(const std::vector<Point3d> &line) {
    std::vector<Point3d> v;
    v.reserve(line.size());
    for (const Point3d &p : line) v.push_back(Patient2Voxel(p));
    return SetCPRLineVoxel(v);
}

bool Engine::CPRStretched(std::vector<Point3d> &pts, std::vector<Direction3d> &dirs, int &w, int &h) const {
    if (cprLine_.size() < 2) return false;
    w = (float)cprStretchedRadius_ * 2.0 + 1;
    if (w % 2) w += 1;
    const Point3d start = cprLine_.front();
    const Point3d rot = rotate_point(cprOriginStretched_, cprDirStretched_, start, cprAngleStretched_ * PI / 180.0);
    const Direction3d dir(rot, start);
    pts.assign(1, project_to_plane(start, dir, rot));
    dirs.assign(1, dir);
    Point3d pre = pts[0];
    for (size_t i = 1; i < cprLine_.size(); ++i) {
        const Point3d cur = project_to_plane(cprLine_[i], dir, rot);
        if (cur.PatientDistanceTo(pre, cprSpacing_) >= cprMinSpacing_) {
            pre = cur;
            pts.push_back(pre);
            dirs.push_back(dir);
        }
    }
    h = (int)pts.size();
    return true;
}

bool Engine::CPRStraightened(std::vector<Point3d> &pts, std::vector<Direction3d> &dirs, int &w, int &h) const {
    if (cprLine_.size() < 2) return false;
    w = (float)cprStraightenedRadius_ * 2.0 + 1;
    if (w % 2) w += 1;
    h = (int)cprLine_.size();
    pts.assign(h, Point3d());          // the last row keeps its default (origin, +x)
    dirs.assign(h, Direction3d());
    const Point3d start = cprLine_.front();
    const Direction3d path(start, cprLine_[1]);
    const Point3d rot = rotate_point(cprOriginStraightened_, path, start, cprAngleStraightened_ * PI / 180.0);
    const Direction3d dir(rot, start);
    pts[0] = rot;
    dirs[0] = dir;
    const double r = rot.DistanceTo(start);
    for (int i = 1; i < h - 1; ++i) {
        const Point3d pre = cprLine_[i - 1], cur = cprLine_[i], nxt = cprLine_[i + 1];
        const Direction3d d1 = dirs[i - 1];
        const Direction3d d2(pre, cur);
        const Direction3d d3(cur, nxt);
        const Direction3d tmp = d1.cross(d2);
        Direction3d d = d3.cross(tmp);
        if (d.Length() < 0.99f) d = d1;
        if (d.dot(d1) < 0) d = d.negative();
        dirs[i] = d;
        pts[i] = cur - dirs[i] * r;
    }
    return true;
}

bool Engine::CPRRows(std::vector<double> &pts, std::vector<double> &dirs, int &w, int &h, PlaneType t) const {
    if (!LayerEnabled(LayerTypeImage)) return false;
    std::vector<Point3d> p;
    std::vector<Direction3d> d;
    bool ok = false;
    if (t == PlaneStretchedCPR) ok = CPRStretched(p, d, w, h);
    else if (t == PlaneStraightenedCPR) ok = CPRStraightened(p, d, w, h);
    if (!ok) return false;
    pts.resize(3 * (size_t)h);
    dirs.resize(3 * (size_t)h);
    for (int i = 0; i < h; ++i) {
        pts[3 * i] = p[i].x();
        pts[3 * i + 1] = p[i].y();
        pts[3 * i + 2] = p[i].z();
        dirs[3 * i] = d[i].x();
        dirs[3 * i + 1] = d[i].y();
        dirs[3 * i + 2] = d[i].z();
    }
    return true;
}

// ---- layers, annotations, planes in VR -------------------------------------

bool Engine::LayerEnabled(LayerType t) const {
    auto it = layers_.find(t);
    return it == layers_.end() ? true : it->second;
}

// MonkeyGL files every annotation under PlaneVR (core/DataManager.cpp:820-823)
bool Engine::AddAnnotation(PlaneType, const std::string &txt, int x, int y, FontSize s, AnnotationFormat f,
                           RGBA c) {
    annotations_.push_back(Annotation{PlaneVR, txt, x, y, s, f, c});
    return true;
}

bool Engine::RemovePlaneAnnotations(PlaneType t) {
    annotations_.erase(std::remove_if(annotations_.begin(), annotations_.end(),
                                      [t](const Annotation &a) { return a.plane == t; }),
                       annotations_.end());
    return true;
}

bool Engine::RemoveAllAnnotations() {
    annotations_.clear();
    return true;
}

// DataManager::ShowPlaneInVR (core/DataManager.cpp:769-818): three 3-voxel
// slabs (z 200-202, y 200-202, x 250-252) as a new object, window 1000/-40,
// alpha 0.6; slabs beyond the volume are left out.
void Engine::ShowPlaneInVR(bool show) {
    if (!show || !vol_) return;
    const int w = dims_[0], h = dims_[1], d = dims_[2];
    const size_t n = (size_t)w * h * d;
    std::shared_ptr<unsigned char> m(new unsigned char[n], std::default_delete<unsigned char[]>());
    std::memset(m.get(), 0, n);
    for (int z = 200; z < 203 && z < d; ++z) std::memset(m.get() + (size_t)z * w * h, 1, (size_t)w * h);
    for (int z = 0; z < d; ++z)
        for (int y = 200; y < 203 && y < h; ++y) std::memset(m.get() + ((size_t)z * h + y) * w, 1, w);
    for (int z = 0; z < d; ++z)
        for (int y = 0; y < h; ++y)
            for (int x = 250; x < 253 && x < w; ++x) m.get()[((size_t)z * h + y) * w + x] = 1;
    planeLabel_ = AddNewObjectMask(m, w, h, d);
    SetVRWWWL(1000, -40, activeLabel_);
    SetObjectAlpha(0.6f, planeLabel_);
}

// ---- device ----------------------------------------------------------------

bool Engine::SyncDevice() {
    if (!vol_) return false;
    if (!dev_ || volumeDirty_) {
        if (dev_) {
            mk_volume_destroy(dev_);
            dev_ = nullptr;
        }
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess) {
            cudaGetLastError();
            device = 0;
        }
        if (mk_volume_create(&dev_, vol_.get(), dims_[0], dims_[1], dims_[2], device) != MK_OK) {
            dev_ = nullptr;
            return false;
        }
        volumeDirty_ = false;
        maskDirty_ = true;
        maskOnDevice_ = false;      // a new device volume: the whole mask goes up
        tfDirty_ = true;
        tableDirty_ = true;
    }
    if (maskDirty_) {
        // a mask already on the device is updated in the box that changed
        // (MonkeyGL re-uploads the whole mask, CuDataManager.cu:75-120)
        if (maskOnDevice_ && mask_) {
            if (maskBox_[0] < maskBox_[3] && mk_volume_update_mask(dev_, mask_.get(), maskBox_) != MK_OK)
                return false;
        } else if (mk_volume_set_mask(dev_, mask_ ? mask_.get() : nullptr) != MK_OK) {
            return false;
        }
        maskOnDevice_ = mask_ != nullptr;
        maskBox_[0] = maskBox_[3] = 0;
        maskDirty_ = false;
    }
    if (tfDirty_) {
        // every label with an ObjectInfo gets its table (DataManager.cpp:372-388)
        for (int l = 0; l < MK_MAX_LABELS; ++l) {
            auto it = objects_.find((unsigned char)l);
            std::vector<RGBA> lut;
            if (it != objects_.end() && BuildTransferFunction(it->second.idx2rgba, it->second.idx2alpha, lut)) {
                if (mk_volume_set_transfer_function(dev_, l, &lut[0].red, (int)lut.size()) != MK_OK) return false;
            } else if (it == objects_.end()) {
                mk_volume_set_transfer_function(dev_, l, nullptr, 0);
            }
        }
        tfDirty_ = false;
    }
    if (tableDirty_) {
        // entries never refreshed are (0, 0, 0): alpha 0 never composites, so
        // their window does not matter; the C ABI wants a positive width
        float t[MK_MAX_LABELS][3];
        std::memcpy(t, table_, sizeof(t));
        for (int l = 0; l < MK_MAX_LABELS; ++l)
            if (!(t[l][1] > 0.0f)) t[l][1] = 1.0f;
        if (mk_volume_set_label_params(dev_, &t[0][0], MK_MAX_LABELS) != MK_OK) return false;
        tableDirty_ = false;
    }
    return true;
}

// The VR provider's layers in MonkeyGL's order (core/VRProvider.cpp:30-36):
// the ray-cast image with the orientation box in its bottom-right corner
// (core/VRImageLayer.cpp:64-145), then the CPR path as a 1-pixel polyline in
// the line colour (core/CPRLineLayer.cpp:40-65).
bool Engine::RenderVR(std::shared_ptr<unsigned char> &out, int &w, int &h) {
    if (!LayerEnabled(LayerTypeImage)) return false;
    mk_vr_params p;
    if (!VRParams(p) || !SyncDevice()) return false;
    w = p.width;
    h = p.height;
    out.reset(new unsigned char[(size_t)w * h * 3], std::default_delete<unsigned char[]>());
    // the orientation box is host work: it is drawn into a 65x65 scratch
    // image (the box fills its bottom-right 64x64) on another thread while
    // the GPU renders, then its drawn pixels (never black) are copied over
    const bool box = mesh_ && w > 64 && h > 64;
    std::vector<unsigned char> scratch;
    std::thread worker;
    if (box) {
        scratch.assign(65 * 65 * 3, 0);
        std::array<float, 9> rot;
        std::memcpy(rot.data(), rot_, sizeof(rot_));
        worker = std::thread([this, rot, &scratch] {
            mk_merge_orientation_box(mesh_, rot.data(), scratch.data(), 65, 65);
        });
    }
    const int rc = mk_render_vr(dev_, &p, out.get(), 0, nullptr);
    if (worker.joinable()) worker.join();
    if (rc != MK_OK) return false;
    if (box) {
        for (int j = 0; j < 64; ++j) {
            const unsigned char *src = &scratch[((size_t)(j + 1) * 65 + 1) * 3];
            unsigned char *dst = out.get() + ((size_t)(h - 64 + j) * w + (w - 64)) * 3;
            for (int i = 0; i < 64; ++i)
                if (src[3 * i] | src[3 * i + 1] | src[3 * i + 2]) {
                    dst[3 * i] = src[3 * i];
                    dst[3 * i + 1] = src[3 * i + 1];
                    dst[3 * i + 2] = src[3 * i + 2];
                }
        }
    }
    // AnnotationLayer::GetRGBData (core/AnnotationLayer.cpp:41-61): every VR
    // annotation in the order added, on images larger than 10x10
    if (LayerEnabled(LayerTypeAnnotation) && font_ && w > 10 && h > 10) {
        for (const Annotation &a : annotations_) {
            if (a.plane != PlaneVR || a.format < AnnotationFormatLeft) continue;
            const float clr[3] = {a.color.red, a.color.green, a.color.blue};
            mk_draw_text_rgb(font_, out.get(), w, h, a.text.c_str(), a.x, a.y, (int)a.size, (int)a.format, clr);
        }
    }
    if (LayerEnabled(LayerTypeCPRLine) && cprLine_.size() >= 2) {
        const float clr[3] = {cprColor_.red, cprColor_.green, cprColor_.blue};
        float x0 = 0, y0 = 0, x1 = 0, y1 = 0;
        TransferVoxel2ImageInVR(x0, y0, w, h, cprLine_[0]);
        for (size_t i = 1; i < cprLine_.size(); ++i) {
            TransferVoxel2ImageInVR(x1, y1, w, h, cprLine_[i]);
            mk_draw_line_rgb(out.get(), w, h, x0, y0, x1, y1, 1, clr);
            x0 = x1;
            y0 = y1;
        }
    }
    return true;
}

bool Engine::RenderPlane(std::shared_ptr<short> &out, int &w, int &h, PlaneType t) {
    if (t >= PlaneAxial && t <= PlaneCoronalOblique) {
        mk_plane_params p;
        if (!PlaneParams(p, t) || !SyncDevice()) return false;
        w = p.width;
        h = p.height;
        out.reset(new short[(size_t)w * h], std::default_delete<short[]>());
        return mk_render_plane(dev_, &p, out.get(), 0, nullptr) == MK_OK;
    }
    if (t == PlaneStretchedCPR || t == PlaneStraightenedCPR) {
        std::vector<double> pts, dirs;
        if (!CPRRows(pts, dirs, w, h, t) || !SyncDevice()) return false;
        out.reset(new short[(size_t)w * h], std::default_delete<short[]>());
        return mk_render_cpr(dev_, w, h, pts.data(), dirs.data(), Need2InvertZ() ? 1 : 0, out.get(), 0,
                             nullptr) == MK_OK;
    }
    return false;
}

// Batch MPR (MonkeyGL declares GetBatchData and BatchInfo but returns false,
// core/Render.cpp:117-120): m_nNum parallel planes m_fSliceDistance apart,
// centred on m_ptCenter, each Width() x Height() int16, allocated with new[]
// and appended to `out` (the caller owns them).
bool Engine::RenderBatch(std::vector<short *> &out, const BatchInfo &b) {
    if (b.m_nNum <= 0 || !(b.m_fPixelSpacing > 0) || !SyncDevice()) return false;
    const int w = b.Width(), h = b.Height();
    if (w <= 0 || h <= 0) return false;
    const Direction3d n = b.m_dirH.cross(b.m_dirV);
    int nSlice = b.m_fSliceThickness / b.m_fPixelSpacing;
    nSlice = nSlice < 1 ? 1 : nSlice;
    for (int i = 0; i < b.m_nNum; ++i) {
        const double off = (i - (b.m_nNum - 1) / 2.0) * b.m_fSliceDistance;
        Point3d c = b.m_ptCenter + n * off;
        Point3d lt = c - b.m_dirH * (0.5 * w * b.m_fPixelSpacing);
        lt = lt - b.m_dirV * (0.5 * h * b.m_fPixelSpacing);
        mk_plane_params p;
        std::memset(&p, 0, sizeof(p));
        p.width = w;
        p.height = h;
        p.mpr_type = b.m_MPRType == MPRTypeNotDefined ? 0 : (int)b.m_MPRType;
        p.sampling = MK_SAMPLE_LINEAR;
        for (int k = 0; k < 3; ++k) {
            p.spacing[k] = f3Spacing_[k];
            p.left_top[k] = lt[k];
        }
        p.dir_h[0] = b.m_dirH.x();
        p.dir_h[1] = b.m_dirH.y();
        p.dir_h[2] = b.m_dirH.z();
        p.dir_v[0] = b.m_dirV.x();
        p.dir_v[1] = b.m_dirV.y();
        p.dir_v[2] = b.m_dirV.z();
        p.dir_n[0] = n.x();
        p.dir_n[1] = n.y();
        p.dir_n[2] = n.z();
        p.pixel_spacing = b.m_fPixelSpacing;
        p.invert_z = Need2InvertZ() ? 1 : 0;
        p.half_num = 1.0f * (nSlice - 1) / 2;
        short *buf = new short[(size_t)w * h];
        if (mk_render_plane(dev_, &p, buf, 0, nullptr) != MK_OK) {
            delete[] buf;
            return false;
        }
        out.push_back(buf);
    }
    return true;
}

}  // namespace detail
}  // namespace MonkeyGL
