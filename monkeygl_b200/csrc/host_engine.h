// host_engine.h -- the per-instance host state behind HelloMonkey / IRender:
// volume and labels, transfer functions, label windows, VR camera, MPR planes
// and crosshair, CPR path, layers and annotations, and the resident device
// volume.  It restates MonkeyGL's DataManager and the Info classes it owns
// (core/DataManager.cpp, VolumeInfo.cpp, RenderInfo.cpp, MPRInfo.cpp,
// CPRInfo.cpp, TransferFunction.cpp, ObjectInfo.h, Methods.cpp) in the same
// arithmetic: FP32 for the camera and volume factors, FP64 for plane and CPR
// frames, so the kernel arguments it produces equal MonkeyGL's.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/monkeygl/Defines.h"
#include "../../include/monkeygl_b200.h"

namespace MonkeyGL {
namespace detail {

// Per-label rendering state (core/ObjectInfo.h:19-43).
struct ObjectInfo {
    float alpha = 1.0f;
    float ww = 400.0f;
    float wl = 40.0f;
    std::map<int, RGBA> idx2rgba{{5, RGBA(0.8f, 0.8f, 0.8f, 0.0f)}, {95, RGBA(0.8f, 0.8f, 0.8f, 0.8f)}};
    std::map<int, float> idx2alpha;
};

// Control points -> 100-entry RGBA table (core/TransferFunction.cpp:38-140).
bool BuildTransferFunction(std::map<int, RGBA> rgb, std::map<int, float> alpha, std::vector<RGBA> &lut);

// TF text file (core/ObjectInfo.h:45-95).
bool WriteObjectInfo(const char *file, const ObjectInfo &info);
bool ReadObjectInfo(const char *file, ObjectInfo &info);

struct PlaneInfo {
    float crossHairAngle = 0.0f;
    PlaneType type = PlaneNotDefined;
    Direction3d dirH;
    Direction3d dirV;
    int width = 0;
    int height = 0;
    int number = 0;
    double pixelSpacing = 0.0;
    double sliceThickness = 0.0;
    MPRType mprType = MPRTypeAverage;

    Direction3d Normal() const { return dirH.cross(dirV); }
    Point3d LeftTop(Point3d center) const {
        Point3d p = center - dirH * (0.5 * width * pixelSpacing);
        return p - dirV * (0.5 * height * pixelSpacing);
    }
};

struct Annotation {
    PlaneType plane;
    std::string text;
    int x, y;
    FontSize size;
    AnnotationFormat format;
    RGBA color;
};

class Engine {
public:
    Engine();
    ~Engine();

    // ---- volume and labels (DataManager.cpp:144-335) ----
    bool SetVolumeData(std::shared_ptr<short> data, int w, int h, int d);
    unsigned char AddNewObjectMask(std::shared_ptr<unsigned char> data, int w, int h, int d);
    bool UpdateObjectMask(std::shared_ptr<unsigned char> data, int w, int h, int d, unsigned char label);
    std::shared_ptr<short> GetVolumeData(int &w, int &h, int &d);
    std::shared_ptr<unsigned char> GetMaskData() { return mask_; }
    void SetDirection(Direction3d x, Direction3d y, Direction3d z);
    void SetSpacing(double x, double y, double z);
    void SetOrigin(Point3d p) { origin_ = p; }
    void Reset() { ResetPlaneInfos(); }
    void SetColorBackground(RGBA c) { background_ = c; }
    bool Need2InvertZ() const;
    int Dim(int i) const { return dims_[i]; }
    double Spacing(int i) const { return spacing_[i]; }
    double MinSpacing() const;
    Point3d Patient2Voxel(Point3d p) const;

    // ---- transfer functions and windows (DataManager.cpp:337-611) ----
    bool SetControlPoints(std::map<int, RGBA> rgb, int label);
    bool SetControlPoints(std::map<int, RGBA> rgb, std::map<int, float> alpha, int label);
    bool SetVRWWWL(float ww, float wl, int label);
    bool SetObjectAlpha(float alpha, int label);
    int ActiveLabel() const { return activeLabel_; }
    bool LoadTransferFunction(const char *file);
    bool SaveTransferFunction(const char *file);
    bool TransferFunctionLUT(unsigned char label, std::vector<RGBA> &lut);
    std::vector<float> LabelTable() const;

    // ---- VR camera (RenderInfo.cpp, Methods.cpp:52-132) ----
    bool SetVRSize(int w, int h);
    void GetVRSize(int &w, int &h) const {
        w = vrWidth_;
        h = vrHeight_;
    }
    void Rotate(float fx, float fy);
    float Zoom(float ratio);
    float ZoomRatio() const { return scale_; }
    void Pan(float dx, float dy);
    void Orientation(int which);   // 0 anterior .. 5 foot
    void SetRenderType(RenderType t) { renderType_ = t; }
    bool TransferVoxel2ImageInVR(float &fx, float &fy, int w, int h, Point3d voxel) const;
    bool VRParams(mk_vr_params &p) const;
    const float *RotateMatrix() const { return rot_; }

    // ---- MPR (MPRInfo.cpp, MPRImageLayer.cpp:84-201) ----
    void ResetPlaneInfos();
    bool PlaneSize(int &w, int &h, PlaneType t) const;
    bool PlaneMaxSize(int &w, int &h, PlaneType t) const;
    bool PlaneParams(mk_plane_params &p, PlaneType t) const;
    void SetMPRType(MPRType t);
    void UpdateThickness(double v);
    void SetThickness(double v, PlaneType t);
    double Thickness(PlaneType t) const;
    double PixelSpacing(PlaneType t) const;
    void Browse(float delta, PlaneType t);
    void PanCrossHair(float x, float y, PlaneType t);
    void RotateCrossHair(float angle, PlaneType t);
    void SetPlaneIndex(int index, PlaneType t);
    bool PlaneIndex(int &index, PlaneType t) const;
    bool PlaneNumber(int &n, PlaneType t) const;
    bool PlaneRotateMatrix(float *m, PlaneType t) const;
    bool CrossHairPoint(double &x, double &y, PlaneType t) const;
    bool TransferImage2Voxel(Point3d &voxel, double x, double y, PlaneType t) const;
    bool Direction2D(Direction2d &h, Direction2d &v, PlaneType t) const;
    bool Direction3D(Direction3d &h, Direction3d &v, PlaneType t) const;
    bool BatchDirection3D(Direction3d &h, Direction3d &v, double angle, PlaneType t) const;
    Point3d CrossHair() const { return crossHair_; }

    // ---- CPR (CPRInfo.cpp) ----
    bool SetCPRLinePatient(const std::vector<Point3d> &line);
    bool SetCPRLineVoxel(const std::vector<Point3d> &line);
    std::vector<Point3d> CPRLineVoxel() const { return cprLine_; }
    bool RotateCPR(float angle, PlaneType t);
    void SetCPRLineColor(RGBA c) { cprColor_ = c; }
    bool CPRRows(std::vector<double> &pts, std::vector<double> &dirs, int &w, int &h, PlaneType t) const;

    // ---- layers and annotations ----
    bool EnableLayer(LayerType t, bool on) {
        layers_[t] = on;
        return true;
    }
    bool LayerEnabled(LayerType t) const;
    bool AddAnnotation(PlaneType t, const std::string &txt, int x, int y, FontSize s, AnnotationFormat f, RGBA c);
    bool RemovePlaneAnnotations(PlaneType t);
    bool RemoveAllAnnotations();
    void ShowPlaneInVR(bool show);

    // ---- rendering through the C ABI ----
    bool RenderVR(std::shared_ptr<unsigned char> &out, int &w, int &h);
    bool RenderPlane(std::shared_ptr<short> &out, int &w, int &h, PlaneType t);
    bool RenderBatch(std::vector<short *> &out, const BatchInfo &info);
    mk_volume DeviceVolume() const { return dev_; }

private:
    void InitCommon();
    void ComputeTransform(float fx, float fz, float scale);
    void ResetCamera();
    void UpdateAlphaWWWL();
    void UploadTransferFunctions();
    void UploadMask();
    bool SyncDevice();
    void UpdateCPRInfo();
    bool CPRStretched(std::vector<Point3d> &pts, std::vector<Direction3d> &dirs, int &w, int &h) const;
    bool CPRStraightened(std::vector<Point3d> &pts, std::vector<Direction3d> &dirs, int &w, int &h) const;
    Point3d CenterPointPlane(Direction3d n) const;
    std::vector<PlaneType> CrossPlaneTypes(PlaneType t) const;
    void UpdatePlaneSize(PlaneType t);
    bool GroupPlanesExist(PlaneType t) const;

    // volume
    std::shared_ptr<short> vol_;
    std::shared_ptr<unsigned char> mask_;
    int dims_[3] = {0, 0, 0};
    double spacing_[3] = {1.0, 1.0, 1.0};
    Direction3d dirX_{1, 0, 0}, dirY_{0, 1, 0}, dirZ_{0, 0, -1};
    Point3d origin_;
    RGBA background_;
    // factors of InitCommon, float (set by SetSpacing)
    float f3Spacing_[3] = {0, 0, 0}, f3SpacingVoxel_[3] = {0, 0, 0}, f3MaxLenSpacing_[3] = {0, 0, 0};

    // labels
    int activeLabel_ = -1;
    std::map<unsigned char, ObjectInfo> objects_;
    float table_[MK_MAX_LABELS][3] = {};   // AlphaAndWWWLInfo as the kernel receives it

    // camera
    float xT_ = 0, yT_ = 0, scale_ = 1;
    float rot_[9], rotT_[9], xf_[9], xfT_[9];
    float kernelMatrix_[9];                // the copy the kernel receives (CuDataManager)
    int vrWidth_ = 512, vrHeight_ = 512;
    RenderType renderType_ = RenderTypeVR;

    // MPR
    std::map<PlaneType, PlaneInfo> planes_;
    Point3d crossHair_, center_;

    // CPR
    std::vector<Point3d> cprLine_;
    Direction3d cprDirStretched_{0, 0, 1};
    Point3d cprOriginStretched_, cprOriginStraightened_;
    double cprAngleStretched_ = 0, cprAngleStraightened_ = 0;
    double cprMinSpacing_ = 1.0;
    Point3d cprSpacing_;
    double cprStretchedRadius_ = 0.0, cprStraightenedRadius_ = 50.0;
    RGBA cprColor_{1.0f, 1.0f, 1.0f};

    // layers / annotations
    std::map<LayerType, bool> layers_;
    std::vector<Annotation> annotations_;
    int planeLabel_ = 0;

    // orientation box mesh (./resources/human.stl at construction, as
    // MonkeyGL's MarchingCube loads it); null when the file is absent
    mk_mesh mesh_ = nullptr;
    mk_font font_ = nullptr;          // annotation glyphs (./resources/annotation_glyphs.bin)

    // device
    mk_volume dev_ = nullptr;
    bool tfDirty_ = true, tableDirty_ = true, maskDirty_ = false, volumeDirty_ = false;
    // the device holds the mask as of the last upload; voxels changed since
    // lie in maskBox_ (x0, y0, z0, x1, y1, z1, exclusive; empty when x0 >= x1)
    bool maskOnDevice_ = false;
    int maskBox_[6] = {0, 0, 0, 0, 0, 0};
    void GrowMaskBox(int x, int y, int z);
};

}  // namespace detail
}  // namespace MonkeyGL
