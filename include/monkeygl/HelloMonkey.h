// HelloMonkey.h -- the MonkeyGL C++ API (namespace MonkeyGL), implemented on
// the B200 kernels of include/monkeygl_b200.h.
//
// Every virtual method of MonkeyGL's HelloMonkey (core/HelloMonkey.h:36-139)
// is present with the same signature and meaning.  Differences:
//   * each HelloMonkey instance owns its own state and resident volume
//     (MonkeyGL shares one process-wide DataManager between all instances,
//     core/DataManager.cpp:46-54);
//   * errors are reported through the documented return values, never by
//     exiting the process;
//   * the methods below "Introspection" are additions: they return the exact
//     kernel arguments a render call would use.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../monkeygl_b200.h"
#include "Defines.h"

namespace MonkeyGL {

class IRender;

class HelloMonkey {
public:
    HelloMonkey();
    virtual ~HelloMonkey();

    virtual void SetLogLevel(LogLevel level);
    virtual void LoadVolumeFile(const char *szFile);
    virtual void SetDirection(Direction3d dirX, Direction3d dirY, Direction3d dirZ);
    virtual void SetSpacing(double x, double y, double z);
    virtual void SetOrigin(Point3d pt);
    virtual void Reset();
    virtual void SetColorBackground(RGBA clrBG);
    virtual bool SetVolumeData(std::shared_ptr<short> pData, int nWidth, int nHeight, int nDepth);
    virtual unsigned char AddNewObjectMask(std::shared_ptr<unsigned char> pData, int nWidth, int nHeight,
                                           int nDepth);
    virtual unsigned char AddObjectMaskFile(const char *szFile);
    virtual bool UpdateObjectMask(std::shared_ptr<unsigned char> pData, int nWidth, int nHeight, int nDepth,
                                  const unsigned char &nLabel);

    // output
    virtual std::shared_ptr<short> GetVolumeData(int &nWidth, int &nHeight, int &nDepth);
    virtual bool GetPlaneMaxSize(int &nWidth, int &nHeight, const PlaneType &planeType);
    virtual bool GetPlaneData(std::shared_ptr<short> &pData, int &nWidth, int &nHeight,
                              const PlaneType &planeType);
    virtual std::string GetPlaneData_pngString(const PlaneType &planeType);
    virtual std::string GetOriginData_pngString(int slice);

    virtual bool GetCrossHairPoint(double &x, double &y, const PlaneType &planeType);
    virtual Point2d GetCrossHairPoint(const PlaneType &planeType);
    virtual bool TransferImage2Voxel(double &x, double &y, double &z, double xImage, double yImage,
                                     PlaneType planeType);
    virtual bool GetCrossHairPoint3D(Point3d &pt);
    virtual bool GetDirection(Direction2d &dirH, Direction2d &dirV, const PlaneType &planeType);
    virtual bool GetDirection3D(Direction3d &dir3dH, Direction3d &dir3dV, const PlaneType &planeType);
    virtual bool GetBatchDirection3D(Direction3d &dir3dH, Direction3d &dir3dV, double fAngle,
                                     const PlaneType &planeType);

    virtual double GetPixelSpacing(PlaneType planeType);

    virtual bool SetVRSize(int nWidth, int nHeight);
    virtual bool GetVRData(std::shared_ptr<unsigned char> &pData, int nWidth, int nHeight);
    virtual std::string GetVRData_pngString();
    virtual std::vector<uint8_t> GetVRData_png(int nWidth, int nHeight);
    virtual void SaveVR2Png(const char *szFile, int nWidth, int nHeight);

    virtual bool GetBatchData(std::vector<short *> &vecBatchData, const BatchInfo &batchInfo);

    virtual bool GetPlaneIndex(int &index, const PlaneType &planeType);
    virtual int GetPlaneIndex(const PlaneType &planeType);
    virtual bool GetPlaneNumber(int &nTotalNum, const PlaneType &planeType);
    virtual int GetPlaneNumber(const PlaneType &planeType);

    virtual bool GetPlaneRotateMatrix(float *pMatrix, PlaneType planeType);

    // interactions
    virtual void Anterior();
    virtual void Posterior();
    virtual void Left();
    virtual void Right();
    virtual void Head();
    virtual void Foot();

    virtual void SetRenderType(RenderType type);
    virtual void Rotate(float fxRotate, float fyRotate);
    virtual float Zoom(float ratio);
    virtual float GetZoomRatio();
    virtual void Pan(float fxShift, float fyShift);
    virtual bool SetVRWWWL(float fWW, float fWL);
    virtual bool SetVRWWWL(float fWW, float fWL, unsigned char nLabel);
    virtual bool SetObjectAlpha(float fAlpha);
    virtual bool SetObjectAlpha(float fAlpha, unsigned char nLabel);
    virtual bool SetTransferFunc(std::map<int, RGBA> ctrlPoints);
    virtual bool SetTransferFunc(std::map<int, RGBA> ctrlPoints, unsigned char nLabel);
    virtual bool SetTransferFunc(std::map<int, RGBA> rgbPoints, std::map<int, float> alphaPoints);
    virtual bool SetTransferFunc(std::map<int, RGBA> rgbPoints, std::map<int, float> alphaPoints,
                                 unsigned char nLabel);
    virtual bool LoadTransferFunction(const char *szFile);
    virtual bool SaveTransferFunction(const char *szFile);

    virtual void Browse(float fDelta, PlaneType planeType);
    virtual void PanCrossHair(float fx, float fy, PlaneType planeType);
    virtual void RotateCrossHair(float fAngle, PlaneType planeType);
    virtual void SetPlaneIndex(int index, PlaneType planeType);

    virtual void UpdateThickness(double val);
    virtual void SetThickness(double val, PlaneType planeType);
    virtual double GetThickness(PlaneType planeType);
    virtual void SetMPRType(MPRType type);

    virtual bool AddAnnotation(PlaneType planeType, std::string txt, int x, int y, FontSize fontSize,
                               AnnotationFormat annoFormat, RGBA clr);
    virtual bool RemovePlaneAnnotations(PlaneType planeType);
    virtual bool RemoveAllAnnotations();
    virtual bool EnableLayer(LayerType layerType, bool bEnable);

    // cpr
    virtual bool SetCPRLinePatient(std::vector<Point3d> cprLine);
    virtual bool SetCPRLineVoxel(std::vector<Point3d> cprLine);
    virtual bool RotateCPR(float angle, PlaneType planeType);
    virtual void SetCPRLineColor(RGBA clr);

    // plane in VR
    virtual void ShowPlaneInVR(bool bShow);

    virtual void Transfer2Base64(unsigned char *pData, int nWidth, int nHeight);

    // ---- Introspection (additions) ---------------------------------------
    // VR size after SetVRSize's reduction (what GetVRData renders).
    void GetVRSize(int &nWidth, int &nHeight);
    // Kernel arguments of the next GetVRData call.
    bool GetVRParams(mk_vr_params &params);
    // Per-label (alpha, ww, wl) table as the kernel receives it (65 rows).
    std::vector<float> GetLabelTable();
    // Kernel arguments of GetPlaneData for an MPR plane.
    bool GetPlaneParams(mk_plane_params &params, PlaneType planeType);
    // Rows of GetPlaneData for a CPR plane: points and directions (voxel
    // units, 3 doubles per row) and the image size.
    bool GetCPRRows(std::vector<double> &points, std::vector<double> &dirs, int &nWidth, int &nHeight,
                    PlaneType planeType);
    // The 100-entry RGBA LUT built from a label's control points.
    bool GetTransferFunctionLUT(std::vector<float> &rgba, unsigned char nLabel);
    // The resident device volume (nullptr before SetVolumeData or without a GPU).
    mk_volume GetDeviceVolume();

private:
    std::shared_ptr<IRender> m_pRender;
};

}  // namespace MonkeyGL
