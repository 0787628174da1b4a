// pymonkeygl.cpp -- the pyMonkeyGL Python module (pybind11) over the MonkeyGL
// C++ API of this library.  Names, enumerations and array conventions follow
// MonkeyGL's module (pybind11_interface/PybindInterface.cpp:112-351):
//   * SetVolumeArray / AddNewObjectMaskArray / UpdateMaskArray take an array
//     whose shape[0..2] is (width, height, depth) and whose raw buffer is
//     x-fastest (a (z, y, x) numpy array viewed with swapaxes(2, 0));
//   * GetVRArray returns a (3, w, h) array over the interleaved RGB bytes of
//     the VR image; GetVolumeArray returns the volume as (w, h, d).
// Additions beyond MonkeyGL's module: GetPlaneArray (int16 plane as (h, w)),
// GetVRImage ((h, w, 3) RGB), and introspection of the kernel arguments.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstring>

#include "../../include/monkeygl/HelloMonkey.h"
#include "../../include/monkeygl_b200.h"

namespace py = pybind11;
using namespace MonkeyGL;

namespace {

template <typename T>
std::shared_ptr<T> array3d_to_ptr(py::array_t<T> a, int &w, int &h, int &d) {
    py::buffer_info b = a.request();
    if (b.ndim != 3) throw std::invalid_argument("expected a 3-D array");
    w = (int)b.shape[0];
    h = (int)b.shape[1];
    d = (int)b.shape[2];
    std::shared_ptr<T> p(new T[b.size], std::default_delete<T[]>());
    // the buffer is copied as it lies in memory (MonkeyGL's _arrays_3d_to_ptr)
    py::array_t<T, py::array::c_style | py::array::forcecast> flat(a);
    if (!(a.flags() & py::array::c_style) && !(a.flags() & py::array::f_style)) {
        std::memcpy(p.get(), flat.data(), b.size * sizeof(T));
    } else {
        std::memcpy(p.get(), b.ptr, b.size * sizeof(T));
    }
    return p;
}

// (N, 3) points; float32 input converts exactly, float64 keeps full precision
// (MonkeyGL's binding rounds every point to float32)
std::vector<Point3d> points_from_array(py::array_t<double> a) {
    std::vector<Point3d> out;
    py::buffer_info b = a.request();
    if (b.ndim != 2 || b.shape[1] != 3) return out;
    py::array_t<double, py::array::c_style | py::array::forcecast> c(a);
    const double *p = c.data();
    for (ssize_t i = 0; i < b.shape[0]; ++i) out.emplace_back(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    return out;
}

class PyHelloMonkey : public HelloMonkey {
public:
    bool SetVolumeArray(py::array_t<short> a) {
        int w, h, d;
        auto p = array3d_to_ptr<short>(a, w, h, d);
        return SetVolumeData(p, w, h, d);
    }
    unsigned char AddNewObjectMaskArray(py::array_t<unsigned char> a) {
        int w, h, d;
        auto p = array3d_to_ptr<unsigned char>(a, w, h, d);
        return AddNewObjectMask(p, w, h, d);
    }
    bool UpdateMaskArray(py::array_t<unsigned char> a, const unsigned char &label) {
        int w, h, d;
        auto p = array3d_to_ptr<unsigned char>(a, w, h, d);
        return UpdateObjectMask(p, w, h, d, label);
    }
    py::array_t<short> GetVolumeArray() {
        int w = 0, h = 0, d = 0;
        auto p = GetVolumeData(w, h, d);
        py::array_t<short> out({(ssize_t)w, (ssize_t)h, (ssize_t)d});
        if (p) std::memcpy(out.mutable_data(), p.get(), (size_t)w * h * d * sizeof(short));
        return out;
    }
    // (3, w, h) over the interleaved RGB bytes, as MonkeyGL returns it
    py::array_t<unsigned char> GetVRArray(int, int) {
        int w = 0, h = 0;
        GetVRSize(w, h);
        std::shared_ptr<unsigned char> p;
        py::array_t<unsigned char> out({(ssize_t)3, (ssize_t)w, (ssize_t)h});
        if (GetVRData(p, w, h) && p) std::memcpy(out.mutable_data(), p.get(), (size_t)w * h * 3);
        else std::memset(out.mutable_data(), 0, (size_t)w * h * 3);
        return out;
    }
    // addition: the same image as (h, w, 3)
    py::array_t<unsigned char> GetVRImage() {
        int w = 0, h = 0;
        GetVRSize(w, h);
        std::shared_ptr<unsigned char> p;
        py::array_t<unsigned char> out({(ssize_t)h, (ssize_t)w, (ssize_t)3});
        if (!GetVRData(p, w, h) || !p) throw std::runtime_error(std::string("GetVRData failed: ") + mk_last_error());
        std::memcpy(out.mutable_data(), p.get(), (size_t)w * h * 3);
        return out;
    }
    // addition: int16 plane (MPR or CPR) as (h, w)
    py::array_t<short> GetPlaneArray(PlaneType t) {
        int w = 0, h = 0;
        std::shared_ptr<short> p;
        if (!GetPlaneData(p, w, h, t) || !p)
            throw std::runtime_error(std::string("GetPlaneData failed: ") + mk_last_error());
        py::array_t<short> out({(ssize_t)h, (ssize_t)w});
        std::memcpy(out.mutable_data(), p.get(), (size_t)w * h * sizeof(short));
        return out;
    }
    py::array_t<uint8_t> GetVRDataArray_png(int w, int h) {
        std::vector<uint8_t> v = GetVRData_png(w, h);
        py::array_t<uint8_t> out((ssize_t)v.size());
        if (!v.empty()) std::memcpy(out.mutable_data(), v.data(), v.size());
        return out;
    }
    void Transfer2Base64Array(py::array_t<unsigned char> a) {
        py::buffer_info b = a.request();
        if (b.ndim != 2) throw std::invalid_argument("expected a 2-D array");
        py::array_t<unsigned char, py::array::c_style | py::array::forcecast> c(a);
        Transfer2Base64(const_cast<unsigned char *>(c.data()), (int)b.shape[0], (int)b.shape[1]);
    }
    bool SetCPRLinePatientArray(py::array_t<double> a) { return SetCPRLinePatient(points_from_array(a)); }
    bool SetCPRLineVoxelArray(py::array_t<double> a) { return SetCPRLineVoxel(points_from_array(a)); }
    int GetPlaneCurrentIndex(PlaneType t) {
        int i = -1;
        GetPlaneIndex(i, t);
        return i;
    }
    int GetPlaneTotalNumber(PlaneType t) {
        int n = 0;
        GetPlaneNumber(n, t);
        return n;
    }
    // ---- introspection -------------------------------------------------
    py::dict VRParams() {
        mk_vr_params p;
        py::dict d;
        if (!GetVRParams(p)) return d;
        d["width"] = p.width;
        d["height"] = p.height;
        d["render_type"] = p.render_type;
        d["max_len_spacing"] = std::vector<float>(p.max_len_spacing, p.max_len_spacing + 3);
        d["spacing"] = std::vector<float>(p.spacing, p.spacing + 3);
        d["spacing_voxel"] = std::vector<float>(p.spacing_voxel, p.spacing_voxel + 3);
        d["x_translate"] = p.x_translate;
        d["y_translate"] = p.y_translate;
        d["scale"] = p.scale;
        d["transform"] = std::vector<float>(p.transform, p.transform + 9);
        d["invert_z"] = p.invert_z;
        d["voi"] = std::vector<int>(p.voi, p.voi + 6);
        d["background"] = std::vector<float>(p.background, p.background + 4);
        return d;
    }
    py::dict PlaneParams(PlaneType t) {
        mk_plane_params p;
        py::dict d;
        if (!GetPlaneParams(p, t)) return d;
        d["width"] = p.width;
        d["height"] = p.height;
        d["mpr_type"] = p.mpr_type;
        d["spacing"] = std::vector<float>(p.spacing, p.spacing + 3);
        d["dir_h"] = std::vector<float>(p.dir_h, p.dir_h + 3);
        d["dir_v"] = std::vector<float>(p.dir_v, p.dir_v + 3);
        d["dir_n"] = std::vector<float>(p.dir_n, p.dir_n + 3);
        d["left_top"] = std::vector<float>(p.left_top, p.left_top + 3);
        d["pixel_spacing"] = p.pixel_spacing;
        d["invert_z"] = p.invert_z;
        d["half_num"] = p.half_num;
        return d;
    }
    py::tuple CPRRows(PlaneType t) {
        std::vector<double> pts, dirs;
        int w = 0, h = 0;
        if (!GetCPRRows(pts, dirs, w, h, t)) return py::make_tuple();
        py::array_t<double> P({(ssize_t)h, (ssize_t)3}), D({(ssize_t)h, (ssize_t)3});
        std::memcpy(P.mutable_data(), pts.data(), pts.size() * sizeof(double));
        std::memcpy(D.mutable_data(), dirs.data(), dirs.size() * sizeof(double));
        return py::make_tuple(w, h, P, D);
    }
    py::array_t<float> LabelTable() {
        std::vector<float> t = GetLabelTable();
        py::array_t<float> out({(ssize_t)MK_MAX_LABELS, (ssize_t)3});
        std::memcpy(out.mutable_data(), t.data(), t.size() * sizeof(float));
        return out;
    }
    py::object TransferFunctionLUT(unsigned char label) {
        std::vector<float> v;
        if (!GetTransferFunctionLUT(v, label)) return py::none();
        py::array_t<float> out({(ssize_t)(v.size() / 4), (ssize_t)4});
        std::memcpy(out.mutable_data(), v.data(), v.size() * sizeof(float));
        return out;
    }
    py::tuple CrossHairPoint3D() {
        Point3d p;
        GetCrossHairPoint3D(p);
        return py::make_tuple(p.x(), p.y(), p.z());
    }
    py::tuple Direction3D(PlaneType t) {
        Direction3d h, v;
        if (!GetDirection3D(h, v, t)) return py::make_tuple();
        return py::make_tuple(py::make_tuple(h.x(), h.y(), h.z()), py::make_tuple(v.x(), v.y(), v.z()));
    }
};

}  // namespace

PYBIND11_MODULE(pyMonkeyGL, m) {
    m.doc() = "MonkeyGL API on the B200 ray-casting kernels";

    py::enum_<LogLevel>(m, "LogLevel")
        .value("LogLevelNotDefined", LogLevelNotDefined)
        .value("LogLevelInfo", LogLevelInfo)
        .value("LogLevelWarn", LogLevelWarn)
        .value("LogLevelError", LogLevelError)
        .export_values();
    py::enum_<PlaneType>(m, "PlaneType")
        .value("PlaneNotDefined", PlaneNotDefined)
        .value("PlaneAxial", PlaneAxial)
        .value("PlaneSagittal", PlaneSagittal)
        .value("PlaneCoronal", PlaneCoronal)
        .value("PlaneAxialOblique", PlaneAxialOblique)
        .value("PlaneSagittalOblique", PlaneSagittalOblique)
        .value("PlaneCoronalOblique", PlaneCoronalOblique)
        .value("PlaneVR", PlaneVR)
        .value("PlaneStretchedCPR", PlaneStretchedCPR)
        .value("PlaneStraightenedCPR", PlaneStraightenedCPR)
        .export_values();
    py::enum_<Orientation>(m, "Orientation")
        .value("OrientationNotDefined", OrientationNotDefined)
        .value("OrientationAnterior", OrientationAnterior)
        .value("OrientationPosterior", OrientationPosterior)
        .value("OrientationLeft", OrientationLeft)
        .value("OrientationRight", OrientationRight)
        .value("OrientationHead", OrientationHead)
        .value("OrientationFoot", OrientationFoot)
        .export_values();
    py::enum_<MPRType>(m, "MPRType")
        .value("MPRTypeNotDefined", MPRTypeNotDefined)
        .value("MPRTypeAverage", MPRTypeAverage)
        .value("MPRTypeMIP", MPRTypeMIP)
        .value("MPRTypeMinIP", MPRTypeMinIP)
        .export_values();
    py::enum_<RenderType>(m, "RenderType")
        .value("RenderTypeNotDefined", RenderTypeNotDefined)
        .value("RenderTypeVR", RenderTypeVR)
        .value("RenderTypeMIP", RenderTypeMIP)
        .value("RenderTypeSurface", RenderTypeSurface)
        .export_values();
    py::enum_<LayerType>(m, "LayerType")
        .value("LayerTypeNotDefined", LayerTypeNotDefined)
        .value("LayerTypeImage", LayerTypeImage)
        .value("LayerTypeAnnotation", LayerTypeAnnotation)
        .value("LayerTypeCPRLine", LayerTypeCPRLine)
        .export_values();
    py::enum_<FontSize>(m, "FontSize")
        .value("FontSizeNotDefined", FontSizeNotDefined)
        .value("FontSizeSmall", FontSizeSmall)
        .value("FontSizeMiddle", FontSizeMiddle)
        .value("FontSizeBig", FontSizeBig)
        .export_values();
    py::enum_<AnnotationFormat>(m, "AnnotationFormat")
        .value("AnnotationFormatNotDefined", AnnotationFormatNotDefined)
        .value("AnnotationFormatLeft", AnnotationFormatLeft)
        .value("AnnotationFormatRight", AnnotationFormatRight)
        .value("AnnotationFormatCenter", AnnotationFormatCenter)
        .export_values();

    struct DeviceInfo {
        int GetCount() {
            int n = 0;
            mk_device_count(&n);
            return n;
        }
    };
    py::class_<DeviceInfo>(m, "DeviceInfo").def(py::init<>()).def("GetCount", &DeviceInfo::GetCount);

    py::class_<RGBA>(m, "RGBA")
        .def(py::init<>())
        .def(py::init<float, float, float>())
        .def(py::init<float, float, float, float>())
        .def_readwrite("red", &RGBA::red)
        .def_readwrite("green", &RGBA::green)
        .def_readwrite("blue", &RGBA::blue)
        .def_readwrite("alpha", &RGBA::alpha)
        .def("Print", &RGBA::Print);
    py::class_<Direction3d>(m, "Direction3d")
        .def(py::init<>())
        .def(py::init<double, double, double>())
        .def("x", &Direction3d::x)
        .def("y", &Direction3d::y)
        .def("z", &Direction3d::z);
    py::class_<Point2d>(m, "Point2d")
        .def(py::init<>())
        .def(py::init<double, double>())
        .def("x", &Point2d::x)
        .def("y", &Point2d::y)
        .def("SetX", &Point2d::SetX)
        .def("SetY", &Point2d::SetY);
    py::class_<Point3d>(m, "Point3d")
        .def(py::init<>())
        .def(py::init<double, double, double>())
        .def("x", &Point3d::x)
        .def("y", &Point3d::y)
        .def("z", &Point3d::z)
        .def("SetX", &Point3d::SetX)
        .def("SetY", &Point3d::SetY)
        .def("SetZ", &Point3d::SetZ);

    using H = PyHelloMonkey;
    py::class_<H>(m, "HelloMonkey")
        .def(py::init<>())
        .def("SetLogLevel", &H::SetLogLevel)
        .def("LoadVolumeFile", &H::LoadVolumeFile)
        .def("SetVolumeArray", &H::SetVolumeArray)
        .def("AddObjectMaskFile", &H::AddObjectMaskFile)
        .def("AddNewObjectMaskArray", &H::AddNewObjectMaskArray)
        .def("UpdateMaskArray", &H::UpdateMaskArray)
        .def("SetSpacing", &H::SetSpacing)
        .def("SetDirection", &H::SetDirection)
        .def("SetOrigin", &H::SetOrigin)
        .def("SetTransferFunc", static_cast<bool (H::*)(std::map<int, RGBA>)>(&H::SetTransferFunc))
        .def("SetTransferFunc", static_cast<bool (H::*)(std::map<int, RGBA>, unsigned char)>(&H::SetTransferFunc))
        .def("SetTransferFunc",
             static_cast<bool (H::*)(std::map<int, RGBA>, std::map<int, float>)>(&H::SetTransferFunc))
        .def("SetTransferFunc", static_cast<bool (H::*)(std::map<int, RGBA>, std::map<int, float>, unsigned char)>(
                                    &H::SetTransferFunc))
        .def("LoadTransferFunction", &H::LoadTransferFunction)
        .def("SaveTransferFunction", &H::SaveTransferFunction)
        .def("SetColorBackground", &H::SetColorBackground)
        .def("Reset", &H::Reset)
        .def("Anterior", &H::Anterior)
        .def("Posterior", &H::Posterior)
        .def("Left", &H::Left)
        .def("Right", &H::Right)
        .def("Head", &H::Head)
        .def("Foot", &H::Foot)
        .def("SetVRWWWL", static_cast<bool (H::*)(float, float)>(&H::SetVRWWWL))
        .def("SetVRWWWL", static_cast<bool (H::*)(float, float, unsigned char)>(&H::SetVRWWWL))
        .def("SetObjectAlpha", static_cast<bool (H::*)(float)>(&H::SetObjectAlpha))
        .def("SetObjectAlpha", static_cast<bool (H::*)(float, unsigned char)>(&H::SetObjectAlpha))
        .def("SetRenderType", &H::SetRenderType)
        .def("Rotate", &H::Rotate)
        .def("Pan", &H::Pan)
        .def("Zoom", &H::Zoom)
        .def("UpdateThickness", &H::UpdateThickness)
        .def("SetThickness", &H::SetThickness)
        .def("GetThickness", &H::GetThickness)
        .def("SetMPRType", &H::SetMPRType)
        .def("Browse", &H::Browse)
        .def("PanCrossHair", &H::PanCrossHair)
        .def("RotateCrossHair", &H::RotateCrossHair)
        .def("SetCPRLinePatientArray", &H::SetCPRLinePatientArray)
        .def("SetCPRLineVoxelArray", &H::SetCPRLineVoxelArray)
        .def("RotateCPR", &H::RotateCPR)
        .def("SetCPRLineColor", &H::SetCPRLineColor)
        .def("SetVRSize", &H::SetVRSize)
        .def("ShowPlaneInVR", &H::ShowPlaneInVR)
        .def("SetPlaneIndex", &H::SetPlaneIndex)
        .def("Transfer2Base64Array", &H::Transfer2Base64Array)
        .def("AddAnnotation", &H::AddAnnotation)
        .def("RemovePlaneAnnotations", &H::RemovePlaneAnnotations)
        .def("RemoveAllAnnotations", &H::RemoveAllAnnotations)
        .def("EnableLayer", &H::EnableLayer)
        .def("GetZoomRatio", &H::GetZoomRatio)
        .def("GetPlaneCurrentIndex", &H::GetPlaneCurrentIndex)
        .def("GetPlaneTotalNumber", &H::GetPlaneTotalNumber)
        .def("GetVolumeArray", &H::GetVolumeArray)
        .def("GetVRArray", &H::GetVRArray)
        .def("GetVRData_pngString", &H::GetVRData_pngString)
        .def("GetVRData_png", &H::GetVRDataArray_png)
        .def("SaveVR2Png", &H::SaveVR2Png)
        .def("GetPlaneData_pngString", &H::GetPlaneData_pngString)
        .def("GetOriginData_pngString", &H::GetOriginData_pngString)
        .def("GetCrossHairPoint", static_cast<Point2d (H::*)(const PlaneType &)>(&H::GetCrossHairPoint))
        .def("GetPlaneIndex", static_cast<int (H::*)(const PlaneType &)>(&H::GetPlaneIndex))
        .def("GetPlaneNumber", static_cast<int (H::*)(const PlaneType &)>(&H::GetPlaneNumber))
        .def("GetPixelSpacing", &H::GetPixelSpacing)
        // additions
        .def("GetVRImage", &H::GetVRImage)
        .def("GetPlaneArray", &H::GetPlaneArray)
        .def("GetVRParams", &H::VRParams)
        .def("GetPlaneParams", &H::PlaneParams)
        .def("GetCPRRows", &H::CPRRows)
        .def("GetLabelTable", &H::LabelTable)
        .def("GetTransferFunctionLUT", &H::TransferFunctionLUT)
        .def("GetCrossHairPoint3D", &H::CrossHairPoint3D)
        .def("GetDirection3D", &H::Direction3D);
}
