// Defines.h -- value types and enumerations of the MonkeyGL C++ API
// (namespace MonkeyGL), as used by HelloMonkey / IRender.  Names, enumerator
// values and member semantics match MonkeyGL's core/Defines.h, core/Point.h
// and core/Direction.h so that code written against MonkeyGL compiles and
// behaves the same against this library.
#pragma once

#include <cmath>
#include <cstring>
#include <iostream>
#include <string>

namespace MonkeyGL {

constexpr int MAXOBJECTCOUNT = 64;   // labels 1..64 plus background 0
constexpr double PI = 3.141592654;   // MonkeyGL's value of pi

// RGBA colour with components in [0, 1]; the three-component constructor
// sets alpha to 1, arithmetic results are clamped to [0, 1].
struct RGBA {
    float red = 0.0f, green = 0.0f, blue = 0.0f, alpha = 0.0f;

    RGBA() = default;
    RGBA(float r, float g, float b) : red(r), green(g), blue(b), alpha(1.0f) {}
    RGBA(float r, float g, float b, float a) : red(r), green(g), blue(b), alpha(a) {}

    void trim() {
        auto c = [](float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); };
        red = c(red);
        green = c(green);
        blue = c(blue);
        alpha = c(alpha);
    }
    RGBA operator*(float r) const {
        RGBA o(red * r, green * r, blue * r, alpha * r);
        o.trim();
        return o;
    }
    RGBA operator*=(float r) {
        *this = *this * r;
        return *this;
    }
    RGBA operator+(float d) const {
        RGBA o(red + d, green + d, blue + d, alpha + d);
        o.trim();
        return o;
    }
    void Print() const {
        std::cout << "red: " << red << "\ngreen: " << green << "\nblue: " << blue
                  << "\nalpha: " << alpha << std::endl;
    }
};

enum Orientation {
    OrientationNotDefined = -1,
    OrientationAnterior,
    OrientationPosterior,
    OrientationLeft,
    OrientationRight,
    OrientationHead,
    OrientationFoot
};

enum PlaneType {
    PlaneNotDefined = -1,
    PlaneAxial,
    PlaneSagittal,
    PlaneCoronal,
    PlaneAxialOblique,
    PlaneSagittalOblique,
    PlaneCoronalOblique,
    PlaneVR,
    PlaneStretchedCPR,
    PlaneStraightenedCPR
};

std::string PlaneTypeName(PlaneType planeType);

enum MPRType { MPRTypeNotDefined = -1, MPRTypeAverage, MPRTypeMIP, MPRTypeMinIP };

enum RenderType { RenderTypeNotDefined = -1, RenderTypeVR, RenderTypeMIP, RenderTypeSurface };

enum LogLevel { LogLevelNotDefined = -1, LogLevelInfo, LogLevelWarn, LogLevelError };

enum FontSize { FontSizeNotDefined = -1, FontSizeSmall, FontSizeMiddle, FontSizeBig };

enum AnnotationFormat {
    AnnotationFormatNotDefined = -1,
    AnnotationFormatLeft,
    AnnotationFormatRight,
    AnnotationFormatCenter
};

enum LayerType {
    LayerTypeNotDefined = -1,
    LayerTypeImage,
    LayerTypeAnnotation,
    LayerTypeCPRLine
};

// Point in dim dimensions (zero-initialised).
template <class T, unsigned char dim>
class Point {
public:
    Point() { std::memset(c_, 0, sizeof(c_)); }
    Point(T x, T y) {
        std::memset(c_, 0, sizeof(c_));
        c_[0] = x;
        c_[1] = y;
    }
    Point(T x, T y, T z) {
        c_[0] = x;
        c_[1] = y;
        if (dim == 3) c_[dim - 1] = z;
    }
    T x() const { return c_[0]; }
    T y() const { return c_[1]; }
    T z() const { return dim == 3 ? c_[dim - 1] : T(0); }
    void SetX(T v) { c_[0] = v; }
    void SetY(T v) { c_[1] = v; }
    void SetZ(T v) {
        if (dim == 3) c_[dim - 1] = v;
    }
    void Set(T x, T y) {
        c_[0] = x;
        c_[1] = y;
    }
    void Set(T x, T y, T z) {
        c_[0] = x;
        c_[1] = y;
        SetZ(z);
    }
    T &operator[](int i) { return c_[i]; }
    T operator[](int i) const { return c_[i]; }
    double DistanceTo(const Point &p) const {
        double s = 0;
        for (int i = 0; i < dim; ++i) s += (double)(c_[i] - p.c_[i]) * (c_[i] - p.c_[i]);
        return std::sqrt(s);
    }
    // distance with per-axis scale factors (voxel -> millimetre)
    double PatientDistanceTo(const Point &p, const Point &spacing) const {
        double s = 0;
        for (int i = 0; i < dim; ++i)
            s += (double)(c_[i] - p.c_[i]) * (c_[i] - p.c_[i]) * spacing.c_[i] * spacing.c_[i];
        return std::sqrt(s);
    }
    Point operator+(const Point &p) const {
        Point o;
        for (int i = 0; i < dim; ++i) o.c_[i] = c_[i] + p.c_[i];
        return o;
    }
    Point operator-(const Point &p) const {
        Point o;
        for (int i = 0; i < dim; ++i) o.c_[i] = c_[i] - p.c_[i];
        return o;
    }
    Point operator*(T f) const {
        Point o;
        for (int i = 0; i < dim; ++i) o.c_[i] = c_[i] * f;
        return o;
    }
    Point operator/(const Point &p) const {
        Point o;
        for (int i = 0; i < dim; ++i) o.c_[i] = c_[i] / p.c_[i];
        return o;
    }
    Point &operator+=(const Point &p) {
        for (int i = 0; i < dim; ++i) c_[i] += p.c_[i];
        return *this;
    }
    Point &operator-=(const Point &p) {
        for (int i = 0; i < dim; ++i) c_[i] -= p.c_[i];
        return *this;
    }
    Point &operator/=(const Point &p) {
        for (int i = 0; i < dim; ++i) c_[i] /= p.c_[i];
        return *this;
    }

private:
    T c_[dim];
};

// Unit direction: every constructor from components or from two points
// normalises; the default direction is +x.
template <class T, unsigned char dim>
class Direction {
public:
    Direction() {
        std::memset(c_, 0, sizeof(c_));
        c_[0] = 1;
    }
    Direction(T x, T y) {
        std::memset(c_, 0, sizeof(c_));
        c_[0] = x;
        c_[1] = y;
        normalize();
    }
    Direction(T x, T y, T z) {
        c_[0] = x;
        c_[1] = y;
        if (dim == 3) c_[dim - 1] = z;
        normalize();
    }
    Direction(const Point<T, dim> &from, const Point<T, dim> &to) {
        for (int i = 0; i < dim; ++i) c_[i] = to[i] - from[i];
        normalize();
    }
    T x() const { return c_[0]; }
    T y() const { return c_[1]; }
    T z() const { return dim == 3 ? c_[dim - 1] : T(0); }
    void SetX(T v) { c_[0] = v; }
    void SetY(T v) { c_[1] = v; }
    void SetZ(T v) {
        if (dim == 3) c_[dim - 1] = v;
    }
    T Length() const {
        T s = 0;
        for (int i = 0; i < dim; ++i) s += c_[i] * c_[i];
        return std::sqrt(s);
    }
    T dot(const Direction &d) const {
        T v = 0;
        for (int i = 0; i < dim; ++i) v += c_[i] * d.c_[i];
        return v;
    }
    Direction cross(const Direction &d) const {
        if (dim != 3) return Direction();
        return Direction(y() * d.z() - z() * d.y(), z() * d.x() - x() * d.z(), x() * d.y() - y() * d.x());
    }
    Direction negative() const {
        if (dim != 3) return Direction();
        return Direction(-x(), -y(), -z());
    }
    Point<T, dim> operator*(T f) const {
        Point<T, dim> p;
        p.SetX(x() * f);
        p.SetY(y() * f);
        if (dim == 3) p.SetZ(z() * f);
        return p;
    }

private:
    void normalize() {
        T n = Length();
        for (int i = 0; i < dim; ++i) c_[i] /= n;
    }
    T c_[dim];
};

typedef Point<double, 3> Point3d;
typedef Point<double, 2> Point2d;
typedef Point<float, 3> Point3f;
typedef Point<float, 2> Point2f;
typedef Direction<double, 3> Direction3d;
typedef Direction<double, 2> Direction2d;
typedef Direction<float, 3> Direction3f;
typedef Direction<float, 2> Direction2f;

// Batch reslice request (core/BatchInfo.h): a stack of parallel planes.
struct BatchInfo {
    Direction3d m_dirH;
    Direction3d m_dirV;
    Point3d m_ptCenter;
    double m_fLengthH = 0.0;
    double m_fLengthV = 0.0;
    double m_fPixelSpacing = 0.0;
    double m_fSliceThickness = 0.0;
    double m_fSliceDistance = 0.0;
    int m_nNum = 0;
    MPRType m_MPRType = MPRTypeAverage;

    int Width() const { return int(m_fLengthH / m_fPixelSpacing); }
    int Height() const { return int(m_fLengthV / m_fPixelSpacing); }
};

}  // namespace MonkeyGL
