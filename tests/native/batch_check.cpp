// GPU check of HelloMonkey::GetBatchData, driven from C++ as a caller of the
// MonkeyGL API would.  MonkeyGL declares GetBatchData with its BatchInfo
// (core/HelloMonkey.cpp:415-419, core/BatchInfo.h:29-54) but its Render
// returns false (core/Render.cpp:117-120); this library renders the stack:
// m_nNum parallel planes m_fSliceDistance apart along dirH x dirV, centred on
// m_ptCenter, each Width() x Height() int16, slab of
// max(1, int(thickness / pixel spacing)) samples.  Checks:
//   1. a one-plane batch with the axial plane's geometry equals
//      GetPlaneData(PlaneAxial) value for value;
//   2. every plane of a 5-plane oblique MIP-slab batch equals mk_render_plane
//      called with that plane's parameters, built here independently.
// Exit status: 0 pass, 1 mismatch, 77 no CUDA device.
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <memory>
#include <vector>

#include "monkeygl/HelloMonkey.h"
#include "monkeygl_b200.h"

using namespace MonkeyGL;

static int compare(const short *a, const short *b, size_t n, const char *what) {
    size_t bad = 0;
    for (size_t i = 0; i < n; ++i) bad += a[i] != b[i];
    printf("%s: %zu of %zu values differ\n", what, bad, n);
    return bad == 0 ? 0 : 1;
}

int main() {
    int ndev = 0;
    if (mk_device_count(&ndev) != MK_OK || ndev == 0) {
        printf("no CUDA device\n");
        return 77;
    }
    const int X = 160, Y = 128, Z = 96;
    const double sp[3] = {0.7, 0.6, 0.9};
    std::shared_ptr<short> vox(new short[(size_t)X * Y * Z], std::default_delete<short[]>());
    uint32_t s = 12345u;
    for (size_t i = 0; i < (size_t)X * Y * Z; ++i) {
        s = s * 1664525u + 1013904223u;
        const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((size_t)X * Y));
        // smooth structure plus noise, so that trilinear reads differ from voxels
        vox.get()[i] = (short)(400.0 * sin(0.11 * x) * cos(0.07 * y + 0.05 * z) + (int)(s >> 24) - 128);
    }
    HelloMonkey hm;
    if (!hm.SetVolumeData(vox, X, Y, Z)) {
        printf("SetVolumeData failed\n");
        return 1;
    }
    hm.SetDirection(Direction3d(1, 0, 0), Direction3d(0, 1, 0), Direction3d(0, 0, -1));
    hm.SetSpacing(sp[0], sp[1], sp[2]);
    const double ps = sp[1];   // the minimum spacing: MPRInfo's pixel spacing and thickness

    int rc = 0;
    // 1. one plane = the axial MPR plane
    {
        std::shared_ptr<short> axial;
        int w = 0, h = 0;
        if (!hm.GetPlaneData(axial, w, h, PlaneAxial)) {
            printf("GetPlaneData failed\n");
            return 1;
        }
        Point3d c;
        hm.GetCrossHairPoint3D(c);
        BatchInfo b;
        b.m_dirH = Direction3d(1, 0, 0);
        b.m_dirV = Direction3d(0, 1, 0);
        b.m_ptCenter = c;
        b.m_fLengthH = (w + 0.5) * ps;
        b.m_fLengthV = (h + 0.5) * ps;
        b.m_fPixelSpacing = ps;
        b.m_fSliceThickness = ps;
        b.m_fSliceDistance = 1.0;
        b.m_nNum = 1;
        b.m_MPRType = MPRTypeAverage;
        std::vector<short *> out;
        if (!hm.GetBatchData(out, b) || out.size() != 1 || b.Width() != w || b.Height() != h) {
            printf("GetBatchData (one plane) failed: %zu planes, %dx%d vs %dx%d\n", out.size(), b.Width(),
                   b.Height(), w, h);
            return 1;
        }
        rc |= compare(out[0], axial.get(), (size_t)w * h, "one-plane batch vs GetPlaneData(PlaneAxial)");
        for (short *p : out) delete[] p;
    }
    // 2. an oblique stack of MIP slabs against mk_render_plane
    {
        const Direction3d dh(0.8, 0.36, 0.48), dv0(-0.2, 0.9, -0.3);
        const Direction3d dv = dh.cross(dv0).cross(dh);   // in the plane, orthogonal to dh
        const Direction3d n = dh.cross(dv);
        BatchInfo b;
        b.m_dirH = dh;
        b.m_dirV = dv;
        b.m_ptCenter = Point3d(0.5 * X * sp[0] + 3.0, 0.5 * Y * sp[1] - 2.0, 0.5 * Z * sp[2] + 1.0);
        b.m_fLengthH = 97.3;
        b.m_fLengthV = 61.9;
        b.m_fPixelSpacing = 0.45;
        b.m_fSliceThickness = 1.85;   // int(1.85 / 0.45) = 4 samples: half width 1.5
        b.m_fSliceDistance = 1.3;
        b.m_nNum = 5;
        b.m_MPRType = MPRTypeMIP;
        std::vector<short *> out;
        if (!hm.GetBatchData(out, b) || out.size() != 5) {
            printf("GetBatchData (stack) failed: %zu planes\n", out.size());
            return 1;
        }
        const int w = b.Width(), h = b.Height();
        std::vector<short> want((size_t)w * h);
        for (int i = 0; i < 5; ++i) {
            const double off = (i - 2.0) * b.m_fSliceDistance;
            mk_plane_params p = {};
            p.width = w;
            p.height = h;
            p.mpr_type = MK_MPR_MIP;
            p.sampling = MK_SAMPLE_LINEAR;
            const double hh[3] = {dh.x(), dh.y(), dh.z()}, vv[3] = {dv.x(), dv.y(), dv.z()},
                         nn[3] = {n.x(), n.y(), n.z()}, cc[3] = {b.m_ptCenter.x(), b.m_ptCenter.y(),
                                                                 b.m_ptCenter.z()};
            for (int k = 0; k < 3; ++k) {
                p.spacing[k] = (float)sp[k];
                p.dir_h[k] = (float)hh[k];
                p.dir_v[k] = (float)vv[k];
                p.dir_n[k] = (float)nn[k];
                const double ck = cc[k] + nn[k] * off;
                p.left_top[k] = (float)((ck - hh[k] * (0.5 * w * b.m_fPixelSpacing)) - vv[k] * (0.5 * h * b.m_fPixelSpacing));
            }
            p.pixel_spacing = (float)b.m_fPixelSpacing;
            p.invert_z = 0;
            p.half_num = 1.5f;
            if (mk_render_plane(hm.GetDeviceVolume(), &p, want.data(), 0, nullptr) != MK_OK) {
                printf("mk_render_plane failed: %s\n", mk_last_error());
                return 1;
            }
            char what[64];
            snprintf(what, sizeof(what), "stack plane %d (%dx%d)", i, w, h);
            rc |= compare(out[i], want.data(), want.size(), what);
        }
        for (short *p : out) delete[] p;
    }
    printf(rc == 0 ? "batch ok\n" : "batch MISMATCH\n");
    return rc;
}
