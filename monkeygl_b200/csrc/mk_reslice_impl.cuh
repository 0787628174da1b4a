// mk_reslice_impl.cuh -- device code of the planar reslice: one output pixel
// of MonkeyGL's d_renderPlane_{MIP,MinIP,Average} (core/kernel.cu:570-793),
// shared by the one-plane kernel (mk_reslice.cu) and the serving kernel
// (mk_server.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mk_internal.h"
#include "mk_math.h"

namespace mk {

struct PlaneParams {
    int W, H;
    float sp[3];
    float fdim[3];
    float h[3], v[3], n[3], lt[3];
    float ps;
    int invertZ;
    float halfNum;
    int mode;
    const uint8_t *voi_lut;   // u8 epilogue: display value of int16 v at [v + 32768]
};

template <int MODE>
__device__ __forceinline__ short reslice_pixel(const PlaneParams &P, cudaTextureObject_t tex, int x,
                                               int y) {
    short acc = (MODE == MK_MPR_MIP) ? (short)-32768 : (short)32767;
    double sum = 0.0;          // MonkeyGL's double accumulator (core/kernel.cu:773)
    // The contraction of MonkeyGL's sums pt + x*ps*h + y*ps*v into fused
    // multiply-adds is spelled out, left to right: of the fused and unfused
    // orders, this one reproduces MonkeyGL's kernel pixel for pixel, and
    // writing it out keeps every kernel that inlines this function on it.
    const float xs = __fmul_rn((float)x, P.ps), ys = __fmul_rn((float)y, P.ps);
    for (float t = -P.halfNum; t <= P.halfNum; t += 1) {
        const float fLength = __fmul_rn(t, P.ps);
        const float pt_x = __fmaf_rn(fLength, P.n[0], P.lt[0]);
        const float pt_y = __fmaf_rn(fLength, P.n[1], P.lt[1]);
        const float pt_z = __fmaf_rn(fLength, P.n[2], P.lt[2]);
        const float fx = __fdiv_rn(__fmaf_rn(ys, P.v[0], __fmaf_rn(xs, P.h[0], pt_x)), __fmul_rn(P.sp[0], P.fdim[0]));
        const float fy = __fdiv_rn(__fmaf_rn(ys, P.v[1], __fmaf_rn(xs, P.h[1], pt_y)), __fmul_rn(P.sp[1], P.fdim[1]));
        float fz = __fdiv_rn(__fmaf_rn(ys, P.v[2], __fmaf_rn(xs, P.h[2], pt_z)), __fmul_rn(P.sp[2], P.fdim[2]));
        // "fz = 1.0 - fz" in double, then rounded to float: identical to the
        // float subtraction for every float fz (the exact difference rounds once)
        if (!P.invertZ) fz = 1.0f - fz;
        const bool inside = fx >= 0 && fx <= 1 && fy >= 0 && fy <= 1 && fz >= 0 && fz <= 1;
        if (MODE == MK_MPR_AVERAGE) {
            sum = __dadd_rn(sum, (double)(inside ? 32768 * tex3D<float>(tex, fx, fy, fz) : -32768.0f));
        } else {
            const short val = inside ? f2s_sat(32768 * tex3D<float>(tex, fx, fy, fz)) : (short)-32768;
            if (MODE == MK_MPR_MIP) acc = acc > val ? acc : val;
            else acc = acc < val ? acc : val;
        }
    }
    if (MODE == MK_MPR_AVERAGE) {
        // fSum / (2 * halfNum + 1) in double, converted to short (truncated,
        // saturated as the conversion instruction does)
        const double q = __ddiv_rn(sum, (double)(2 * P.halfNum + 1));
        return (short)min(max(__double2int_rz(q), -32768), 32767);
    }
    return acc;
}

// One 32x8 tile (bx, by) of a plane by a 256-thread block: thread t covers
// pixel (t % 32, t / 32) of the tile.
template <int MODE, bool U8>
__device__ __forceinline__ void plane_tile(const PlaneParams &P, cudaTextureObject_t tex, void *out, int bx, int by) {
    const int x = bx * 32 + (threadIdx.x & 31);
    const int y = by * 8 + (threadIdx.x >> 5);
    if (x >= P.W || y >= P.H) return;
    const short r = reslice_pixel<MODE>(P, tex, x, y);
    if (U8) {
        // display window: one table read per pixel (the table is built on
        // the host; 64 KB, resident in L1/L2)
        static_cast<uint8_t *>(out)[(size_t)y * P.W + x] = __ldg(P.voi_lut + ((int)r + 32768));
    } else {
        static_cast<short *>(out)[(size_t)y * P.W + x] = r;
    }
}

// Host: kernel parameters of one plane (validates the request).
int fill_plane_params(const VolumeState &v, const mk_plane_params *p, PlaneParams &P);

}  // namespace mk
