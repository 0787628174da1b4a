// mk_math.h -- scalar expressions of MonkeyGL's kernels shared by the CUDA
// kernels and host code.
//
// MonkeyGL evaluates a few expressions in double precision on the device (a
// double literal promotes the whole expression).  They are evaluated here in
// double too, operation for operation, with explicit roundings on the device
// so that no multiply-add is contracted differently from MonkeyGL's build:
// FP64 runs at half the FP32 rate on sm_100, and the values then equal
// MonkeyGL's by construction.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define MK_HD __host__ __device__ __forceinline__
#else
#define MK_HD inline
#endif

namespace mk {

// (float)(((double)a - 0.866) * (double)scale): the ray parameter of
// core/kernel.cu:197 (and :313, :415), whose 0.866 literal makes the
// expression double: the difference and the product are rounded to double,
// then the product to float.  Host builds are compiled with
// -ffp-contract=off, and a difference times a factor has no multiply-add to
// contract anyway.
MK_HD float ray_fy(float a, float scale) {
#if defined(__CUDA_ARCH__)
    return __double2float_rn(__dmul_rn(__dsub_rn((double)a, 0.866), (double)scale));
#else
    return (float)(((double)a - 0.866) * (double)scale);
#endif
}

// float -> int16 with truncation and saturation (PTX cvt.rzi.s16.f32
// semantics, which MonkeyGL's "short v = 32768 * tex3D(...)" compiles to).
MK_HD short f2s_sat(float v) {
    if (!(v == v)) return 0;
    if (v >= 32767.0f) return 32767;
    if (v <= -32768.0f) return -32768;
    return (short)v;
}

}  // namespace mk
