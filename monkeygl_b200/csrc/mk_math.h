// mk_math.h -- float arithmetic shared by the CUDA kernels and host code.
//
// MonkeyGL evaluates a few expressions in double precision on the device
// (a double literal promotes the whole expression).  These kernels keep all
// device arithmetic in FP32 and reproduce those double expressions with
// error-free float transformations (Knuth's TwoSum, Dekker/FMA TwoProduct),
// which return the correctly rounded float of the exact value.  MonkeyGL's
// double evaluation rounds to double first and then to float, so the two agree
// except when the exact value lies within 2^-29 relative of a float rounding
// midpoint.
//
// Every function here is __host__ __device__ so the host-side tests can check
// the very code the kernels run.  Products that must stay separately rounded
// go through MK_MUL_RN so that -fmad contraction cannot fuse them.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define MK_HD __host__ __device__ __forceinline__
#else
#define MK_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define MK_MUL_RN(a, b) __fmul_rn((a), (b))
#define MK_ADD_RN(a, b) __fadd_rn((a), (b))
#define MK_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#else
// Host builds of this header are compiled with -ffp-contract=off.
#define MK_MUL_RN(a, b) ((a) * (b))
#define MK_ADD_RN(a, b) ((a) + (b))
#define MK_FMA(a, b, c) fmaf((a), (b), (c))
#endif

namespace mk {

// s + e == a + b exactly (Knuth TwoSum, 6 flops, no ordering requirement).
MK_HD void two_sum(float a, float b, float &s, float &e) {
    s = MK_ADD_RN(a, b);
    float bb = MK_ADD_RN(s, -a);
    float aa = MK_ADD_RN(s, -bb);
    e = MK_ADD_RN(MK_ADD_RN(a, -aa), MK_ADD_RN(b, -bb));
}

// p + e == a * b exactly (FMA TwoProduct).
MK_HD void two_prod(float a, float b, float &p, float &e) {
    p = MK_MUL_RN(a, b);
    e = MK_FMA(a, b, -p);
}

// A double constant split into three floats: c == hi + mid + lo exactly
// (24 + 24 + 5 significant bits).
struct dconst {
    float hi;
    float mid;
    float lo;
};

#define MK_DCONST(c)                                                        \
    ::mk::dconst {                                                          \
        (float)(c), (float)((c) - (double)(float)(c)),                      \
            (float)((c) - (double)(float)(c) -                              \
                    (double)(float)((c) - (double)(float)(c)))              \
    }

// x - c for a float x and a double constant c, as an unevaluated float pair
// (h + l) that is exact to ~2^-48 relative.
MK_HD void sub_dconst(float x, dconst c, float &h, float &l) {
    float s, e;
    two_sum(x, -c.hi, s, e);                   // x - hi exactly
    float t, te;
    two_sum(e, -c.mid, t, te);                 // e - mid exactly
    float t2 = MK_ADD_RN(te, -c.lo);
    float u, ue;
    two_sum(s, t, u, ue);
    two_sum(u, MK_ADD_RN(ue, t2), h, l);
}

// (float)(((double)a - 0.866) * (double)scale): the ray parameter of
// core/kernel.cu:197 (and :313, :415), whose 0.866 literal is a double.
MK_HD float ray_fy(float a, float scale) {
    float h, l;
    sub_dconst(a, MK_DCONST(0.866), h, l);
    float p, pe;
    two_prod(h, scale, p, pe);
    pe = MK_FMA(l, scale, pe);
    return MK_ADD_RN(p, pe);
}

// (float)((double)x + c) for a double constant c, e.g. the "+0.05" of
// core/kernel.cu:460.
MK_HD float add_dconst(float x, dconst c) {
    float h, l;
    dconst nc = {-c.hi, -c.mid, -c.lo};
    sub_dconst(x, nc, h, l);
    return MK_ADD_RN(h, l);
}

// Correctly rounded float of (hi + lo) / d, for |lo| <= ulp(hi).
MK_HD float div_pair(float hi, float lo, float d) {
    float q = hi / d;
    float r = MK_FMA(-q, d, hi);               // exact remainder of hi / d
    r = MK_ADD_RN(r, lo);
    return MK_ADD_RN(q, r / d);
}

// (float)(((double)p + (double)x * (double)dir) / (double)n) where p and dir
// are doubles supplied as float pairs and x is a small integer: the CPR
// coordinate of core/kernel.cu:860-862.
MK_HD float cpr_coord(float p_hi, float p_lo, float d_hi, float d_lo, float x, float n) {
    float m, me;
    two_prod(x, d_hi, m, me);                  // x * d_hi exactly
    float s, se;
    two_sum(p_hi, m, s, se);                   // p_hi + m exactly
    float lo = MK_ADD_RN(MK_ADD_RN(se, me), MK_FMA(x, d_lo, p_lo));
    float h, l;
    two_sum(s, lo, h, l);
    return div_pair(h, l, n);
}

// Running sum of floats kept as an unevaluated pair (hi + lo), for the
// double accumulator of core/kernel.cu:773.
struct fsum {
    float hi;
    float lo;
};

MK_HD void fsum_add(fsum &acc, float v) {
    float s, e;
    two_sum(acc.hi, v, s, e);
    acc.hi = s;
    acc.lo = MK_ADD_RN(acc.lo, e);
}

// Truncate (hi + lo) / n toward zero and saturate to int16: the
// "short = double / float" conversion of core/kernel.cu:791.
MK_HD short fsum_div_to_short(fsum acc, float n) {
    float s, e;
    two_sum(acc.hi, acc.lo, s, e);             // renormalise
    float q = s / n;
    float r = MK_FMA(-q, n, s);
    r = MK_ADD_RN(r, e);
    float ql = r / n;                          // quotient = q + ql (+ tiny)
    float ti = truncf(q);
    float f = MK_ADD_RN(MK_ADD_RN(q, -ti), ql); // fractional part, sign exact
    float res = ti;
    float qq = MK_ADD_RN(q, ql);
    if (qq >= 0.0f) {
        if (f < 0.0f) res = MK_ADD_RN(ti, -1.0f);
        else if (f >= 1.0f) res = MK_ADD_RN(ti, 1.0f);
    } else {
        if (f > 0.0f) res = MK_ADD_RN(ti, 1.0f);
        else if (f <= -1.0f) res = MK_ADD_RN(ti, -1.0f);
    }
    if (res > 32767.0f) res = 32767.0f;
    if (res < -32768.0f) res = -32768.0f;
    return (short)res;
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
