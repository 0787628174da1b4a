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
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define MK_HD __host__ __device__ __forceinline__
#else
#define MK_HD inline
#endif

// Device ray parameter in native double (1) or by the float evaluation (0).
#ifndef MK_FY_NATIVE
#define MK_FY_NATIVE 1
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

// float <-> bits and leading zeros, on both sides of the compiler.
MK_HD uint32_t float_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, sizeof(u));
    return u;
#endif
}

MK_HD float bits_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, sizeof(f));
    return f;
#endif
}

MK_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// Round the unsigned integer q (q > 0) to `bits` significant bits, ties to
// even; the result is m * 2^e with m < 2^bits.
MK_HD void round_bits(unsigned __int128 q, int bits, unsigned __int128 &m, int &e) {
    const uint64_t hi = (uint64_t)(q >> 64), lo = (uint64_t)q;
    const int len = hi ? 128 - clz64(hi) : 64 - clz64(lo);
    if (len <= bits) {
        m = q;
        e = 0;
        return;
    }
    const int sh = len - bits;
    unsigned __int128 r = q >> sh;
    const unsigned __int128 rem = q & ((((unsigned __int128)1) << sh) - 1);
    const unsigned __int128 half = ((unsigned __int128)1) << (sh - 1);
    if (rem > half || (rem == half && (r & 1))) r += 1;
    e = sh;
    if (r >> bits) {   // carried into a new bit
        r >>= 1;
        e += 1;
    }
    m = r;
}

// The same product by integers: for a == 0 or a >= 2^-30 (every
// accuLength of the schedule) (double)a - 0.866 is exactly N * 2^-53 with
// |N| < 2^53, so with scale = S * 2^k (24-bit S) the product is the integer
// N * S * 2^(k - 53), at most 77 bits; rounding it to 53 and then to 24
// significant bits, ties to even each time, reproduces both of MonkeyGL's
// roundings exactly.  Returns false for other a (never produced).
MK_HD bool ray_fy_exact(float a, float scale, float &out) {
    const uint32_t ab = float_bits(a), sb = float_bits(scale);
    const int ea = (int)((ab >> 23) & 255), es = (int)((sb >> 23) & 255);
    if (!((a == 0.0f || (ea >= 127 - 30 && ea < 255)) && es > 0 && es < 255)) return false;
    // 0.866 = C * 2^-53 exactly (its double significand)
    const int64_t C = (int64_t)(0.866 * 9007199254740992.0);
    int64_t n = -C;
    if (a != 0.0f) {
        const int64_t ma = (int64_t)((ab & 0x7fffff) | 0x800000);   // a = ma * 2^(ea - 150)
        const int64_t va = ma << (ea - 150 + 53);                    // a * 2^53, exact
        n = ((ab >> 31) ? -va : va) - C;
    }
    const bool neg = (n < 0) != ((sb >> 31) != 0);
    const uint64_t un = (uint64_t)(n < 0 ? -n : n);
    const uint64_t ms = (uint64_t)((sb & 0x7fffff) | 0x800000);   // scale = ms * 2^(es - 150)
    const unsigned __int128 q = (unsigned __int128)un * ms;       // |product| = q * 2^(es - 150 - 53)
    unsigned __int128 m53, m24;
    int e53, e24;
    round_bits(q, 53, m53, e53);
    round_bits(m53, 24, m24, e24);
    const float r = ldexpf((float)(uint32_t)m24, e53 + e24 + es - 150 - 53);
    out = neg ? -r : r;
    return true;
}

// (float)(((double)a - 0.866) * (double)scale): the ray parameter of
// core/kernel.cu:197 (and :313, :415), whose 0.866 literal makes the
// expression double: the product is rounded to 53 bits, then to 24.  The
// float evaluation below carries the product to within 2^-47 of its value
// and rounds once.  Where the carried product lies more than 2^-20 half-ulps
// (2^-44 relative, eight times that error) from a float rounding midpoint,
// the exact product is on the same side of it and outside the 2^-53 window
// where rounding to double first could land on the midpoint, so both
// evaluations give this float; the residual of the final rounding measures
// that distance.  The rest (about one product in 2^20) take the exact
// integer route.
MK_HD float ray_fy(float a, float scale) {
#if defined(__CUDA_ARCH__) && MK_FY_NATIVE
    // On the device the double expression itself, operation for operation
    // (FP64 runs at half the FP32 rate on sm_100, cheaper than the float
    // evaluation below); explicit roundings so that nothing is contracted.
    return __double2float_rn(__dmul_rn(__dsub_rn((double)a, 0.866), (double)scale));
#endif
    float h, l;
    sub_dconst(a, MK_DCONST(0.866), h, l);
    float p, pe;
    two_prod(h, scale, p, pe);
    pe = MK_FMA(l, scale, pe);
    const float r = MK_ADD_RN(p, pe);
    // residual of that rounding (|pe| <= ulp(p), so this is exact)
    const float e = MK_ADD_RN(MK_ADD_RN(p, -r), pe);
    const float half_ulp = MK_MUL_RN(mk::bits_float(float_bits(r) & 0x7f800000u), 5.9604645e-08f);   // 2^-24
    const float d = fabsf(MK_ADD_RN(fabsf(e), -half_ulp));
    if (d > MK_MUL_RN(half_ulp, 9.5367432e-07f)) return r;   // 2^-20 half-ulps from a midpoint
    float x;
    return ray_fy_exact(a, scale, x) ? x : r;
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
