// Host build of monkeygl_b200/csrc/mk_math.h for the emulation tests: each
// function evaluates, over arrays, both the FP32 emulation the kernels run
// and the double expression MonkeyGL evaluates, so the test can count
// disagreements.
#include <stdint.h>
#include "mk_math.h"

extern "C" {

// fy = (float)(((double)a - 0.866) * (double)scale)
int64_t check_ray_fy(const float *a, const float *scale, int64_t n, float *emul, float *ref) {
    int64_t bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        emul[i] = mk::ray_fy(a[i], scale[i]);
        ref[i] = (float)(((double)a[i] - 0.866) * (double)scale[i]);
        bad += emul[i] != ref[i];
    }
    return bad;
}

// the exact integer route alone (ray_fy takes it near rounding midpoints)
int64_t check_ray_fy_exact(const float *a, const float *scale, int64_t n, float *emul, float *ref) {
    int64_t bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        float x = 0.0f;
        if (!mk::ray_fy_exact(a[i], scale[i], x)) x = -1e30f;
        emul[i] = x;
        ref[i] = (float)(((double)a[i] - 0.866) * (double)scale[i]);
        bad += emul[i] != ref[i];
    }
    return bad;
}

// (float)((double)x + 0.05)
int64_t check_add005(const float *x, int64_t n, float *emul, float *ref) {
    int64_t bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        emul[i] = mk::add_dconst(x[i], MK_DCONST(0.05));
        ref[i] = (float)((double)x[i] + 0.05);
        bad += emul[i] != ref[i];
    }
    return bad;
}

// (float)((p + x * d) / dim) with double p, d
int64_t check_cpr(const double *p, const double *d, const int *x, const int *dim, int64_t n, float *emul,
                  float *ref) {
    int64_t bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        const float ph = (float)p[i], pl = (float)(p[i] - (double)ph);
        const float dh = (float)d[i], dl = (float)(d[i] - (double)dh);
        emul[i] = mk::cpr_coord(ph, pl, dh, dl, (float)x[i], (float)dim[i]);
        ref[i] = (float)((p[i] + x[i] * d[i]) / (double)dim[i]);
        bad += emul[i] != ref[i];
    }
    return bad;
}

// short(sum_double(v) / n) with truncation and saturation
int64_t check_mean(const float *v, int64_t rows, int64_t k, short *emul, short *ref) {
    int64_t bad = 0;
    for (int64_t r = 0; r < rows; ++r) {
        mk::fsum acc = {0.0f, 0.0f};
        double s = 0.0;
        for (int64_t j = 0; j < k; ++j) {
            mk::fsum_add(acc, v[r * k + j]);
            s += (double)v[r * k + j];
        }
        emul[r] = mk::fsum_div_to_short(acc, (float)k);
        double q = s / (double)k;
        short qs = q >= 32767.0 ? 32767 : (q <= -32768.0 ? -32768 : (short)q);
        ref[r] = qs;
        bad += emul[r] != ref[r];
    }
    return bad;
}
}
