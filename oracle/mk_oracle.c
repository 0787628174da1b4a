/*
 * mk_oracle.c -- TEST INFRASTRUCTURE: CPU restatement of MonkeyGL's
 * ray-casting path (see mk_oracle.h).  Each function names the lines of
 * MonkeyGL's core/kernel.cu it follows.  Compiled with -ffp-contract=off so
 * that every float operation is rounded separately.
 */
#include "mk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_wmode = 0;

void mko_set_weight_mode(int mode) { g_wmode = mode; }

/* ---------------------------------------------------------------- */
/* texture unit emulation (core/CuDataManager.cu:54-72, 101-119, 132-163) */

static float quantize_weight(float a) {
    if (g_wmode == 2) return a;
    float s = a * 256.0f;
    s = (g_wmode == 0) ? floorf(s + 0.5f) : floorf(s);
    return s / 256.0f;
}

static inline int clampi(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }

/* cudaReadModeNormalizedFloat of int16: max(v / 32767, -1). */
static inline float texel_f(const mko_volume *v, int x, int y, int z) {
    x = clampi(x, 0, v->dim[0] - 1);
    y = clampi(y, 0, v->dim[1] - 1);
    z = clampi(z, 0, v->dim[2] - 1);
    float f = (float)v->vox[((size_t)z * v->dim[1] + y) * v->dim[0] + x] / 32767.0f;
    return f < -1.0f ? -1.0f : f;
}

static inline double texel_d(const mko_volume *v, int x, int y, int z) {
    x = clampi(x, 0, v->dim[0] - 1);
    y = clampi(y, 0, v->dim[1] - 1);
    z = clampi(z, 0, v->dim[2] - 1);
    double f = (double)v->vox[((size_t)z * v->dim[1] + y) * v->dim[0] + x] / 32767.0;
    return f < -1.0 ? -1.0 : f;
}

/* Split a texel coordinate into integer index and quantised fraction. */
static inline void split_coord(float xb, int *i, float *a) {
    float f = floorf(xb);
    float w = quantize_weight(xb - f);
    if (w >= 1.0f) {
        f += 1.0f;
        w = 0.0f;
    }
    *i = (int)f;
    *a = w;
}

/* tex3D<float> with normalized coordinates and linear filtering. */
float mko_tex3d_linear(const mko_volume *v, float x, float y, float z) {
    int i, j, k;
    float a, b, c;
    split_coord(x * (float)v->dim[0] - 0.5f, &i, &a);
    split_coord(y * (float)v->dim[1] - 0.5f, &j, &b);
    split_coord(z * (float)v->dim[2] - 0.5f, &k, &c);
    float c00 = texel_f(v, i, j, k) * (1.0f - a) + texel_f(v, i + 1, j, k) * a;
    float c10 = texel_f(v, i, j + 1, k) * (1.0f - a) + texel_f(v, i + 1, j + 1, k) * a;
    float c01 = texel_f(v, i, j, k + 1) * (1.0f - a) + texel_f(v, i + 1, j, k + 1) * a;
    float c11 = texel_f(v, i, j + 1, k + 1) * (1.0f - a) + texel_f(v, i + 1, j + 1, k + 1) * a;
    float c0 = c00 * (1.0f - b) + c10 * b;
    float c1 = c01 * (1.0f - b) + c11 * b;
    return c0 * (1.0f - c) + c1 * c;
}

static double tex3d_linear_d(const mko_volume *v, double x, double y, double z) {
    double xb = x * v->dim[0] - 0.5, yb = y * v->dim[1] - 0.5, zb = z * v->dim[2] - 0.5;
    double fi = floor(xb), fj = floor(yb), fk = floor(zb);
    double a = xb - fi, b = yb - fj, c = zb - fk;
    int i = (int)fi, j = (int)fj, k = (int)fk;
    double c00 = texel_d(v, i, j, k) * (1 - a) + texel_d(v, i + 1, j, k) * a;
    double c10 = texel_d(v, i, j + 1, k) * (1 - a) + texel_d(v, i + 1, j + 1, k) * a;
    double c01 = texel_d(v, i, j, k + 1) * (1 - a) + texel_d(v, i + 1, j, k + 1) * a;
    double c11 = texel_d(v, i, j + 1, k + 1) * (1 - a) + texel_d(v, i + 1, j + 1, k + 1) * a;
    double c0 = c00 * (1 - b) + c10 * b;
    double c1 = c01 * (1 - b) + c11 * b;
    return c0 * (1 - c) + c1 * c;
}

/* tex3D<float> with normalized coordinates and point filtering. */
float mko_tex3d_point(const mko_volume *v, float x, float y, float z) {
    return texel_f(v, (int)floorf(x * (float)v->dim[0]), (int)floorf(y * (float)v->dim[1]),
                   (int)floorf(z * (float)v->dim[2]));
}

/* tex1D<float4> with normalized coordinates, linear filter, clamp. */
void mko_tex1d_lut(const float *lut, int n, float t, float out[4]) {
    int i;
    float a;
    split_coord(t * (float)n - 0.5f, &i, &a);
    int i0 = clampi(i, 0, n - 1), i1 = clampi(i + 1, 0, n - 1);
    for (int c = 0; c < 4; ++c) out[c] = lut[4 * i0 + c] * (1.0f - a) + lut[4 * i1 + c] * a;
}

static void tex1d_lut_d(const float *lut, int n, double t, double out[4]) {
    double xb = t * n - 0.5;
    double f = floor(xb);
    double a = xb - f;
    int i = (int)f;
    int i0 = clampi(i, 0, n - 1), i1 = clampi(i + 1, 0, n - 1);
    for (int c = 0; c < 4; ++c) out[c] = lut[4 * i0 + c] * (1.0 - a) + lut[4 * i1 + c] * a;
}

/* Label texture: unnormalized integer coordinates, point filter, clamp
 * (core/CuDataManager.cu:107-117). */
static inline int mask_at(const mko_volume *v, int x, int y, int z) {
    if (!v->mask) return 0;
    x = clampi(x, 0, v->dim[0] - 1);
    y = clampi(y, 0, v->dim[1] - 1);
    z = clampi(z, 0, v->dim[2] - 1);
    int l = v->mask[((size_t)z * v->dim[1] + y) * v->dim[0] + x];
    return l > MKO_LABELS - 1 ? MKO_LABELS - 1 : l; /* labels above 64 never come from the API */
}

/* ---------------------------------------------------------------- */
/* ray casting, FP32 (core/kernel.cu:133-469)                       */

typedef struct {
    float mls[3], sp[3], sv[3], xT, yT, scale, M[9];
    int invertZ, voi[6];
    float bg[4];
    float alpha[MKO_LABELS], ww[MKO_LABELS], wl[MKO_LABELS];
} vrp;

static void unpack_vr(const float *p, vrp *q) {
    for (int k = 0; k < 3; ++k) {
        q->mls[k] = p[k];
        q->sp[k] = p[3 + k];
        q->sv[k] = p[6 + k];
    }
    q->xT = p[9];
    q->yT = p[10];
    q->scale = p[11];
    for (int i = 0; i < 9; ++i) q->M[i] = p[12 + i];
    q->invertZ = p[21] != 0.0f;
    for (int i = 0; i < 6; ++i) q->voi[i] = (int)p[22 + i];
    for (int i = 0; i < 4; ++i) q->bg[i] = p[28 + i];
    for (int l = 0; l < MKO_LABELS; ++l) {
        q->alpha[l] = p[32 + 3 * l];
        q->ww[l] = p[33 + 3 * l];
        q->wl[l] = p[34 + 3 * l];
    }
}

/* helper_math dot() as three separately rounded products and two sums */
static inline float dotf(float ax, float ay, float az, float bx, float by, float bz) {
    return ax * bx + ay * by + az * bz;
}

static inline float satf(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

/* rgbaFloatToInt + byte stores (core/kernel.cu:40-47, 258-262) */
static void store_rgb(uint8_t *o, const float c[4]) {
    o[0] = (uint8_t)(unsigned)(satf(c[0]) * 255);
    o[1] = (uint8_t)(unsigned)(satf(c[1]) * 255);
    o[2] = (uint8_t)(unsigned)(satf(c[2]) * 255);
}

static inline int outside_voi(const vrp *q, int x, int y, int z) {
    return x < q->voi[0] || x > q->voi[1] || y < q->voi[2] || y > q->voi[3] || z < q->voi[4] ||
           z > q->voi[5];
}

/* pos for accuLength a (core/kernel.cu:197-206) */
static void ray_pos_f(const vrp *q, float u, float vv, float a, float pos[3]) {
    float fy = (float)(((double)a - 0.866) * (double)q->scale);
    float px = dotf(u, fy, vv, q->M[0], q->M[1], q->M[2]);
    float py = dotf(u, fy, vv, q->M[3], q->M[4], q->M[5]);
    float pz = dotf(u, fy, vv, q->M[6], q->M[7], q->M[8]);
    pos[0] = px * q->mls[0] + 0.5f;
    pos[1] = py * q->mls[1] + 0.5f;
    pos[2] = pz * q->mls[2] + 0.5f;
    if (q->invertZ) pos[2] = 1.0f - pos[2];
}

static void light_dir_f(const vrp *q, float L[3]) {
    float lx = dotf(0.0f, 1.0f, 0.0f, q->M[0], q->M[1], q->M[2]);
    float ly = dotf(0.0f, 1.0f, 0.0f, q->M[3], q->M[4], q->M[5]);
    float lz = dotf(0.0f, 1.0f, 0.0f, q->M[6], q->M[7], q->M[8]);
    float inv = 1.0f / sqrtf(lx * lx + ly * ly + lz * lz);
    L[0] = lx * inv;
    L[1] = ly * inv;
    L[2] = lz * inv;
}

/* tracing (core/kernel.cu:49-81) */
static void tracing_f(const mko_volume *v, const vrp *q, float sum[4], float alphaAcc, const float pos[3],
                      const float col[4], const float L[3]) {
    float N[3];
    N[0] = mko_tex3d_linear(v, pos[0] + q->sv[0], pos[1], pos[2]) -
           mko_tex3d_linear(v, pos[0] - q->sv[0], pos[1], pos[2]);
    N[1] = mko_tex3d_linear(v, pos[0], pos[1] + q->sv[1], pos[2]) -
           mko_tex3d_linear(v, pos[0], pos[1] - q->sv[1], pos[2]);
    N[2] = mko_tex3d_linear(v, pos[0], pos[1], pos[2] + q->sv[2]) -
           mko_tex3d_linear(v, pos[0], pos[1], pos[2] - q->sv[2]);
    if (q->invertZ) N[2] = -N[2];
    float inv = 1.0f / sqrtf(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    for (int k = 0; k < 3; ++k) N[k] *= inv;
    float diffuse = N[0] * L[0] + N[1] * L[1] + N[2] * L[2];
    float clr[4], t4[4] = {0, 0, 0, 0};
    for (int c = 0; c < 4; ++c) clr[c] = col[c] * 0.35f;
    if (diffuse > 0.0f) {
        float s = diffuse * 0.8f + 0.16f * powf(diffuse, 8.0f);
        for (int c = 0; c < 4; ++c) t4[c] = col[c] * s;
    }
    for (int c = 0; c < 4; ++c) clr[c] += t4[c];
    float w = (1.0f - alphaAcc) * col[3];
    for (int c = 0; c < 4; ++c) sum[c] = sum[c] + w * clr[c];
}

static void lut_lookup_f(const mko_volume *v, int label, float t, float col[4]) {
    if (!v->lut[label] || v->lut_len[label] <= 0) {
        col[0] = col[1] = col[2] = col[3] = 0.0f;
        return;
    }
    mko_tex1d_lut(v->lut[label], v->lut_len[label], t, col);
}

/* d_render (core/kernel.cu:133-264) for one pixel */
static void vr_pixel_f(const mko_volume *v, const vrp *q, int w, int h, int x, int y, uint8_t *o,
                       uint64_t *ns) {
    float u = 1.0f * (x - w / 2.0f - q->xT) / h;
    float vv = 1.0f * (y - h / 2.0f - q->yT) / h;
    float sum[4] = {0, 0, 0, 0};
    float L[3];
    light_dir_f(q, L);
    const float L1 = 1.0f / (float)v->dim[2], L4 = L1 / 4.0f, L8 = L1 / 8.0f;
    float step = L1;
    float accObj[MKO_LABELS];
    memset(accObj, 0, sizeof(accObj));
    float alphaAcc = 0.0f, accu = 0.0f, aPre = 0.0f;
    uint64_t n = 0;
    while ((double)accu < 1.732) {
        float pos[3];
        ray_pos_f(q, u, vv, accu, pos);
        int ix = (int)(pos[0] * (float)v->dim[0]);
        int iy = (int)(pos[1] * (float)v->dim[1]);
        int iz = (int)(pos[2] * (float)v->dim[2]);
        if (outside_voi(q, ix, iy, iz)) {
            accu += step;
            continue;
        }
        ++n;
        int label = mask_at(v, ix, iy, iz);
        float temp = 32768 * mko_tex3d_linear(v, pos[0], pos[1], pos[2]);
        temp = (float)((double)((temp - q->wl[label]) / q->ww[label]) + 0.5);
        if (temp > 1) temp = 1;
        float col[4];
        lut_lookup_f(v, label, temp, col);
        float alpha = col[3];
        /* getNextStep (core/kernel.cu:84-125) */
        if (step == L4) alpha = 1 - powf(1 - alpha, 0.25f);
        else if (step == L8) alpha = 1 - powf(1 - alpha, 0.125f);
        if (accu > 0.0f) {
            if ((alpha > aPre ? alpha : aPre) > 0.001f) {
                if (step == L1) {
                    accu -= (L1 - L4);
                    step = L4;
                    continue;
                } else if (step == L4) {
                    accu -= (L4 - L8);
                    step = L8;
                    continue;
                }
            } else {
                step = (step == L8) ? L4 : L1;
            }
        }
        aPre = alpha;
        accu += step;
        col[3] = alpha;
        if (col[3] > 0.0005f && accObj[label] < q->alpha[label]) {
            tracing_f(v, q, sum, alphaAcc, pos, col, L);
            accObj[label] += (1.0f - alphaAcc) * col[3];
            alphaAcc += (1.0f - alphaAcc) * col[3];
        }
        if (alphaAcc > 0.995f) break;
    }
    if (sum[0] == 0.0f && sum[1] == 0.0f && sum[2] == 0.0f && sum[3] == 0.0f)
        memcpy(sum, q->bg, sizeof(sum));
    store_rgb(o, sum);
    if (ns) *ns = n;
}

/* d_renderMIP (core/kernel.cu:266-364) for one pixel */
static void mip_pixel_f(const mko_volume *v, const vrp *q, int w, int h, int x, int y, uint8_t *o,
                        uint64_t *ns) {
    float u = 1.0f * (x - w / 2.0f - q->xT) / h;
    float vv = 1.0f * (y - h / 2.0f - q->yT) / h;
    const float fStep = 1.0f / (float)v->dim[2];
    float A = 0.0f, accu = 0.0f;
    uint64_t n = 0;
    while ((double)accu < 1.732) {
        float pos[3];
        ray_pos_f(q, u, vv, accu, pos);
        int ix = (int)(pos[0] * (float)v->dim[0]);
        int iy = (int)(pos[1] * (float)v->dim[1]);
        int iz = (int)(pos[2] * (float)v->dim[2]);
        if (outside_voi(q, ix, iy, iz)) {
            accu += fStep;
            continue;
        }
        int label = mask_at(v, ix, iy, iz);
        if (q->alpha[label] > 0) {
            ++n;
            float temp = 32768 * mko_tex3d_linear(v, pos[0], pos[1], pos[2]);
            temp = (float)((double)((temp - q->wl[label]) / q->ww[label]) + 0.5);
            if (A < temp) A = temp;
        }
        accu += fStep;
    }
    float sum[4];
    if (A <= 0.0f) memcpy(sum, q->bg, sizeof(sum));
    else sum[0] = sum[1] = sum[2] = sum[3] = A;
    store_rgb(o, sum);
    if (ns) *ns = n;
}

/* d_renderSurface (core/kernel.cu:366-469) for one pixel */
static void surf_pixel_f(const mko_volume *v, const vrp *q, int w, int h, int x, int y, uint8_t *o,
                         uint64_t *ns) {
    float u = 1.0f * (x - w / 2.0f - q->xT) / h;
    float vv = 1.0f * (y - h / 2.0f - q->yT) / h;
    const float fStep = 1.0f / (float)v->dim[2];
    float L[3];
    light_dir_f(q, L);
    float A = 0.0f, accu = 0.0f;
    uint64_t n = 0;
    while ((double)accu < 1.732) {
        float pos[3];
        ray_pos_f(q, u, vv, accu, pos);
        int ix = (int)(pos[0] * (float)v->dim[0]);
        int iy = (int)(pos[1] * (float)v->dim[1]);
        int iz = (int)(pos[2] * (float)v->dim[2]);
        if (outside_voi(q, ix, iy, iz)) {
            accu += fStep;
            continue;
        }
        ++n;
        float temp = 32768 * mko_tex3d_linear(v, pos[0], pos[1], pos[2]);
        if (temp <= 400) {
            accu += fStep;
            continue;
        }
        float N[3];
        N[0] = mko_tex3d_linear(v, pos[0] + q->sv[0], pos[1], pos[2]) -
               mko_tex3d_linear(v, pos[0] - q->sv[0], pos[1], pos[2]);
        N[1] = mko_tex3d_linear(v, pos[0], pos[1] + q->sv[1], pos[2]) -
               mko_tex3d_linear(v, pos[0], pos[1] - q->sv[1], pos[2]);
        N[2] = mko_tex3d_linear(v, pos[0], pos[1], pos[2] + q->sv[2]) -
               mko_tex3d_linear(v, pos[0], pos[1], pos[2] - q->sv[2]);
        if (q->invertZ) N[2] = -N[2];
        float inv = 1.0f / sqrtf(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
        for (int k = 0; k < 3; ++k) N[k] *= inv;
        A = N[0] * L[0] + N[1] * L[1] + N[2] * L[2];
        if (A > 0) break;
        accu += fStep;
    }
    float sum[4];
    if (A <= 0.0f) {
        memcpy(sum, q->bg, sizeof(sum));
    } else {
        float g = (float)((double)A + 0.05);
        sum[0] = sum[1] = sum[2] = g;
        sum[3] = 1.0f;
    }
    store_rgb(o, sum);
    if (ns) *ns = n;
}

/* ---------------------------------------------------------------- */
/* the same method in FP64 with exact filtering                     */

static void ray_pos_d(const vrp *q, double u, double vv, double a, double pos[3]) {
    double fy = (a - 0.866) * q->scale;
    for (int r = 0; r < 3; ++r)
        pos[r] = (u * q->M[3 * r] + fy * q->M[3 * r + 1] + vv * q->M[3 * r + 2]) * q->mls[r] + 0.5;
    if (q->invertZ) pos[2] = 1.0 - pos[2];
}

static void pixel_d(const mko_volume *v, const vrp *q, int type, int w, int h, int x, int y, uint8_t *o) {
    double u = (x - w / 2.0 - q->xT) / h;
    double vv = (y - h / 2.0 - q->yT) / h;
    double L[3] = {q->M[1], q->M[4], q->M[7]};
    double ln = sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]);
    for (int k = 0; k < 3; ++k) L[k] /= ln;
    const double L1 = 1.0 / v->dim[2], L4 = L1 / 4, L8 = L1 / 8;
    double step = L1, accu = 0, aPre = 0, A = 0;
    double sum[4] = {0, 0, 0, 0};
    double accObj[MKO_LABELS];
    memset(accObj, 0, sizeof(accObj));
    while (accu < 1.732) {
        double pos[3];
        ray_pos_d(q, u, vv, accu, pos);
        int ix = (int)(pos[0] * v->dim[0]), iy = (int)(pos[1] * v->dim[1]), iz = (int)(pos[2] * v->dim[2]);
        if (outside_voi(q, ix, iy, iz)) {
            accu += step;
            continue;
        }
        int label = mask_at(v, ix, iy, iz);
        double val = 32768 * tex3d_linear_d(v, pos[0], pos[1], pos[2]);
        if (type == MKO_MIP) {
            if (q->alpha[label] > 0) {
                double t = (val - q->wl[label]) / q->ww[label] + 0.5;
                if (A < t) A = t;
            }
            accu += step;
            continue;
        }
        double N[3] = {0, 0, 0};
        if (type == MKO_SURFACE) {
            if (val <= 400) {
                accu += step;
                continue;
            }
        } else {
            double t = (val - q->wl[label]) / q->ww[label] + 0.5;
            if (t > 1) t = 1;
            double col[4] = {0, 0, 0, 0};
            if (v->lut[label]) tex1d_lut_d(v->lut[label], v->lut_len[label], t, col);
            double alpha = col[3];
            if (step == L4) alpha = 1 - pow(1 - alpha, 0.25);
            else if (step == L8) alpha = 1 - pow(1 - alpha, 0.125);
            if (accu > 0) {
                if ((alpha > aPre ? alpha : aPre) > 0.001) {
                    if (step == L1) { accu -= (L1 - L4); step = L4; continue; }
                    else if (step == L4) { accu -= (L4 - L8); step = L8; continue; }
                } else {
                    step = (step == L8) ? L4 : L1;
                }
            }
            aPre = alpha;
            accu += step;
            col[3] = alpha;
            if (col[3] > 0.0005 && accObj[label] < q->alpha[label]) {
                double g[3];
                for (int k = 0; k < 3; ++k) {
                    double pp[3] = {pos[0], pos[1], pos[2]}, pm[3] = {pos[0], pos[1], pos[2]};
                    pp[k] += q->sv[k];
                    pm[k] -= q->sv[k];
                    g[k] = tex3d_linear_d(v, pp[0], pp[1], pp[2]) - tex3d_linear_d(v, pm[0], pm[1], pm[2]);
                }
                if (q->invertZ) g[2] = -g[2];
                double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
                double d = gn > 0 ? (g[0] * L[0] + g[1] * L[1] + g[2] * L[2]) / gn : -1;
                double s = d > 0 ? d * 0.8 + 0.16 * pow(d, 8.0) : 0.0;
                double wgt = (1 - A) * col[3];
                for (int c = 0; c < 4; ++c) sum[c] += wgt * (col[c] * 0.35 + col[c] * s);
                accObj[label] += (1 - A) * col[3];
                A += (1 - A) * col[3];
            }
            if (A > 0.995) break;
            continue;
        }
        /* surface candidate */
        for (int k = 0; k < 3; ++k) {
            double pp[3] = {pos[0], pos[1], pos[2]}, pm[3] = {pos[0], pos[1], pos[2]};
            pp[k] += q->sv[k];
            pm[k] -= q->sv[k];
            N[k] = tex3d_linear_d(v, pp[0], pp[1], pp[2]) - tex3d_linear_d(v, pm[0], pm[1], pm[2]);
        }
        if (q->invertZ) N[2] = -N[2];
        double nn = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
        A = nn > 0 ? (N[0] * L[0] + N[1] * L[1] + N[2] * L[2]) / nn : 0.0;
        if (A > 0) break;
        accu += step;
    }
    float out[4];
    if (type == MKO_VR) {
        if (sum[0] == 0 && sum[1] == 0 && sum[2] == 0 && sum[3] == 0)
            for (int c = 0; c < 4; ++c) out[c] = q->bg[c];
        else
            for (int c = 0; c < 4; ++c) out[c] = (float)sum[c];
    } else if (type == MKO_MIP) {
        if (A <= 0) for (int c = 0; c < 4; ++c) out[c] = q->bg[c];
        else for (int c = 0; c < 4; ++c) out[c] = (float)A;
    } else {
        if (A <= 0) for (int c = 0; c < 4; ++c) out[c] = q->bg[c];
        else { out[0] = out[1] = out[2] = (float)(A + 0.05); out[3] = 1; }
    }
    store_rgb(o, out);
}

int mko_render_vr(const mko_volume *v, int w, int h, int type, const float *params, int precision,
                  int nthreads, uint8_t *out_rgb, uint64_t *samples) {
    return mko_render_vr_rows(v, w, h, type, params, precision, nthreads, 0, 1, h, out_rgb, samples);
}

int mko_render_vr_rows(const mko_volume *v, int w, int h, int type, const float *params, int precision,
                       int nthreads, int row0, int row_step, int nrows, uint8_t *out_rgb, uint64_t *samples) {
    if (!v || !v->vox || !params || !out_rgb || w <= 0 || h <= 0 || type < 0 || type > 2) return 1;
    if (row0 < 0 || row_step <= 0 || nrows <= 0 || row0 + (nrows - 1) * row_step >= h) return 1;
    vrp q;
    unpack_vr(params, &q);
    uint64_t total = 0;
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : total)
#endif
    for (int r = 0; r < nrows; ++r) {
        const int y = row0 + r * row_step;
        for (int x = 0; x < w; ++x) {
            uint8_t *o = out_rgb + ((size_t)r * w + x) * 3;
            uint64_t n = 0;
            if (precision == MKO_EXACT64) pixel_d(v, &q, type, w, h, x, y, o);
            else if (type == MKO_VR) vr_pixel_f(v, &q, w, h, x, y, o, &n);
            else if (type == MKO_MIP) mip_pixel_f(v, &q, w, h, x, y, o, &n);
            else surf_pixel_f(v, &q, w, h, x, y, o, &n);
            total += n;
        }
    }
    (void)nthreads;
    if (samples) *samples = total;
    return 0;
}

/* ---------------------------------------------------------------- */
/* reslicing (core/kernel.cu:570-873)                               */

static short sat_short_f(float f) {
    if (f != f) return 0;
    if (f >= 32767.0f) return 32767;
    if (f <= -32768.0f) return -32768;
    return (short)f;
}

static short sat_short_d(double f) {
    if (f != f) return 0;
    if (f >= 32767.0) return 32767;
    if (f <= -32768.0) return -32768;
    return (short)f;
}

int mko_render_plane(const mko_volume *v, int w, int h, const float *p, int mpr_type, int nearest,
                     int precision, int nthreads, int16_t *out) {
    if (!v || !v->vox || !p || !out || w <= 0 || h <= 0 || mpr_type < 0 || mpr_type > 2) return 1;
    const float sp[3] = {p[0], p[1], p[2]}, dh[3] = {p[3], p[4], p[5]}, dv[3] = {p[6], p[7], p[8]};
    const float dn[3] = {p[9], p[10], p[11]}, lt[3] = {p[12], p[13], p[14]};
    const float ps = p[15];
    const int inv = p[16] != 0.0f;
    const float half = p[17];
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            short acc = mpr_type == 1 ? -32768 : 32767;
            double fsum = 0;
            for (float t = -half; t <= half; t += 1) {
                if (precision == MKO_EXACT64) {
                    double fl = (double)t * ps;
                    double f[3];
                    for (int k = 0; k < 3; ++k)
                        f[k] = (lt[k] + fl * dn[k] + (double)x * ps * dh[k] + (double)y * ps * dv[k]) /
                               ((double)sp[k] * v->dim[k]);
                    if (!inv) f[2] = 1.0 - f[2];
                    int in = f[0] >= 0 && f[0] <= 1 && f[1] >= 0 && f[1] <= 1 && f[2] >= 0 && f[2] <= 1;
                    double val;
                    if (!in) val = -32768;
                    else if (nearest)
                        val = 32768 * texel_d(v, (int)floor(f[0] * v->dim[0]), (int)floor(f[1] * v->dim[1]),
                                              (int)floor(f[2] * v->dim[2]));
                    else val = 32768 * tex3d_linear_d(v, f[0], f[1], f[2]);
                    if (mpr_type == 0) fsum += val;
                    else {
                        short s = sat_short_d(val);
                        if (mpr_type == 1) acc = acc > s ? acc : s;
                        else acc = acc < s ? acc : s;
                    }
                    continue;
                }
                float fLength = t * ps;
                float ptx = lt[0] + fLength * dn[0];
                float pty = lt[1] + fLength * dn[1];
                float ptz = lt[2] + fLength * dn[2];
                float fx = (ptx + x * ps * dh[0] + y * ps * dv[0]) / (sp[0] * (float)v->dim[0]);
                float fy = (pty + x * ps * dh[1] + y * ps * dv[1]) / (sp[1] * (float)v->dim[1]);
                float fz = (ptz + x * ps * dh[2] + y * ps * dv[2]) / (sp[2] * (float)v->dim[2]);
                if (!inv) fz = (float)(1.0 - (double)fz);
                int in = fx >= 0 && fx <= 1 && fy >= 0 && fy <= 1 && fz >= 0 && fz <= 1;
                float tv = 0.0f;
                if (in) tv = nearest ? mko_tex3d_point(v, fx, fy, fz) : mko_tex3d_linear(v, fx, fy, fz);
                if (mpr_type == 0) {
                    fsum += in ? (double)(32768 * tv) : -32768.0;
                } else {
                    short s = in ? sat_short_f(32768 * tv) : (short)-32768;
                    if (mpr_type == 1) acc = acc > s ? acc : s;
                    else acc = acc < s ? acc : s;
                }
            }
            if (mpr_type == 0) acc = sat_short_d(fsum / (double)(2 * half + 1));
            out[(size_t)y * w + x] = acc;
        }
    }
    (void)nthreads;
    return 0;
}

int mko_render_cpr(const mko_volume *v, int w, int h, const double *pts, const double *dirs, int invert_z,
                   int precision, int nthreads, int16_t *out) {
    if (!v || !v->vox || !pts || !dirs || !out || w <= 0 || h <= 0) return 1;
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
    for (int y = 0; y < h; ++y) {
        const double *pt = pts + 3 * (size_t)y;
        const double *dr = dirs + 3 * (size_t)y;
        for (int x = 0; x < w; ++x) {
            if (precision == MKO_EXACT64) {
                double f[3];
                for (int k = 0; k < 3; ++k) f[k] = (pt[k] + x * dr[k]) / v->dim[k];
                if (!invert_z) f[2] = 1.0 - f[2];
                if (f[0] < 0 || f[0] > 1 || f[1] < 0 || f[1] > 1 || f[2] < 0 || f[2] > 1)
                    out[(size_t)y * w + x] = -2048;
                else
                    out[(size_t)y * w + x] = sat_short_d(32768 * tex3d_linear_d(v, f[0], f[1], f[2]));
                continue;
            }
            float fx = (float)((pt[0] + x * dr[0]) / (double)v->dim[0]);
            float fy = (float)((pt[1] + x * dr[1]) / (double)v->dim[1]);
            float fz = (float)((pt[2] + x * dr[2]) / (double)v->dim[2]);
            if (!invert_z) fz = (float)(1.0 - (double)fz);
            if (fx < 0 || fx > 1 || fy < 0 || fy > 1 || fz < 0 || fz > 1)
                out[(size_t)y * w + x] = -2048;
            else
                out[(size_t)y * w + x] = sat_short_f(32768 * mko_tex3d_linear(v, fx, fy, fz));
        }
    }
    (void)nthreads;
    return 0;
}

/* ---------------------------------------------------------------- */
/* differentiable VR (the method of monkeygl_b200/csrc/mk_dvr.cu) in FP64 */

/* p: [0] w, [1] h, [2..4] dims, [5..7] maxLenSpacing, [8..16] camera matrix,
 * [17] scale, [18] xT, [19] yT, [20] step, [21] t_min, [22] lut_len.
 * vol: dims[0]*dims[1]*dims[2] doubles (x fastest); lut: lut_len*4 doubles;
 * image: w*h*3 doubles. */
int mko_dvr_forward_d(const double *p, const double *vol, const double *lut, int nthreads, double *image) {
    const int w = (int)p[0], h = (int)p[1];
    const int dim[3] = {(int)p[2], (int)p[3], (int)p[4]};
    const double *mls = p + 5, *M = p + 8;
    const double scale = p[17], xT = p[18], yT = p[19], step = p[20], t_min = p[21];
    const int n_lut = (int)p[22];
    if (w <= 0 || h <= 0 || dim[0] <= 0 || dim[1] <= 0 || dim[2] <= 0 || n_lut < 2 || !(step > 0)) return 1;
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const double u = (x - w / 2.0 - xT) / h, v = (y - h / 2.0 - yT) / h;
            double base[3], dir[3], lo = 0.0, hi = 1.732;
            int hit = 1;
            for (int k = 0; k < 3; ++k) {
                base[k] = (M[3 * k] * u + M[3 * k + 1] * (-0.866 * scale) + M[3 * k + 2] * v) * mls[k] + 0.5;
                dir[k] = M[3 * k + 1] * scale * mls[k];
                if (fabs(dir[k]) < 1e-12) {
                    if (base[k] < 0.0 || base[k] > 1.0) hit = 0;
                    continue;
                }
                double t0 = -base[k] / dir[k], t1 = (1.0 - base[k]) / dir[k];
                if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
                if (t0 > lo) lo = t0;
                if (t1 < hi) hi = t1;
            }
            double C[3] = {0, 0, 0}, T = 1.0;
            if (hit && lo < hi) {
                const double a0 = ceil(lo / step) * step;
                const int n = (int)floor((hi - a0) / step) + 1;
                for (int i = 0; i < n; ++i) {
                    const double a = a0 + i * step;
                    double c[3], fr[3];
                    int i0[3];
                    for (int k = 0; k < 3; ++k) {
                        c[k] = (base[k] + a * dir[k]) * dim[k] - 0.5;
                        double f = floor(c[k]);
                        i0[k] = (int)f;
                        fr[k] = c[k] - f;
                    }
                    double s = 0.0;
                    for (int dz = 0; dz < 2; ++dz)
                        for (int dy = 0; dy < 2; ++dy)
                            for (int dx = 0; dx < 2; ++dx) {
                                int ix = clampi(i0[0] + dx, 0, dim[0] - 1);
                                int iy = clampi(i0[1] + dy, 0, dim[1] - 1);
                                int iz = clampi(i0[2] + dz, 0, dim[2] - 1);
                                double wt = (dx ? fr[0] : 1 - fr[0]) * (dy ? fr[1] : 1 - fr[1]) * (dz ? fr[2] : 1 - fr[2]);
                                s += wt * vol[((size_t)iz * dim[1] + iy) * dim[0] + ix];
                            }
                    double xx = s * n_lut - 0.5, f = floor(xx), wgt = xx - f;
                    int k = (int)f, k0, k1;
                    if (k < 0) { k0 = k1 = 0; wgt = 0; }
                    else if (k >= n_lut - 1) { k0 = k1 = n_lut - 1; wgt = 0; }
                    else { k0 = k; k1 = k + 1; }
                    double q[4];
                    for (int ch = 0; ch < 4; ++ch) q[ch] = lut[4 * k0 + ch] + wgt * (lut[4 * k1 + ch] - lut[4 * k0 + ch]);
                    for (int ch = 0; ch < 3; ++ch) C[ch] += T * q[3] * q[ch];
                    T *= 1.0 - q[3];
                    if (T < t_min) break;
                }
            }
            for (int ch = 0; ch < 3; ++ch) image[((size_t)y * w + x) * 3 + ch] = C[ch];
        }
    }
    (void)nthreads;
    return 0;
}

/* Conditioning of a reverse march for the differentiable method: per ray, the
 * forward transmittances T_i in FP32, then T reconstructed backwards from the
 * final T by T_i = T_{i+1} / (1 - a_i) (the division a checkpoint-free
 * backward would make), compared with the forward values.  stats receives:
 * [0] rays with samples, [1] rays whose reconstruction is off by more than
 * 1e-3 relative at some sample (or divides by zero), [2] rays that meet an
 * opaque sample (1 - a_i == 0 in FP32), [3] the largest relative error over
 * the rays that stay finite, [4] samples in all rays.  Test infrastructure:
 * it measures the method, it renders nothing. */
int mko_dvr_reverse_stats(const double *p, const float *vol, const float *lut, int nthreads, double *stats) {
    const int w = (int)p[0], h = (int)p[1];
    const int dim[3] = {(int)p[2], (int)p[3], (int)p[4]};
    const double *mls = p + 5, *M = p + 8;
    const double scale = p[17], xT = p[18], yT = p[19], step = p[20], t_min = p[21];
    const int n_lut = (int)p[22];
    if (w <= 0 || h <= 0 || dim[0] <= 0 || dim[1] <= 0 || dim[2] <= 0 || n_lut < 2 || !(step > 0)) return 1;
    long long rays = 0, bad = 0, opaque = 0, samples = 0;
    double worst = 0.0;
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(+ : rays, bad, opaque, samples) reduction(max : worst)
#endif
    for (int y = 0; y < h; ++y) {
        float *Ts = (float *)malloc(sizeof(float) * 8192), *as = (float *)malloc(sizeof(float) * 8192);
        for (int x = 0; x < w; ++x) {
            const double u = (x - w / 2.0 - xT) / h, v = (y - h / 2.0 - yT) / h;
            double base[3], dir[3], lo = 0.0, hi = 1.732;
            int hit = 1;
            for (int k = 0; k < 3; ++k) {
                base[k] = (M[3 * k] * u + M[3 * k + 1] * (-0.866 * scale) + M[3 * k + 2] * v) * mls[k] + 0.5;
                dir[k] = M[3 * k + 1] * scale * mls[k];
                if (fabs(dir[k]) < 1e-12) {
                    if (base[k] < 0.0 || base[k] > 1.0) hit = 0;
                    continue;
                }
                double t0 = -base[k] / dir[k], t1 = (1.0 - base[k]) / dir[k];
                if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
                if (t0 > lo) lo = t0;
                if (t1 < hi) hi = t1;
            }
            if (!hit || !(lo < hi)) continue;
            const double a0 = ceil(lo / step) * step;
            int n = (int)floor((hi - a0) / step) + 1;
            if (n > 8190) n = 8190;
            float T = 1.0f;
            int m = 0;
            for (int i = 0; i < n; ++i) {
                const double a = a0 + i * step;
                float c[3], fr[3];
                int i0[3];
                for (int k = 0; k < 3; ++k) {
                    c[k] = (float)((base[k] + a * dir[k]) * dim[k] - 0.5);
                    float f = floorf(c[k]);
                    i0[k] = (int)f;
                    fr[k] = c[k] - f;
                }
                float s = 0.0f;
                for (int dz = 0; dz < 2; ++dz)
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) {
                            int ix = clampi(i0[0] + dx, 0, dim[0] - 1);
                            int iy = clampi(i0[1] + dy, 0, dim[1] - 1);
                            int iz = clampi(i0[2] + dz, 0, dim[2] - 1);
                            float wt = (dx ? fr[0] : 1 - fr[0]) * (dy ? fr[1] : 1 - fr[1]) * (dz ? fr[2] : 1 - fr[2]);
                            s += wt * vol[((size_t)iz * dim[1] + iy) * dim[0] + ix];
                        }
                float xx = s * n_lut - 0.5f, f = floorf(xx), wgt = xx - f;
                int k = (int)f, k0, k1;
                if (k < 0) { k0 = k1 = 0; wgt = 0; }
                else if (k >= n_lut - 1) { k0 = k1 = n_lut - 1; wgt = 0; }
                else { k0 = k; k1 = k + 1; }
                const float al = lut[4 * k0 + 3] + wgt * (lut[4 * k1 + 3] - lut[4 * k0 + 3]);
                Ts[m] = T;
                as[m] = al;
                ++m;
                T *= 1.0f - al;
                if (T < t_min) break;
            }
            if (m == 0) continue;
            ++rays;
            samples += m;
            float Tr = T;
            int is_opaque = 0;
            double e = 0.0;
            for (int i = m - 1; i >= 0; --i) {
                const float d = 1.0f - as[i];
                if (d == 0.0f) {
                    is_opaque = 1;
                    break;
                }
                Tr = Tr / d;
                const double ref = Ts[i] > 1e-30f ? Ts[i] : 1e-30;
                const double r = fabs((double)Tr - Ts[i]) / ref;
                if (!(r <= 1e30)) { is_opaque = 1; break; }
                if (r > e) e = r;
            }
            if (is_opaque) { ++opaque; ++bad; }
            else {
                if (e > 1e-3) ++bad;
                if (e > worst) worst = e;
            }
        }
        free(Ts);
        free(as);
    }
    stats[0] = (double)rays;
    stats[1] = (double)bad;
    stats[2] = (double)opaque;
    stats[3] = worst;
    stats[4] = (double)samples;
    (void)nthreads;
    return 0;
}
