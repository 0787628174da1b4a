// mk_dvr.cu -- differentiable direct volume rendering: forward and a
// hand-written backward of the front-to-back compositing, with respect to the
// transfer-function LUT entries and the voxel values.
//
// This has no counterpart in MonkeyGL.  It uses MonkeyGL's orthographic VR
// camera (the pixel -> ray mapping of core/kernel.cu:161-206) with the method
// made differentiable: a fixed step along the ray (no adaptive refinement), a
// float32 volume in [0, 1] sampled with exact trilinear weights (texel
// centres at (i+0.5)/dim, clamp to edge), the value used directly as the LUT
// coordinate (entry centres at (i+0.5)/n, linear interpolation, clamp), and
// compositing
//     C = sum_i T_i a_i c_i,   T_0 = 1,   T_{i+1} = T_i (1 - a_i),
// stopped after the sample that takes T below t_min.  The image is C (RGB).
//
// Backward.  With g = dL/dC and U_i the colour composited behind sample i
// seen from unit transmittance just after it (U_last = 0,
// U_{i-1} = a_i c_i + (1 - a_i) U_i),
//     dL/dc_i = T_i a_i g,     dL/da_i = T_i g . (c_i - U_i),
// with no division by (1 - a_i).  T_i comes from per-ray checkpoints of T
// every K samples: the backward walks segments of 16 samples from last to
// first, re-marching each forward from its checkpoint into registers.
// dL/dLUT goes through the interpolation weights into shared-memory bins
// (warp-aggregated per bin, then one global atomic per bin and block);
// dL/dvolume goes through the value's LUT slope and the trilinear weights
// into eight global reductions per sample.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "mk_internal.h"

namespace mk {

constexpr int kDvrMaxLut = 1024;
constexpr int kDvrSeg = 16;          // samples per recomputed segment
constexpr int kDvrMaxCkpt = 512;     // checkpoints per ray

struct DvrParams {
    int W, H;
    int dim[3];
    float fdim[3];
    float mls[3];
    float M[9];
    float scale, xT, yT;
    float step;
    float t_min;
    int lut_len;
    int ckpt;                        // samples between checkpoints (multiple of kDvrSeg)
    int max_ckpt;
};

struct Ray {
    float px, py, pz;                // normalized position at a = 0
    float dx, dy, dz;                // change of normalized position per unit a
    float a0;                        // first sample on the grid a0 + i * step
    int n;                           // samples inside the volume
};

__device__ __forceinline__ Ray make_ray(const DvrParams &P, int x, int y) {
    Ray r;
    const float u = (x - P.W / 2.0f - P.xT) / P.H;
    const float v = (y - P.H / 2.0f - P.yT) / P.H;
    float base[3], dir[3];
    for (int k = 0; k < 3; ++k) {
        // pos(a) = M (u, (a - 0.866) s, v) * mls + 0.5
        base[k] = (P.M[3 * k] * u + P.M[3 * k + 1] * (-0.866f * P.scale) + P.M[3 * k + 2] * v) * P.mls[k] + 0.5f;
        dir[k] = P.M[3 * k + 1] * P.scale * P.mls[k];
    }
    float lo = 0.0f, hi = 1.732f;
    bool hit = true;
    for (int k = 0; k < 3; ++k) {
        if (fabsf(dir[k]) < 1e-12f) {
            if (base[k] < 0.0f || base[k] > 1.0f) hit = false;
            continue;
        }
        float t0 = (0.0f - base[k]) / dir[k], t1 = (1.0f - base[k]) / dir[k];
        if (t0 > t1) {
            const float t = t0;
            t0 = t1;
            t1 = t;
        }
        lo = fmaxf(lo, t0);
        hi = fminf(hi, t1);
    }
    r.px = base[0];
    r.py = base[1];
    r.pz = base[2];
    r.dx = dir[0];
    r.dy = dir[1];
    r.dz = dir[2];
    r.a0 = ceilf(lo / P.step) * P.step;
    r.n = (hit && lo < hi) ? max(0, (int)floorf((hi - r.a0) / P.step) + 1) : 0;
    return r;
}

struct Sample {
    int i0[3];
    float w[3];
    float s;
};

__device__ __forceinline__ void trilinear(const DvrParams &P, const float *__restrict__ vol, const Ray &r, int i,
                                          Sample &S) {
    const float a = r.a0 + i * P.step;
    const float c[3] = {(r.px + a * r.dx) * P.fdim[0] - 0.5f, (r.py + a * r.dy) * P.fdim[1] - 0.5f,
                        (r.pz + a * r.dz) * P.fdim[2] - 0.5f};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float f = floorf(c[k]);
        S.i0[k] = (int)f;
        S.w[k] = c[k] - f;
    }
    float acc = 0.0f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int ix = min(max(S.i0[0] + dx, 0), P.dim[0] - 1);
                const int iy = min(max(S.i0[1] + dy, 0), P.dim[1] - 1);
                const int iz = min(max(S.i0[2] + dz, 0), P.dim[2] - 1);
                const float wt = (dx ? S.w[0] : 1.0f - S.w[0]) * (dy ? S.w[1] : 1.0f - S.w[1]) *
                                 (dz ? S.w[2] : 1.0f - S.w[2]);
                acc += wt * __ldg(&vol[((size_t)iz * P.dim[1] + iy) * P.dim[0] + ix]);
            }
    S.s = acc;
}

struct LutHit {
    int k0, k1;
    float w;                         // weight of k1
    float slope;                     // d(LUT coordinate)/d(value): n inside, 0 where clamped
};

__device__ __forceinline__ LutHit lut_index(const DvrParams &P, float s) {
    LutHit h;
    const int n = P.lut_len;
    const float x = s * n - 0.5f;
    const float f = floorf(x);
    const int k = (int)f;
    if (k < 0) {
        h.k0 = h.k1 = 0;
        h.w = 0.0f;
        h.slope = 0.0f;
    } else if (k >= n - 1) {
        h.k0 = h.k1 = n - 1;
        h.w = 0.0f;
        h.slope = 0.0f;
    } else {
        h.k0 = k;
        h.k1 = k + 1;
        h.w = x - f;
        h.slope = (float)n;
    }
    return h;
}

__device__ __forceinline__ float4 lut_fetch(const float4 *lut, const LutHit &h) {
    const float4 a = lut[h.k0], b = lut[h.k1];
    return make_float4(a.x + h.w * (b.x - a.x), a.y + h.w * (b.y - a.y), a.z + h.w * (b.z - a.z),
                       a.w + h.w * (b.w - a.w));
}

__device__ __forceinline__ int pixel_x(int bx, int tile_w) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    return bx * tile_w + (warp % (tile_w / 8)) * 8 + (lane & 7);
}

__device__ __forceinline__ int pixel_y(int by, int tile_w) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    return by * 8 + (warp / (tile_w / 8)) * 4 + (lane >> 3);
}

// ---------------------------------------------------------------------------
// forward: 256 threads = 32x8 pixels as 8x4 warp tiles

__global__ void __launch_bounds__(256) k_dvr_forward(DvrParams P, const float *__restrict__ vol,
                                                     const float4 *__restrict__ lut_g, float *__restrict__ image,
                                                     float *__restrict__ trans, float *__restrict__ work) {
    __shared__ float4 lut[kDvrMaxLut];
    for (int i = threadIdx.x; i < P.lut_len; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    const int x = pixel_x(blockIdx.x, 32), y = pixel_y(blockIdx.y, 32);
    if (x >= P.W || y >= P.H) return;
    const size_t pix = (size_t)y * P.W + x, npix = (size_t)P.W * P.H;
    float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
    const Ray r = make_ray(P, x, y);
    int i = 0;
    for (; i < r.n; ++i) {
        if (work && (i % P.ckpt) == 0) work[(size_t)(i / P.ckpt) * npix + pix] = T;
        Sample S;
        trilinear(P, vol, r, i, S);
        const float4 c = lut_fetch(lut, lut_index(P, S.s));
        const float wgt = T * c.w;
        cr += wgt * c.x;
        cg += wgt * c.y;
        cb += wgt * c.z;
        T *= (1.0f - c.w);
        if (T < P.t_min) {
            ++i;
            break;
        }
    }
    image[3 * pix + 0] = cr;
    image[3 * pix + 1] = cg;
    image[3 * pix + 2] = cb;
    trans[pix] = T;
    if (work) reinterpret_cast<int *>(work + (size_t)P.max_ckpt * npix)[pix] = i;   // samples taken
}

// ---------------------------------------------------------------------------
// backward: 128 threads = 16x8 pixels as 8x4 warp tiles

__device__ __forceinline__ void bin_add(float *bins, int k, float4 v) {
    // lanes that hit the same entry add their values first (warp shuffle),
    // then one lane per entry updates the shared-memory bin
    const unsigned active = __activemask();
    const unsigned same = __match_any_sync(active, k);
    const int leader = __ffs(same) - 1;
    const int lane = threadIdx.x & 31;
    float4 acc = v;
    if (__popc(same) > 1) {
        // sum over the lanes of `same` by walking their bits (groups are small)
        acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (unsigned m = same; m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            acc.x += __shfl_sync(same, v.x, src);
            acc.y += __shfl_sync(same, v.y, src);
            acc.z += __shfl_sync(same, v.z, src);
            acc.w += __shfl_sync(same, v.w, src);
        }
    }
    if (lane == leader) {
        atomicAdd(&bins[4 * k + 0], acc.x);
        atomicAdd(&bins[4 * k + 1], acc.y);
        atomicAdd(&bins[4 * k + 2], acc.z);
        atomicAdd(&bins[4 * k + 3], acc.w);
    }
}

__global__ void __launch_bounds__(128) k_dvr_backward(DvrParams P, const float *__restrict__ vol,
                                                      const float4 *__restrict__ lut_g,
                                                      const float *__restrict__ work,
                                                      const float *__restrict__ grad_image,
                                                      float *__restrict__ grad_lut, float *__restrict__ grad_vol) {
    __shared__ float4 lut[kDvrMaxLut];
    __shared__ float bins[kDvrMaxLut * 4];
    for (int i = threadIdx.x; i < P.lut_len; i += blockDim.x) {
        lut[i] = lut_g[i];
        bins[4 * i] = bins[4 * i + 1] = bins[4 * i + 2] = bins[4 * i + 3] = 0.0f;
    }
    __syncthreads();
    const int x = pixel_x(blockIdx.x, 16), y = pixel_y(blockIdx.y, 16);
    const size_t npix = (size_t)P.W * P.H;
    int n = 0;
    float gr = 0.f, gg = 0.f, gb = 0.f;
    Ray r;
    size_t pix = 0;
    if (x < P.W && y < P.H) {
        pix = (size_t)y * P.W + x;
        n = reinterpret_cast<const int *>(work + (size_t)P.max_ckpt * npix)[pix];
        gr = grad_image[3 * pix];
        gg = grad_image[3 * pix + 1];
        gb = grad_image[3 * pix + 2];
        if (gr == 0.0f && gg == 0.0f && gb == 0.0f) n = 0;
        r = make_ray(P, x, y);
    }
    // lanes with nothing to do still take part in the warp-wide bin updates
    float Ur = 0.f, Ug = 0.f, Ub = 0.f;
    const int nseg = (n + kDvrSeg - 1) / kDvrSeg;
    const int wseg = __reduce_max_sync(0xffffffffu, nseg);
    for (int seg = wseg - 1; seg >= 0; --seg) {
        const bool live = seg < nseg;
        float Ts[kDvrSeg];
        int s1 = 0;
        if (live) {
            const int s0 = seg * kDvrSeg;
            const int c = s0 / P.ckpt;
            float T = work[(size_t)c * npix + pix];
            for (int i = c * P.ckpt; i < s0; ++i) {
                Sample S;
                trilinear(P, vol, r, i, S);
                T *= 1.0f - lut_fetch(lut, lut_index(P, S.s)).w;
            }
            s1 = min(s0 + kDvrSeg, n) - s0;
#pragma unroll
            for (int j = 0; j < kDvrSeg; ++j) {
                Ts[j] = T;
                if (j < s1) {
                    Sample S;
                    trilinear(P, vol, r, s0 + j, S);
                    T *= 1.0f - lut_fetch(lut, lut_index(P, S.s)).w;
                }
            }
        }
#pragma unroll
        for (int j = kDvrSeg - 1; j >= 0; --j) {
            const bool on = live && j < s1;
            LutHit h;
            h.k0 = h.k1 = 0;
            h.w = 0.f;
            h.slope = 0.f;
            float4 d0 = make_float4(0.f, 0.f, 0.f, 0.f), d1 = d0;
            Sample S;
            float d_cr = 0.f, d_cg = 0.f, d_cb = 0.f, d_a = 0.f;
            if (on) {
                trilinear(P, vol, r, seg * kDvrSeg + j, S);
                h = lut_index(P, S.s);
                const float4 q = lut_fetch(lut, h);
                const float Ti = Ts[j];
                d_cr = Ti * q.w * gr;
                d_cg = Ti * q.w * gg;
                d_cb = Ti * q.w * gb;
                d_a = Ti * (gr * (q.x - Ur) + gg * (q.y - Ug) + gb * (q.z - Ub));
                Ur = q.w * q.x + (1.0f - q.w) * Ur;
                Ug = q.w * q.y + (1.0f - q.w) * Ug;
                Ub = q.w * q.z + (1.0f - q.w) * Ub;
                const float w1 = h.w, w0 = 1.0f - h.w;
                d0 = make_float4(w0 * d_cr, w0 * d_cg, w0 * d_cb, w0 * d_a);
                d1 = make_float4(w1 * d_cr, w1 * d_cg, w1 * d_cb, w1 * d_a);
            }
            bin_add(bins, h.k0, d0);
            bin_add(bins, h.k1, d1);
            if (on && grad_vol && h.slope != 0.0f) {
                const float4 L0 = lut[h.k0], L1 = lut[h.k1];
                const float ds = h.slope * (d_cr * (L1.x - L0.x) + d_cg * (L1.y - L0.y) + d_cb * (L1.z - L0.z) +
                                            d_a * (L1.w - L0.w));
                if (ds != 0.0f) {
#pragma unroll
                    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
                        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                            for (int dx = 0; dx < 2; ++dx) {
                                const int ix = min(max(S.i0[0] + dx, 0), P.dim[0] - 1);
                                const int iy = min(max(S.i0[1] + dy, 0), P.dim[1] - 1);
                                const int iz = min(max(S.i0[2] + dz, 0), P.dim[2] - 1);
                                const float wt = (dx ? S.w[0] : 1.0f - S.w[0]) * (dy ? S.w[1] : 1.0f - S.w[1]) *
                                                 (dz ? S.w[2] : 1.0f - S.w[2]);
                                atomicAdd(&grad_vol[((size_t)iz * P.dim[1] + iy) * P.dim[0] + ix], wt * ds);
                            }
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P.lut_len * 4; i += blockDim.x) {
        const float v = bins[i];
        if (v != 0.0f) atomicAdd(&grad_lut[i], v);
    }
}

static int fill(const mk_dvr_params *p, DvrParams &P) {
    if (!p || p->width <= 0 || p->height <= 0 || p->width > 16384 || p->height > 16384 || p->dims[0] <= 0 ||
        p->dims[1] <= 0 || p->dims[2] <= 0 || p->lut_len < 2 || p->lut_len > kDvrMaxLut || !(p->step > 0.0f) ||
        !(p->scale > 0.0f) || p->step < 1e-5f) {
        set_last_error("mk_dvr: bad parameters (image size, dims, 2 <= lut_len <= 1024, 1e-5 <= step, scale > 0)");
        return MK_ERR_INVALID_ARGUMENT;
    }
    P.W = p->width;
    P.H = p->height;
    for (int k = 0; k < 3; ++k) {
        P.dim[k] = p->dims[k];
        P.fdim[k] = (float)p->dims[k];
        P.mls[k] = p->max_len_spacing[k];
    }
    for (int i = 0; i < 9; ++i) P.M[i] = p->transform[i];
    P.scale = p->scale;
    P.xT = p->x_translate;
    P.yT = p->y_translate;
    P.step = p->step;
    P.t_min = p->t_min;
    P.lut_len = p->lut_len;
    const int steps = (int)(1.74f / p->step) + 2;
    int ck = kDvrSeg;
    while ((steps + ck - 1) / ck > kDvrMaxCkpt) ck *= 2;
    P.ckpt = ck;
    P.max_ckpt = (steps + ck - 1) / ck;
    return MK_OK;
}

}  // namespace mk

using namespace mk;

extern "C" int mk_dvr_workspace_floats(const mk_dvr_params *params, size_t *floats) {
    DvrParams P;
    if (!floats) return MK_ERR_INVALID_ARGUMENT;
    int rc = fill(params, P);
    if (rc != MK_OK) return rc;
    *floats = (size_t)(P.max_ckpt + 1) * P.W * P.H;
    return MK_OK;
}

extern "C" int mk_dvr_forward(const mk_dvr_params *params, const float *volume, const float *lut, float *image,
                              float *transmittance, float *workspace, void *stream) {
    DvrParams P;
    int rc = fill(params, P);
    if (rc != MK_OK) return rc;
    if (!volume || !lut || !image || !transmittance) {
        set_last_error("mk_dvr_forward: null pointer");
        return MK_ERR_INVALID_ARGUMENT;
    }
    dim3 grid((P.W + 31) / 32, (P.H + 7) / 8);
    k_dvr_forward<<<grid, 256, 0, (cudaStream_t)stream>>>(P, volume, reinterpret_cast<const float4 *>(lut), image,
                                                         transmittance, workspace);
    MK_CUDA_TRY(cudaGetLastError());
    return MK_OK;
}

extern "C" int mk_dvr_backward(const mk_dvr_params *params, const float *volume, const float *lut,
                               const float *workspace, const float *grad_image, float *grad_lut,
                               float *grad_volume, void *stream) {
    DvrParams P;
    int rc = fill(params, P);
    if (rc != MK_OK) return rc;
    if (!volume || !lut || !workspace || !grad_image || !grad_lut) {
        set_last_error("mk_dvr_backward: null pointer");
        return MK_ERR_INVALID_ARGUMENT;
    }
    dim3 grid((P.W + 15) / 16, (P.H + 7) / 8);
    k_dvr_backward<<<grid, 128, 0, (cudaStream_t)stream>>>(P, volume, reinterpret_cast<const float4 *>(lut), workspace,
                                                          grad_image, grad_lut, grad_volume);
    MK_CUDA_TRY(cudaGetLastError());
    return MK_OK;
}
