// mk_dvr.cu -- differentiable direct volume rendering: forward and a
// hand-written backward of the front-to-back compositing, with respect to the
// transfer-function LUT entries and the voxel values.
//
// This has no counterpart in MonkeyGL.  It uses MonkeyGL's orthographic VR
// camera (the pixel -> ray mapping of core/kernel.cu:161-206) with the method
// made differentiable: a fixed step along the ray (no adaptive refinement), a
// float32 volume in [0, 1] sampled with exact trilinear weights (texel
// centres at (i+0.5)/dim, clamp to edge), the value used directly as the LUT
// coordinate (entry i centred at (i+0.5)/n, linear interpolation, clamp), and
// compositing
//     C = sum_i T_i a_i c_i,   T_0 = 1,   T_{i+1} = T_i (1 - a_i),
// stopped after the sample that takes T below t_min.  The image is C (RGB).
// The texture unit is not used for the volume: its float32 trilinear filter
// combines the x and y weights in fixed point below 8 fractional bits, so a
// backward pass could not reproduce the weights of the forward one.
//
// Backward.  With g = dL/dC and U_i the colour composited behind sample i
// seen from unit transmittance just after it (U_last = 0,
// U_{i-1} = a_i c_i + (1 - a_i) U_i),
//     dL/dc_i = T_i a_i g,     dL/da_i = T_i g . (c_i - U_i).
// The backward reverse-marches each ray from its last sample, reconstructing
// T_i = T_{i+1} / (1 - a_i) from the transmittance the forward saved after
// the last sample; the forward also saves T every K samples (checkpoints),
// which reset the reconstruction at each checkpoint and give T_i where
// a_i = 1 leaves nothing to divide by (a re-march from the checkpoint).  A
// ray accumulates its dL/dLUT in registers while its samples stay in one LUT
// cell and its dL/dvolume while they stay in one voxel cell; a change of
// cell flushes the sums -- the LUT sums of the lanes flushing one cell are
// combined by warp shuffles before the shared-memory bins, which go to global
// memory once per block; the voxel sums take eight global reductions.
#include <cuda_runtime.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "mk_internal.h"

namespace mk {

constexpr int kDvrMaxLut = 1024;
constexpr int kDvrSeg = 16;              // samples per recomputed segment
constexpr int kDvrMaxCkpt = 512;         // checkpoints per ray
constexpr int kDvrViewsPerLaunch = 32;

struct DvrView {
    float M[9];
    float mls[3];
    float scale, xT, yT;
    float step;
    float t_min;
    int ckpt_shift;                      // samples between checkpoints = 1 << ckpt_shift (>= kDvrSeg)
    int max_ckpt;
    unsigned long long work_off;         // floats from the workspace start
};

struct DvrBatch {
    int W, H;
    int lut_len;
    int dim[3];
    int sxy;                             // dim[0] * dim[1]
    float fdim[3];
    DvrView v[kDvrViewsPerLaunch];
};

struct Ray {
    float px, py, pz;                    // normalized position at a = 0
    float dx, dy, dz;                    // change of normalized position per unit a
    float a0;                            // first sample on the grid a0 + i * step
    int n;                               // samples inside the volume
};

__device__ __forceinline__ Ray make_ray(const DvrBatch &B, const DvrView &V, int x, int y) {
    Ray r;
    const float u = (x - B.W / 2.0f - V.xT) / B.H;
    const float v = (y - B.H / 2.0f - V.yT) / B.H;
    float base[3], dir[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        // pos(a) = M (u, (a - 0.866) s, v) * mls + 0.5
        base[k] = (V.M[3 * k] * u + V.M[3 * k + 1] * (-0.866f * V.scale) + V.M[3 * k + 2] * v) * V.mls[k] + 0.5f;
        dir[k] = V.M[3 * k + 1] * V.scale * V.mls[k];
    }
    float lo = 0.0f, hi = 1.732f;
    bool hit = true;
#pragma unroll
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
    r.a0 = ceilf(lo / V.step) * V.step;
    r.n = (hit && lo < hi) ? max(0, (int)floorf((hi - r.a0) / V.step) + 1) : 0;
    return r;
}

// Cell and weights of sample i: texel coordinate pos*dim - 0.5, its integer
// part and fraction.  One expression (explicit fused multiply-adds) serves the
// forward and backward kernels, so both see the same cells and weights.
struct Cell {
    int ix, iy, iz;
    float wx, wy, wz;
};

__device__ __forceinline__ Cell sample_cell(const DvrBatch &B, const Ray &r, float step, int i) {
    const float a = __fmaf_rn((float)i, step, r.a0);
    const float cx = __fmaf_rn(__fmaf_rn(a, r.dx, r.px), B.fdim[0], -0.5f);
    const float cy = __fmaf_rn(__fmaf_rn(a, r.dy, r.py), B.fdim[1], -0.5f);
    const float cz = __fmaf_rn(__fmaf_rn(a, r.dz, r.pz), B.fdim[2], -0.5f);
    const float fx = floorf(cx), fy = floorf(cy), fz = floorf(cz);
    Cell c;
    c.ix = (int)fx;
    c.iy = (int)fy;
    c.iz = (int)fz;
    c.wx = cx - fx;
    c.wy = cy - fy;
    c.wz = cz - fz;
    return c;
}

__device__ __forceinline__ float lerp(float a, float b, float w) { return __fmaf_rn(w, b - a, a); }

// Trilinear value of a cell; cells inside the volume read their eight voxels
// without clamping (the common case), the boundary half-voxel clamps to edge.
__device__ __forceinline__ float trilinear(const DvrBatch &B, const float *__restrict__ vol, const Cell &c) {
    const int X = B.dim[0];
    float v0, v1, v2, v3, v4, v5, v6, v7;
    if ((unsigned)c.ix < (unsigned)(X - 1) && (unsigned)c.iy < (unsigned)(B.dim[1] - 1) &&
        (unsigned)c.iz < (unsigned)(B.dim[2] - 1)) {
        const float *p = vol + (c.iz * B.sxy + c.iy * X + c.ix);
        v0 = __ldg(p);
        v1 = __ldg(p + 1);
        v2 = __ldg(p + X);
        v3 = __ldg(p + X + 1);
        p += B.sxy;
        v4 = __ldg(p);
        v5 = __ldg(p + 1);
        v6 = __ldg(p + X);
        v7 = __ldg(p + X + 1);
    } else {
        const int x0 = min(max(c.ix, 0), X - 1), x1 = min(max(c.ix + 1, 0), X - 1);
        const int y0 = min(max(c.iy, 0), B.dim[1] - 1) * X, y1 = min(max(c.iy + 1, 0), B.dim[1] - 1) * X;
        const int z0 = min(max(c.iz, 0), B.dim[2] - 1) * B.sxy, z1 = min(max(c.iz + 1, 0), B.dim[2] - 1) * B.sxy;
        v0 = __ldg(vol + z0 + y0 + x0);
        v1 = __ldg(vol + z0 + y0 + x1);
        v2 = __ldg(vol + z0 + y1 + x0);
        v3 = __ldg(vol + z0 + y1 + x1);
        v4 = __ldg(vol + z1 + y0 + x0);
        v5 = __ldg(vol + z1 + y0 + x1);
        v6 = __ldg(vol + z1 + y1 + x0);
        v7 = __ldg(vol + z1 + y1 + x1);
    }
    const float a0 = lerp(v0, v1, c.wx), a1 = lerp(v2, v3, c.wx), a2 = lerp(v4, v5, c.wx), a3 = lerp(v6, v7, c.wx);
    return lerp(lerp(a0, a1, c.wy), lerp(a2, a3, c.wy), c.wz);
}

// LUT lookup: x = s*n - 0.5 clamped to [0, n-1]; cell k = floor, weight w of
// entry k+1.  L[k] holds the entries, D[k] = L[k+1] - L[k] (D[n-1] = 0).
struct LutCell {
    int k;
    float w;
    bool inside;                         // 0 <= x < n-1: the value's slope is n
};

__device__ __forceinline__ LutCell lut_cell(float s, int n) {
    LutCell c;
    const float x = __fmaf_rn(s, (float)n, -0.5f);
    c.inside = (x >= 0.0f) && (x < (float)(n - 1));
    const float xc = fminf(fmaxf(x, 0.0f), (float)(n - 1));
    c.k = (int)xc;
    c.w = xc - (float)c.k;
    return c;
}

__device__ __forceinline__ float4 lut_value(const float4 *L, const float4 *D, const LutCell &c) {
    const float4 a = L[c.k], d = D[c.k];
    return make_float4(__fmaf_rn(c.w, d.x, a.x), __fmaf_rn(c.w, d.y, a.y), __fmaf_rn(c.w, d.z, a.z),
                       __fmaf_rn(c.w, d.w, a.w));
}

__device__ __forceinline__ void load_lut(const float4 *__restrict__ lut_g, float4 *L, float4 *D, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 a = lut_g[i];
        L[i] = a;
        if (i + 1 < n) {
            const float4 b = lut_g[i + 1];
            D[i] = make_float4(b.x - a.x, b.y - a.y, b.z - a.z, b.w - a.w);
        } else {
            D[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
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
// forward: 256 threads = 32x8 pixels as 8x4 warp tiles; blockIdx.z = view

__global__ void __launch_bounds__(256) k_dvr_forward(const __grid_constant__ DvrBatch B,
                                                     const float *__restrict__ vol,
                                                     const float4 *__restrict__ lut_g, float *__restrict__ images,
                                                     float *__restrict__ trans, float *__restrict__ work) {
    extern __shared__ float4 sm[];
    float4 *L = sm, *D = sm + B.lut_len;
    load_lut(lut_g, L, D, B.lut_len);
    __syncthreads();
    const DvrView &V = B.v[blockIdx.z];
    const int x = pixel_x(blockIdx.x, 32), y = pixel_y(blockIdx.y, 32);
    if (x >= B.W || y >= B.H) return;
    const size_t npix = (size_t)B.W * B.H, pix = (size_t)y * B.W + x;
    float *wk = work ? work + V.work_off : nullptr;
    const int cmask = (1 << V.ckpt_shift) - 1;
    float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
    const Ray r = make_ray(B, V, x, y);
    int i = 0;
    for (; i < r.n; ++i) {
        if (wk && (i & cmask) == 0) wk[(size_t)(i >> V.ckpt_shift) * npix + pix] = T;
        const float s = trilinear(B, vol, sample_cell(B, r, V.step, i));
        const float4 c = lut_value(L, D, lut_cell(s, B.lut_len));
        const float wgt = T * c.w;
        cr = __fmaf_rn(wgt, c.x, cr);
        cg = __fmaf_rn(wgt, c.y, cg);
        cb = __fmaf_rn(wgt, c.z, cb);
        T *= (1.0f - c.w);
        if (T < V.t_min) {
            ++i;
            break;
        }
    }
    const size_t o = (size_t)blockIdx.z * npix + pix;
    images[3 * o + 0] = cr;
    images[3 * o + 1] = cg;
    images[3 * o + 2] = cb;
    trans[o] = T;
    if (wk) {
        reinterpret_cast<int *>(wk + (size_t)V.max_ckpt * npix)[pix] = i;   // samples taken
        wk[(size_t)(V.max_ckpt + 1) * npix + pix] = T;                      // transmittance after them
    }
}

// ---------------------------------------------------------------------------
// backward: 128 threads = 16x8 pixels as 8x4 warp tiles; blockIdx.z = view

// Adds the LUT-gradient runs that lanes end at this step (cell k: a0 to
// entry k, a1 to entry k + 1) to the block's shared bins.  Every lane of the
// warp calls it.  Lanes ending a run on the same cell are summed by warp
// shuffles first (a butterfly per cell), so a cell takes one set of
// shared-memory atomics per warp and step; a lane alone on its cell adds
// directly.
__device__ __forceinline__ void flush_lut_warp(float *bins, int n, bool flush, int k, const float4 &a0,
                                               const float4 &a1) {
    const unsigned FULL = 0xffffffffu;
    if (__ballot_sync(FULL, flush) == 0u) return;
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(FULL, flush ? k : -1);
    const bool alone = flush && __popc(peers) == 1;
    if (alone) {
        atomicAdd(&bins[4 * k + 0], a0.x);
        atomicAdd(&bins[4 * k + 1], a0.y);
        atomicAdd(&bins[4 * k + 2], a0.z);
        atomicAdd(&bins[4 * k + 3], a0.w);
        if (k + 1 < n) {
            atomicAdd(&bins[4 * k + 4], a1.x);
            atomicAdd(&bins[4 * k + 5], a1.y);
            atomicAdd(&bins[4 * k + 6], a1.z);
            atomicAdd(&bins[4 * k + 7], a1.w);
        }
    }
    unsigned shared = __ballot_sync(FULL, flush && !alone);
    while (shared) {
        const int leader = __ffs(shared) - 1;
        const unsigned grp = __shfl_sync(FULL, peers, leader);
        const bool in = (grp >> lane) & 1u;
        float v[8] = {in ? a0.x : 0.f, in ? a0.y : 0.f, in ? a0.z : 0.f, in ? a0.w : 0.f,
                      in ? a1.x : 0.f, in ? a1.y : 0.f, in ? a1.z : 0.f, in ? a1.w : 0.f};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int c = 0; c < 8; ++c) v[c] += __shfl_xor_sync(FULL, v[c], o);
        }
        if (lane == leader) {
#pragma unroll
            for (int c = 0; c < 4; ++c) atomicAdd(&bins[4 * k + c], v[c]);
            if (k + 1 < n) {
#pragma unroll
                for (int c = 0; c < 4; ++c) atomicAdd(&bins[4 * k + 4 + c], v[4 + c]);
            }
        }
        shared &= ~grp;
    }
}

__device__ __forceinline__ void flush_vol(float *__restrict__ gv, const DvrBatch &B, int ix, int iy, int iz,
                                          const float (&acc)[8]) {
    if (ix == INT_MIN) return;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        if (acc[c] == 0.0f) continue;
        const int x = min(max(ix + (c & 1), 0), B.dim[0] - 1);
        const int y = min(max(iy + ((c >> 1) & 1), 0), B.dim[1] - 1);
        const int z = min(max(iz + (c >> 2), 0), B.dim[2] - 1);
        atomicAdd(&gv[z * B.sxy + y * B.dim[0] + x], acc[c]);
    }
}

// Reverse march.  A ray walks its samples from the last to the first,
// reconstructing T_i = T_{i+1} / (1 - a_i) from the transmittance saved after
// its last sample; at every checkpoint (each 2^ckpt_shift samples) T is taken
// from the forward pass instead, so a reconstruction never runs for more
// than one checkpoint interval.  A sample with a_i = 1 (nothing to divide
// by) takes T_i by re-marching forward from its interval's checkpoint.  Each
// sample is fetched once otherwise.  The walk is warp-uniform (lanes past
// their first sample idle), so the LUT-gradient runs that end in one step
// can be combined across the warp.
template <bool VOLGRAD>
__global__ void __launch_bounds__(128) k_dvr_backward(const __grid_constant__ DvrBatch B,
                                                      const float *__restrict__ vol,
                                                      const float4 *__restrict__ lut_g,
                                                      const float *__restrict__ work,
                                                      const float *__restrict__ grad_images,
                                                      float *__restrict__ grad_lut, float *__restrict__ grad_vol) {
    extern __shared__ float4 sm[];
    const int n = B.lut_len;
    float4 *L = sm, *D = sm + n;
    float *bins = reinterpret_cast<float *>(sm + 2 * n);
    load_lut(lut_g, L, D, n);
    for (int i = threadIdx.x; i < 4 * n; i += blockDim.x) bins[i] = 0.0f;
    __syncthreads();

    const DvrView &V = B.v[blockIdx.z];
    const int x = pixel_x(blockIdx.x, 16), y = pixel_y(blockIdx.y, 16);
    const bool in_image = x < B.W && y < B.H;
    const size_t npix = (size_t)B.W * B.H, pix = in_image ? (size_t)y * B.W + x : 0;
    const float *wk = work + V.work_off;
    const size_t o = (size_t)blockIdx.z * npix + pix;
    float gr = 0.f, gg = 0.f, gb = 0.f, T = 0.f;
    int ns = 0;
    if (in_image) {
        gr = grad_images[3 * o];
        gg = grad_images[3 * o + 1];
        gb = grad_images[3 * o + 2];
        ns = reinterpret_cast<const int *>(wk + (size_t)V.max_ckpt * npix)[pix];
        T = wk[(size_t)(V.max_ckpt + 1) * npix + pix];
        if (gr == 0.0f && gg == 0.0f && gb == 0.0f) ns = 0;
    }
    const Ray r = make_ray(B, V, x, y);
    const int cmask = (1 << V.ckpt_shift) - 1;
    int steps = ns;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) steps = max(steps, __shfl_xor_sync(0xffffffffu, steps, off));
    float Ur = 0.f, Ug = 0.f, Ub = 0.f;
    int lk = -1;
    float4 la0 = make_float4(0.f, 0.f, 0.f, 0.f), la1 = la0;
    int vx = INT_MIN, vy = 0, vz = 0;
    float va[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) va[c] = 0.0f;

    for (int t = 0; t < steps; ++t) {
        const int i = ns - 1 - t;
        const bool live = i >= 0;
        LutCell h;
        h.k = -1;
        h.w = 0.0f;
        h.inside = false;
        float d_cr = 0.f, d_cg = 0.f, d_cb = 0.f, d_a = 0.f;
        Cell c = {};
        if (live) {
            c = sample_cell(B, r, V.step, i);
            h = lut_cell(trilinear(B, vol, c), n);
            const float4 q = lut_value(L, D, h);
            const float d = 1.0f - q.w;
            float Ti;
            if ((i & cmask) == 0) {
                Ti = wk[(size_t)(i >> V.ckpt_shift) * npix + pix];
            } else if (d != 0.0f) {
                Ti = T / d;
            } else {
                Ti = wk[(size_t)(i >> V.ckpt_shift) * npix + pix];
                for (int j = i & ~cmask; j < i; ++j)
                    Ti *= 1.0f - lut_value(L, D, lut_cell(trilinear(B, vol, sample_cell(B, r, V.step, j)), n)).w;
            }
            T = Ti;
            d_cr = Ti * q.w * gr;
            d_cg = Ti * q.w * gg;
            d_cb = Ti * q.w * gb;
            d_a = Ti * (gr * (q.x - Ur) + gg * (q.y - Ug) + gb * (q.z - Ub));
            Ur = q.w * q.x + (1.0f - q.w) * Ur;
            Ug = q.w * q.y + (1.0f - q.w) * Ug;
            Ub = q.w * q.z + (1.0f - q.w) * Ub;
        }
        const bool change = live && h.k != lk;
        flush_lut_warp(bins, n, change && lk >= 0, lk, la0, la1);
        if (change) {
            lk = h.k;
            la0 = make_float4(0.f, 0.f, 0.f, 0.f);
            la1 = la0;
        }
        if (live) {
            const float w1 = h.w, w0 = 1.0f - h.w;
            la0.x += w0 * d_cr;
            la0.y += w0 * d_cg;
            la0.z += w0 * d_cb;
            la0.w += w0 * d_a;
            la1.x += w1 * d_cr;
            la1.y += w1 * d_cg;
            la1.z += w1 * d_cb;
            la1.w += w1 * d_a;
            if (VOLGRAD && h.inside) {
                const float4 dd = D[h.k];
                const float ds = (float)n * (d_cr * dd.x + d_cg * dd.y + d_cb * dd.z + d_a * dd.w);
                if (ds != 0.0f) {
                    if (c.ix != vx || c.iy != vy || c.iz != vz) {
                        flush_vol(grad_vol, B, vx, vy, vz, va);
                        vx = c.ix;
                        vy = c.iy;
                        vz = c.iz;
#pragma unroll
                        for (int k = 0; k < 8; ++k) va[k] = 0.0f;
                    }
                    const float y0z0 = (1.0f - c.wy) * (1.0f - c.wz) * ds, y1z0 = c.wy * (1.0f - c.wz) * ds;
                    const float y0z1 = (1.0f - c.wy) * c.wz * ds, y1z1 = c.wy * c.wz * ds;
                    va[0] += (1.0f - c.wx) * y0z0;
                    va[1] += c.wx * y0z0;
                    va[2] += (1.0f - c.wx) * y1z0;
                    va[3] += c.wx * y1z0;
                    va[4] += (1.0f - c.wx) * y0z1;
                    va[5] += c.wx * y0z1;
                    va[6] += (1.0f - c.wx) * y1z1;
                    va[7] += c.wx * y1z1;
                }
            }
        }
    }
    flush_lut_warp(bins, n, lk >= 0, lk, la0, la1);
    if (VOLGRAD) flush_vol(grad_vol, B, vx, vy, vz, va);
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * n; i += blockDim.x) {
        const float v = bins[i];
        if (v != 0.0f) atomicAdd(&grad_lut[i], v);
    }
}

// ---------------------------------------------------------------------------
// host side

// Checkpoint spacing of a view: 16 samples, doubled until at most 512
// checkpoints cover the longest ray (1.732 in the ray parameter).
static void view_layout(const mk_dvr_params &p, int &ckpt_shift, int &max_ckpt) {
    const int steps = (int)(1.74f / p.step) + 2;
    int sh = 4;
    while (((steps + (1 << sh) - 1) >> sh) > kDvrMaxCkpt) ++sh;
    ckpt_shift = sh;
    max_ckpt = (steps + (1 << sh) - 1) >> sh;
}

// Workspace floats of one view: max_ckpt checkpoint planes, a plane of sample
// counts and a plane of final transmittances.
static size_t view_floats(const mk_dvr_params &p) {
    int sh, mc;
    view_layout(p, sh, mc);
    return (size_t)(mc + 2) * p.width * p.height;
}

static int check_views(const mk_dvr_params *views, int nviews) {
    if (!views || nviews <= 0) {
        set_last_error("mk_dvr: no views");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const mk_dvr_params &a = views[0];
    for (int i = 0; i < nviews; ++i) {
        const mk_dvr_params &p = views[i];
        if (p.width <= 0 || p.height <= 0 || p.width > 16384 || p.height > 16384 || p.dims[0] <= 0 ||
            p.dims[1] <= 0 || p.dims[2] <= 0 || p.lut_len < 2 || p.lut_len > kDvrMaxLut || !(p.step >= 1e-5f) ||
            !(p.scale > 0.0f) || !(p.t_min >= 0.0f)) {
            set_last_error("mk_dvr: bad view parameters (image size 1..16384, dims > 0, 2 <= lut_len <= 1024, "
                           "step >= 1e-5, scale > 0, t_min >= 0)");
            return MK_ERR_INVALID_ARGUMENT;
        }
        if ((double)p.dims[0] * p.dims[1] * p.dims[2] >= 2147483648.0) {
            set_last_error("mk_dvr: the volume must have fewer than 2^31 voxels");
            return MK_ERR_INVALID_ARGUMENT;
        }
        if (p.width != a.width || p.height != a.height || p.lut_len != a.lut_len || p.dims[0] != a.dims[0] ||
            p.dims[1] != a.dims[1] || p.dims[2] != a.dims[2]) {
            set_last_error("mk_dvr: the views of one call must share width, height, dims and lut_len");
            return MK_ERR_INVALID_ARGUMENT;
        }
    }
    return MK_OK;
}

static void fill_batch(const mk_dvr_params *views, int first, int count, size_t work_off0, DvrBatch &B) {
    memset(&B, 0, sizeof(B));
    const mk_dvr_params &a = views[first];
    B.W = a.width;
    B.H = a.height;
    B.lut_len = a.lut_len;
    for (int k = 0; k < 3; ++k) {
        B.dim[k] = a.dims[k];
        B.fdim[k] = (float)a.dims[k];
    }
    B.sxy = a.dims[0] * a.dims[1];
    size_t off = work_off0;
    for (int i = 0; i < count; ++i) {
        const mk_dvr_params &p = views[first + i];
        DvrView &V = B.v[i];
        for (int m = 0; m < 9; ++m) V.M[m] = p.transform[m];
        for (int k = 0; k < 3; ++k) V.mls[k] = p.max_len_spacing[k];
        V.scale = p.scale;
        V.xT = p.x_translate;
        V.yT = p.y_translate;
        V.step = p.step;
        V.t_min = p.t_min;
        view_layout(p, V.ckpt_shift, V.max_ckpt);
        V.work_off = off;
        off += view_floats(p);
    }
}

}  // namespace mk

using namespace mk;

extern "C" int mk_dvr_workspace_floats(const mk_dvr_params *views, int nviews, size_t *floats) {
    if (!floats) {
        set_last_error("mk_dvr_workspace_floats: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    int rc = check_views(views, nviews);
    if (rc != MK_OK) return rc;
    size_t total = 0;
    for (int i = 0; i < nviews; ++i) total += view_floats(views[i]);
    *floats = total;
    return MK_OK;
}

extern "C" int mk_dvr_forward(const mk_dvr_params *views, int nviews, const float *volume, const float *lut,
                              float *images, float *transmittance, float *workspace, void *stream) {
    if (!volume || !lut || !images || !transmittance) {
        set_last_error("mk_dvr_forward: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    int rc = check_views(views, nviews);
    if (rc != MK_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t npix = (size_t)views[0].width * views[0].height;
    const size_t smem = 2 * (size_t)views[0].lut_len * sizeof(float4);
    MK_CUDA_TRY(cudaFuncSetAttribute(k_dvr_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    size_t off = 0;
    DvrBatch B;
    for (int first = 0; first < nviews; first += kDvrViewsPerLaunch) {
        const int count = min(kDvrViewsPerLaunch, nviews - first);
        fill_batch(views, first, count, off, B);
        for (int i = 0; i < count; ++i) off += view_floats(views[first + i]);
        dim3 grid((B.W + 31) / 32, (B.H + 7) / 8, count);
        k_dvr_forward<<<grid, 256, smem, s>>>(B, volume, reinterpret_cast<const float4 *>(lut),
                                              images + (size_t)first * npix * 3, transmittance + (size_t)first * npix,
                                              workspace);
        MK_CUDA_TRY(cudaGetLastError());
    }
    return MK_OK;
}

extern "C" int mk_dvr_backward(const mk_dvr_params *views, int nviews, const float *volume, const float *lut,
                               const float *workspace, const float *grad_images, float *grad_lut,
                               float *grad_volume, void *stream) {
    if (!volume || !lut || !workspace || !grad_images || !grad_lut) {
        set_last_error("mk_dvr_backward: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    int rc = check_views(views, nviews);
    if (rc != MK_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t npix = (size_t)views[0].width * views[0].height;
    const size_t smem = 3 * (size_t)views[0].lut_len * sizeof(float4);
    auto kern = grad_volume ? k_dvr_backward<true> : k_dvr_backward<false>;
    MK_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    size_t off = 0;
    DvrBatch B;
    for (int first = 0; first < nviews; first += kDvrViewsPerLaunch) {
        const int count = min(kDvrViewsPerLaunch, nviews - first);
        fill_batch(views, first, count, off, B);
        for (int i = 0; i < count; ++i) off += view_floats(views[first + i]);
        dim3 grid((B.W + 15) / 16, (B.H + 7) / 8, count);
        kern<<<grid, 128, smem, s>>>(B, volume, reinterpret_cast<const float4 *>(lut), workspace,
                                     grad_images + (size_t)first * npix * 3, grad_lut, grad_volume);
        MK_CUDA_TRY(cudaGetLastError());
    }
    return MK_OK;
}
