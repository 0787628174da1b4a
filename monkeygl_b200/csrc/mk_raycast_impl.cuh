// mk_raycast_impl.cuh -- device code of the orthographic ray caster: the
// per-tile march shared by the one-frame kernel (mk_raycast.cu) and the
// serving kernel (mk_server.cu).  The method and its organisation on the GPU
// are described at the top of mk_raycast.cu.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "mk_internal.h"
#include "mk_math.h"

namespace mk {

enum RayMode { kModeVR = 0, kModeMIP = 1, kModeSurface = 2 };
enum Track { kTrackNone = 0, kTrackShared = 1, kTrackLocal = 2 };

struct RayParams {
    int W, H;
    float fdim[3];               // dims as float (index = trunc(pos * dim))
    int dimi[3];
    float mls[3];                // f3maxLenSpacing
    float sv[3];                 // f3SpacingVoxel
    float xT, yT, scale;
    float M[9];
    int invertZ;
    int voi[6];
    float4 bg;
    float step1;                 // 1 / dim_z
    float limit;                 // smallest float > 1.732
    const float *accu;           // accuLength schedule table
    int accu_len;
    int rgba;                    // 1 = 4 bytes per pixel
    int skip;
    uint8_t *out;
    unsigned long long *counter; // sample counting mode
    uint32_t *vox_bits;          // counting mode: voxels inside trilinear footprints (may be null)
    uint32_t *lab_bits;          // counting mode: label voxels read (may be null)
};

struct LabelSmem {
    cudaTextureObject_t tf[MK_MAX_LABELS];
    float alpha[MK_MAX_LABELS];
    float ww[MK_MAX_LABELS];
    float wl[MK_MAX_LABELS];
    signed char slot[MK_MAX_LABELS];   // >=0 tracked slot, -1 uncapped, -2 never composites
};

// The camera-matrix product of core/kernel.cu:31-38 (helper_math dot()).
// nvcc fuses MonkeyGL's x*x' + y*y' + z*z' left to right into two FMAs; the
// same expression written plainly here is contracted differently in this
// kernel, so the order is spelled out.  Comparing images against MonkeyGL's
// kernel on tilted views, this is the only order of the six fused and one
// unfused forms that reproduces every sample position.
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fmaf_rn(az, bz, __fmaf_rn(ay, by, __fmul_rn(ax, bx)));
}

// One sample position of the reference schedule (core/kernel.cu:197-206).
__device__ __forceinline__ float3 ray_pos(const RayParams &P, float u, float v, float a) {
    const float fy = ray_fy(a, P.scale);
    float3 p;
    p.x = dot3(u, fy, v, P.M[0], P.M[1], P.M[2]);
    p.y = dot3(u, fy, v, P.M[3], P.M[4], P.M[5]);
    p.z = dot3(u, fy, v, P.M[6], P.M[7], P.M[8]);
    p.x = p.x * P.mls[0] + 0.5f;
    p.y = p.y * P.mls[1] + 0.5f;
    p.z = p.z * P.mls[2] + 0.5f;
    if (P.invertZ) p.z = 1.0f - p.z;
    return p;
}

// Interval [a0, a1] of accuLength where the ray may touch the VOI, from the
// affine form pos(fy) = A + fy * B with a two-voxel margin.  Returns false if
// the ray misses.
__device__ inline bool ray_interval(const RayParams &P, float u, float v, float &a0, float &a1) {
    float A[3], B[3];
    for (int k = 0; k < 3; ++k) {
        A[k] = (u * P.M[3 * k + 0] + v * P.M[3 * k + 2]) * P.mls[k] + 0.5f;
        B[k] = P.M[3 * k + 1] * P.mls[k];
    }
    if (P.invertZ) {
        A[2] = 1.0f - A[2];
        B[2] = -B[2];
    }
    float lo = -INFINITY, hi = INFINITY;
    for (int k = 0; k < 3; ++k) {
        const float d = P.fdim[k];
        const float bl = ((float)P.voi[2 * k] - 3.0f) / d;
        const float bh = ((float)P.voi[2 * k + 1] + 3.0f) / d;
        if (fabsf(B[k]) < 1e-30f) {
            if (A[k] < bl || A[k] > bh) return false;
            continue;
        }
        float t0 = (bl - A[k]) / B[k], t1 = (bh - A[k]) / B[k];
        if (t0 > t1) {
            float t = t0;
            t0 = t1;
            t1 = t;
        }
        lo = fmaxf(lo, t0);
        hi = fminf(hi, t1);
    }
    if (!(lo <= hi)) return false;
    a0 = lo / P.scale + 0.866f;
    a1 = hi / P.scale + 0.866f;
    return true;
}

// Index of the last schedule entry <= a (0 if none).
__device__ __forceinline__ int accu_lower(const RayParams &P, float a) {
    int lo = 0, hi = P.accu_len - 1;
    if (!(a > P.accu[0])) return 0;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.accu[mid] <= a) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ bool outside_voi(const RayParams &P, int ix, int iy, int iz) {
    return ix < P.voi[0] || ix > P.voi[1] || iy < P.voi[2] || iy > P.voi[3] || iz < P.voi[4] ||
           iz > P.voi[5];
}

__device__ __forceinline__ int brick_index(const RayParams &P, const BrickView &BV, int ix, int iy,
                                           int iz) {
    ix = min(max(ix, 0), P.dimi[0] - 1);
    iy = min(max(iy, 0), P.dimi[1] - 1);
    iz = min(max(iz, 0), P.dimi[2] - 1);
    return ((iz >> kBrickShift) * BV.nby + (iy >> kBrickShift)) * BV.nbx + (ix >> kBrickShift);
}

// Number of further coarse steps that stay inside brick (bx,by,bz) with a
// 0.05-voxel margin, capped at 64.  Position p is in voxel units.
__device__ __forceinline__ int steps_in_brick(const float3 &pv, const float3 &dv, int ix, int iy,
                                              int iz) {
    float t = 64.0f;
    const float e = 0.05f;
    const float lo[3] = {(float)((ix >> kBrickShift) << kBrickShift),
                         (float)((iy >> kBrickShift) << kBrickShift),
                         (float)((iz >> kBrickShift) << kBrickShift)};
    const float pp[3] = {pv.x, pv.y, pv.z};
    const float dd[3] = {dv.x, dv.y, dv.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (dd[k] > 1e-6f) t = fminf(t, (lo[k] + kBrick - e - pp[k]) / dd[k]);
        else if (dd[k] < -1e-6f) t = fminf(t, (pp[k] - lo[k] - e) / -dd[k]);
    }
    return t > 0.0f ? (int)t : 0;
}

// Counting mode: mark the eight texels of a trilinear fetch at normalized
// position (x, y, z) under clamp addressing.
__device__ inline void mark_footprint(const RayParams &P, float x, float y, float z) {
    if (!P.vox_bits) return;
    int lo[3], hi[3];
    const float c[3] = {x, y, z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int i0 = (int)floorf(c[k] * P.fdim[k] - 0.5f);
        lo[k] = min(max(i0, 0), P.dimi[k] - 1);
        hi[k] = min(max(i0 + 1, 0), P.dimi[k] - 1);
    }
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                const size_t idx = ((size_t)(dz ? hi[2] : lo[2]) * P.dimi[1] + (dy ? hi[1] : lo[1])) *
                                       P.dimi[0] + (dx ? hi[0] : lo[0]);
                atomicOr(&P.vox_bits[idx >> 5], 1u << (idx & 31));
            }
}

__device__ inline void mark_gradient(const RayParams &P, float3 pos) {
    mark_footprint(P, pos.x + P.sv[0], pos.y, pos.z);
    mark_footprint(P, pos.x - P.sv[0], pos.y, pos.z);
    mark_footprint(P, pos.x, pos.y + P.sv[1], pos.z);
    mark_footprint(P, pos.x, pos.y - P.sv[1], pos.z);
    mark_footprint(P, pos.x, pos.y, pos.z + P.sv[2]);
    mark_footprint(P, pos.x, pos.y, pos.z - P.sv[2]);
}

__device__ inline void mark_label(const RayParams &P, int ix, int iy, int iz) {
    if (!P.lab_bits) return;
    ix = min(max(ix, 0), P.dimi[0] - 1);
    iy = min(max(iy, 0), P.dimi[1] - 1);
    iz = min(max(iz, 0), P.dimi[2] - 1);
    const size_t idx = ((size_t)iz * P.dimi[1] + iy) * P.dimi[0] + ix;
    atomicOr(&P.lab_bits[idx >> 5], 1u << (idx & 31));
}

// Central-difference normal and headlight shading (core/kernel.cu:49-81).
__device__ __forceinline__ float4 shade(float4 sum, float alphaAcc, cudaTextureObject_t vol,
                                        float3 pos, float4 col, float3 L, const RayParams &P) {
    float3 N;
    N.x = tex3D<float>(vol, pos.x + P.sv[0], pos.y, pos.z) - tex3D<float>(vol, pos.x - P.sv[0], pos.y, pos.z);
    N.y = tex3D<float>(vol, pos.x, pos.y + P.sv[1], pos.z) - tex3D<float>(vol, pos.x, pos.y - P.sv[1], pos.z);
    N.z = tex3D<float>(vol, pos.x, pos.y, pos.z + P.sv[2]) - tex3D<float>(vol, pos.x, pos.y, pos.z - P.sv[2]);
    if (P.invertZ) N.z = -N.z;
    const float inv = rsqrtf(N.x * N.x + N.y * N.y + N.z * N.z);
    N.x = N.x * inv;
    N.y = N.y * inv;
    N.z = N.z * inv;
    float diffuse = N.x * L.x + N.y * L.y + N.z * L.z;
    float4 clr = make_float4(col.x * 0.35f, col.y * 0.35f, col.z * 0.35f, col.w * 0.35f);
    float4 t4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (diffuse > 0.0f) {
        const float s = diffuse * 0.8f + 0.16f * (powf(diffuse, 8.0f));
        t4 = make_float4(col.x * s, col.y * s, col.z * s, col.w * s);
    }
    clr.x += t4.x;
    clr.y += t4.y;
    clr.z += t4.z;
    clr.w += t4.w;
    diffuse = (1.0f - alphaAcc) * col.w;
    return make_float4(sum.x + diffuse * clr.x, sum.y + diffuse * clr.y, sum.z + diffuse * clr.z,
                       sum.w + diffuse * clr.w);
}

// rgbaFloatToInt (core/kernel.cu:40-47): saturate, scale by 255, truncate.
__device__ __forceinline__ uint32_t pack_rgb(float4 c) {
    const uint32_t r = (uint32_t)(__saturatef(c.x) * 255);
    const uint32_t g = (uint32_t)(__saturatef(c.y) * 255);
    const uint32_t b = (uint32_t)(__saturatef(c.z) * 255);
    return r | (g << 8) | (b << 16);
}

// Label table of one frame in shared memory; slot assignment for the
// per-label opacity accumulators (>= 0 tracked slot, -1 uncapped, -2 never
// composites).  Run by every thread of the block, then __syncthreads().
__device__ __forceinline__ void load_label_smem(LabelSmem &S, const LabelTable &LT, int track) {
    const int tid = threadIdx.x;
    for (int l = tid; l < MK_MAX_LABELS; l += blockDim.x) {
        S.tf[l] = LT.tf[l];
        S.alpha[l] = LT.alpha[l];
        S.ww[l] = LT.ww[l];
        S.wl[l] = LT.wl[l];
    }
    if (tid == 0) {
        int next = 0;
        for (int l = 0; l < MK_MAX_LABELS; ++l) {
            const float a = LT.alpha[l];
            signed char sl;
            if (!(a > 0.0f)) sl = -2;
            else if (a >= 1.0f || track != kTrackShared) sl = -1;
            else sl = (next < kMaxTrackedLabels) ? (signed char)(next++) : -1;
            S.slot[l] = sl;
        }
    }
}

// One 32x8 pixel tile (bx, by) of a frame, by a 256-thread block: eight 8x4
// warp tiles.  s_acc holds the tracked opacity accumulators (kTrackShared),
// s_px the tile's RGB bytes, s_count the counting-mode total (zeroed by the
// caller).  Every thread of the block must call it.
template <int MODE, int TRACK, bool COUNT>
__device__ __forceinline__ void raycast_tile(const RayParams &P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                                             const LabelSmem &S, const BrickView &BV, float (*s_acc)[256],
                                             uint8_t (*s_px)[32 * 3], unsigned long long *s_count, int bx,
                                             int by) {
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int lx = (warp & 3) * 8 + (lane & 7);
    const int ly = (warp >> 2) * 4 + (lane >> 3);
    const int x = bx * 32 + lx;
    const int y = by * 8 + ly;
    const bool active = (x < P.W) && (y < P.H);

    float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    unsigned long long nsamples = 0;
    float A = 0.0f;   // alphaAcc (VR, MIP max, SURFACE last N.L)

    if (active) {
        const float u = 1.0f * (x - P.W / 2.0f - P.xT) / P.H;
        const float v = 1.0f * (y - P.H / 2.0f - P.yT) / P.H;
        float a0, a1;
        const bool hit = ray_interval(P, u, v, a0, a1);
        if (hit) {
            int k0 = accu_lower(P, a0);
            k0 = k0 > 0 ? k0 - 1 : 0;
            float a = P.accu[k0];
            const float a_stop = a1;

            // per-step displacement in voxel units, for runs inside empty bricks
            float3 dv;
            {
                const float ds = P.step1 * P.scale;
                dv.x = P.M[1] * P.mls[0] * ds * P.fdim[0];
                dv.y = P.M[4] * P.mls[1] * ds * P.fdim[1];
                dv.z = P.M[7] * P.mls[2] * ds * P.fdim[2];
                if (P.invertZ) dv.z = -dv.z;
            }

            if (MODE == kModeVR) {
                float3 L;
                {
                    // normalize(mul(M, (0,1,0))) (core/kernel.cu:166-167)
                    float lx_ = dot3(0.0f, 1.0f, 0.0f, P.M[0], P.M[1], P.M[2]);
                    float ly_ = dot3(0.0f, 1.0f, 0.0f, P.M[3], P.M[4], P.M[5]);
                    float lz_ = dot3(0.0f, 1.0f, 0.0f, P.M[6], P.M[7], P.M[8]);
                    const float inv = rsqrtf(lx_ * lx_ + ly_ * ly_ + lz_ * lz_);
                    L = make_float3(lx_ * inv, ly_ * inv, lz_ * inv);
                }
                const float L1 = P.step1;
                const float L4 = L1 / 4.0f;
                const float L8 = L1 / 8.0f;
                float step = L1;
                float aPre = 0.0f;
                float accLocal[TRACK == kTrackLocal ? MK_MAX_LABELS : 1];
                if (TRACK == kTrackShared) {
                    for (int i = 0; i < kMaxTrackedLabels; ++i) s_acc[i][tid] = 0.0f;
                } else if (TRACK == kTrackLocal) {
                    for (int i = 0; i < MK_MAX_LABELS; ++i) accLocal[i] = 0.0f;
                }
                while (a < P.limit) {
                    if (a > a_stop) break;
                    const float3 pos = ray_pos(P, u, v, a);
                    const int ix = pos.x * P.fdim[0];
                    const int iy = pos.y * P.fdim[1];
                    const int iz = pos.z * P.fdim[2];
                    if (outside_voi(P, ix, iy, iz)) {
                        a += step;
                        continue;
                    }
                    if (!COUNT && P.skip && step == L1 && aPre <= 0.001f) {
                        const int b = brick_index(P, BV, ix, iy, iz);
                        if (!((BV.visible_bits[b >> 5] >> (b & 31)) & 1u)) {
                            aPre = 0.0f;
                            a += step;
                            const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1],
                                                          pos.z * P.fdim[2]);
                            int n = steps_in_brick(pv, dv, ix, iy, iz);
                            for (; n > 0; --n) a += step;
                            continue;
                        }
                    }
                    if (COUNT) {
                        ++nsamples;
                        mark_footprint(P, pos.x, pos.y, pos.z);
                        if (mask) mark_label(P, ix, iy, iz);
                    }
                    const int label = mask ? min((int)tex3D<unsigned char>(mask, ix, iy, iz), MK_MAX_LABELS - 1) : 0;
                    float temp = 32768 * tex3D<float>(vol, pos.x, pos.y, pos.z);
                    temp = (temp - S.wl[label]) / S.ww[label] + 0.5f;
                    if (temp > 1) temp = 1;
                    const cudaTextureObject_t tf = S.tf[label];
                    float4 col = tf ? tex1D<float4>(tf, temp) : make_float4(0.f, 0.f, 0.f, 0.f);
                    float alpha = col.w;
                    // getNextStep (core/kernel.cu:84-125)
                    if (step == L4) alpha = 1 - powf(1 - alpha, 0.25f);
                    else if (step == L8) alpha = 1 - powf(1 - alpha, 0.125f);
                    if (a > 0.0f) {
                        if ((alpha > aPre ? alpha : aPre) > 0.001f) {
                            if (step == L1) {
                                a -= (L1 - L4);
                                step = L4;
                                continue;
                            } else if (step == L4) {
                                a -= (L4 - L8);
                                step = L8;
                                continue;
                            }
                        } else {
                            if (step == L8) step = L4;
                            else step = L1;
                        }
                    }
                    aPre = alpha;
                    a += step;
                    col.w = alpha;
                    if (COUNT) {
                        // counting pass: composite decisions still matter for termination
                        if (col.w > 0.0005f) {
                            const signed char sl = S.slot[label];
                            bool ok;
                            if (TRACK == kTrackLocal) ok = (sl != -2) && accLocal[label] < S.alpha[label];
                            else if (sl == -2) ok = false;
                            else if (sl == -1) ok = true;
                            else ok = s_acc[sl][tid] < S.alpha[label];
                            if (ok) {
                                mark_gradient(P, pos);
                                if (TRACK == kTrackLocal) accLocal[label] += (1.0f - A) * col.w;
                                else if (TRACK == kTrackShared && sl >= 0) s_acc[sl][tid] += (1.0f - A) * col.w;
                                A += (1.0f - A) * col.w;
                            }
                        }
                    } else if (col.w > 0.0005f) {
                        const signed char sl = S.slot[label];
                        bool ok;
                        if (TRACK == kTrackLocal) ok = (sl != -2) && accLocal[label] < S.alpha[label];
                        else if (sl == -2) ok = false;
                        else if (sl == -1) ok = true;
                        else ok = s_acc[sl][tid] < S.alpha[label];
                        if (ok) {
                            sum = shade(sum, A, vol, pos, col, L, P);
                            if (TRACK == kTrackLocal) accLocal[label] += (1.0f - A) * col.w;
                            else if (TRACK == kTrackShared && sl >= 0) s_acc[sl][tid] += (1.0f - A) * col.w;
                            A += (1.0f - A) * col.w;
                        }
                    }
                    if (A > 0.995f) break;
                }
                if (sum.x == 0.0f && sum.y == 0.0f && sum.z == 0.0f && sum.w == 0.0f) sum = P.bg;
            } else if (MODE == kModeMIP) {
                const float fStep = P.step1;
                while (a < P.limit) {
                    if (a > a_stop) break;
                    const float3 pos = ray_pos(P, u, v, a);
                    const int ix = pos.x * P.fdim[0];
                    const int iy = pos.y * P.fdim[1];
                    const int iz = pos.z * P.fdim[2];
                    if (outside_voi(P, ix, iy, iz)) {
                        a += fStep;
                        continue;
                    }
                    if (!COUNT && P.skip) {
                        const int b = brick_index(P, BV, ix, iy, iz);
                        if (BV.mip_tmax[b] <= A) {
                            a += fStep;
                            const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1],
                                                          pos.z * P.fdim[2]);
                            int n = steps_in_brick(pv, dv, ix, iy, iz);
                            for (; n > 0; --n) a += fStep;
                            continue;
                        }
                    }
                    const int label = mask ? min((int)tex3D<unsigned char>(mask, ix, iy, iz), MK_MAX_LABELS - 1) : 0;
                    if (COUNT && mask) mark_label(P, ix, iy, iz);
                    if (S.alpha[label] > 0) {
                        if (COUNT) {
                            ++nsamples;
                            mark_footprint(P, pos.x, pos.y, pos.z);
                        }
                        float temp = 32768 * tex3D<float>(vol, pos.x, pos.y, pos.z);
                        temp = (temp - S.wl[label]) / S.ww[label] + 0.5f;
                        if (A < temp) A = temp;
                    }
                    a += fStep;
                    // the output saturates at 1.0 (core/kernel.cu:351-358)
                    if (!COUNT && P.skip && A >= 1.0f) break;
                }
                if (A <= 0.0f) sum = P.bg;
                else sum = make_float4(A, A, A, A);
            } else {   // kModeSurface
                const float fStep = P.step1;
                float3 L;
                {
                    float lx_ = dot3(0.0f, 1.0f, 0.0f, P.M[0], P.M[1], P.M[2]);
                    float ly_ = dot3(0.0f, 1.0f, 0.0f, P.M[3], P.M[4], P.M[5]);
                    float lz_ = dot3(0.0f, 1.0f, 0.0f, P.M[6], P.M[7], P.M[8]);
                    const float inv = rsqrtf(lx_ * lx_ + ly_ * ly_ + lz_ * lz_);
                    L = make_float3(lx_ * inv, ly_ * inv, lz_ * inv);
                }
                while (a < P.limit) {
                    if (a > a_stop) break;
                    const float3 pos = ray_pos(P, u, v, a);
                    const int ix = pos.x * P.fdim[0];
                    const int iy = pos.y * P.fdim[1];
                    const int iz = pos.z * P.fdim[2];
                    if (outside_voi(P, ix, iy, iz)) {
                        a += fStep;
                        continue;
                    }
                    if (!COUNT && P.skip) {
                        const int b = brick_index(P, BV, ix, iy, iz);
                        const short2 mm = BV.minmax[b];
                        // 32768 * (v / 32767) <= 400 for every tap
                        if ((float)mm.y * (32768.0f / 32767.0f) + 0.01f <= 400.0f) {
                            a += fStep;
                            const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1],
                                                          pos.z * P.fdim[2]);
                            int n = steps_in_brick(pv, dv, ix, iy, iz);
                            for (; n > 0; --n) a += fStep;
                            continue;
                        }
                    }
                    if (COUNT) {
                        ++nsamples;
                        mark_footprint(P, pos.x, pos.y, pos.z);
                    }
                    const float temp = 32768 * tex3D<float>(vol, pos.x, pos.y, pos.z);
                    if (temp <= 400) {
                        a += fStep;
                        continue;
                    }
                    if (COUNT) mark_gradient(P, pos);
                    float3 N;
                    N.x = tex3D<float>(vol, pos.x + P.sv[0], pos.y, pos.z) - tex3D<float>(vol, pos.x - P.sv[0], pos.y, pos.z);
                    N.y = tex3D<float>(vol, pos.x, pos.y + P.sv[1], pos.z) - tex3D<float>(vol, pos.x, pos.y - P.sv[1], pos.z);
                    N.z = tex3D<float>(vol, pos.x, pos.y, pos.z + P.sv[2]) - tex3D<float>(vol, pos.x, pos.y, pos.z - P.sv[2]);
                    if (P.invertZ) N.z = -N.z;
                    const float inv = rsqrtf(N.x * N.x + N.y * N.y + N.z * N.z);
                    N.x = N.x * inv;
                    N.y = N.y * inv;
                    N.z = N.z * inv;
                    A = N.x * L.x + N.y * L.y + N.z * L.z;
                    if (A > 0) break;
                    a += fStep;
                }
                if (A <= 0.0f) {
                    sum = P.bg;
                } else {
                    const float g = add_dconst(A, MK_DCONST(0.05));
                    sum = make_float4(g, g, g, 1.0f);
                }
            }
        } else {
            // ray misses the VOI: MonkeyGL composites nothing and paints the background
            if (MODE == kModeVR) sum = P.bg;
            else if (MODE == kModeMIP) sum = P.bg;
            else sum = P.bg;
        }
    }

    if (COUNT) {
        if (nsamples) atomicAdd(s_count, nsamples);
        __syncthreads();
        if (tid == 0 && *s_count) atomicAdd(P.counter, *s_count);
        return;
    }

    // output: RGB8 staged through shared memory, RGBA8 stored directly
    const uint32_t rgb = pack_rgb(sum);
    if (P.rgba) {
        if (active)
            reinterpret_cast<uint32_t *>(P.out)[(size_t)y * P.W + x] = rgb | 0xff000000u;
        return;
    }
    s_px[ly][lx * 3 + 0] = rgb & 0xff;
    s_px[ly][lx * 3 + 1] = (rgb >> 8) & 0xff;
    s_px[ly][lx * 3 + 2] = (rgb >> 16) & 0xff;
    __syncthreads();
    const int x0 = bx * 32, y0 = by * 8;
    const bool full = (x0 + 32 <= P.W) && (y0 + 8 <= P.H) && ((P.W & 3) == 0) &&
                      ((reinterpret_cast<uintptr_t>(P.out) & 3) == 0);   // word stores need an aligned row
    if (full) {
        if (tid < 8 * 24) {
            const int r = tid / 24, w = tid % 24;
            const uint32_t word = (uint32_t)s_px[r][4 * w] | ((uint32_t)s_px[r][4 * w + 1] << 8) |
                                  ((uint32_t)s_px[r][4 * w + 2] << 16) |
                                  ((uint32_t)s_px[r][4 * w + 3] << 24);
            uint8_t *row = P.out + ((size_t)(y0 + r) * P.W + x0) * 3;
            reinterpret_cast<uint32_t *>(row)[w] = word;
        }
    } else if (active) {
        uint8_t *p = P.out + ((size_t)y * P.W + x) * 3;
        p[0] = s_px[ly][lx * 3 + 0];
        p[1] = s_px[ly][lx * 3 + 1];
        p[2] = s_px[ly][lx * 3 + 2];
    }
}

// Host: kernel parameters of one frame (validates the request; the output
// pointer is left null), and the opacity-accumulator mode for the labels
// present in a volume under a table of (alpha, ww, wl) rows.
int fill_ray_params(const VolumeState &v, const mk_vr_params *p, RayParams &P);
int tracking_mode_for(const uint64_t present[2], const float (*params)[3]);
// Host: the 32x8 tiles of a W x H frame (index by * tiles_x + bx) sorted by
// the distance of their centre to (W/2 + xT, H/2 + yT), where the volume
// centre projects: launching them in this order starts the long rays first.
std::vector<int> centre_first_tiles(int W, int H, int xT, int yT);

}  // namespace mk
