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

// A VR ray handed from a frame's tile launch to its tail launch: the march
// state of MonkeyGL's loop at a sample boundary and the ray's opacity
// accumulators, restored bit for bit by the tail launch.
struct __align__(16) SpillRay {
    float4 sum;
    float u, v, a, a_stop;
    float step, aPre, A;
    int lat;
    int pix;                     // y * W + x
    int pad[3];
    float acc[kMaxTrackedLabels];
};

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
    const float *fy_tab;         // ray parameter of each table entry at this scale (null: compute)
    int accu_len;
    int rgba;                    // 1 = 4 bytes per pixel
    int skip;
    int coop_rays;               // VR: a warp with at most this many rays left marches them cooperatively
    uint8_t *out;
    unsigned long long *counter; // sample counting mode
    uint32_t *vox_bits;          // counting mode: voxels inside trilinear footprints (may be null)
    uint32_t *lab_bits;          // counting mode: label voxels read (may be null)
    // VR frame tail (null: rays are marched to the end where they start):
    // {tiles finished, rays spilled, rays taken, tail blocks finished}
    unsigned *tail;
    SpillRay *spill;             // rays handed to the tail launch
    int spill_cap;
    int tail_trigger;            // rays still marching spill once this many tiles have finished
    // tail launch with host output: its pixels go to this (pix, rgb) list
    // (word 0: the count, pairs from word 2) instead of `out`; null: `out`
    uint32_t *patch;
    // MIP: 1 when every label present in the mask is visible (alpha > 0) and
    // shares one window (mip_ww > 0, mip_wl); the label fetch is then not
    // needed and the window is applied only to a new raw maximum
    int mip_uniform;
    float mip_ww, mip_wl;
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

// One sample position of the reference schedule (core/kernel.cu:197-206)
// from the ray parameter fy = (accuLength - 0.866) * scale.
__device__ __forceinline__ float3 ray_pos_fy(const RayParams &P, float u, float v, float fy) {
    float3 p;
    p.x = dot3(u, fy, v, P.M[0], P.M[1], P.M[2]);
    p.y = dot3(u, fy, v, P.M[3], P.M[4], P.M[5]);
    p.z = dot3(u, fy, v, P.M[6], P.M[7], P.M[8]);
    // pos * maxLenSpacing + 0.5: fused, as nvcc compiles MonkeyGL's
    // expression (a separate multiply and add misplaces samples); written
    // out so that no inlining context can change it
    p.x = __fmaf_rn(p.x, P.mls[0], 0.5f);
    p.y = __fmaf_rn(p.y, P.mls[1], 0.5f);
    p.z = __fmaf_rn(p.z, P.mls[2], 0.5f);
    if (P.invertZ) p.z = 1.0f - p.z;
    return p;
}

__device__ __forceinline__ float3 ray_pos(const RayParams &P, float u, float v, float a) {
    return ray_pos_fy(P, u, v, ray_fy(a, P.scale));
}

// The position of a sample that lies on the schedule table (a == accu[k]).
// Rendering launches carry the frame's fy table; counting passes evaluate.
template <bool COUNT>
__device__ __forceinline__ float3 ray_pos_at(const RayParams &P, float u, float v, int k, float a) {
    return COUNT ? ray_pos(P, u, v, a) : ray_pos_fy(P, u, v, P.fy_tab[k]);
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

// Per-step displacement of a ray in voxel units (dv) and its reciprocal
// (rdv, 0 where the ray is parallel to an axis), for runs inside empty
// bricks.
struct StepVec {
    float3 dv;
    float3 rdv;
};

__device__ __forceinline__ StepVec step_vec(const RayParams &P) {
    StepVec S;
    const float ds = P.step1 * P.scale;
    S.dv.x = P.M[1] * P.mls[0] * ds * P.fdim[0];
    S.dv.y = P.M[4] * P.mls[1] * ds * P.fdim[1];
    S.dv.z = P.M[7] * P.mls[2] * ds * P.fdim[2];
    if (P.invertZ) S.dv.z = -S.dv.z;
    S.rdv.x = fabsf(S.dv.x) > 1e-6f ? 1.0f / S.dv.x : 0.0f;
    S.rdv.y = fabsf(S.dv.y) > 1e-6f ? 1.0f / S.dv.y : 0.0f;
    S.rdv.z = fabsf(S.dv.z) > 1e-6f ? 1.0f / S.dv.z : 0.0f;
    return S;
}

// Number of further coarse steps that stay inside brick (bx,by,bz) with a
// 0.05-voxel margin, capped at 64.  Position p is in voxel units.  Any
// count that keeps those samples inside the brick is valid (they are all
// skippable); the margin covers the rounding of the linear model.
__device__ __forceinline__ int steps_in_brick(const float3 &pv, const StepVec &sv, int ix, int iy, int iz) {
    float t = 64.0f;
    const float e = 0.05f;
    const float lo[3] = {(float)((ix >> kBrickShift) << kBrickShift),
                         (float)((iy >> kBrickShift) << kBrickShift),
                         (float)((iz >> kBrickShift) << kBrickShift)};
    const float pp[3] = {pv.x, pv.y, pv.z};
    const float rd[3] = {sv.rdv.x, sv.rdv.y, sv.rdv.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (rd[k] > 0.0f) t = fminf(t, (lo[k] + kBrick - e - pp[k]) * rd[k]);
        else if (rd[k] < 0.0f) t = fminf(t, (pp[k] - lo[k] - e) * -rd[k]);
    }
    return t > 0.0f ? (int)t : 0;
}

// Advance accuLength by n coarse steps: n float additions of L1, as
// MonkeyGL's loop makes them.  While a ray has never refined its step it
// stays on the schedule table (a == accu[lat]), whose entry lat + n holds
// the same sum; lat < 0 once the ray has left it.
__device__ __forceinline__ void advance_coarse(const RayParams &P, float &a, int &lat, float step, int n) {
    if (lat >= 0) {
        lat = min(lat + n, P.accu_len - 1);
        a = P.accu[lat];
    } else {
        for (; n > 0; --n) a += step;
    }
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

// Central-difference normal and headlight shading (core/kernel.cu:49-81):
// the shaded colour of a sample, before it is weighted by the remaining
// transparency.  It depends only on the sample, not on the ray's state.
// The six central-difference taps (core/kernel.cu:61-63): +x, -x, +y, -y,
// +z, -z, one spacing voxel away.
struct GradTaps {
    float xp, xm, yp, ym, zp, zm;
};

__device__ __forceinline__ GradTaps fetch_taps(cudaTextureObject_t vol, float3 pos, const RayParams &P) {
    GradTaps g;
    g.xp = tex3D<float>(vol, pos.x + P.sv[0], pos.y, pos.z);
    g.xm = tex3D<float>(vol, pos.x - P.sv[0], pos.y, pos.z);
    g.yp = tex3D<float>(vol, pos.x, pos.y + P.sv[1], pos.z);
    g.ym = tex3D<float>(vol, pos.x, pos.y - P.sv[1], pos.z);
    g.zp = tex3D<float>(vol, pos.x, pos.y, pos.z + P.sv[2]);
    g.zm = tex3D<float>(vol, pos.x, pos.y, pos.z - P.sv[2]);
    return g;
}

__device__ __forceinline__ float4 shade_taps(const GradTaps &g, float4 col, float3 L, const RayParams &P) {
    float3 N;
    N.x = g.xp - g.xm;
    N.y = g.yp - g.ym;
    N.z = g.zp - g.zm;
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
    return clr;
}

// sum + (1 - alphaAcc) * alpha * clr, the return value of tracing()
// (core/kernel.cu:78-80).
__device__ __forceinline__ float4 composite(float4 sum, float alphaAcc, float alpha, float4 clr) {
    const float w = (1.0f - alphaAcc) * alpha;
    return make_float4(sum.x + w * clr.x, sum.y + w * clr.y, sum.z + w * clr.z, sum.w + w * clr.w);
}

__device__ __forceinline__ float4 shade_color(cudaTextureObject_t vol, float3 pos, float4 col, float3 L,
                                              const RayParams &P) {
    return shade_taps(fetch_taps(vol, pos, P), col, L, P);
}

__device__ __forceinline__ float4 shade(float4 sum, float alphaAcc, cudaTextureObject_t vol,
                                        float3 pos, float4 col, float3 L, const RayParams &P) {
    return composite(sum, alphaAcc, col.w, shade_color(vol, pos, col, L, P));
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

// ---------------------------------------------------------------------------
// VR march of one warp's rays with a cooperative tail.
//
// A ray is a chain of dependent steps (sample position, texture fetch, LUT
// fetch, opacity correction, shading fetches), so a warp whose last few rays
// are long runs at the latency of that chain with most lanes idle; on a
// 1024^2 frame one such warp can take three times as long as the average SM
// is busy.  When at most P.coop_rays rays of a warp are left, its 32 lanes
// are split into groups of G = 32/rays (a power of two) and each group takes
// one ray: lane j of a group evaluates the sample j steps ahead at the
// current step size (position, label, value, LUT, opacity correction and,
// for alpha > 0.0005, the shaded colour), all in parallel, and then every
// lane of the group walks MonkeyGL's schedule over those samples in order
// (refinement, coarsening, empty-brick runs, opacity caps, compositing,
// termination).  The walk stops at the first sample whose successor was not
// evaluated at the right place (the step changed) and the next round starts
// there.  A sample depends only on its accuLength, and the walk applies the
// same float operations in the same order as the one-lane march, so the
// image is unchanged.

// Result of evaluating one sample.  meta: bits 0-3 kCoop* flags, 4-11 label,
// 12-19 further steps of an empty-brick run.
struct __align__(16) CoopSample {
    float4 clr;      // shaded colour (alpha > 0.0005)
    float4 res;      // final colour of the ray whose pixel is this lane's
    float alpha;     // opacity-corrected alpha at the round's step
    int meta;
    int pad[2];
};
constexpr int kCoopEnd = 1;        // past the end of the ray (a >= limit or a > a_stop)
constexpr int kCoopOutside = 2;    // outside the VOI: no fetch
constexpr int kCoopEmpty = 4;      // in a brick with its visibility bit clear (step L1)
constexpr int kCoopFetched = 8;    // label, value and LUT fetched
constexpr int kCoopRaysDefault = 16;

struct VrRay {
    float u, v, a, a_stop, step, aPre, A;
    float4 sum;
    int lat;         // index of a in the schedule table while the step was never refined, else -1
    int pix;         // y * W + x of the ray's pixel
    bool done;
};

// Frame tail.  Tiles of long rays set the length of a frame: near its end a
// few warps march alone on otherwise idle SMs, at the latency of their sample
// chains.  Once P.tail_trigger tiles have finished, a warp hands its rays that
// are still marching to the spill list (state at a sample boundary, opacity
// accumulators included) and stops; the tail launch (k_vr_tail) resumes them
// with several lanes per ray on every SM.  Where a ray is handed over does
// not change its samples or their order, so the image is unchanged.
// Warp-uniform: lane 0 reads the finished-tile count.
__device__ __forceinline__ bool tail_reached(const RayParams &P) {
    unsigned t = 0;
    if ((threadIdx.x & 31) == 0) t = *(volatile const unsigned *)P.tail;
    t = __shfl_sync(0xffffffffu, t, 0);
    return t >= (unsigned)P.tail_trigger;
}

// Write ray R (opacity accumulators at s_acc[.][acc_tid]) to the spill list;
// false when the list is full (the ray then keeps marching).
template <int TRACK, int NT>
__device__ __forceinline__ bool spill_ray(const RayParams &P, const VrRay &R, const float (*s_acc)[NT],
                                          int acc_tid) {
    const unsigned i = atomicAdd(&P.tail[1], 1u);
    if (i >= (unsigned)P.spill_cap) return false;
    SpillRay &o = P.spill[i];
    o.sum = R.sum;
    o.u = R.u;
    o.v = R.v;
    o.a = R.a;
    o.a_stop = R.a_stop;
    o.step = R.step;
    o.aPre = R.aPre;
    o.A = R.A;
    o.lat = R.lat;
    o.pix = R.pix;
    if (TRACK == kTrackShared) {
#pragma unroll
        for (int k = 0; k < kMaxTrackedLabels; ++k) o.acc[k] = s_acc[k][acc_tid];
    }
    return true;
}

template <int TRACK, int NT>
__device__ __forceinline__ bool vr_cap_ok(const LabelSmem &S, const float (*s_acc)[NT], const float *accLocal,
                                          int label, int owner) {
    const signed char sl = S.slot[label];
    if (TRACK == kTrackLocal) return (sl != -2) && accLocal[label] < S.alpha[label];
    if (sl == -2) return false;
    if (sl == -1) return true;
    return s_acc[sl][owner] < S.alpha[label];
}

template <int TRACK, int NT>
__device__ __forceinline__ void vr_cap_add(const LabelSmem &S, float (*s_acc)[NT], float *accLocal, int label,
                                           int owner, float A, float alpha) {
    const signed char sl = S.slot[label];
    if (TRACK == kTrackLocal) accLocal[label] += (1.0f - A) * alpha;
    else if (TRACK == kTrackShared && sl >= 0) s_acc[sl][owner] += (1.0f - A) * alpha;
}

// The cooperative tail: every lane of the warp calls it with the warp's
// mask of unfinished rays `act`; on return each lane of `act` holds its
// ray's final colour in R.sum.  Groups widen as rays finish: whenever the
// unfinished rays fit into groups twice as large, their states move to new
// groups, so a warp's last ray is marched by all 32 lanes.
template <int TRACK, bool EARLY_TAPS = false, int NT = 256>
__device__ void vr_coop_tail(const RayParams &P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                             const LabelSmem &S, const BrickView &BV, float (*s_acc)[NT], CoopSample *ws,
                             unsigned act, VrRay &R, const StepVec &dv, float3 L, bool may_spill) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const float L1 = P.step1, L4 = L1 / 4.0f, L8 = L1 / 8.0f;
    VrRay Q = R;            // the ray this lane works on; initially its own
    int owner = lane;       // lane of Q's pixel (and of its opacity caps)
    unsigned cur = act;     // lanes whose Q is an unfinished ray, to be grouped
    while (cur) {
        const int nrays = __popc(cur);
        int G = 32;
        while (G * nrays > 32) G >>= 1;
        const int g = lane / G, j = lane - g * G;
        const bool member = g < nrays;
        int src = lane;     // holder of ray g: the g-th set bit of cur
        if (member) {
            unsigned m = cur;
            for (int i = 0; i < g; ++i) m &= m - 1u;
            src = __ffs(m) - 1;
        }
        {
            VrRay T;
            T.u = __shfl_sync(FULL, Q.u, src);
            T.v = __shfl_sync(FULL, Q.v, src);
            T.a = __shfl_sync(FULL, Q.a, src);
            T.a_stop = __shfl_sync(FULL, Q.a_stop, src);
            T.step = __shfl_sync(FULL, Q.step, src);
            T.aPre = __shfl_sync(FULL, Q.aPre, src);
            T.A = __shfl_sync(FULL, Q.A, src);
            T.sum.x = __shfl_sync(FULL, Q.sum.x, src);
            T.sum.y = __shfl_sync(FULL, Q.sum.y, src);
            T.sum.z = __shfl_sync(FULL, Q.sum.z, src);
            T.sum.w = __shfl_sync(FULL, Q.sum.w, src);
            T.lat = __shfl_sync(FULL, Q.lat, src);
            T.pix = __shfl_sync(FULL, Q.pix, src);
            // masked to a lane: a shuffled value indexes the warp's own
            // slices of s_acc and ws, so even a value from a lane that did
            // not take part cannot address outside them
            owner = __shfl_sync(FULL, owner, src) & 31;
            T.done = !member;
            Q = T;
        }
        const int owner_tid = (threadIdx.x & ~31) | owner;
        bool reported = false;
        int round = 0;
        while (true) {
            // A round on step L1/4 always stops at its first sample: MonkeyGL
            // either refines there (to L1/8, from a - (L1/4 - L1/8)) or
            // composites it and coarsens (to L1, from a + L1).  Such a round
            // evaluates both continuations: lane 0 the sample itself, lanes
            // 1..hA the refined run, lanes hA+1.. the coarsened run; the
            // sample's test picks the run that is walked.
            const bool two = G >= 8 && !Q.done && Q.step == L4 && Q.a > 0.0f;
            const int hA = G / 2 - 1;
            // 1. this lane's sample: j steps ahead, or its place in its run
            float4 clr = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            float alpha_j = 0.0f;
            int flags = 0, label = 0, nskip = 0;
            float aj = Q.a, sj = Q.step;
            int jj = j;
            if (two && j > 0) {
                if (j <= hA) {
                    sj = L8;
                    aj = Q.a - (L4 - L8);
                    jj = j - 1;
                } else {
                    sj = L1;
                    aj = Q.a + L1;
                    jj = j - hA - 1;
                }
            }
            if (!Q.done) {
                const int kj = Q.lat >= 0 ? min(Q.lat + j, P.accu_len - 1) : -1;
                if (kj >= 0) {
                    aj = P.accu[kj];
                } else {
                    // sequential additions, as the walk makes them
#pragma unroll
                    for (int k = 0; k < 31; ++k)
                        if (k < jj) aj += sj;
                }
                if (!(aj < P.limit) || aj > Q.a_stop) {
                    flags = kCoopEnd;
                } else {
                    const float3 pos = kj >= 0 ? ray_pos_at<false>(P, Q.u, Q.v, kj, aj) : ray_pos(P, Q.u, Q.v, aj);
                    const int ix = pos.x * P.fdim[0];
                    const int iy = pos.y * P.fdim[1];
                    const int iz = pos.z * P.fdim[2];
                    if (outside_voi(P, ix, iy, iz)) {
                        flags = kCoopOutside;
                    } else {
                        bool empty = false;
                        if (P.skip && sj == L1) {
                            const int b = brick_index(P, BV, ix, iy, iz);
                            empty = !((BV.visible_bits[b >> 5] >> (b & 31)) & 1u);
                            if (empty) {
                                const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1], pos.z * P.fdim[2]);
                                nskip = steps_in_brick(pv, dv, ix, iy, iz);
                                flags |= kCoopEmpty;
                            }
                        }
                        // an empty-brick sample is fetched only where the walk may not skip it
                        if (!empty || (j == 0 && !(Q.aPre <= 0.001f))) {
                            label = mask ? min((int)tex3D<unsigned char>(mask, ix, iy, iz), MK_MAX_LABELS - 1) : 0;
                            float temp = 32768 * tex3D<float>(vol, pos.x, pos.y, pos.z);
                            // (tail launch) a ray on a refined step is inside
                            // something that composites: its shading taps are
                            // fetched with the value, not after the LUT (one
                            // texture round trip less, more registers)
                            const bool early = EARLY_TAPS && sj != L1;
                            GradTaps taps = {};
                            if (early) taps = fetch_taps(vol, pos, P);
                            temp = (temp - S.wl[label]) / S.ww[label] + 0.5f;
                            if (temp > 1) temp = 1;
                            const cudaTextureObject_t tf = S.tf[label];
                            const float4 col = tf ? tex1D<float4>(tf, temp) : make_float4(0.f, 0.f, 0.f, 0.f);
                            float alpha = col.w;
                            if (sj == L4) alpha = 1 - powf(1 - alpha, 0.25f);
                            else if (sj == L8) alpha = 1 - powf(1 - alpha, 0.125f);
                            alpha_j = alpha;
                            if (alpha > 0.0005f) {
                                if (!early) taps = fetch_taps(vol, pos, P);
                                clr = shade_taps(taps, make_float4(col.x, col.y, col.z, alpha), L, P);
                            }
                            flags |= kCoopFetched;
                        }
                    }
                }
            }
            ws[lane].clr = clr;
            ws[lane].alpha = alpha_j;
            ws[lane].meta = flags | (label << 4) | (nskip << 12);
            __syncwarp();

            // 2. MonkeyGL's schedule over the group's samples, in order.
            // In a round whose samples are all fetched (none outside the VOI,
            // past the end or in a skipped brick) the step can change only
            // where MonkeyGL's refinement test says so, and that test needs
            // only sample j's alpha and the previous one: every lane decides
            // whether the walk stops at its sample, the first stop ends the
            // round, and only the compositing of the samples before it stays
            // serial.  The ray's new position, step and previous alpha come
            // from the stopping lane (the same float operations as the walk).
            // Other rounds take the sample-by-sample walk.
            const float alpha_up = __shfl_up_sync(FULL, alpha_j, 1);
            const float alpha_0 = __shfl_sync(FULL, alpha_j, lane & ~(G - 1));   // the group's lane 0
            float pre_j = j == 0 ? Q.aPre : alpha_up;
            if (two && j == 1) pre_j = Q.aPre;           // a refinement keeps aPre
            if (two && j == hA + 1) pre_j = alpha_0;     // after sample 0 was walked
            const bool busy = (pre_j > alpha_j ? pre_j : alpha_j) > 0.001f;  // (alpha > aPre ? alpha : aPre) > 0.001
            const bool pos_a = aj > 0.0f;
            const bool refine_j = pos_a && busy && sj != L8;
            const bool stop_j = !pos_a || sj == L4 || (sj == L1 ? busy : !busy);
            const bool plain_j = (flags & (kCoopEnd | kCoopOutside | kCoopFetched)) == kCoopFetched;
            const unsigned plain_m = __ballot_sync(FULL, plain_j);
            const unsigned stop_m = __ballot_sync(FULL, stop_j);
            const unsigned refine_m = __ballot_sync(FULL, refine_j);
            const unsigned gbits = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
            const unsigned gplain = (plain_m >> (g * G)) & gbits;
            const unsigned gstop = (stop_m >> (g * G)) & gbits;
            const unsigned grefine = (refine_m >> (g * G)) & gbits;
            // the lanes of the run walked this round, [r_lo, r_hi]; in a
            // two-continuation round the coarsened run follows sample 0
            // (lead0), the refined one replaces it
            int r_lo = 0, r_hi = G - 1;
            bool lead0 = false;
            if (two) {
                if (grefine & 1u) {
                    r_lo = 1;
                    r_hi = hA;
                } else {
                    r_lo = hA + 1;
                    lead0 = true;
                }
            }
            const int r_n = r_hi - r_lo + 1;
            const unsigned rmask = (r_n == 32 ? 0xffffffffu : ((1u << r_n) - 1u)) << r_lo;
            const unsigned need = rmask | (two ? 1u : 0u);
            const bool simple = member && !Q.done && (gplain & need) == need;
            const unsigned rstop = gstop & rmask;
            const int s_at = rstop ? __ffs(rstop) - 1 : r_hi + 1;  // first stopping sample, r_hi + 1: none
            const bool none = s_at > r_hi;
            const bool s_refine = !none && ((grefine >> s_at) & 1u);
            {
                // values of the stopping lane (or of the run's last lane when none stops)
                const float ns = pos_a ? (sj == L8 ? L4 : L1) : sj;
                float a_out, pre_out, step_out;
                int lat_out;
                if (none) {                         // all samples walked: a += step
                    a_out = aj + sj;
                    pre_out = alpha_j;
                    step_out = sj;
                    lat_out = Q.lat >= 0 ? Q.lat + j + 1 : Q.lat;
                } else if (refine_j) {              // refine before compositing sample j
                    a_out = sj == L1 ? aj - (L1 - L4) : aj - (L4 - L8);
                    pre_out = pre_j;
                    step_out = sj == L1 ? L4 : L8;
                    lat_out = -1;
                } else {                            // sample j walked, then the step coarsens
                    a_out = aj + ns;
                    pre_out = alpha_j;
                    step_out = ns;
                    lat_out = Q.lat >= 0 ? Q.lat + j + 1 : Q.lat;
                }
                const int src = g * G + (none ? r_hi : s_at);
                const float a_new = __shfl_sync(FULL, a_out, src);
                const float pre_new = __shfl_sync(FULL, pre_out, src);
                const float step_new = __shfl_sync(FULL, step_out, src);
                const int lat_new = __shfl_sync(FULL, lat_out, src);
                if (simple) {
                    const CoopSample *gs = ws + g * G;
                    // walked samples: sample 0 first if lead0, then [r_lo, c_end)
                    const int c_end = none ? r_hi + 1 : (s_refine ? s_at : s_at + 1);
                    int c_lab = -1, c_slot = -2;
                    float c_cap = 0.0f, c_acc = 0.0f;
                    bool ended = false;
                    int k = lead0 ? 0 : r_lo;
                    float alpha_n = gs[k].alpha;
                    int meta_n = gs[k].meta;
                    float4 clr_n = gs[k].clr;
                    while (k < c_end) {
                        const float alpha = alpha_n;
                        const int lab = (meta_n >> 4) & 255;
                        const float4 clr = clr_n;
                        const int kn = (lead0 && k == 0) ? r_lo : k + 1;
                        if (kn < c_end) {
                            alpha_n = gs[kn].alpha;
                            meta_n = gs[kn].meta;
                            clr_n = gs[kn].clr;
                        }
                        k = kn;
                        if (alpha > 0.0005f) {
                            if (lab != c_lab) {
                                if (TRACK == kTrackShared && c_slot >= 0) s_acc[c_slot][owner_tid] = c_acc;
                                c_lab = lab;
                                c_slot = S.slot[lab];
                                c_cap = S.alpha[lab];
                                c_acc = (TRACK == kTrackShared && c_slot >= 0) ? s_acc[c_slot][owner_tid] : 0.0f;
                            }
                            const bool ok = c_slot != -2 && (c_slot == -1 || TRACK != kTrackShared || c_acc < c_cap);
                            if (ok) {
                                Q.sum = composite(Q.sum, Q.A, alpha, clr);
                                if (TRACK == kTrackShared && c_slot >= 0) c_acc += (1.0f - Q.A) * alpha;
                                Q.A += (1.0f - Q.A) * alpha;
                                if (Q.A > 0.995f) {
                                    ended = true;
                                    break;
                                }
                            }
                        }
                    }
                    if (TRACK == kTrackShared && c_slot >= 0) s_acc[c_slot][owner_tid] = c_acc;
                    if (ended) {
                        Q.done = true;
                    } else {
                        Q.a = a_new;
                        Q.aPre = pre_new;
                        Q.step = step_new;
                        Q.lat = lat_new;
                    }
                }
            }
            if (!simple && !Q.done) {
                // The walk is the serial part of a round, so nothing on its
                // chain waits for shared memory: the next sample is read
                // while this one is walked, and the opacity cap of the label
                // last composited stays in registers (written back once).
                const CoopSample *gs = ws + g * G;
                int c_lab = -1, c_slot = -2;
                float c_cap = 0.0f, c_acc = 0.0f;
                int k = 0;
                int meta = gs[0].meta;
                float alpha_n = gs[0].alpha;
                float4 clr_n = gs[0].clr;
                // the lanes after sample 0 of a two-continuation round hold
                // runs that start elsewhere: the walk takes sample 0 only
                const int walk_end = two ? 1 : G;
                while (k < walk_end) {
                    const int f = meta & 15;
                    if (f & kCoopEnd) {
                        Q.done = true;
                        break;
                    }
                    if (f & kCoopOutside) {
                        Q.a += Q.step;
                        if (Q.lat >= 0) ++Q.lat;
                        if (++k < walk_end) {
                            meta = gs[k].meta;
                            alpha_n = gs[k].alpha;
                            clr_n = gs[k].clr;
                        }
                        continue;
                    }
                    if ((f & kCoopEmpty) && P.skip && Q.step == L1 && Q.aPre <= 0.001f) {
                        const int n = 1 + ((meta >> 12) & 255);
                        Q.aPre = 0.0f;
                        advance_coarse(P, Q.a, Q.lat, Q.step, n);
                        k += n;
                        if (k < walk_end) {
                            meta = gs[k].meta;
                            alpha_n = gs[k].alpha;
                            clr_n = gs[k].clr;
                        }
                        continue;
                    }
                    if (!(f & kCoopFetched)) break;   // evaluate it in the next round
                    const float alpha = alpha_n;
                    const float4 clr = clr_n;
                    const int lab = (meta >> 4) & 255;
                    if (k + 1 < walk_end) {
                        meta = gs[k + 1].meta;
                        alpha_n = gs[k + 1].alpha;
                        clr_n = gs[k + 1].clr;
                    }
                    bool last = false;
                    if (Q.a > 0.0f) {
                        if ((alpha > Q.aPre ? alpha : Q.aPre) > 0.001f) {
                            if (Q.step == L1) {
                                Q.a -= (L1 - L4);
                                Q.step = L4;
                                Q.lat = -1;
                                break;
                            } else if (Q.step == L4) {
                                Q.a -= (L4 - L8);
                                Q.step = L8;
                                break;
                            }
                        } else {
                            const float ns = (Q.step == L8) ? L4 : L1;
                            last = ns != Q.step;
                            Q.step = ns;
                        }
                    } else {
                        last = true;
                    }
                    Q.aPre = alpha;
                    Q.a += Q.step;
                    if (Q.lat >= 0) ++Q.lat;
                    if (alpha > 0.0005f) {
                        if (lab != c_lab) {
                            if (TRACK == kTrackShared && c_slot >= 0) s_acc[c_slot][owner_tid] = c_acc;
                            c_lab = lab;
                            c_slot = S.slot[lab];
                            c_cap = S.alpha[lab];
                            c_acc = (TRACK == kTrackShared && c_slot >= 0) ? s_acc[c_slot][owner_tid] : 0.0f;
                        }
                        // vr_cap_ok / vr_cap_add on the cached accumulator
                        const bool ok = c_slot != -2 && (c_slot == -1 || TRACK != kTrackShared || c_acc < c_cap);
                        if (ok) {
                            Q.sum = composite(Q.sum, Q.A, alpha, clr);
                            if (TRACK == kTrackShared && c_slot >= 0) c_acc += (1.0f - Q.A) * alpha;
                            Q.A += (1.0f - Q.A) * alpha;
                        }
                    }
                    if (Q.A > 0.995f) {
                        Q.done = true;
                        break;
                    }
                    if (last) break;
                    ++k;
                }
                if (TRACK == kTrackShared && c_slot >= 0) s_acc[c_slot][owner_tid] = c_acc;
            }
            if (may_spill && (++round & 3) == 0 && tail_reached(P)) {
                may_spill = false;
                bool moved = false;
                if (member && j == 0 && !Q.done) moved = spill_ray<TRACK>(P, Q, s_acc, owner_tid);
                moved = __shfl_sync(FULL, moved, member ? g * G : lane);
                if (member && moved) {
                    Q.done = true;      // finished by the tail launch: no colour from here
                    reported = true;
                }
            }
            if (member && Q.done && !reported) {
                if (j == 0) ws[owner].res = Q.sum;
                reported = true;
            }
            __syncwarp();
            const unsigned live = __ballot_sync(FULL, member && j == 0 && !Q.done);
            if (live == 0u) {
                cur = 0u;
                break;
            }
            if (G < 32 && __popc(live) * 2 * G <= 32) {
                cur = live;          // regroup the unfinished rays into wider groups
                break;
            }
        }
    }
    __syncwarp();
    if ((act >> lane) & 1u) R.sum = ws[lane].res;
    __syncwarp();
}

// The headlight direction normalize(mul(M, (0,1,0))) (core/kernel.cu:166-167).
__device__ __forceinline__ float3 vr_light(const RayParams &P) {
    const float lx = dot3(0.0f, 1.0f, 0.0f, P.M[0], P.M[1], P.M[2]);
    const float ly = dot3(0.0f, 1.0f, 0.0f, P.M[3], P.M[4], P.M[5]);
    const float lz = dot3(0.0f, 1.0f, 0.0f, P.M[6], P.M[7], P.M[8]);
    const float inv = rsqrtf(lx * lx + ly * ly + lz * lz);
    return make_float3(lx * inv, ly * inv, lz * inv);
}

// MonkeyGL's d_render march (core/kernel.cu:156-256) for the ray of this
// lane, called by every lane of the warp; returns the composited colour
// (the background where nothing composited).
template <int TRACK, int NT>
__device__ __forceinline__ float4 vr_march(const RayParams &P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                                           const LabelSmem &S, const BrickView &BV, float (*s_acc)[NT],
                                           CoopSample *ws, bool active, int x, int y) {
    const int tid = threadIdx.x;
    VrRay R;
    R.u = R.v = R.a = R.a_stop = 0.0f;
    R.step = P.step1;
    R.aPre = 0.0f;
    R.A = 0.0f;
    R.sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    R.lat = -1;
    R.pix = y * P.W + x;
    R.done = true;
    if (active) {
        R.u = 1.0f * (x - P.W / 2.0f - P.xT) / P.H;
        R.v = 1.0f * (y - P.H / 2.0f - P.yT) / P.H;
        float a0, a1;
        if (ray_interval(P, R.u, R.v, a0, a1)) {
            int k0 = accu_lower(P, a0);
            k0 = k0 > 0 ? k0 - 1 : 0;
            R.a = P.accu[k0];
            R.lat = k0;
            R.a_stop = a1;
            R.done = false;
        }
    }
    const StepVec dv = step_vec(P);
    const float3 L = vr_light(P);
    const float L1 = P.step1;
    const float L4 = L1 / 4.0f;
    const float L8 = L1 / 8.0f;
    float accLocal[TRACK == kTrackLocal ? MK_MAX_LABELS : 1];
    if (TRACK == kTrackShared) {
        for (int i = 0; i < kMaxTrackedLabels; ++i) s_acc[i][tid] = 0.0f;
    } else if (TRACK == kTrackLocal) {
        for (int i = 0; i < MK_MAX_LABELS; ++i) accLocal[i] = 0.0f;
    }
    bool may_spill = TRACK != kTrackLocal && P.tail != nullptr;
    int iter = 0;
    // Every lane passes the loop's votes in the same iteration: a lane whose
    // ray is done skips only the body (no early continue), so the warp meets
    // at one ballot per iteration.
    while (true) {
        unsigned act = __ballot_sync(0xffffffffu, !R.done);
        if (act == 0u) break;
        if (may_spill && (++iter & 15) == 0 && tail_reached(P)) {
            may_spill = false;
            if (!R.done && spill_ray<TRACK>(P, R, s_acc, tid)) R.done = true;
            act = __ballot_sync(0xffffffffu, !R.done);
            if (act == 0u) break;
        }
        if (TRACK != kTrackLocal && __popc(act) <= P.coop_rays) {
            vr_coop_tail<TRACK>(P, vol, mask, S, BV, s_acc, ws + (tid & ~31), act, R, dv, L, may_spill);
            break;
        }
        if (!R.done) {
            // one step of the schedule: a sample outside the VOI, a run of
            // samples in an empty brick, or a fetched sample (lanes that take
            // different ones diverge only within this iteration)
            do {
                if (!(R.a < P.limit) || R.a > R.a_stop) {
                    R.done = true;
                    break;
                }
                const float3 pos = R.lat >= 0 ? ray_pos_at<false>(P, R.u, R.v, R.lat, R.a) : ray_pos(P, R.u, R.v, R.a);
                const int ix = pos.x * P.fdim[0];
                const int iy = pos.y * P.fdim[1];
                const int iz = pos.z * P.fdim[2];
                if (outside_voi(P, ix, iy, iz)) {
                    R.a += R.step;
                    if (R.lat >= 0) ++R.lat;
                    break;
                }
                if (P.skip && R.step == L1 && R.aPre <= 0.001f) {
                    const int b = brick_index(P, BV, ix, iy, iz);
                    if (!((BV.visible_bits[b >> 5] >> (b & 31)) & 1u)) {
                        R.aPre = 0.0f;
                        const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1], pos.z * P.fdim[2]);
                        advance_coarse(P, R.a, R.lat, R.step, 1 + steps_in_brick(pv, dv, ix, iy, iz));
                        break;
                    }
                }
                const int label = mask ? min((int)tex3D<unsigned char>(mask, ix, iy, iz), MK_MAX_LABELS - 1) : 0;
                float temp = 32768 * tex3D<float>(vol, pos.x, pos.y, pos.z);
                temp = (temp - S.wl[label]) / S.ww[label] + 0.5f;
                if (temp > 1) temp = 1;
                const cudaTextureObject_t tf = S.tf[label];
                float4 col = tf ? tex1D<float4>(tf, temp) : make_float4(0.f, 0.f, 0.f, 0.f);
                float alpha = col.w;
                // getNextStep (core/kernel.cu:84-125)
                if (R.step == L4) alpha = 1 - powf(1 - alpha, 0.25f);
                else if (R.step == L8) alpha = 1 - powf(1 - alpha, 0.125f);
                if (R.a > 0.0f) {
                    if ((alpha > R.aPre ? alpha : R.aPre) > 0.001f) {
                        if (R.step == L1) {
                            R.a -= (L1 - L4);
                            R.step = L4;
                            R.lat = -1;
                            break;
                        } else if (R.step == L4) {
                            R.a -= (L4 - L8);
                            R.step = L8;
                            break;
                        }
                    } else {
                        if (R.step == L8) R.step = L4;
                        else R.step = L1;
                    }
                }
                R.aPre = alpha;
                R.a += R.step;
                if (R.lat >= 0) ++R.lat;
                col.w = alpha;
                if (col.w > 0.0005f && vr_cap_ok<TRACK>(S, s_acc, accLocal, label, tid)) {
                    R.sum = composite(R.sum, R.A, col.w, shade_color(vol, pos, col, L, P));
                    vr_cap_add<TRACK>(S, s_acc, accLocal, label, tid, R.A, col.w);
                    R.A += (1.0f - R.A) * col.w;
                }
                if (R.A > 0.995f) R.done = true;
            } while (0);
        }
    }
    float4 sum = R.sum;
    if (sum.x == 0.0f && sum.y == 0.0f && sum.z == 0.0f && sum.w == 0.0f) sum = P.bg;
    return sum;
}

// One 32x8 pixel tile (bx, by) of a frame, by a 256-thread block: eight 8x4
// warp tiles.  s_acc holds the tracked opacity accumulators (kTrackShared),
// s_px the tile's RGB bytes, s_count the counting-mode total (zeroed by the
// caller).  Every thread of the block must call it.
template <int MODE, int TRACK, bool COUNT>
__device__ __forceinline__ void raycast_tile(const RayParams &P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                                             const LabelSmem &S, const BrickView &BV, float (*s_acc)[256],
                                             CoopSample *s_coop, uint8_t (*s_px)[32 * 3],
                                             unsigned long long *s_count, int bx, int by) {
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

    if (MODE == kModeVR && !COUNT) {
        sum = vr_march<TRACK>(P, vol, mask, S, BV, s_acc, s_coop, active, x, y);
    } else if (active) {
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
            const StepVec dv = step_vec(P);

            if (MODE == kModeVR) {
                // counting pass over MonkeyGL's schedule: every sample is
                // fetched (no skipping); rendering goes through vr_march
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
                    ++nsamples;
                    mark_footprint(P, pos.x, pos.y, pos.z);
                    if (mask) mark_label(P, ix, iy, iz);
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
                    // composite decisions still matter for termination
                    if (col.w > 0.0005f && vr_cap_ok<TRACK>(S, s_acc, accLocal, label, tid)) {
                        mark_gradient(P, pos);
                        vr_cap_add<TRACK>(S, s_acc, accLocal, label, tid, A, col.w);
                        A += (1.0f - A) * col.w;
                    }
                    if (A > 0.995f) break;
                }
                if (sum.x == 0.0f && sum.y == 0.0f && sum.z == 0.0f && sum.w == 0.0f) sum = P.bg;
            } else if (MODE == kModeMIP && !COUNT && P.mip_uniform) {
                // Every label the ray can meet is visible and has the same
                // window w(t) = (32768 t - wl) / ww + 0.5 with ww > 0.  Each of
                // its operations is rounded monotonically (a product by a
                // power of two, a difference, a quotient by a positive
                // number, a sum), so w is non-decreasing and the maximum of
                // w over the samples is w of the largest raw sample: the
                // label fetch is dropped and w is evaluated only when a
                // sample exceeds the raw maximum so far.  A holds the same
                // value as in the general loop below after every sample.
                // The loop below visits the entries k0 .. k_end - 1: those with
                // accu[k] <= a_stop and accu[k] < limit (the table's last entry
                // is its first >= limit), the entries the general loop visits.
                int k_end = accu_lower(P, a_stop);
                if (P.accu[k_end] <= a_stop) ++k_end;
                k_end = min(k_end, P.accu_len - 1);
                float vmax = -INFINITY;
                for (int k = k0; k < k_end;) {
                    const float3 pos = ray_pos_fy(P, u, v, P.fy_tab[k]);
                    const int ix = pos.x * P.fdim[0];
                    const int iy = pos.y * P.fdim[1];
                    const int iz = pos.z * P.fdim[2];
                    if (outside_voi(P, ix, iy, iz)) {
                        ++k;
                        continue;
                    }
                    if (P.skip) {
                        const int b = brick_index(P, BV, ix, iy, iz);
                        if (BV.mip_tmax[b] <= A) {
                            const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1],
                                                          pos.z * P.fdim[2]);
                            k += 1 + steps_in_brick(pv, dv, ix, iy, iz);
                            continue;
                        }
                    }
                    const float raw = tex3D<float>(vol, pos.x, pos.y, pos.z);
                    if (raw > vmax) {
                        vmax = raw;
                        float temp = 32768 * raw;
                        temp = (temp - P.mip_wl) / P.mip_ww + 0.5f;
                        if (A < temp) A = temp;
                    }
                    ++k;
                    // the output saturates at 1.0 (core/kernel.cu:351-358)
                    if (P.skip && A >= 1.0f) break;
                }
                if (A <= 0.0f) sum = P.bg;
                else sum = make_float4(A, A, A, A);
            } else if (MODE == kModeMIP) {
                // fixed step 1/dim_z from a table entry: every sample is
                // table entry k, a == accu[k]
                int k = k0;
                while (a < P.limit) {
                    if (a > a_stop) break;
                    const float3 pos = ray_pos_at<COUNT>(P, u, v, k, a);
                    const int ix = pos.x * P.fdim[0];
                    const int iy = pos.y * P.fdim[1];
                    const int iz = pos.z * P.fdim[2];
                    if (outside_voi(P, ix, iy, iz)) {
                        k = min(k + 1, P.accu_len - 1);
                        a = P.accu[k];
                        continue;
                    }
                    if (!COUNT && P.skip) {
                        const int b = brick_index(P, BV, ix, iy, iz);
                        if (BV.mip_tmax[b] <= A) {
                            const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1],
                                                          pos.z * P.fdim[2]);
                            k = min(k + 1 + steps_in_brick(pv, dv, ix, iy, iz), P.accu_len - 1);
                            a = P.accu[k];
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
                    k = min(k + 1, P.accu_len - 1);
                    a = P.accu[k];
                    // the output saturates at 1.0 (core/kernel.cu:351-358)
                    if (!COUNT && P.skip && A >= 1.0f) break;
                }
                if (A <= 0.0f) sum = P.bg;
                else sum = make_float4(A, A, A, A);
            } else {   // kModeSurface
                float3 L;
                {
                    float lx_ = dot3(0.0f, 1.0f, 0.0f, P.M[0], P.M[1], P.M[2]);
                    float ly_ = dot3(0.0f, 1.0f, 0.0f, P.M[3], P.M[4], P.M[5]);
                    float lz_ = dot3(0.0f, 1.0f, 0.0f, P.M[6], P.M[7], P.M[8]);
                    const float inv = rsqrtf(lx_ * lx_ + ly_ * ly_ + lz_ * lz_);
                    L = make_float3(lx_ * inv, ly_ * inv, lz_ * inv);
                }
                // fixed step from a table entry, as for MIP
                int k = k0;
                while (a < P.limit) {
                    if (a > a_stop) break;
                    const float3 pos = ray_pos_at<COUNT>(P, u, v, k, a);
                    const int ix = pos.x * P.fdim[0];
                    const int iy = pos.y * P.fdim[1];
                    const int iz = pos.z * P.fdim[2];
                    if (outside_voi(P, ix, iy, iz)) {
                        k = min(k + 1, P.accu_len - 1);
                        a = P.accu[k];
                        continue;
                    }
                    if (!COUNT && P.skip) {
                        const int b = brick_index(P, BV, ix, iy, iz);
                        const short2 mm = BV.minmax[b];
                        // 32768 * (v / 32767) <= 400 for every tap
                        if ((float)mm.y * (32768.0f / 32767.0f) + 0.01f <= 400.0f) {
                            const float3 pv = make_float3(pos.x * P.fdim[0], pos.y * P.fdim[1],
                                                          pos.z * P.fdim[2]);
                            k = min(k + 1 + steps_in_brick(pv, dv, ix, iy, iz), P.accu_len - 1);
                            a = P.accu[k];
                            continue;
                        }
                    }
                    if (COUNT) {
                        ++nsamples;
                        mark_footprint(P, pos.x, pos.y, pos.z);
                    }
                    const float temp = 32768 * tex3D<float>(vol, pos.x, pos.y, pos.z);
                    if (temp <= 400) {
                        k = min(k + 1, P.accu_len - 1);
                        a = P.accu[k];
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
                    k = min(k + 1, P.accu_len - 1);
                    a = P.accu[k];
                }
                if (A <= 0.0f) {
                    sum = P.bg;
                } else {
                    // A + 0.05 in double, rounded to float (core/kernel.cu:460)
                    const float g = __double2float_rn(__dadd_rn((double)A, 0.05));
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
// Host: the ray parameter of every schedule entry at `scale` (cached on the
// volume); rendering kernels read it for the samples on the table.
// The caller records its launch that reads table *idx with note_table_use.
int fy_table(VolumeState &v, float scale, cudaStream_t s, const float **out, int *idx);
// Host: build that table into `out` (v.accu_len floats) on stream s.
int launch_fy_table(const VolumeState &v, float scale, float *out, cudaStream_t s);
int tracking_mode_for(const uint64_t present[2], const float (*params)[3]);
// Host: P.mip_uniform / mip_ww / mip_wl for the labels present in a volume
// under a table of (alpha, ww, wl) rows.
void set_mip_window(RayParams &P, const uint64_t present[2], const float (*params)[3]);
// Host: the 32x8 tiles of a W x H frame (index by * tiles_x + bx) sorted by
// the distance of their centre to (W/2 + xT, H/2 + yT), where the volume
// centre projects: launching them in this order starts the long rays first.
std::vector<int> centre_first_tiles(int W, int H, int xT, int yT);

}  // namespace mk
