// mk_raycast.cu -- orthographic ray casting: direct volume rendering with
// front-to-back compositing (VR), maximum intensity projection (MIP) and
// first-hit shaded surface (SURFACE).
//
// Method: MonkeyGL's d_render / d_renderMIP / d_renderSurface
// (core/kernel.cu:133-469).  Every sample position, window, LUT lookup,
// adaptive-step decision, opacity correction, shading term and the
// termination test follow that method step for step, so an image from
// these kernels equals MonkeyGL's on the same inputs.  What differs is how
// the work is organised on the GPU:
//
//  * Ray clipping.  MonkeyGL walks accuLength from 0 to 1.732 for every
//    pixel (about 1.7 * dim_z iterations, most of them outside the volume).
//    Here each ray computes, from the camera matrix, the parameter interval
//    where it can touch the VOI (with a two-voxel margin), starts at the
//    last schedule point before it (all rays share the accuLength sequence
//    a_{k+1} = fl(a_k + 1/dim_z) up to their first in-volume sample, kept in
//    a table) and stops once past it.  Samples outside that interval are
//    provably outside the VOI, where MonkeyGL only advances accuLength.
//  * Empty-space skipping.  While the ray is at the coarse step with a small
//    previous alpha, a sample inside a brick whose visibility bit is clear
//    cannot composite or refine the step (its alpha is <= kEmptyAlpha), so
//    the texture fetches are skipped; accuLength still advances by the same
//    float additions, and runs of such samples up to the brick exit are
//    advanced with additions only.  MIP skips bricks whose bound cannot
//    raise the running maximum and stops at 1.0 (the 8-bit output
//    saturates); SURFACE skips bricks whose voxels are all <= 400 HU.
//  * Warp-coherent tiles.  A 256-thread block covers a 32x8 pixel tile as
//    eight 8x4 warp tiles, so each warp's rays are spatially adjacent and
//    share texture cache lines; RGB output is staged in shared memory and
//    stored as aligned 32-bit words.
//  * Per-label opacity caps live in shared memory (or registers when no
//    label needs one) instead of a 65-float local array per thread.
//  * FP32 only: MonkeyGL's double-promoted expressions are reproduced with
//    error-free float transformations (mk_math.h).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <utility>
#include <vector>

#include "mk_internal.h"
#include "mk_math.h"
#include "mk_raycast_impl.cuh"

namespace mk {

// One 32x8 tile per block.  With `order`, block i renders tile order[i]
// (index by * tiles_x + bx): the launch takes tiles centre first, where the
// projected volume -- and the longest rays -- usually are, so they start in
// the first wave instead of forming the tail of the launch.  Register
// budgets, measured on 1024^2 frames: VR 48 (five blocks per SM; four and
// six were slower on the body and cardiac frames), MIP and surface 40 (six;
// eight, at 32 registers, was slower).
constexpr int kVrBlocksPerSm = 5;
constexpr int kRayBlocksPerSm = 6;
// The hand-off launch: two blocks per SM (up to 128 registers); three and
// four (80 and 64 registers) were slower on the body frame.
constexpr int kTailBlocksPerSm = 2;
template <int MODE, int TRACK, bool COUNT>
__global__ void __launch_bounds__(256, MODE == kModeVR ? kVrBlocksPerSm : kRayBlocksPerSm) k_raycast(RayParams P, cudaTextureObject_t vol,
                                                 cudaTextureObject_t mask, LabelTable LT,
                                                 BrickView BV, const int *__restrict__ order) {
    __shared__ LabelSmem S;
    __shared__ float s_acc[TRACK == kTrackShared ? kMaxTrackedLabels : 1][256];
    __shared__ CoopSample s_coop[MODE == kModeVR && !COUNT ? 256 : 1];
    __shared__ uint8_t s_px[8][32 * 3];
    __shared__ unsigned long long s_count;
    load_label_smem(S, LT, TRACK);
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    int bx = blockIdx.x, by = blockIdx.y;
    if (order) {
        const int t = order[blockIdx.x], tx = (P.W + 31) / 32;
        bx = t % tx;
        by = t / tx;
    }
    raycast_tile<MODE, TRACK, COUNT>(P, vol, mask, S, BV, s_acc, s_coop, s_px, &s_count, bx, by);
    if (MODE == kModeVR && !COUNT && P.tail) {
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(&P.tail[0], 1u);
    }
}

// The tail launch of a VR frame: resumes the rays that the tile launch
// spilled (same P, same tables), one ray per warp at a time so that each
// gets all 32 lanes of vr_coop_tail (measured faster than packing several
// rays into a warp when there are more rays than warps: body 1024^2 frames
// +1.1%, cardiac +1.9%), writes their pixels, and resets the frame's tail
// counters for the next frame.
template <int TRACK>
__global__ void __launch_bounds__(256, kTailBlocksPerSm) k_vr_tail(RayParams P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                                                 LabelTable LT, BrickView BV) {
    __shared__ LabelSmem S;
    __shared__ float s_acc[TRACK == kTrackShared ? kMaxTrackedLabels : 1][256];
    __shared__ CoopSample s_coop[256];
    __shared__ unsigned s_n;
    load_label_smem(S, LT, TRACK);
    if (threadIdx.x == 0) s_n = min(*(volatile unsigned *)&P.tail[1], (unsigned)P.spill_cap);
    __syncthreads();
    const unsigned n = s_n;
    const int tid = threadIdx.x, lane = tid & 31;
    if (P.patch && blockIdx.x == 0 && tid == 0) P.patch[0] = n;
    const unsigned per = 1;    // rays a warp takes at a time
    const StepVec dv = step_vec(P);
    const float3 L = vr_light(P);
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&P.tail[2], per);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const unsigned cnt = min(per, n - base);
        VrRay R;
        R.done = true;
        R.sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if ((unsigned)lane < cnt) {
            const SpillRay &q = P.spill[base + lane];
            R.sum = q.sum;
            R.u = q.u;
            R.v = q.v;
            R.a = q.a;
            R.a_stop = q.a_stop;
            R.step = q.step;
            R.aPre = q.aPre;
            R.A = q.A;
            R.lat = q.lat;
            R.pix = q.pix;
            R.done = false;
            if (TRACK == kTrackShared) {
#pragma unroll
                for (int k = 0; k < kMaxTrackedLabels; ++k) s_acc[k][tid] = q.acc[k];
            }
        }
        const unsigned act = __ballot_sync(0xffffffffu, (unsigned)lane < cnt);
        __syncwarp();
        vr_coop_tail<TRACK, true>(P, vol, mask, S, BV, s_acc, s_coop + (tid & ~31), act, R, dv, L, false);
        // the pixel index comes from the spill list: it is checked against
        // the frame before the store, so a corrupt entry cannot write
        // outside the image
        if ((unsigned)lane < cnt && (unsigned)R.pix < (unsigned)P.W * (unsigned)P.H) {
            float4 sum = R.sum;
            if (sum.x == 0.0f && sum.y == 0.0f && sum.z == 0.0f && sum.w == 0.0f) sum = P.bg;
            const uint32_t rgb = pack_rgb(sum);
            if (P.patch) {
                // host output: the image is being copied while this launch
                // runs; the host applies these pixels after both finish
                P.patch[2 + 2 * (size_t)(base + lane)] = (uint32_t)R.pix;
                P.patch[3 + 2 * (size_t)(base + lane)] = rgb;
            } else if (P.rgba) {
                reinterpret_cast<uint32_t *>(P.out)[R.pix] = rgb | 0xff000000u;
            } else {
                uint8_t *o = P.out + (size_t)R.pix * 3;
                o[0] = rgb & 0xff;
                o[1] = (rgb >> 8) & 0xff;
                o[2] = (rgb >> 16) & 0xff;
            }
        }
    }
    // the last block to finish resets the counters for the next frame
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&P.tail[3], 1u) == gridDim.x - 1) {
            P.tail[0] = 0;
            P.tail[1] = 0;
            P.tail[2] = 0;
            P.tail[3] = 0;
        }
    }
}

template <int MODE, int TRACK, bool COUNT>
static void launch_mode(const RayParams &P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                        const LabelTable &LT, const BrickView &BV, const int *order, cudaStream_t s) {
    const int tx = (P.W + 31) / 32, ty = (P.H + 7) / 8;
    const dim3 grid = order ? dim3(tx * ty) : dim3(tx, ty);
    k_raycast<MODE, TRACK, COUNT><<<grid, 256, 0, s>>>(P, vol, mask, LT, BV, order);
}

template <bool COUNT>
static void launch_raycast(int mode, int track, const RayParams &P, cudaTextureObject_t vol,
                           cudaTextureObject_t mask, const LabelTable &LT, const BrickView &BV,
                           const int *order, cudaStream_t s) {
    if (mode == kModeVR) {
        if (track == kTrackNone) launch_mode<kModeVR, kTrackNone, COUNT>(P, vol, mask, LT, BV, order, s);
        else if (track == kTrackShared) launch_mode<kModeVR, kTrackShared, COUNT>(P, vol, mask, LT, BV, order, s);
        else launch_mode<kModeVR, kTrackLocal, COUNT>(P, vol, mask, LT, BV, order, s);
    } else if (mode == kModeMIP) {
        launch_mode<kModeMIP, kTrackNone, COUNT>(P, vol, mask, LT, BV, order, s);
    } else {
        launch_mode<kModeSurface, kTrackNone, COUNT>(P, vol, mask, LT, BV, order, s);
    }
}

// Tiles still unfinished when rays start to spill to the tail launch:
// two thirds of the SM count (measured on 1024^2 body frames on 148 SMs:
// 16, 48, 96, 148, 296 tiles gave 2699, 2907, 2989, 2761, 2445 frames/s).
// MONKEYGL_B200_TAIL_TILES overrides it (0: rays never spill).
static int tail_tiles() {
    static const int k = [] {
        const char *e = getenv("MONKEYGL_B200_TAIL_TILES");
        if (e) return std::max(0, atoi(e));
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 148;
        return std::max(1, 2 * sms / 3);
    }();
    return k;
}

// The tail buffers of stream s (created on first use, grown for larger
// frames) and the frame's tail fields of P.  Four streams per volume have
// their own; a fifth renders without a tail launch.
static int tail_params(VolumeState &v, RayParams &P, cudaStream_t s) {
    const int ntiles = ((P.W + 31) / 32) * ((P.H + 7) / 8);
    const int K = tail_tiles();
    if (K == 0) return MK_OK;                      // no hand-off: P.tail stays null
    const int want = (int)std::min<long long>((long long)P.W * P.H, std::max(4LL * K * 256, 65536LL));
    int i = 0;
    while (i < v.n_tails && v.tails[i].stream != s) ++i;
    if (i == v.n_tails) {
        if (v.n_tails == 4) return MK_OK;
        VolumeState::TailBuf t = {};
        t.stream = s;
        MK_CUDA_TRY(cudaMalloc(&t.d_tail, 4 * sizeof(unsigned)));
        if (cudaMemsetAsync(t.d_tail, 0, 4 * sizeof(unsigned), s) != cudaSuccess) {
            cudaFree(t.d_tail);
            set_last_error("tail counters: memset failed");
            return MK_ERR_CUDA;
        }
        v.tails[v.n_tails++] = t;
    }
    VolumeState::TailBuf &t = v.tails[i];
    if (t.cap < want) {
        MK_CUDA_TRY(cudaStreamSynchronize(s));     // the last frame on s is done with the list
        cudaFree(t.d_rays);
        t.d_rays = nullptr;
        t.cap = 0;
        MK_CUDA_TRY(cudaMalloc(&t.d_rays, (size_t)want * sizeof(SpillRay)));
        t.cap = want;
    }
    P.tail = t.d_tail;
    P.spill = static_cast<SpillRay *>(t.d_rays);
    P.spill_cap = t.cap;
    P.tail_trigger = std::max(0, ntiles - K);
    return MK_OK;
}

// Host output of a frame with a tail launch: the (pix, rgb) list that the
// tail launch writes instead of the image, and the stream and event that
// let the image's copy to the host run while the tail launch does.  Sets
// *tb to null (and leaves P.patch null: the plain readback) when stream s
// has no tail buffer or the mapped allocation fails.
static int tail_patch(VolumeState &v, RayParams &P, cudaStream_t s, VolumeState::TailBuf **tb) {
    *tb = nullptr;
    if (!P.tail) return MK_OK;
    int i = 0;
    while (i < v.n_tails && v.tails[i].stream != s) ++i;
    if (i == v.n_tails) return MK_OK;
    VolumeState::TailBuf &t = v.tails[i];
    if (!t.copy_stream) {
        MK_CUDA_TRY(cudaStreamCreateWithFlags(&t.copy_stream, cudaStreamNonBlocking));
        if (cudaEventCreateWithFlags(&t.tiles_done, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            cudaStreamDestroy(t.copy_stream);
            t.copy_stream = nullptr;
            return MK_OK;
        }
    }
    if (t.patch_cap < P.spill_cap) {
        if (t.h_patch) cudaFreeHost(t.h_patch);      // the last frame on s has finished (host output)
        t.h_patch = t.d_patch = nullptr;
        t.patch_cap = 0;
        void *h = nullptr, *d = nullptr;
        const size_t words = 2 + 2 * (size_t)P.spill_cap;
        if (cudaHostAlloc(&h, words * sizeof(uint32_t), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
            cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
            cudaGetLastError();
            if (h) cudaFreeHost(h);
            return MK_OK;
        }
        t.h_patch = static_cast<uint32_t *>(h);
        t.d_patch = static_cast<uint32_t *>(d);
        t.patch_cap = P.spill_cap;
    }
    P.patch = t.d_patch;
    *tb = &t;
    return MK_OK;
}

template <int TRACK>
static int launch_tail_track(const RayParams &P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                             const LabelTable &LT, const BrickView &BV, cudaStream_t s) {
    // one resident grid; computed once (threads that race here compute the
    // same value)
    static std::atomic<int> cached{0};
    int grid = cached.load(std::memory_order_relaxed);
    if (grid == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        MK_CUDA_TRY(cudaGetDevice(&dev));
        MK_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        MK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vr_tail<TRACK>, 256, 0));
        grid = std::max(1, sms * std::max(1, per_sm));
        cached.store(grid, std::memory_order_relaxed);
    }
    k_vr_tail<TRACK><<<grid, 256, 0, s>>>(P, vol, mask, LT, BV);
    MK_CUDA_TRY(cudaGetLastError());
    return MK_OK;
}

static int launch_vr_tail(int track, const RayParams &P, cudaTextureObject_t vol, cudaTextureObject_t mask,
                          const LabelTable &LT, const BrickView &BV, cudaStream_t s) {
    if (!P.tail) return MK_OK;
    if (track == kTrackShared) return launch_tail_track<kTrackShared>(P, vol, mask, LT, BV, s);
    return launch_tail_track<kTrackNone>(P, vol, mask, LT, BV, s);
}

std::vector<int> centre_first_tiles(int W, int H, int xT, int yT) {
    const int tx = (W + 31) / 32, ty = (H + 7) / 8, n = tx * ty;
    const double cx = W / 2.0 + xT, cy = H / 2.0 + yT;
    std::vector<std::pair<double, int>> d((size_t)n);
    for (int t = 0; t < n; ++t) {
        const double dx = (t % tx) * 32 + 16 - cx, dy = (t / tx) * 8 + 4 - cy;
        d[t] = {dx * dx + dy * dy, t};
    }
    std::stable_sort(d.begin(), d.end());
    std::vector<int> h((size_t)n);
    for (int t = 0; t < n; ++t) h[t] = d[t].second;
    return h;
}

int note_table_use(TableUses &u, cudaStream_t s) {
    int i = 0;
    while (i < u.n && u.stream[i] != s) ++i;
    if (i == u.n) {
        if (u.n == kTableStreams) {
            u.many = true;                  // reuse will wait for the device
            return MK_OK;
        }
        MK_CUDA_TRY(cudaEventCreateWithFlags(&u.done[i], cudaEventDisableTiming));
        u.stream[i] = s;
        ++u.n;
    }
    MK_CUDA_TRY(cudaEventRecord(u.done[i], s));
    return MK_OK;
}

int wait_table_uses(TableUses &u) {
    if (u.many) {
        MK_CUDA_TRY(cudaDeviceSynchronize());
    } else {
        for (int i = 0; i < u.n; ++i) MK_CUDA_TRY(cudaEventSynchronize(u.done[i]));
    }
    free_table_uses(u);
    return MK_OK;
}

void free_table_uses(TableUses &u) {
    for (int i = 0; i < u.n; ++i) cudaEventDestroy(u.done[i]);
    u.n = 0;
    u.many = false;
}

// The centre-first tile order of a W x H image whose volume centre projects
// to (W/2 + xT, H/2 + yT) (core/kernel.cu:161-162 with u = v = 0), cached on
// the volume (16 keys).  A new table is uploaded on `s` without a host wait;
// launches on other streams that find it wait for its `ready` event.  The
// caller records the launch that reads it with note_table_use(*idx); a
// replaced table's memory is reused once those launches have finished.
static int tile_order(VolumeState &v, const RayParams &P, cudaStream_t s, const int **out, int *idx) {
    const int key[4] = {P.W, P.H, (int)lrintf(P.xT), (int)lrintf(P.yT)};
    for (int i = 0; i < v.n_orders; ++i) {
        VolumeState::TileOrder &o = v.orders[i];
        if (o.key[0] == key[0] && o.key[1] == key[1] && o.key[2] == key[2] && o.key[3] == key[3]) {
            MK_CUDA_TRY(cudaStreamWaitEvent(s, o.ready, 0));
            o.stamp = ++v.order_clock;
            *out = o.d_tiles;
            *idx = i;
            return MK_OK;
        }
    }
    const std::vector<int> h = centre_first_tiles(P.W, P.H, key[2], key[3]);
    const int n = (int)h.size();
    int i = v.n_orders;
    if (i == 16) {                               // replace the least recently used
        i = 0;
        for (int j = 1; j < 16; ++j)
            if (v.orders[j].stamp < v.orders[i].stamp) i = j;
        int rc = wait_table_uses(v.orders[i].uses);
        if (rc != MK_OK) return rc;
    } else {
        VolumeState::TileOrder o = {};
        MK_CUDA_TRY(cudaEventCreateWithFlags(&o.ready, cudaEventDisableTiming));
        v.orders[v.n_orders++] = o;
    }
    VolumeState::TileOrder &o = v.orders[i];
    if (o.cap < n) {
        cudaFree(o.d_tiles);
        o.d_tiles = nullptr;
        o.cap = 0;
        MK_CUDA_TRY(cudaMalloc(&o.d_tiles, (size_t)n * sizeof(int)));
        o.cap = n;
    }
    // pageable source: the call returns once `h` is staged
    MK_CUDA_TRY(cudaMemcpyAsync(o.d_tiles, h.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
    MK_CUDA_TRY(cudaEventRecord(o.ready, s));
    for (int k = 0; k < 4; ++k) o.key[k] = key[k];
    o.stamp = ++v.order_clock;
    *out = o.d_tiles;
    *idx = i;
    return MK_OK;
}

// fy = (accu[k] - 0.866) * scale for every schedule entry, by the same
// device function the kernels evaluate per sample (core/kernel.cu:197).
__global__ void k_fy_table(const float *__restrict__ accu, int n, float scale, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = ray_fy(accu[i], scale);
}

int launch_fy_table(const VolumeState &v, float scale, float *out, cudaStream_t s) {
    k_fy_table<<<(v.accu_len + 255) / 256, 256, 0, s>>>(v.d_accu, v.accu_len, scale, out);
    MK_CUDA_TRY(cudaGetLastError());
    return MK_OK;
}

// The fy table of volume v at `scale`, cached on the volume (8 scales).  A
// new table is built on `s` without waiting: launches on `s` follow it in
// stream order, and a launch on another stream that finds it in the cache
// waits for its `ready` event.  The caller records the launch that reads it
// with note_table_use(*idx); replacing the least recently used table (a
// ninth scale) waits on the host for the launches recorded on it.
int fy_table(VolumeState &v, float scale, cudaStream_t s, const float **out, int *idx) {
    for (int i = 0; i < v.n_fy_tables; ++i) {
        VolumeState::FyTable &t = v.fy_tables[i];
        if (memcmp(&t.scale, &scale, sizeof(float)) == 0) {
            MK_CUDA_TRY(cudaStreamWaitEvent(s, t.ready, 0));
            t.stamp = ++v.fy_clock;
            *out = t.d_fy;
            *idx = i;
            return MK_OK;
        }
    }
    int i = v.n_fy_tables;
    if (i == 8) {
        i = 0;
        for (int j = 1; j < 8; ++j)
            if (v.fy_tables[j].stamp < v.fy_tables[i].stamp) i = j;
        int rc = wait_table_uses(v.fy_tables[i].uses);
        if (rc != MK_OK) return rc;
    } else {
        VolumeState::FyTable t = {};
        MK_CUDA_TRY(cudaMalloc(&t.d_fy, (size_t)v.accu_len * sizeof(float)));
        if (cudaEventCreateWithFlags(&t.ready, cudaEventDisableTiming) != cudaSuccess) {
            cudaFree(t.d_fy);
            set_last_error("fy table: event creation failed");
            return MK_ERR_CUDA;
        }
        v.fy_tables[v.n_fy_tables++] = t;
    }
    VolumeState::FyTable &t = v.fy_tables[i];
    int rc = launch_fy_table(v, scale, t.d_fy, s);
    if (rc != MK_OK) return rc;
    MK_CUDA_TRY(cudaEventRecord(t.ready, s));
    t.scale = scale;
    t.stamp = ++v.fy_clock;
    *out = t.d_fy;
    *idx = i;
    return MK_OK;
}

// Labels that need a per-ray opacity accumulator: present in the mask and
// with a cap strictly between 0 and 1.
int tracking_mode_for(const uint64_t present[2], const float (*params)[3]) {
    int n = 0;
    for (int l = 0; l < MK_MAX_LABELS; ++l) {
        const bool pres = (present[l >> 6] >> (l & 63)) & 1ull;
        const float a = params[l][0];
        if (pres && a > 0.0f && a < 1.0f) ++n;
    }
    if (n == 0) return kTrackNone;
    // slots are assigned in label order over all labels with 0 < alpha < 1
    int all = 0;
    for (int l = 0; l < MK_MAX_LABELS; ++l) {
        const float a = params[l][0];
        if (a > 0.0f && a < 1.0f) ++all;
    }
    return all <= kMaxTrackedLabels ? kTrackShared : kTrackLocal;
}

static int tracking_mode(const VolumeState &v) { return tracking_mode_for(v.present_labels, v.params); }

// MIP takes the uniform-window loop when every label present in the mask
// has alpha > 0 and all of them share one window with ww > 0.
void set_mip_window(RayParams &P, const uint64_t present[2], const float (*params)[3]) {
    P.mip_uniform = 0;
    int first = -1;
    for (int l = 0; l < MK_MAX_LABELS; ++l) {
        if (!((present[l >> 6] >> (l & 63)) & 1ull)) continue;
        if (!(params[l][0] > 0.0f)) return;
        if (first < 0) {
            first = l;
        } else if (params[l][1] != params[first][1] || params[l][2] != params[first][2]) {
            return;
        }
    }
    if (first < 0 || !(params[first][1] > 0.0f)) return;
    P.mip_uniform = 1;
    P.mip_ww = params[first][1];
    P.mip_wl = params[first][2];
}

int fill_ray_params(const VolumeState &v, const mk_vr_params *p, RayParams &P) {
    if (!p || p->width <= 0 || p->height <= 0 || p->width > 16384 || p->height > 16384) {
        set_last_error("mk_render_vr: image size must be in [1, 16384]");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (!(p->scale > 0.0f)) {
        set_last_error("mk_render_vr: scale must be > 0");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (p->render_type < MK_RENDER_VR || p->render_type > MK_RENDER_SURFACE) {
        set_last_error("mk_render_vr: unknown render type");
        return MK_ERR_INVALID_ARGUMENT;
    }
    P.W = p->width;
    P.H = p->height;
    for (int k = 0; k < 3; ++k) {
        P.fdim[k] = (float)v.dims[k];
        P.dimi[k] = v.dims[k];
        P.mls[k] = p->max_len_spacing[k];
        P.sv[k] = p->spacing_voxel[k];
    }
    P.xT = p->x_translate;
    P.yT = p->y_translate;
    P.scale = p->scale;
    for (int i = 0; i < 9; ++i) P.M[i] = p->transform[i];
    P.invertZ = p->invert_z ? 1 : 0;
    for (int i = 0; i < 6; ++i) P.voi[i] = p->voi[i];
    P.bg = make_float4(p->background[0], p->background[1], p->background[2], p->background[3]);
    P.step1 = 1.0f / (float)v.dims[2];
    P.limit = float_bound_above(1.732);
    P.accu = v.d_accu;
    P.fy_tab = nullptr;
    P.accu_len = v.accu_len;
    P.rgba = (p->pixel_format == MK_PIXEL_RGBA8) ? 1 : 0;
    P.skip = (p->flags & MK_VR_NO_SKIP) ? 0 : 1;
    P.coop_rays = (p->flags & MK_VR_NO_COOP) ? 0 : kCoopRaysDefault;
    P.out = nullptr;
    P.counter = nullptr;
    P.vox_bits = nullptr;
    P.lab_bits = nullptr;
    P.tail = nullptr;
    P.spill = nullptr;
    P.spill_cap = 0;
    P.tail_trigger = 0;
    P.patch = nullptr;
    P.mip_uniform = 0;
    P.mip_ww = 1.0f;
    P.mip_wl = 0.0f;
    return MK_OK;
}

}  // namespace mk

using namespace mk;

extern "C" int mk_render_vr(mk_volume vol, const mk_vr_params *params, void *out,
                            int out_on_device, void *stream) {
    if (!vol || !out) {
        set_last_error("mk_render_vr: null volume or output");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &v = vol->st;
    RayParams P;
    int rc = fill_ray_params(v, params, P);
    if (rc != MK_OK) return rc;
    cudaSetDevice(v.device);
    cudaStream_t s = stream ? (cudaStream_t)stream : v.stream;
    const size_t bytes = (size_t)P.W * P.H * (P.rgba ? 4 : 3);
    if (out_on_device) {
        P.out = (uint8_t *)out;
    } else {
        rc = ensure_device_buffer(&v, bytes);
        if (rc != MK_OK) return rc;
        P.out = (uint8_t *)v.d_out;
    }
    rc = rebuild_brick_maps(&v, s);
    if (rc != MK_OK) return rc;
    const int *order = nullptr;
    int order_idx = 0, fy_idx = 0;
    rc = tile_order(v, P, s, &order, &order_idx);
    if (rc != MK_OK) return rc;
    rc = fy_table(v, P.scale, s, &P.fy_tab, &fy_idx);
    if (rc != MK_OK) return rc;
    const int track = tracking_mode(v);
    if (params->render_type == MK_RENDER_MIP) set_mip_window(P, v.present_labels, v.params);
    const bool tail = params->render_type == MK_RENDER_VR && track != kTrackLocal &&
                      !(params->flags & (MK_VR_NO_TAIL | MK_VR_NO_COOP));
    VolumeState::TailBuf *tb = nullptr;
    if (tail) {
        rc = tail_params(v, P, s);
        if (rc == MK_OK && !out_on_device) rc = tail_patch(v, P, s, &tb);
        if (rc != MK_OK) return rc;
    }
    uint8_t *dst = nullptr;                    // host copy of the image (tb: overlapping the tail launch)
    if (tb) {
        if (is_pinned_host(out)) {
            dst = static_cast<uint8_t *>(out);
        } else {
            rc = ensure_pinned_buffer(&v, bytes);
            if (rc != MK_OK) return rc;
            dst = static_cast<uint8_t *>(v.h_pinned);
        }
    }
    launch_raycast<false>(params->render_type, track, P, v.tex_linear, v.tex_mask, label_table(&v),
                          brick_view(&v), order, s);
    MK_CUDA_TRY(cudaGetLastError());
    if (tb) {
        // every pixel but the tail launch's is final once the tiles are done
        MK_CUDA_TRY(cudaEventRecord(tb->tiles_done, s));
        MK_CUDA_TRY(cudaStreamWaitEvent(tb->copy_stream, tb->tiles_done, 0));
        MK_CUDA_TRY(cudaMemcpyAsync(dst, P.out, bytes, cudaMemcpyDeviceToHost, tb->copy_stream));
    }
    if (tail) {
        rc = launch_vr_tail(track, P, v.tex_linear, v.tex_mask, label_table(&v), brick_view(&v), s);
        if (rc != MK_OK) return rc;
    }
    rc = note_table_use(v.orders[order_idx].uses, s);
    if (rc == MK_OK) rc = note_table_use(v.fy_tables[fy_idx].uses, s);
    if (rc != MK_OK) return rc;
    if (!tb) return finish_output(&v, out, bytes, out_on_device, s);
    MK_CUDA_TRY(cudaStreamSynchronize(tb->copy_stream));
    MK_CUDA_TRY(cudaStreamSynchronize(s));
    if (dst != out) memcpy(out, dst, bytes);
    // the tail launch's pixels, from its (pix, rgb) list in mapped memory
    const volatile uint32_t *pl = tb->h_patch;
    const uint32_t n_listed = pl[0];
    const uint32_t n = std::min<uint32_t>(n_listed, (uint32_t)tb->patch_cap);
    const uint32_t npix = (uint32_t)P.W * (uint32_t)P.H;
    uint8_t *o = static_cast<uint8_t *>(out);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t pix = pl[2 + 2 * (size_t)i], rgb = pl[3 + 2 * (size_t)i];
        if (pix >= npix) continue;
        if (P.rgba) {
            const uint32_t w = rgb | 0xff000000u;
            memcpy(o + (size_t)pix * 4, &w, 4);
        } else {
            o[(size_t)pix * 3 + 0] = rgb & 0xff;
            o[(size_t)pix * 3 + 1] = (rgb >> 8) & 0xff;
            o[(size_t)pix * 3 + 2] = (rgb >> 16) & 0xff;
        }
    }
    return MK_OK;
}

__global__ void k_popcount(const uint32_t *__restrict__ bits, size_t nwords, unsigned long long *out) {
    unsigned long long c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nwords; i += (size_t)gridDim.x * blockDim.x)
        c += __popc(bits[i]);
    c = __reduce_add_sync(0xffffffffu, (unsigned)c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

extern "C" int mk_count_vr_samples(mk_volume vol, const mk_vr_params *params, uint64_t *samples) {
    if (!vol || !samples) {
        set_last_error("mk_count_vr_samples: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &v = vol->st;
    RayParams P;
    int rc = fill_ray_params(v, params, P);
    if (rc != MK_OK) return rc;
    cudaSetDevice(v.device);
    cudaStream_t s = v.stream;
    P.skip = 0;
    P.counter = v.d_counter;
    MK_CUDA_TRY(cudaMemsetAsync(v.d_counter, 0, sizeof(unsigned long long), s));
    rc = rebuild_brick_maps(&v, s);
    if (rc != MK_OK) return rc;
    launch_raycast<true>(params->render_type, tracking_mode(v), P, v.tex_linear, v.tex_mask,
                         label_table(&v), brick_view(&v), nullptr, s);
    MK_CUDA_TRY(cudaGetLastError());
    unsigned long long h = 0;
    MK_CUDA_TRY(cudaMemcpyAsync(&h, v.d_counter, sizeof(h), cudaMemcpyDeviceToHost, s));
    MK_CUDA_TRY(cudaStreamSynchronize(s));
    *samples = h;
    return MK_OK;
}

extern "C" int mk_count_vr_footprint(mk_volume vol, const mk_vr_params *params, uint64_t *samples,
                                     uint64_t *voxels, uint64_t *label_voxels) {
    if (!vol || !samples || !voxels || !label_voxels) {
        set_last_error("mk_count_vr_footprint: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &v = vol->st;
    RayParams P;
    int rc = fill_ray_params(v, params, P);
    if (rc != MK_OK) return rc;
    cudaSetDevice(v.device);
    cudaStream_t s = v.stream;
    const size_t nvox = (size_t)v.dims[0] * v.dims[1] * v.dims[2];
    const size_t nwords = (nvox + 31) / 32;
    uint32_t *bits = nullptr;
    unsigned long long *cnt = nullptr;
    MK_CUDA_TRY(cudaMalloc(&bits, 2 * nwords * sizeof(uint32_t)));
    if (cudaMalloc(&cnt, 3 * sizeof(unsigned long long)) != cudaSuccess) {
        cudaFree(bits);
        set_last_error("mk_count_vr_footprint: allocation failed");
        return MK_ERR_OUT_OF_MEMORY;
    }
    cudaMemsetAsync(bits, 0, 2 * nwords * sizeof(uint32_t), s);
    cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned long long), s);
    P.skip = 0;
    P.counter = cnt;
    P.vox_bits = bits;
    P.lab_bits = bits + nwords;
    rc = rebuild_brick_maps(&v, s);
    if (rc == MK_OK) {
        launch_raycast<true>(params->render_type, tracking_mode(v), P, v.tex_linear, v.tex_mask,
                             label_table(&v), brick_view(&v), nullptr, s);
        k_popcount<<<1184, 256, 0, s>>>(bits, nwords, cnt + 1);
        k_popcount<<<1184, 256, 0, s>>>(bits + nwords, nwords, cnt + 2);
        unsigned long long h[3] = {0, 0, 0};
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_last_error(std::string("mk_count_vr_footprint: ") + cudaGetErrorString(e));
            rc = MK_ERR_CUDA;
        } else {
            *samples = h[0];
            *voxels = h[1];
            *label_voxels = h[2];
        }
    }
    cudaFree(bits);
    cudaFree(cnt);
    return rc;
}
