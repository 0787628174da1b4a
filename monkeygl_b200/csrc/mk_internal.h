// mk_internal.h -- device-side state of a resident volume and the parameter
// blocks the kernels receive.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/monkeygl_b200.h"

namespace mk {

// Bricks are 8^3 voxels.  A brick "owns" the sample positions whose integer
// voxel index (trunc(pos * dim), core/kernel.cu:208-210) falls inside it; its
// value footprint is the owned voxels plus a one-voxel apron, which covers
// every trilinear tap of an owned sample.
constexpr int kBrickShift = 3;
constexpr int kBrick = 1 << kBrickShift;

// Transfer-function alpha at or below this bound counts as empty.  MonkeyGL
// composites only samples with alpha > 0.0005 and refines the step only for
// alpha > 0.001 (core/kernel.cu:101, 242); the margin absorbs the rounding of
// the linear LUT filter.
constexpr float kEmptyAlpha = 0.0004f;

// Labels whose opacity cap needs a running per-ray accumulator, tracked in
// shared memory; volumes with more such labels use the local-memory path.
constexpr int kMaxTrackedLabels = 16;

struct LabelTable {
    cudaTextureObject_t tf[MK_MAX_LABELS];   // 0 = no table (transparent)
    float alpha[MK_MAX_LABELS];
    float ww[MK_MAX_LABELS];
    float wl[MK_MAX_LABELS];
};

// Per-frame view of the brick maps handed to the ray-casting kernels.
struct BrickView {
    const uint32_t *visible_bits;   // VR: 1 = some sample may have alpha > kEmptyAlpha
    const float *mip_tmax;          // MIP: upper bound of the windowed value over labels with alpha > 0
    const short2 *minmax;           // raw voxel min/max of the footprint
    int nbx, nby, nbz;
};

// The launches that read a cached device table, one event per reading
// stream (recorded after the launch): before the table's memory is reused,
// the host waits for those launches only.  A table read from more than
// kTableStreams streams falls back to waiting for the device.
constexpr int kTableStreams = 4;
struct TableUses {
    cudaStream_t stream[kTableStreams];
    cudaEvent_t done[kTableStreams];
    int n;
    bool many;
};
// Record, on stream s, the end of the launches queued so far that read the table.
int note_table_use(TableUses &u, cudaStream_t s);
// Wait on the host until every recorded reader has finished, then forget them.
int wait_table_uses(TableUses &u);
void free_table_uses(TableUses &u);

struct VolumeState {
    int device = 0;
    int dims[3] = {0, 0, 0};
    cudaStream_t stream = nullptr;

    cudaArray_t vol_array = nullptr;
    cudaTextureObject_t tex_linear = 0;   // normalized coords, trilinear, clamp, normalized float
    cudaTextureObject_t tex_point = 0;    // same array, nearest
    cudaArray_t mask_array = nullptr;
    cudaTextureObject_t tex_mask = 0;     // unnormalized coords, nearest, element type

    cudaArray_t tf_array[MK_MAX_LABELS] = {};
    cudaTextureObject_t tf_tex[MK_MAX_LABELS] = {};
    float *d_tf_alpha[MK_MAX_LABELS] = {};   // LUT alpha column, for the visibility pass
    int tf_len[MK_MAX_LABELS] = {};
    float params[MK_MAX_LABELS][3];          // alpha, ww, wl

    // brick maps
    int nb[3] = {0, 0, 0};
    short2 *d_minmax = nullptr;
    uint32_t *d_labels = nullptr;            // 3 words (labels 0..64) per brick
    uint32_t *d_visible = nullptr;           // 1 bit per brick
    float *d_mip_tmax = nullptr;
    bool maps_dirty = true;
    uint64_t present_labels[2] = {1, 0};     // labels occurring anywhere in the mask

    // ray schedule: accuLength after k plain steps of 1/dim_z
    float *d_accu = nullptr;
    int accu_len = 0;

    // output staging
    void *d_out = nullptr;
    size_t d_out_bytes = 0;
    void *h_pinned = nullptr;
    size_t h_pinned_bytes = 0;
    unsigned long long *d_counter = nullptr;

    // launch orders of the ray-casting tiles (centre first), per image size
    // and pan: {W, H, x pan, y pan} -> device table of tile indices
    struct TileOrder {
        int key[4];
        int *d_tiles;
        int cap;                // ints the table holds
        cudaEvent_t ready;      // recorded after the upload
        TableUses uses;
        uint64_t stamp;         // last use (least recently used is replaced)
    };
    TileOrder orders[16] = {};
    int n_orders = 0;
    uint64_t order_clock = 0;

    // ray parameter (accu[k] - 0.866) * scale of every schedule entry, per
    // camera scale: samples on the table read it instead of evaluating it
    struct FyTable {
        float scale;
        float *d_fy;
        cudaEvent_t ready;      // recorded after the table is built
        TableUses uses;
        uint64_t stamp;         // last use (least recently used is replaced)
    };
    FyTable fy_tables[8] = {};
    int n_fy_tables = 0;
    uint64_t fy_clock = 0;

    // display window of mk_render_plane_u8: the uint8 value of every int16
    // (index value + 32768) under the last (ww, wl) asked for
    uint8_t *d_voi_lut = nullptr;
    float voi_key[2] = {0.0f, 0.0f};
    bool voi_valid = false;
    cudaEvent_t voi_ready = nullptr;     // recorded after the table's upload
    TableUses voi_uses = {};

    // VR frame tail: counters and spill list, one set per rendering stream
    // (the tile launch and the tail launch of a frame use them in stream
    // order; the tail launch leaves the counters at zero)
    struct TailBuf {
        cudaStream_t stream;
        unsigned *d_tail;       // 4 counters
        void *d_rays;           // spill list
        int cap;                // rays it holds
        // host output: the tail launch's pixels as (pix, rgb) pairs in
        // mapped pinned memory, read while the image copy overlaps the tail
        // launch; 2 + 2 * cap words (word 0: the number of pairs)
        uint32_t *h_patch;
        uint32_t *d_patch;      // the same memory seen from the device
        int patch_cap;
        cudaStream_t copy_stream;
        cudaEvent_t tiles_done;
    };
    TailBuf tails[4] = {};
    int n_tails = 0;

    size_t device_bytes = 0;
};

// Thread-local last-error text (set by the C ABI on failure).
void set_last_error(const std::string &msg);

#define MK_CUDA_TRY(expr)                                                        \
    do {                                                                         \
        cudaError_t _e = (expr);                                                 \
        if (_e != cudaSuccess) {                                                 \
            ::mk::set_last_error(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
            return (_e == cudaErrorMemoryAllocation) ? MK_ERR_OUT_OF_MEMORY      \
                                                     : MK_ERR_CUDA;              \
        }                                                                        \
    } while (0)

// Smallest float strictly greater than the double bound c; for a float a,
// a < c  <=>  a < float_bound_above(c) when c is not itself a float.
float float_bound_above(double c);

// Host helpers shared by the entry points.
int ensure_device_buffer(VolumeState *v, size_t bytes);
int ensure_pinned_buffer(VolumeState *v, size_t bytes);
int rebuild_brick_maps(VolumeState *v, cudaStream_t s);
// Brick visibility bits and MIP bounds of volume v for the given per-label
// LUT alpha columns (device pointers, nullptr = no table), LUT lengths and
// (alpha, ww, wl) rows, written to vis_bits / mip_tmax on stream s.
int launch_brick_visibility(const VolumeState *v, const float *const *lut_alpha, const int *lut_len,
                            const float (*params)[3], uint32_t *vis_bits, float *mip_tmax, cudaStream_t s);
// Words of visibility bits / floats of MIP bounds of a volume's brick maps.
inline size_t brick_count(const VolumeState *v) { return (size_t)v->nb[0] * v->nb[1] * v->nb[2]; }
int finish_output(VolumeState *v, void *out, size_t bytes, int out_on_device, cudaStream_t s);
// True for page-locked host memory the device can copy to directly.
bool is_pinned_host(const void *p);
BrickView brick_view(const VolumeState *v);
LabelTable label_table(const VolumeState *v);
// Host-to-device copy of a large pageable buffer on stream s, pipelined
// through two pinned staging buffers shared by the process (host_stage.cpp);
// returns once the copy is done.  Below 8 MB: one cudaMemcpyAsync.
cudaError_t stage_to_device(void *dst, const void *src, size_t bytes, cudaStream_t s);

}  // namespace mk

struct mk_volume_s {
    mk::VolumeState st;
};
