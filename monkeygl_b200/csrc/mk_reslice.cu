// mk_reslice.cu -- planar (MPR) and curved (CPR) reslicing of a resident
// volume into int16 images.
//
// Method: MonkeyGL's d_renderPlane_{MIP,MinIP,Average} and d_renderCPR
// (core/kernel.cu:570-873): each output pixel maps to a point in volume
// millimetres (planes) or voxel units (CPR), is normalised by the volume
// extent, z-flipped unless the volume is already inverted, and read through
// the trilinear texture scaled by 32768; slabs reduce 2*halfNum+1 samples
// along the plane normal by max, min or mean.  The coordinate expressions keep
// MonkeyGL's operation order; its FP64 pieces (the CPR point arithmetic and
// the slab-mean accumulator) are evaluated in double, operation for
// operation (FP64 runs at half the FP32 rate on sm_100).  MK_SAMPLE_NEAREST reads the same voxels through a
// point-filtered texture view.
//
// Layout: 256-thread blocks cover 32x8 output tiles so each warp stores one
// 64-byte row segment; CPR rows share their (point, direction) pair through
// shared memory.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "mk_internal.h"
#include "mk_math.h"
#include "mk_reslice_impl.cuh"

namespace mk {

template <int MODE, bool U8>
__global__ void __launch_bounds__(256) k_plane(PlaneParams P, cudaTextureObject_t tex, void *out) {
    plane_tile<MODE, U8>(P, tex, out, blockIdx.x, blockIdx.y);
}

// CPR row data: the point and direction of each row, as MonkeyGL passes them.
struct CprRow {
    double p[3], d[3];
};

// (float)((p + x * dir) / n) in double, operation for operation as nvcc
// compiles core/kernel.cu:860-862 (the multiply-add fused; the CPR parity
// tests compare every pixel with MonkeyGL's kernel).
__device__ __forceinline__ float cpr_coord_d(double p, double d, int x, float n) {
    return __double2float_rn(__ddiv_rn(__fma_rn((double)x, d, p), (double)n));
}

__global__ void __launch_bounds__(256) k_cpr(int W, int H, float3 fdim, int invertZ,
                                             const CprRow *__restrict__ rows,
                                             cudaTextureObject_t tex, short *out) {
    __shared__ CprRow s_rows[8];
    const int ly = threadIdx.x >> 5;
    const int y = blockIdx.y * 8 + ly;
    if ((threadIdx.x & 31) == 0 && y < H) s_rows[ly] = rows[y];
    __syncthreads();
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    if (x >= W || y >= H) return;
    const CprRow &R = s_rows[ly];
    const float fx = cpr_coord_d(R.p[0], R.d[0], x, fdim.x);
    const float fy = cpr_coord_d(R.p[1], R.d[1], x, fdim.y);
    float fz = cpr_coord_d(R.p[2], R.d[2], x, fdim.z);
    // "fz = 1.0 - fz" in double, then rounded to float: the float
    // subtraction rounds the same exact difference once
    if (!invertZ) fz = 1.0f - fz;
    short r;
    if (fx < 0 || fx > 1 || fy < 0 || fy > 1 || fz < 0 || fz > 1) r = -2048;
    else r = f2s_sat(32768 * tex3D<float>(tex, fx, fy, fz));
    out[(size_t)y * W + x] = r;
}

int fill_plane_params(const VolumeState &v, const mk_plane_params *p, PlaneParams &P) {
    if (!p || p->width <= 0 || p->height <= 0 || p->width > 32768 || p->height > 32768) {
        set_last_error("mk_render_plane: plane size must be in [1, 32768]");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (p->mpr_type < MK_MPR_AVERAGE || p->mpr_type > MK_MPR_MINIP ||
        (p->sampling != MK_SAMPLE_LINEAR && p->sampling != MK_SAMPLE_NEAREST)) {
        set_last_error("mk_render_plane: unknown MPR type or sampling");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (!(p->half_num >= 0.0f) || p->half_num > 4096.0f) {
        set_last_error("mk_render_plane: half_num must be in [0, 4096]");
        return MK_ERR_INVALID_ARGUMENT;
    }
    P.W = p->width;
    P.H = p->height;
    for (int k = 0; k < 3; ++k) {
        P.sp[k] = p->spacing[k];
        P.fdim[k] = (float)v.dims[k];
        P.h[k] = p->dir_h[k];
        P.v[k] = p->dir_v[k];
        P.n[k] = p->dir_n[k];
        P.lt[k] = p->left_top[k];
    }
    P.ps = p->pixel_spacing;
    P.invertZ = p->invert_z ? 1 : 0;
    P.halfNum = p->half_num;
    P.mode = p->mpr_type;
    P.voi_lut = nullptr;
    return MK_OK;
}

// The display window MonkeyGL's HTML client applies to an int16 plane:
// decodeMPR (examples/html/js/utils.js:62-118) hands window width 400 and
// centre 40 to cornerstone 0.12.2, whose generateLut
// (examples/html/js/libs/cornerstone@0.12.2.js:688-733) evaluates
// ((x - wc) / ww + 0.5) * 255 in double for every stored value x and keeps it
// in a Uint8ClampedArray: NaN and values <= 0 give 0, values >= 255 give 255,
// the rest round to nearest with ties to even.
uint8_t voi_window_u8(int x, double ww, double wc) {
    const double v = (((double)x - wc) / ww + 0.5) * 255.0;
    if (!(v > 0.0)) return 0;
    if (v >= 255.0) return 255;
    const double f = floor(v);
    if (f + 0.5 < v) return (uint8_t)(f + 1.0);
    if (v < f + 0.5) return (uint8_t)f;
    return (uint8_t)((((long)f) & 1) ? f + 1.0 : f);
}

// The table of that window for every int16 value, on the device: rebuilt
// when (ww, wl) changes, after the launches that read the old one.
static int voi_table(VolumeState &v, float ww, float wl, cudaStream_t s, const uint8_t **out) {
    if (!v.d_voi_lut) {
        MK_CUDA_TRY(cudaEventCreateWithFlags(&v.voi_ready, cudaEventDisableTiming));
        MK_CUDA_TRY(cudaMalloc(&v.d_voi_lut, 65536));
        v.device_bytes += 65536;
        v.voi_valid = false;
    }
    if (v.voi_valid && v.voi_key[0] == ww && v.voi_key[1] == wl) {
        MK_CUDA_TRY(cudaStreamWaitEvent(s, v.voi_ready, 0));
        *out = v.d_voi_lut;
        return MK_OK;
    }
    int rc = wait_table_uses(v.voi_uses);
    if (rc != MK_OK) return rc;
    std::vector<uint8_t> h(65536);
    for (int i = 0; i < 65536; ++i) h[i] = voi_window_u8(i - 32768, (double)ww, (double)wl);
    v.voi_valid = false;
    // pageable source: the call returns once `h` is staged
    MK_CUDA_TRY(cudaMemcpyAsync(v.d_voi_lut, h.data(), 65536, cudaMemcpyHostToDevice, s));
    MK_CUDA_TRY(cudaEventRecord(v.voi_ready, s));
    v.voi_key[0] = ww;
    v.voi_key[1] = wl;
    v.voi_valid = true;
    *out = v.d_voi_lut;
    return MK_OK;
}

template <bool U8>
static void launch_plane(const PlaneParams &P, cudaTextureObject_t tex, void *out, cudaStream_t s) {
    dim3 grid((P.W + 31) / 32, (P.H + 7) / 8);
    if (P.mode == MK_MPR_AVERAGE) k_plane<MK_MPR_AVERAGE, U8><<<grid, 256, 0, s>>>(P, tex, out);
    else if (P.mode == MK_MPR_MIP) k_plane<MK_MPR_MIP, U8><<<grid, 256, 0, s>>>(P, tex, out);
    else k_plane<MK_MPR_MINIP, U8><<<grid, 256, 0, s>>>(P, tex, out);
}

}  // namespace mk

using namespace mk;

extern "C" int mk_render_plane(mk_volume vol, const mk_plane_params *params, int16_t *out,
                               int out_on_device, void *stream) {
    if (!vol || !out) {
        set_last_error("mk_render_plane: null volume or output");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &v = vol->st;
    PlaneParams P;
    int rc = fill_plane_params(v, params, P);
    if (rc != MK_OK) return rc;
    cudaSetDevice(v.device);
    cudaStream_t s = stream ? (cudaStream_t)stream : v.stream;
    const size_t bytes = (size_t)P.W * P.H * sizeof(short);
    void *dst = out;
    if (!out_on_device) {
        rc = ensure_device_buffer(&v, bytes);
        if (rc != MK_OK) return rc;
        dst = v.d_out;
    }
    const cudaTextureObject_t tex = params->sampling == MK_SAMPLE_NEAREST ? v.tex_point : v.tex_linear;
    launch_plane<false>(P, tex, dst, s);
    MK_CUDA_TRY(cudaGetLastError());
    return finish_output(&v, out, bytes, out_on_device, s);
}

extern "C" int mk_render_plane_u8(mk_volume vol, const mk_plane_params *params, float ww, float wl,
                                  uint8_t *out, int out_on_device, void *stream) {
    if (!vol || !out || !(ww > 0.0f)) {
        set_last_error("mk_render_plane_u8: null volume/output or ww <= 0");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &v = vol->st;
    PlaneParams P;
    int rc = fill_plane_params(v, params, P);
    if (rc != MK_OK) return rc;
    cudaSetDevice(v.device);
    cudaStream_t s = stream ? (cudaStream_t)stream : v.stream;
    rc = voi_table(v, ww, wl, s, &P.voi_lut);
    if (rc != MK_OK) return rc;
    const size_t bytes = (size_t)P.W * P.H;
    void *dst = out;
    if (!out_on_device) {
        rc = ensure_device_buffer(&v, bytes);
        if (rc != MK_OK) return rc;
        dst = v.d_out;
    }
    const cudaTextureObject_t tex = params->sampling == MK_SAMPLE_NEAREST ? v.tex_point : v.tex_linear;
    launch_plane<true>(P, tex, dst, s);
    MK_CUDA_TRY(cudaGetLastError());
    rc = note_table_use(v.voi_uses, s);
    if (rc != MK_OK) return rc;
    return finish_output(&v, out, bytes, out_on_device, s);
}

extern "C" int mk_render_cpr(mk_volume vol, int width, int height, const double *points,
                             const double *dirs, int invert_z, int16_t *out, int out_on_device,
                             void *stream) {
    if (!vol || !out || !points || !dirs || width <= 0 || height <= 0 || width > 32768 ||
        height > 32768) {
        set_last_error("mk_render_cpr: bad arguments");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &v = vol->st;
    cudaSetDevice(v.device);
    cudaStream_t s = stream ? (cudaStream_t)stream : v.stream;
    std::vector<CprRow> rows(height);
    for (int y = 0; y < height; ++y) {
        for (int k = 0; k < 3; ++k) {
            rows[y].p[k] = points[3 * y + k];
            rows[y].d[k] = dirs[3 * y + k];
        }
    }
    const size_t out_bytes = (size_t)width * height * sizeof(short);
    const size_t row_bytes = (size_t)height * sizeof(CprRow);
    const size_t row_off = (out_bytes + 255) & ~(size_t)255;
    int rc = ensure_device_buffer(&v, row_off + row_bytes);
    if (rc != MK_OK) return rc;
    CprRow *d_rows = reinterpret_cast<CprRow *>(static_cast<char *>(v.d_out) + row_off);
    rc = ensure_pinned_buffer(&v, row_bytes);
    if (rc != MK_OK) return rc;
    memcpy(v.h_pinned, rows.data(), row_bytes);
    MK_CUDA_TRY(cudaMemcpyAsync(d_rows, v.h_pinned, row_bytes, cudaMemcpyHostToDevice, s));
    short *dst = out_on_device ? out : static_cast<short *>(v.d_out);
    dim3 grid((width + 31) / 32, (height + 7) / 8);
    const float3 fdim = make_float3((float)v.dims[0], (float)v.dims[1], (float)v.dims[2]);
    k_cpr<<<grid, 256, 0, s>>>(width, height, fdim, invert_z ? 1 : 0, d_rows, v.tex_linear, dst);
    MK_CUDA_TRY(cudaGetLastError());
    if (out_on_device) {
        // the row table in the staging buffer must outlive the kernel
        MK_CUDA_TRY(cudaStreamSynchronize(s));
        return MK_OK;
    }
    return finish_output(&v, out, out_bytes, 0, s);
}

// ---------------------------------------------------------------------------
// CPR without allocation.
//
// Some callers cannot call cudaMalloc: hosts that hand the GPU a fixed,
// pre-planned memory budget (certified medical viewers, embedded consoles),
// frameworks whose own caching allocator has reserved the device memory, and
// render loops that must not stall on the device-wide synchronisation that
// cudaMalloc/cudaFree can imply.  mk_render_cpr_noalloc serves them: the
// caller passes the path (host doubles) and a device output buffer, and the
// per-row table the kernel reads lives in the fixed array below, which every
// GPU that loads this library holds until the process exits.
constexpr int kNoAllocCprRows = 4096;   // 4096 rows x 48 B = 192 KiB
static __device__ __align__(256) CprRow g_noalloc_cpr_rows[kNoAllocCprRows];

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;                         // guards the two tables below
void *g_noalloc_rows_dev[kNoAllocMaxDevices] = {};  // device address of the array, per device
CprRow g_noalloc_rows_host[kNoAllocCprRows];        // host staging of one call's rows
}  // namespace

extern "C" int mk_render_cpr_noalloc(mk_volume vol, int width, int height, const double *points,
                                     const double *dirs, int invert_z, int16_t *out_device,
                                     void *stream) {
    if (!vol || !out_device || !points || !dirs || width <= 0 || width > 32768 || height <= 0) {
        set_last_error("mk_render_cpr_noalloc: bad arguments");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (height > kNoAllocCprRows) {
        set_last_error("mk_render_cpr_noalloc: height " + std::to_string(height) +
                       " exceeds its fixed table of " + std::to_string(kNoAllocCprRows) + " rows");
        return MK_ERR_INVALID_ARGUMENT;
    }
    VolumeState &v = vol->st;
    if (v.device < 0 || v.device >= kNoAllocMaxDevices) {
        set_last_error("mk_render_cpr_noalloc: device index beyond the per-device table");
        return MK_ERR_INVALID_ARGUMENT;
    }
    MK_CUDA_TRY(cudaSetDevice(v.device));
    cudaStream_t s = stream ? (cudaStream_t)stream : v.stream;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    // first call on this device: look up the array's device address (the
    // host-side name of a __device__ variable is not a device pointer).  The
    // address belongs to the device's current context and is kept for the
    // life of the process; a device reset (cudaDeviceReset) ends that context
    // together with every volume created in it, and this entry point is not
    // to be called on that device after a reset.
    if (!g_noalloc_rows_dev[v.device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_cpr_rows);
        if (e != cudaSuccess || !ptr) {
            set_last_error(std::string("mk_render_cpr_noalloc: cudaGetSymbolAddress: ") +
                           cudaGetErrorString(e));
            return MK_ERR_CUDA;
        }
        g_noalloc_rows_dev[v.device] = ptr;
    }
    CprRow *d_rows = static_cast<CprRow *>(g_noalloc_rows_dev[v.device]);
    for (int y = 0; y < height; ++y) {
        for (int k = 0; k < 3; ++k) {
            CprRow &r = g_noalloc_rows_host[y];
            r.p[k] = points[3 * y + k];
            r.d[k] = dirs[3 * y + k];
        }
    }
    // pageable source: the call returns once the rows are staged, so the host
    // table may be refilled by the next call
    MK_CUDA_TRY(cudaMemcpyAsync(d_rows, g_noalloc_rows_host, (size_t)height * sizeof(CprRow),
                                cudaMemcpyHostToDevice, s));
    dim3 grid((width + 31) / 32, (height + 7) / 8);
    const float3 fdim = make_float3((float)v.dims[0], (float)v.dims[1], (float)v.dims[2]);
    k_cpr<<<grid, 256, 0, s>>>(width, height, fdim, invert_z ? 1 : 0, d_rows, v.tex_linear, out_device);
    MK_CUDA_TRY(cudaGetLastError());
    return MK_OK;
}
