/*
 * monkeygl_b200.h -- C ABI of the B200 (sm_100a) volume ray-casting library.
 *
 * This is the seam between host code (the C++ HelloMonkey/IRender API, the
 * pyMonkeyGL module, ctypes callers) and the hand-written CUDA kernels.  Every
 * entry point takes plain pointers, sizes and POD structs; nothing here needs
 * CUDA or torch headers.  Each declaration names the MonkeyGL interface it
 * replaces (paths relative to the MonkeyGL source tree).
 *
 * Conventions
 *   - Every function returns an mk_status (0 = MK_OK).  No entry point exits
 *     the process; CUDA errors come back as MK_ERR_CUDA and the text of the
 *     last error is available from mk_last_error().
 *   - Volumes are x-fastest int16 arrays (dim_x * dim_y * dim_z), exactly the
 *     buffer MonkeyGL's SetVolumeData takes (core/VolumeInfo.cpp:78-91).
 *   - `stream` is a cudaStream_t passed as void* (NULL = the library's own
 *     per-volume stream).  Calls with host output pointers are synchronous with
 *     respect to that stream; calls with device output pointers are
 *     asynchronous.
 *   - Outputs are caller-owned.  The library allocates device memory only at
 *     volume creation and when an output larger than any before is requested.
 */
#ifndef MONKEYGL_B200_H
#define MONKEYGL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Labels 0..64: MAXOBJECTCOUNT + 1 (core/Defines.h:34). */
#define MK_MAX_LABELS 65

typedef enum mk_status {
    MK_OK = 0,
    MK_ERR_INVALID_ARGUMENT = 1,
    MK_ERR_CUDA = 2,
    MK_ERR_OUT_OF_MEMORY = 3,
    MK_ERR_NOT_READY = 4,
    MK_ERR_BUDGET = 5,
    MK_ERR_TIMEOUT = 6,
    MK_ERR_NO_DEVICE = 7,
    MK_ERR_QUEUE_FULL = 8
} mk_status;

/* RenderType (core/Defines.h:224-230). */
typedef enum mk_render_type {
    MK_RENDER_VR = 0,
    MK_RENDER_MIP = 1,
    MK_RENDER_SURFACE = 2
} mk_render_type;

/* MPRType (core/Defines.h:216-222). */
typedef enum mk_mpr_type {
    MK_MPR_AVERAGE = 0,
    MK_MPR_MIP = 1,
    MK_MPR_MINIP = 2
} mk_mpr_type;

/* Volume sampling for planes.  MonkeyGL only has LINEAR (its texture is
 * created with cudaFilterModeLinear, core/CuDataManager.cu:64); NEAREST is the
 * same reslice read through a point-filtered view of the same voxels. */
typedef enum mk_sampling {
    MK_SAMPLE_LINEAR = 0,
    MK_SAMPLE_NEAREST = 1
} mk_sampling;

/* VR output pixel layout.  MonkeyGL returns 3 bytes per pixel, R,G,B
 * (core/kernel.cu:258-262); RGBA8 is the same colour with A = 255. */
typedef enum mk_pixel_format {
    MK_PIXEL_RGB8 = 0,
    MK_PIXEL_RGBA8 = 1
} mk_pixel_format;

/* mk_vr_params.flags */
#define MK_VR_NO_SKIP 0x1 /* march every reference sample (no empty-space skipping) */
#define MK_VR_NO_COOP 0x2 /* VR: one lane per ray to the end (no cooperative tail, no tail launch; same image) */
#define MK_VR_NO_TAIL 0x4 /* VR: no tail launch (rays finish in the tile launch; same image) */

typedef struct mk_volume_s *mk_volume;

/*
 * Ray-casting parameters: the scalar arguments of MonkeyGL's cu_render
 * (core/kernel.cu:471-492), in the same meaning and units.
 */
typedef struct mk_vr_params {
    int width;
    int height;
    int render_type;             /* mk_render_type */
    float max_len_spacing[3];    /* f3maxLenSpacing (core/DataManager.h:201-216) */
    float spacing[3];            /* f3Spacing */
    float spacing_voxel[3];      /* f3SpacingVoxel = 1/dim */
    float x_translate;           /* RenderInfo total pan, pixels */
    float y_translate;
    float scale;                 /* RenderInfo total zoom */
    float transform[9];          /* row-major 3x3 camera matrix (float3x3 m[3]) */
    int invert_z;
    int voi[6];                  /* left, right, posterior, anterior, head, foot */
    float background[4];         /* RGBA background, used only where nothing composited */
    int pixel_format;            /* mk_pixel_format */
    int flags;                   /* MK_VR_* */
} mk_vr_params;

/*
 * MPR parameters: the arguments of cu_renderPlane_{Average,MIP,MinIP}
 * (core/kernel.cu:616-631, 706-721, 795-810), plus the reslice mode.
 */
typedef struct mk_plane_params {
    int width;
    int height;
    int mpr_type;                /* mk_mpr_type */
    int sampling;                /* mk_sampling */
    float spacing[3];            /* voxel spacing, mm */
    float dir_h[3];              /* unit row direction */
    float dir_v[3];              /* unit column direction */
    float dir_n[3];              /* unit slab normal */
    float left_top[3];           /* plane corner, mm from the volume corner */
    float pixel_spacing;         /* mm per output pixel */
    int invert_z;
    float half_num;              /* slab half width in samples: (n - 1) / 2 */
} mk_plane_params;

/* ------------------------------------------------------------------ */
/* Library / device                                                    */
/* ------------------------------------------------------------------ */

/* Text for a status code. */
const char *mk_status_string(int status);
/* Text of the last error recorded on the calling thread ("" if none). */
const char *mk_last_error(void);
/* Number of visible CUDA devices (0 when none).  Replaces DeviceInfo::GetCount
 * (core/DeviceInfo.cpp:91-97). */
int mk_device_count(int *count);
/* Library version string, "major.minor.patch". */
const char *mk_version(void);

/* ------------------------------------------------------------------ */
/* Volume residency                                                    */
/* ------------------------------------------------------------------ */

/*
 * Upload an int16 volume to `device` and build its brick occupancy map.
 * Replaces cu_copyVolumeData (core/CuDataManager.cu:28-73).  The host buffer
 * may be freed after the call returns.  A volume handle is used from one host
 * thread at a time (its per-frame caches -- tile orders, ray parameter
 * tables, hand-off lists -- are not locked); concurrent renders of one volume
 * go through several streams from that thread, or through mk_server_*.
 * The brick maps are built by kernels whose waits are bounded: a wait that
 * runs out (never expected) is reported as MK_ERR_TIMEOUT and no volume is
 * returned.
 */
int mk_volume_create(mk_volume *out, const int16_t *voxels, int dim_x, int dim_y,
                     int dim_z, int device);
/* Release every device resource of the volume. */
int mk_volume_destroy(mk_volume vol);
/* Device bytes held by the volume (textures, maps, buffers). */
int mk_volume_device_bytes(mk_volume vol, size_t *bytes);
/* Dimensions of the volume. */
int mk_volume_dims(mk_volume vol, int *dim_x, int *dim_y, int *dim_z);

/*
 * Introspection of the occupancy maps built at upload (no counterpart in
 * MonkeyGL, which has none): nb = bricks along x, y, z (8^3 voxels each,
 * numbered x fastest); minmax = 2 int16 per brick, the minimum and maximum
 * voxel of the brick grown by one voxel on every side (clamped to the
 * volume); labels = 3 words per brick, bit l set when label l (0..64)
 * occurs among the brick's own voxels; present = 2 words, the labels
 * occurring anywhere.  Any output pointer may be NULL; host memory.
 */
int mk_volume_brick_maps(mk_volume vol, int *nb, int16_t *minmax, uint32_t *labels, uint64_t *present);

/*
 * Upload (labels != NULL) or remove (labels == NULL) the uint8 label volume,
 * same dims and layout as the voxels.  Replaces cu_copyMaskData
 * (core/CuDataManager.cu:75-120).  MK_ERR_TIMEOUT as for mk_volume_create
 * (the label sets' bounded waits); the volume then has no mask.
 */
int mk_volume_set_mask(mk_volume vol, const uint8_t *labels);

/*
 * Incremental form of mk_volume_set_mask for a mask that changed only inside
 * box = {x0, y0, z0, x1, y1, z1} (voxels x0 <= x < x1 etc.): `labels` is the
 * whole updated uint8 label volume (same dims and layout), of which only the
 * box, widened to whole 8^3 bricks, is copied to the device and re-bricked.
 * MonkeyGL re-uploads the whole mask on every object added or updated
 * (DataManager.cpp:280-335, CuDataManager.cu:75-120).  The volume must have
 * a mask already (MK_ERR_INVALID_ARGUMENT otherwise); labels that the update
 * removed everywhere stay listed as present (the per-ray state they size is
 * then larger than needed, never smaller).
 */
int mk_volume_update_mask(mk_volume vol, const uint8_t *labels, const int box[6]);

/*
 * Set the RGBA lookup table of one label: `n_entries` float4 (r,g,b,a) in
 * [0,1], filtered linearly over t in [0,1] with entry centres at (i+0.5)/n.
 * Replaces cu_setTransferFunc (core/CuDataManager.cu:122-163).  A label with
 * no table renders as fully transparent.
 */
int mk_volume_set_transfer_function(mk_volume vol, int label, const float *rgba,
                                    int n_entries);

/*
 * Per-label opacity cap, window width and window level: `n_labels` rows of
 * (alpha, ww, wl).  Replaces the AlphaAndWWWLInfo argument of cu_render
 * (core/Defines.h:123-149, core/DataManager.cpp:602-611).  ww must be > 0.
 */
int mk_volume_set_label_params(mk_volume vol, const float *alpha_ww_wl, int n_labels);

/* ------------------------------------------------------------------ */
/* Rendering                                                           */
/* ------------------------------------------------------------------ */

/*
 * Ray-cast the volume (VR, MIP or first-hit surface) into an image of
 * width*height pixels, 3 (RGB8) or 4 (RGBA8) bytes each, row-major.
 * Replaces cu_render (core/kernel.cu:471-568).  `out` is host memory when
 * out_on_device == 0 (the call then returns with the image in `out`), else a
 * device pointer (the call returns after queuing the work on `stream`).
 * A VR frame is two launches on `stream`: the tiles, then the rays still
 * marching when all but a few tiles have finished (MK_VR_NO_TAIL: one
 * launch).  The hand-off list is kept per volume and stream (four streams;
 * created on a stream's first frame, grown for larger frames).
 */
int mk_render_vr(mk_volume vol, const mk_vr_params *params, void *out,
                 int out_on_device, void *stream);

/*
 * Count the samples of MonkeyGL's own ray schedule for this frame (positions
 * inside the volume where its d_render/d_renderMIP/d_renderSurface would
 * fetch a voxel, core/kernel.cu:195-252, 311-349, 413-453).  This is the unit
 * of the Gsamples/s figure; it does not render.
 */
int mk_count_vr_samples(mk_volume vol, const mk_vr_params *params, uint64_t *samples);

/*
 * Measurement pass over the same schedule as mk_count_vr_samples: besides the
 * sample count, the number of distinct int16 voxels inside the trilinear
 * footprints of every fetch (value and gradient taps) and of distinct label
 * voxels read.  These give the algorithmic bytes of a frame
 * (2 * voxels + label_voxels + output bytes).  Allocates two temporary bitsets
 * of one bit per voxel; does not render.
 */
int mk_count_vr_footprint(mk_volume vol, const mk_vr_params *params, uint64_t *samples,
                          uint64_t *voxels, uint64_t *label_voxels);

/*
 * Reslice a plane (MPR) into width*height int16 values.  Replaces
 * cu_renderPlane_{Average,MIP,MinIP} (core/kernel.cu:570-837).
 */
int mk_render_plane(mk_volume vol, const mk_plane_params *params, int16_t *out,
                    int out_on_device, void *stream);

/*
 * Optional display epilogue for planes: the int16 plane of mk_render_plane
 * windowed into uint8 exactly as MonkeyGL's HTML client displays it.  Its
 * decodeMPR (examples/html/js/utils.js:62-118) hands ww 400 / wl 40 to
 * cornerstone 0.12.2, which maps every value x to
 * ((x - wl) / ww + 0.5) * 255 in double precision, clamped to [0, 255] and
 * rounded to nearest with ties to even (a Uint8ClampedArray store,
 * examples/html/js/libs/cornerstone@0.12.2.js:688-733).  The library builds
 * that table for all 65536 int16 values on the host (64 KB of device memory
 * per volume, allocated on the first call, rebuilt when ww or wl changes).
 */
int mk_render_plane_u8(mk_volume vol, const mk_plane_params *params, float ww, float wl,
                       uint8_t *out, int out_on_device, void *stream);

/*
 * Curved planar reformation: row y samples points[y] + x * dirs[y] (voxel
 * units, x = 0..width-1); out-of-volume pixels are -2048.  `points` and
 * `dirs` are height*3 doubles each, as built by CPRInfo (core/CPRInfo.cpp:81-160).
 * Replaces cu_renderCPR (core/kernel.cu:839-918).
 */
int mk_render_cpr(mk_volume vol, int width, int height, const double *points,
                  const double *dirs, int invert_z, int16_t *out, int out_on_device,
                  void *stream);

/* ------------------------------------------------------------------ */
/* Differentiable volume rendering (no counterpart in MonkeyGL)        */
/* ------------------------------------------------------------------ */

/*
 * MonkeyGL's orthographic VR camera (the pixel -> ray mapping of
 * core/kernel.cu:161-206) with a differentiable method: fixed step, float32
 * volume in [0,1] (x-fastest, dims[0]*dims[1]*dims[2], fewer than 2^31
 * voxels) sampled with exact trilinear weights (texel centres at
 * (i+0.5)/dim, clamp to edge), the value used directly as the LUT coordinate
 * (lut_len float4 entries, entry i centred at (i+0.5)/lut_len, linear,
 * clamp), front-to-back compositing stopped after the sample that takes
 * transmittance below t_min.  All pointers are device pointers; calls are
 * asynchronous on `stream`.
 */
typedef struct mk_dvr_params {
    int width;
    int height;
    int dims[3];
    float max_len_spacing[3];
    float transform[9];
    float scale;
    float x_translate;
    float y_translate;
    float step;                  /* in MonkeyGL's ray parameter: 1/dim_z is one voxel of the longest axis */
    float t_min;                 /* early termination threshold on transmittance (0 = never) */
    int lut_len;                 /* 2..1024 */
} mk_dvr_params;

/* A call renders `nviews` views (any number; one launch per 32).  The views
 * share width, height, dims and lut_len; the camera, spacing, scale,
 * translation, step and t_min are per view. */

/* Floats of workspace mk_dvr_forward needs to support a backward pass
 * (per-ray transmittance checkpoints and sample counts). */
int mk_dvr_workspace_floats(const mk_dvr_params *views, int nviews, size_t *floats);

/* images: nviews*height*width*3 floats (RGB); transmittance:
 * nviews*height*width floats; workspace: mk_dvr_workspace_floats floats, or
 * NULL for inference only. */
int mk_dvr_forward(const mk_dvr_params *views, int nviews, const float *volume, const float *lut,
                   float *images, float *transmittance, float *workspace, void *stream);

/* Accumulates (adds) dL/dLUT into grad_lut (lut_len*4 floats) and, when
 * grad_volume is not NULL, dL/dvolume into grad_volume (dims floats, x
 * fastest), given grad_images = dL/dimages and the workspace of the matching
 * forward call. */
int mk_dvr_backward(const mk_dvr_params *views, int nviews, const float *volume, const float *lut,
                    const float *workspace, const float *grad_images, float *grad_lut,
                    float *grad_volume, void *stream);

/*
 * mk_render_cpr without any device allocation.  It has no counterpart in
 * MonkeyGL: it is for callers that cannot call cudaMalloc (a host with a
 * fixed, pre-planned device-memory budget, a framework whose caching
 * allocator already holds the memory, a render loop that must not stall on
 * the synchronisation cudaMalloc/cudaFree can imply).  Same rows, pixels and
 * fill value as mk_render_cpr; the caller provides the device output buffer
 * (width*height int16) and the path as host doubles.
 *   - The per-row table lives in a fixed device array of 4096 rows (192 KiB)
 *     that every GPU loading this library holds until the process exits;
 *     height > 4096 is rejected with MK_ERR_INVALID_ARGUMENT and a message.
 *   - The first call on a device looks up that array's device address.  The
 *     address is kept until the process exits, so the call is not for use on
 *     a device after a cudaDeviceReset in the same process.
 *   - The rows reach the device by a copy from one process-wide host table,
 *     so the call must not be recorded under stream capture: a replayed
 *     graph would copy whatever rows the latest call left there.
 *   - The call is asynchronous on `stream` (NULL = the volume's stream).
 *     Every call shares the one array (each call overwrites the rows it
 *     uses; nothing needs to start at zero), so calls that overlap on the
 *     GPU, e.g. on two streams, race; calls on one stream are ordered.
 *   - It calls no cudaMalloc, cudaFree or other allocating routine.
 */
int mk_render_cpr_noalloc(mk_volume vol, int width, int height, const double *points,
                          const double *dirs, int invert_z, int16_t *out_device, void *stream);

/* Wait for all work queued on `stream` (NULL = the volume's stream). */
int mk_volume_synchronize(mk_volume vol, void *stream);

/* ------------------------------------------------------------------ */
/* VR image overlays (host)                                            */
/* ------------------------------------------------------------------ */

/* The orientation mesh: a binary STL, centred, scaled by the larger of its
 * x and z extents and mirrored in z, as MonkeyGL's MarchingCube loads
 * ./resources/human.stl (core/MarchingCube.cpp:305-354).  MK_ERR_INVALID_ARGUMENT
 * for a missing, short or truncated file. */
typedef struct mk_mesh_s *mk_mesh;
int mk_mesh_load_stl(const char *path, mk_mesh *out);
int mk_mesh_destroy(mk_mesh mesh);
int mk_mesh_facet_count(mk_mesh mesh);

/* VRImageLayer::MergeOrientationBox (core/VRImageLayer.cpp:99-194): the mesh,
 * turned by the camera's 3x3 rotation (RenderInfo's rotate matrix, row-major),
 * flat-shaded and z-buffered on a 512x512 raster, drawn every 8th pixel into
 * the bottom-right 64x64 pixels of an RGB8 image (colour (0.902, 0.902,
 * 0.302) * shade + 0.05).  Nothing is drawn when either side is <= 64.
 * Host memory; pixels equal MonkeyGL's. */
int mk_merge_orientation_box(mk_mesh mesh, const float rotate[9], uint8_t *rgb, int width, int height);

/* Methods::DrawLineInImage24Bit (core/Methods.cpp:183-200): a line of
 * `line_width` parallel strokes, one dot every half pixel, in colour
 * (r, g, b) in [0, 1]; the CPR line layer draws the projected CPR path with
 * it (core/CPRLineLayer.cpp:40-65).  Host memory. */
int mk_draw_line_rgb(uint8_t *rgb, int width, int height, float x0, float y0, float x1, float y1,
                     int line_width, const float color[3]);

/* PNG + Base64, the output form of MonkeyGL's GetVRData_pngString and
 * GetPlaneData_pngString (core/HelloMonkey.cpp:212-259, 333-413, which use
 * fpng): an 8-bit PNG of `channels` = 3 (RGB) or 4 (RGBA; MonkeyGL packs an
 * int16 plane of width W as W/2 RGBA pixels) compressed in parallel row
 * bands, then Base64, NUL-terminated, into `out` (`capacity` bytes, at least
 * mk_encoded_capacity).  The decoded pixels equal the input; the bytes are
 * not fpng's. */
int mk_encoded_capacity(int width, int height, int channels, size_t *bytes);
int mk_encode_png_base64(const uint8_t *pixels, int width, int height, int channels, char *out,
                         size_t capacity, size_t *length);

/* Text annotations (core/AnnotationLayer.cpp:41-61 ->
 * AnnotationUtils::Textout2Image, core/AnnotationUtils.cpp:419-458).  The
 * glyph masks are loaded from a glyph file ("MKGLYPH1": uint32 count, then per
 * glyph uint8 font size 0..2, uint8 key length, the key bytes, uint16 width,
 * uint16 height, width*height mask bytes); MonkeyGL's own masks are
 * extracted into such a file by the oracle build (oracle/make_glyphs.py).
 * The text is drawn byte by byte: a byte without a glyph moves the pen back
 * one pixel and draws nothing; mask m > 0 sets each channel to the truncated
 * m * colour; format 0 left, 1 right, 2 centred on x (MonkeyGL's
 * AnnotationFormat); images below 10x10 are refused. */
typedef struct mk_font_s *mk_font;
int mk_font_load(const char *path, mk_font *out);
int mk_font_destroy(mk_font font);
/* AnnotationUtils::GetSize: total width (unknown bytes count -1) and the
 * height of the last glyph. */
int mk_text_size(mk_font font, const char *text, int font_size, int *width, int *height);
int mk_draw_text_rgb(mk_font font, uint8_t *rgb, int width, int height, const char *text, int x, int y,
                     int font_size, int format, const float color[3]);

/* ------------------------------------------------------------------ */
/* Serving: continuous batching of VR/MIP/MPR requests                 */
/* ------------------------------------------------------------------ */

/*
 * No counterpart in MonkeyGL, which serves one request at a time through a
 * process-wide singleton holding one volume (core/DataManager.cpp:46-54,
 * server.py).  A server keeps several volumes resident on one device,
 * admitted against an HBM budget, and renders requests for any of them:
 * requests take free slots (their LUTs, label parameters, brick visibility
 * and output buffer), and every step one persistent kernel, launched from a
 * CUDA graph, pulls 32x8-pixel tiles of all requests in flight from a device
 * work queue.  A request larger than one step's tile quota spans several
 * steps; requests arriving meanwhile join the next step.  Each request's
 * image is the one mk_render_vr / mk_render_plane produce for the same
 * volume, parameters and tables.  The calls are thread-safe.
 */
typedef struct mk_server_s *mk_server;

typedef struct mk_server_config {
    int device;
    size_t hbm_budget_bytes;     /* resident volumes + slot buffers; 0 = 90% of the free memory */
    int max_slots;               /* requests on the device at once, 1..256 */
    int max_pending;             /* requests waiting for a slot (>= 1); more are refused (MK_ERR_QUEUE_FULL) */
    int max_pixels;              /* largest image of a request (width * height) */
    int lut_len;                 /* entries of every LUT of a request, 2..4096 */
    int max_labels;              /* LUTs per request (labels 0..max_labels-1), 1..65 */
    int max_bricks;              /* largest volume, in 8^3 bricks; 0 = 512 x 512 x 2048 voxels */
    int tiles_per_step;          /* tiles of one batched launch; 0 = 8192 */
    int evict_idle;              /* 0: a volume over the budget is refused (MK_ERR_BUDGET).
                                    1: the server keeps a host copy of every volume; a volume that
                                    does not fit, or a request for a volume evicted earlier, makes
                                    room by evicting resident volumes that no admitted request
                                    uses (least recently used first, those with no queued request
                                    before those with one) and is uploaded on a loader thread
                                    while requests for resident volumes keep running */
} mk_server_config;

enum { MK_REQUEST_VR = 0, MK_REQUEST_MIP = 1, MK_REQUEST_SURFACE = 2, MK_REQUEST_MPR = 3 };

typedef struct mk_request {
    int volume;                  /* id returned by mk_server_add_volume */
    int kind;                    /* MK_REQUEST_* */
    mk_vr_params vr;             /* ray casting (render_type is taken from kind) */
    mk_plane_params plane;       /* MPR */
    const float *luts;           /* n_luts tables of lut_len RGBA floats for labels 0..n_luts-1 */
    int n_luts;                  /* 0..max_labels; labels without a table are transparent */
    const float *label_params;   /* n_luts rows of (alpha, ww, wl), ww > 0; others (0, 1, 0) */
    void *out;                   /* host image: W*H*3 (RGB8) or *4 (RGBA8) bytes, W*H int16 for MPR */
    char *encoded;               /* optional (NULL: none): also the image as MonkeyGL's *_pngString form,
                                    a NUL-terminated Base64 PNG (mk_encode_png_base64; an MPR plane as
                                    W/2 RGBA pixels, W even), written by the server's encoder thread
                                    while later steps run; mk_server_wait returns once it is written */
    size_t encoded_capacity;     /* bytes at `encoded`: at least mk_encoded_capacity of the image */
} mk_request;

typedef struct mk_request_times {
    double submitted_ms;         /* on the server's clock (ms since mk_server_create) */
    double started_ms;           /* first step holding its tiles was launched */
    double completed_ms;         /* image copied to `out` (and encoded, if asked for) */
    size_t encoded_length;       /* characters written to `encoded` (0: not asked for) */
} mk_request_times;

typedef struct mk_server_stats {
    uint64_t submitted, completed, rejected, steps, tiles;
    uint64_t evictions, loads;   /* volumes evicted / uploaded again (evict_idle) */
    size_t resident_bytes, budget_bytes;
    int volumes, slots_busy, pending;
} mk_server_stats;

int mk_server_create(const mk_server_config *config, mk_server *out);
/* Finish the work in flight, then release everything. */
int mk_server_destroy(mk_server srv);
/* Upload a volume (and its label volume, or NULL); MK_ERR_BUDGET when it does
 * not fit the budget beside the volumes already resident (with evict_idle:
 * only when it exceeds the budget on its own; otherwise idle volumes are
 * evicted, or it is registered evicted and uploaded on its first request). */
int mk_server_add_volume(mk_server srv, const int16_t *voxels, int dim_x, int dim_y, int dim_z,
                         const uint8_t *labels, int *volume_id);
/* MK_ERR_NOT_READY while requests for the volume are queued or in flight, or
 * while it is being uploaded. */
int mk_server_remove_volume(mk_server srv, int volume_id);
/* Queue a request (its tables are copied); MK_ERR_QUEUE_FULL when max_pending
 * requests already wait for a slot. */
int mk_server_submit(mk_server srv, const mk_request *req, uint64_t *ticket);
/* Wait up to timeout_ms (< 0: no limit) for a request.  MK_OK: the image is
 * in `out` and the ticket is released; MK_ERR_TIMEOUT: still running. */
int mk_server_wait(mk_server srv, uint64_t ticket, int timeout_ms, mk_request_times *times);
int mk_server_get_stats(mk_server srv, mk_server_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* MONKEYGL_B200_H */
