// Test infrastructure (oracle): a C-ABI harness around MonkeyGL's own CUDA
// code, built from the unmodified sources core/kernel.cu and
// core/CuDataManager.cu (see oracle/Makefile).  It lets the parity tests and
// the reference arm of bench.py drive MonkeyGL's kernels with plain pointers:
//
//   mkref_volume / mkref_mask / mkref_tf   -> cu_copyVolumeData, cu_copyMaskData,
//                                             cu_setTransferFunc (CuDataManager.cu:28-163)
//   mkref_render                           -> cu_render (kernel.cu:471-568)
//   mkref_plane                            -> cu_renderPlane_{Average,MIP,MinIP} (kernel.cu:616-837)
//   mkref_cpr                              -> cu_renderCPR (kernel.cu:875-918)
//   mkref_render_kernel_ms                 -> d_render/d_renderMIP/d_renderSurface timed alone
//
// Nearest-neighbour planes use the same cudaArray through a harness-built
// point-filtered texture; the reslice kernels take the texture as an argument
// (kernel.cu:574), so MonkeyGL's code stays unchanged.
//
// MonkeyGL's checkCudaErrors exits the process on a CUDA error; the harness
// validates its inputs first so that only genuine device failures reach it.
#include <cuda_runtime.h>
#include <string.h>

#include "CuDataManager.h"
#include "Defines.h"

using namespace MonkeyGL;

extern "C" void cu_copyVolumeData(short *h_volumeData, cudaExtent volumeSize, cudaArray *&d_volumeArray,
                                  cudaTextureObject_t &volumeTexture);
extern "C" void cu_copyMaskData(unsigned char *h_maskData, cudaExtent volumeSize, cudaArray *&d_maskArray,
                                cudaTextureObject_t &maskTexture);
extern "C" void cu_setTransferFunc(float *pTransferFunc, int nLenTransferFunc,
                                   cudaArray *&d_transferFuncArray,
                                   cudaTextureObject_t &transferFuncTexture);
extern "C" void cu_render(unsigned char *pVR, int width, int height, cudaTextureObject_t volumeTexture,
                          cudaExtent volumeSize, cudaTextureObject_t maskTexture,
                          cudaTextureObjects transferFuncTextures, AlphaAndWWWLInfo alphaAndWWWLInfo,
                          float3 f3maxLenSpacing, float3 f3Spacing, float3 f3SpacingVoxel,
                          float xTranslate, float yTranslate, float scale, float3x3 transformMatrix,
                          bool invertZ, VOI voi, RGBA colorBG, RenderType type);
extern "C" void cu_renderPlane_MIP(short *, int, int, cudaTextureObject_t, cudaExtent, float3, float3,
                                   float3, float3, float3, float, bool, float);
extern "C" void cu_renderPlane_MinIP(short *, int, int, cudaTextureObject_t, cudaExtent, float3, float3,
                                     float3, float3, float3, float, bool, float);
extern "C" void cu_renderPlane_Average(short *, int, int, cudaTextureObject_t, cudaExtent, float3,
                                       float3, float3, float3, float3, float, bool, float);
extern "C" void cu_renderCPR(short *, int, int, cudaTextureObject_t, cudaExtent, double *, double *,
                             bool);

// MonkeyGL's kernels (kernel.cu:133, 266, 366), launched directly for the
// kernel-only timing.
__global__ void d_render(unsigned char *, int, int, cudaTextureObject_t, cudaExtent, cudaTextureObject_t,
                         cudaTextureObjects, AlphaAndWWWLInfo, float3, float3, float3, float, float,
                         float, float3x3, bool, VOI, float4);
__global__ void d_renderMIP(unsigned char *, int, int, cudaTextureObject_t, cudaExtent,
                            cudaTextureObject_t, AlphaAndWWWLInfo, float3, float3, float3, float,
                            float, float, float3x3, bool, VOI, float4);
__global__ void d_renderSurface(unsigned char *, int, int, cudaTextureObject_t, cudaExtent,
                                cudaTextureObject_t, float3, float3, float3, float, float, float,
                                float3x3, bool, VOI, float4);

namespace {

struct RefState {
    cudaExtent ext = make_cudaExtent(0, 0, 0);
    cudaArray *vol = nullptr;
    cudaTextureObject_t tex = 0;
    cudaTextureObject_t tex_point = 0;
    cudaArray *mask = nullptr;
    cudaTextureObject_t mask_tex = 0;
    cudaArray *tf[MAXOBJECTCOUNT + 1] = {};
    cudaTextureObjects tfs;
};

// Several volumes can stay resident at once (the serving comparison runs
// MonkeyGL's launchers over the same resident volumes as the server);
// mkref_select chooses the one the other calls use.  MonkeyGL itself holds
// one volume per process.
constexpr int kRefSlots = 8;
RefState g_slots[kRefSlots];
RefState *g_cur = &g_slots[0];

}  // namespace

#define g (*g_cur)

extern "C" int mkref_select(int slot) {
    if (slot < 0 || slot >= kRefSlots) return 1;
    g_cur = &g_slots[slot];
    return 0;
}

// Flat VR parameter block (floats), in cu_render's argument order:
//  [0..2] maxLenSpacing, [3..5] spacing, [6..8] spacingVoxel, [9] xT, [10] yT,
//  [11] scale, [12..20] matrix rows, [21] invertZ, [22..27] VOI, [28..31] bg RGBA,
//  [32 + 3*l .. ] alpha, ww, wl of label l (65 labels)
#define MKREF_VR_FLOATS (32 + 3 * (MAXOBJECTCOUNT + 1))

extern "C" int mkref_vr_param_count(void) { return MKREF_VR_FLOATS; }

extern "C" int mkref_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" int mkref_volume(const short *vox, int w, int h, int d) {
    if (!vox || w <= 0 || h <= 0 || d <= 0) return 1;
    if (g.tex_point) {
        cudaDestroyTextureObject(g.tex_point);
        g.tex_point = 0;
    }
    g.ext = make_cudaExtent(w, h, d);
    cu_copyVolumeData(const_cast<short *>(vox), g.ext, g.vol, g.tex);
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = g.vol;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.normalizedCoords = true;
    td.filterMode = cudaFilterModePoint;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.readMode = cudaReadModeNormalizedFloat;
    return cudaCreateTextureObject(&g.tex_point, &rd, &td, nullptr) == cudaSuccess ? 0 : 2;
}

extern "C" int mkref_mask(const unsigned char *m) {
    if (!g.vol) return 1;
    if (!m) {
        if (g.mask) cudaFreeArray(g.mask);
        g.mask = nullptr;
        g.mask_tex = 0;
        return 0;
    }
    cu_copyMaskData(const_cast<unsigned char *>(m), g.ext, g.mask, g.mask_tex);
    return 0;
}

extern "C" int mkref_tf(int label, const float *rgba, int n) {
    if (label < 0 || label > MAXOBJECTCOUNT || !rgba || n <= 0) return 1;
    cudaTextureObject_t t = 0;
    cu_setTransferFunc(const_cast<float *>(rgba), n, g.tf[label], t);
    g.tfs.m[label] = t;
    return 0;
}

extern "C" int mkref_clear_tfs(void) {
    for (int l = 0; l <= MAXOBJECTCOUNT; ++l) g.tfs.m[l] = 0;
    return 0;
}

static void unpack_vr(const float *p, float3 &mls, float3 &sp, float3 &sv, float &xT, float &yT,
                      float &scale, float3x3 &M, bool &inv, VOI &voi, RGBA &bg, AlphaAndWWWLInfo &info) {
    mls = make_float3(p[0], p[1], p[2]);
    sp = make_float3(p[3], p[4], p[5]);
    sv = make_float3(p[6], p[7], p[8]);
    xT = p[9];
    yT = p[10];
    scale = p[11];
    for (int r = 0; r < 3; ++r) M.m[r] = make_float3(p[12 + 3 * r], p[13 + 3 * r], p[14 + 3 * r]);
    inv = p[21] != 0.0f;
    voi.left = (int)p[22];
    voi.right = (int)p[23];
    voi.posterior = (int)p[24];
    voi.anterior = (int)p[25];
    voi.head = (int)p[26];
    voi.foot = (int)p[27];
    bg = RGBA(p[28], p[29], p[30], p[31]);
    for (int l = 0; l <= MAXOBJECTCOUNT; ++l)
        info.m[l] = AlphaAndWWWL(p[32 + 3 * l], p[33 + 3 * l], p[34 + 3 * l]);
}

// cu_render: host output of w*h*3 bytes.
extern "C" int mkref_render(unsigned char *out, int w, int h, const float *p, int type) {
    if (!g.vol || !out || w <= 0 || h <= 0 || !p || type < 0 || type > 2) return 1;
    float3 mls, sp, sv;
    float xT, yT, scale;
    float3x3 M;
    bool inv;
    VOI voi;
    RGBA bg;
    AlphaAndWWWLInfo info;
    unpack_vr(p, mls, sp, sv, xT, yT, scale, M, inv, voi, bg, info);
    cu_render(out, w, h, g.tex, g.ext, g.mask_tex, g.tfs, info, mls, sp, sv, xT, yT, scale, M, inv, voi,
              bg, (RenderType)type);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// MonkeyGL's ray-casting kernel alone (its own 32x32 launch shape,
// kernel.cu:497-498), timed with CUDA events over `reps` launches into a
// device buffer; returns the mean milliseconds per launch (negative on error).
extern "C" double mkref_render_kernel_ms(int w, int h, const float *p, int type, int reps) {
    if (!g.vol || w <= 0 || h <= 0 || !p || reps <= 0) return -1.0;
    float3 mls, sp, sv;
    float xT, yT, scale;
    float3x3 M;
    bool inv;
    VOI voi;
    RGBA bg;
    AlphaAndWWWLInfo info;
    unpack_vr(p, mls, sp, sv, xT, yT, scale, M, inv, voi, bg, info);
    const float4 clrBG = make_float4(bg.red, bg.green, bg.blue, bg.alpha);
    unsigned char *d = nullptr;
    if (cudaMalloc(&d, (size_t)w * h * 3) != cudaSuccess) return -2.0;
    dim3 block(32, 32);
    dim3 grid((w - 1) / block.x + 1, (h - 1) / block.y + 1);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int i = 0; i < reps; ++i) {
        if (type == 0)
            d_render<<<grid, block>>>(d, w, h, g.tex, g.ext, g.mask_tex, g.tfs, info, mls, sp, sv, xT, yT,
                                      scale, M, inv, voi, clrBG);
        else if (type == 1)
            d_renderMIP<<<grid, block>>>(d, w, h, g.tex, g.ext, g.mask_tex, info, mls, sp, sv, xT, yT,
                                         scale, M, inv, voi, clrBG);
        else
            d_renderSurface<<<grid, block>>>(d, w, h, g.tex, g.ext, g.mask_tex, mls, sp, sv, xT, yT, scale,
                                             M, inv, voi, clrBG);
    }
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (err != cudaSuccess || cudaGetLastError() != cudaSuccess) return -3.0;
    return (double)ms / reps;
}

// Flat plane parameter block (floats): [0..2] spacing, [3..5] dirH, [6..8] dirV,
// [9..11] dirN, [12..14] ptLeftTop, [15] pixel spacing, [16] invertZ, [17] halfNum.
extern "C" int mkref_plane(short *out, int w, int h, const float *p, int mpr_type, int nearest) {
    if (!g.vol || !out || w <= 0 || h <= 0 || !p || mpr_type < 0 || mpr_type > 2) return 1;
    const float3 sp = make_float3(p[0], p[1], p[2]);
    const float3 dh = make_float3(p[3], p[4], p[5]);
    const float3 dv = make_float3(p[6], p[7], p[8]);
    const float3 dn = make_float3(p[9], p[10], p[11]);
    const float3 lt = make_float3(p[12], p[13], p[14]);
    const float ps = p[15];
    const bool inv = p[16] != 0.0f;
    const float half = p[17];
    const cudaTextureObject_t t = nearest ? g.tex_point : g.tex;
    if (mpr_type == 0) cu_renderPlane_Average(out, w, h, t, g.ext, sp, dh, dv, dn, lt, ps, inv, half);
    else if (mpr_type == 1) cu_renderPlane_MIP(out, w, h, t, g.ext, sp, dh, dv, dn, lt, ps, inv, half);
    else cu_renderPlane_MinIP(out, w, h, t, g.ext, sp, dh, dv, dn, lt, ps, inv, half);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int mkref_cpr(short *out, int w, int h, const double *pts, const double *dirs, int invert_z) {
    if (!g.vol || !out || w <= 0 || h <= 0 || !pts || !dirs) return 1;
    cu_renderCPR(out, w, h, g.tex, g.ext, const_cast<double *>(pts), const_cast<double *>(dirs),
                 invert_z != 0);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
