/*
 * mk_oracle.h -- TEST INFRASTRUCTURE, not part of the product.
 *
 * A CPU restatement, in plain C, of MonkeyGL's volume ray-casting path
 * (core/kernel.cu:31-918 with the texture semantics of
 * core/CuDataManager.cu:28-163).  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py use it, as the checker and as the timed host
 * baseline; the library never calls it.
 *
 * Two precisions:
 *   MKO_TEX32  FP32 arithmetic in MonkeyGL's operation order with the CUDA
 *              texture unit emulated: texel coordinate x*N - 0.5, weights
 *              quantised to 8 fractional bits, clamp-to-edge, int16 read as
 *              max(v/32767, -1), LUT filtered linearly with entry centres at
 *              (i+0.5)/N.  MonkeyGL's double-promoted expressions are evaluated
 *              in double as in the original.
 *   MKO_EXACT64 the same method in FP64 with exact trilinear and LUT weights
 *              (the "method" reference for error statements).
 *
 * Parameter blocks are flat float arrays:
 *   VR (MKO_VR_FLOATS = 227): [0..2] maxLenSpacing, [3..5] spacing,
 *     [6..8] spacingVoxel, [9] xTranslate, [10] yTranslate, [11] scale,
 *     [12..20] camera matrix rows, [21] invertZ, [22..27] VOI (left, right,
 *     posterior, anterior, head, foot), [28..31] background RGBA,
 *     [32+3l .. 34+3l] alpha, ww, wl of label l (l = 0..64).
 *   Plane (MKO_PLANE_FLOATS = 18): [0..2] spacing, [3..5] dirH, [6..8] dirV,
 *     [9..11] dirN, [12..14] ptLeftTop, [15] pixel spacing, [16] invertZ,
 *     [17] halfNum.
 */
#ifndef MK_ORACLE_H
#define MK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MKO_LABELS 65
#define MKO_VR_FLOATS (32 + 3 * MKO_LABELS)
#define MKO_PLANE_FLOATS 18

enum { MKO_TEX32 = 0, MKO_EXACT64 = 1 };
enum { MKO_VR = 0, MKO_MIP = 1, MKO_SURFACE = 2 };

typedef struct mko_volume {
    const int16_t *vox;             /* x-fastest dim[0]*dim[1]*dim[2] */
    int dim[3];
    const uint8_t *mask;            /* NULL = no label volume */
    const float *lut[MKO_LABELS];   /* RGBA float4 tables, NULL = none */
    int lut_len[MKO_LABELS];
} mko_volume;

/* Texture weight quantisation: 0 = round to nearest 1/256 (default),
 * 1 = truncate, 2 = no quantisation. */
void mko_set_weight_mode(int mode);

/* d_render / d_renderMIP / d_renderSurface (core/kernel.cu:133-469) into
 * w*h RGB8.  `samples` (may be NULL) receives the number of volume fetches of
 * the schedule.  nthreads <= 0 uses all OpenMP threads. */
int mko_render_vr(const mko_volume *v, int w, int h, int type, const float *params,
                  int precision, int nthreads, uint8_t *out_rgb, uint64_t *samples);

/* The same for the rows row0, row0 + row_step, ... (nrows of them) of a
 * w*h frame, written consecutively to out_rgb (nrows*w*3 bytes). */
int mko_render_vr_rows(const mko_volume *v, int w, int h, int type, const float *params,
                       int precision, int nthreads, int row0, int row_step, int nrows,
                       uint8_t *out_rgb, uint64_t *samples);

/* d_renderPlane_{Average,MIP,MinIP} (core/kernel.cu:570-793). mpr_type: 0
 * Average, 1 MIP, 2 MinIP; nearest selects point sampling. */
int mko_render_plane(const mko_volume *v, int w, int h, const float *params, int mpr_type,
                     int nearest, int precision, int nthreads, int16_t *out);

/* d_renderCPR (core/kernel.cu:839-873). */
int mko_render_cpr(const mko_volume *v, int w, int h, const double *pts, const double *dirs,
                   int invert_z, int precision, int nthreads, int16_t *out);

/* The differentiable method of monkeygl_b200/csrc/mk_dvr.cu in FP64 (for
 * central finite differences).  p: [0] width, [1] height, [2..4] dims,
 * [5..7] maxLenSpacing, [8..16] camera matrix, [17] scale, [18] xT, [19] yT,
 * [20] step, [21] t_min, [22] lut_len; vol and lut are doubles; image is
 * width*height*3 doubles. */
int mko_dvr_forward_d(const double *p, const double *vol, const double *lut, int nthreads, double *image);
/* Conditioning of a reverse march from the final transmittance (FP32); see mk_oracle.c. */
int mko_dvr_reverse_stats(const double *p, const float *vol, const float *lut, int nthreads, double *stats);

/* Single texture fetches, exposed for known-answer tests. */
float mko_tex3d_linear(const mko_volume *v, float x, float y, float z);
float mko_tex3d_point(const mko_volume *v, float x, float y, float z);
void mko_tex1d_lut(const float *lut, int n, float t, float out[4]);

#ifdef __cplusplus
}
#endif

#endif
