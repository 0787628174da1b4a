// host_overlay.cpp -- the overlays MonkeyGL's VR provider draws over the
// ray-cast image (core/VRProvider.cpp:30-36):
//
//  * the orientation box: a human mesh (binary STL, normally
//    ./resources/human.stl) turned with the camera rotation, flat-shaded by
//    N.(0,-1,0), rasterised with a z-buffer at 512x512 and sampled every 8th
//    pixel into the bottom-right 64x64 pixels (core/VRImageLayer.cpp:99-194,
//    core/MarchingCube.cpp:305-354, core/Methods.cpp:202-219, 308-368);
//  * the CPR line: the CPR path projected into the image and drawn as a
//    1-pixel polyline (core/CPRLineLayer.cpp:40-65, core/Methods.cpp:163-200).
//
// Both run on the host, as in MonkeyGL, and reproduce its pixels: every
// expression keeps MonkeyGL's mix of float and double arithmetic (products
// of floats are rounded to float before a double accumulates them, scalings
// by a double happen in double, and so on), which is what makes the edges
// of the rasterised triangles land on the same pixels.
//
// The orientation box reads only 64x64 of the 512x512 raster (every 8th
// pixel of every 8th row), so this version keeps the image and z-buffer at
// those sample points only, rasterises a triangle only if its bounding box
// contains one, and turns each distinct mesh vertex once per frame.  Each
// triangle still goes through MonkeyGL's exact rule: its three edges are
// drawn as dotted lines over its bounding box, and a row of the box is
// filled from its first to its last edge pixel; a pixel takes the triangle
// when its z-buffer entry is unset or smaller, in mesh order.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>
#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "mk_internal.h"
#include "monkeygl_b200.h"

namespace {

struct V3 {
    float x, y, z;
};
struct V2 {
    float x, y;
};
struct Facet {
    V3 v1, v2, v3;
};

// Direction<float, 3> (core/Direction.h): normalised on construction with a
// float length.
V3 direction(float x, float y, float z) {
    const float n = sqrtf(x * x + y * y + z * z);
    return V3{x / n, y / n, z / n};
}

V3 direction_from(const V3 &a, const V3 &b) { return direction(b.x - a.x, b.y - a.y, b.z - a.z); }

// Methods::GetTransferPointf: float products accumulated in double.
V3 rotate_point(const float m[9], const V3 &p) {
    const float c[3] = {p.x, p.y, p.z};
    double r[3];
    for (int i = 0; i < 3; ++i) {
        r[i] = 0;
        for (int j = 0; j < 3; ++j) {
            const float prod = m[i * 3 + j] * c[j];
            r[i] += prod;
        }
    }
    return V3{(float)r[0], (float)r[1], (float)r[2]};
}

// Point2f scaled by the image height (a double scale) and moved to the
// image centre.
V2 to_image(float x, float y, int w, int h) {
    const double r = (float)h;
    V2 p{(float)(x * r), (float)(y * r)};
    p.x = p.x + (float)(w / 2.0);
    p.y = p.y + (float)(h / 2.0);
    return p;
}

// Methods::DrawLineInImage*Bit: points every half pixel along the segment,
// nLineWidth parallel strokes, rounded by int(v + 0.5).  `dot` receives the
// pixel (x, y) of every point (callers clip).
template <class Dot>
void draw_line(float x0, float y0, float x1, float y1, int line_width, Dot dot) {
    const float dxf = x1 - x0, dyf = y1 - y0;
    const double len = sqrtf(dxf * dxf + dyf * dyf);
    // Direction<double, 2>
    double dx = dxf, dy = dyf;
    {
        const double n = sqrt(dx * dx + dy * dy);
        dx /= n;
        dy /= n;
    }
    double nx = -dy, ny = dx;
    {
        const double n = sqrt(nx * nx + ny * ny);
        nx /= n;
        ny /= n;
    }
    const float half = 1.0 * line_width / 2;
    const float xs = x0 - (half - 0.5) * nx;
    const float ys = y0 - (half - 0.5) * ny;
    const int steps = int(len + 0.5) * 2;
    for (int k = 0; k < line_width; ++k) {
        const float xk = xs + k * nx;
        const float yk = ys + k * ny;
        for (int i = 0; i <= steps; ++i) {
            const int x = int(xk + i * dx / 2.0 + 0.5);
            const int y = int(yk + i * dy / 2.0 + 0.5);
            dot(x, y);
        }
    }
}

}  // namespace

// Facets as index triples into the mesh's distinct vertices (STL files
// repeat every shared vertex; each is turned once per frame).
struct mk_mesh_s {
    std::vector<V3> verts;
    std::vector<uint32_t> tri;   // 3 per facet, file order
};

namespace {

constexpr int kRaster = 512;   // side of MonkeyGL's orientation raster
constexpr int kBox = 64;       // side of the box in the image
constexpr int kStride = kRaster / kBox;

// The 64x64 samples of the raster: image value (the winning triangle's
// diffuse term) and z-buffer.
struct BoxRaster {
    float img[kBox * kBox];
    float zb[kBox * kBox];
};

// Methods::FillHoleInImage_Ch1 restricted to the sample points.  MonkeyGL
// draws the three edges into a mask over the triangle's bounding box, marks
// each row outside from both ends up to the first edge pixel, and fills
// what is left: on a row with an edge pixel, everything from its first to
// its last edge pixel.  Only rows on the sample grid are read, so only
// their first and last edge pixels are kept.
struct RowSpan {
    int first[kBox], last[kBox];
};

// Sample rows rlo..rhi-1 only (one thread's band).
void fill_triangle(BoxRaster &R, float diffuse, float z, const V2 &v1, const V2 &v2, const V2 &v3, RowSpan &span,
                   int rlo, int rhi) {
    const float fxmin = fminf(v1.x, fminf(v2.x, v3.x));
    const float fymin = fminf(v1.y, fminf(v2.y, v3.y));
    const float fxmax = fmaxf(v1.x, fmaxf(v2.x, v3.x));
    const float fymax = fmaxf(v1.y, fmaxf(v2.y, v3.y));
    const int xmin = int(fxmin);
    const int ymin = int(fymin);
    const int xmax = int(fxmax + 0.5);
    const int ymax = int(fymax + 0.5);
    if (xmin >= kRaster || ymin >= kRaster || xmax < 0 || ymax < 0) return;
    // sample points (multiples of 8 inside the raster) in the box
    const int gx0 = xmin <= 0 ? 0 : (xmin + kStride - 1) / kStride * kStride;
    const int gy0 = ymin <= 0 ? 0 : (ymin + kStride - 1) / kStride * kStride;
    if (gx0 > xmax || gx0 >= kRaster || gy0 > ymax || gy0 >= kRaster) return;
    const int nw = xmax - xmin + 1, nh = ymax - ymin + 1;
    const int gy1 = ymax < kRaster - 1 ? ymax : kRaster - 1;
    const int r0 = std::max(gy0 / kStride, rlo), r1 = std::min(gy1 / kStride, rhi - 1);
    if (r0 > r1) return;
    for (int r = r0; r <= r1; ++r) {
        span.first[r] = nw;
        span.last[r] = -1;
    }
    // an edge point lands in mask pixel (x, y) when both are inside the mask
    auto dot = [&](int x, int y) {
        if (y < 0 || y >= nh || x < 0 || x >= nw) return;
        const int yy = y + ymin;
        if (yy % kStride != 0 || yy < r0 * kStride || yy > r1 * kStride) return;
        const int r = yy / kStride;
        if (x < span.first[r]) span.first[r] = x;
        if (x > span.last[r]) span.last[r] = x;
    };
    draw_line(v1.x - xmin, v1.y - ymin, v2.x - xmin, v2.y - ymin, 1, dot);
    draw_line(v1.x - xmin, v1.y - ymin, v3.x - xmin, v3.y - ymin, 1, dot);
    draw_line(v2.x - xmin, v2.y - ymin, v3.x - xmin, v3.y - ymin, 1, dot);
    for (int r = r0; r <= r1; ++r) {
        if (span.last[r] < 0) continue;   // no edge pixel: the whole row is outside
        const int gy = r * kStride;
        for (int gx = gx0; gx <= xmax && gx < kRaster; gx += kStride) {
            const int x = gx - xmin;
            if (x < span.first[r] || x > span.last[r]) continue;
            const int s = r * kBox + gx / kStride;
            if (R.zb[s] <= 0 || R.zb[s] < z) {
                R.img[s] = diffuse;
                R.zb[s] = z;
            }
        }
        (void)gy;
    }
}

// A facet after culling and projection: its diffuse term, depth, image
// corners and the band [rlo, rhi) of sample rows its box reaches (empty
// when culled or missing every sample).
struct Shaded {
    float d, z;
    V2 v1, v2, v3;
    int rlo, rhi;
};

// Host threads for the overlay: all the process may use, at most 16.
int overlay_threads() {
    const int n = omp_get_max_threads();
    return n < 1 ? 1 : (n > 16 ? 16 : n);
}

void set_err(const std::string &m) { mk::set_last_error(m); }

}  // namespace

extern "C" int mk_mesh_load_stl(const char *path, mk_mesh *out) {
    if (!path || !out) {
        set_err("mk_mesh_load_stl: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    struct stat fs;
    if (stat(path, &fs) != 0 || (unsigned long)fs.st_size <= 80 + 4 + 50) {
        set_err(std::string("mk_mesh_load_stl: missing or too short: ") + path);
        return MK_ERR_INVALID_ARGUMENT;
    }
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        set_err(std::string("mk_mesh_load_stl: cannot open ") + path);
        return MK_ERR_INVALID_ARGUMENT;
    }
    unsigned char header[84];
    if (fread(header, 1, 84, fp) != 84) {
        fclose(fp);
        set_err("mk_mesh_load_stl: short header");
        return MK_ERR_INVALID_ARGUMENT;
    }
    uint32_t n = 0;
    memcpy(&n, header + 80, 4);
    if ((unsigned long)fs.st_size < 84ul + 50ul * n) {
        fclose(fp);
        set_err("mk_mesh_load_stl: file shorter than its facet count");
        return MK_ERR_INVALID_ARGUMENT;
    }
    std::unique_ptr<mk_mesh_s> m(new mk_mesh_s);
    std::vector<Facet> facets(n);
    // MonkeyGL starts the maxima at FLT_MIN (the smallest positive float)
    float xmin = FLT_MAX, xmax = FLT_MIN, ymin = FLT_MAX, ymax = FLT_MIN, zmin = FLT_MAX, zmax = FLT_MIN;
    for (uint32_t i = 0; i < n; ++i) {
        unsigned char rec[50];
        if (fread(rec, 1, 50, fp) != 50) {
            fclose(fp);
            set_err("mk_mesh_load_stl: truncated facet");
            return MK_ERR_INVALID_ARGUMENT;
        }
        float v[9];
        memcpy(v, rec + 12, sizeof(v));   // skip the stored normal
        Facet &f = facets[i];
        f.v1 = V3{v[0], v[1], v[2]};
        f.v2 = V3{v[3], v[4], v[5]};
        f.v3 = V3{v[6], v[7], v[8]};
        xmin = fminf(xmin, fminf(f.v1.x, fminf(f.v2.x, f.v3.x)));
        xmax = fmaxf(xmax, fmaxf(f.v1.x, fmaxf(f.v2.x, f.v3.x)));
        ymin = fminf(ymin, fminf(f.v1.y, fminf(f.v2.y, f.v3.y)));
        ymax = fmaxf(ymax, fmaxf(f.v1.y, fmaxf(f.v2.y, f.v3.y)));
        zmin = fminf(zmin, fminf(f.v1.z, fminf(f.v2.z, f.v3.z)));
        zmax = fmaxf(zmax, fmaxf(f.v1.z, fmaxf(f.v2.z, f.v3.z)));
    }
    fclose(fp);
    // centre, scale by the larger of the x and z extents (a double scale),
    // flip z (core/MarchingCube.cpp:339-353)
    const float xlen = xmax - xmin, zlen = zmax - zmin;
    const float maxlen = fmaxf(xlen, zlen);
    const V3 c{(xmin + xmax) / 2, (ymin + ymax) / 2, (zmin + zmax) / 2};
    const double r = maxlen;
    auto norm = [&](V3 &p) {
        p.x = p.x - c.x;
        p.y = p.y - c.y;
        p.z = p.z - c.z;
        p.x = (float)(p.x / r);
        p.y = (float)(p.y / r);
        p.z = (float)(p.z / r);
        p.z = -p.z;
    };
    // distinct vertices (by bit pattern), normalised once
    std::unordered_map<std::string, uint32_t> index;
    index.reserve(facets.size());
    m->tri.reserve(3 * facets.size());
    for (Facet &f : facets) {
        for (V3 *p : {&f.v1, &f.v2, &f.v3}) {
            const std::string key(reinterpret_cast<const char *>(p), sizeof(V3));
            auto it = index.find(key);
            if (it == index.end()) {
                V3 q = *p;
                norm(q);
                it = index.emplace(key, (uint32_t)m->verts.size()).first;
                m->verts.push_back(q);
            }
            m->tri.push_back(it->second);
        }
    }
    *out = m.release();
    return MK_OK;
}

extern "C" int mk_mesh_destroy(mk_mesh mesh) {
    delete mesh;
    return MK_OK;
}

extern "C" int mk_mesh_facet_count(mk_mesh mesh) { return mesh ? (int)(mesh->tri.size() / 3) : 0; }

extern "C" int mk_merge_orientation_box(mk_mesh mesh, const float rotate[9], uint8_t *rgb, int width, int height) {
    if (!mesh || !rotate || !rgb || width <= 0 || height <= 0) {
        set_err("mk_merge_orientation_box: bad arguments");
        return MK_ERR_INVALID_ARGUMENT;
    }
    if (width <= kBox || height <= kBox) return MK_OK;   // MonkeyGL draws no box on small images
    std::unique_ptr<BoxRaster> R(new BoxRaster);
    memset(R.get(), 0, sizeof(BoxRaster));
    float m[9];
    memcpy(m, rotate, sizeof(m));
    const size_t nv = mesh->verts.size(), nf = mesh->tri.size() / 3;
    std::vector<V3> rv(nv);
    std::vector<Shaded> sf(nf);
    const V3 view = direction(0.0f, -1.0f, 0.0f);
    const int nthreads = overlay_threads();
    // phase 1, over vertices and then facets: turn, cull and project
    // (VRImageLayer::GetMeshPoints, core/VRImageLayer.cpp:166-194)
#pragma omp parallel num_threads(nthreads)
    {
#pragma omp for schedule(static)
        for (long i = 0; i < (long)nv; ++i) rv[i] = rotate_point(m, mesh->verts[i]);
#pragma omp for schedule(static)
        for (long f = 0; f < (long)nf; ++f) {
            Shaded &o = sf[f];
            o.rlo = 1;
            o.rhi = 0;   // empty: culled or no sample point
            const V3 &a = rv[mesh->tri[3 * f]], &b = rv[mesh->tri[3 * f + 1]], &c = rv[mesh->tri[3 * f + 2]];
            const V3 e1 = direction_from(c, a), e2 = direction_from(c, b);
            const float cx = e1.y * e2.z - e1.z * e2.y;
            const float cy = e1.z * e2.x - e1.x * e2.z;
            const float cz = e1.x * e2.y - e1.y * e2.x;
            // N.(0,-1,0) < 0 exactly when the unnormalised cross product
            // points along +y (its length is then positive), so those
            // facets go before the normalisation
            if (cy > 0) continue;
            const V3 n = direction(cx, cy, cz);
            float d = 0;
            d += n.x * view.x;
            d += n.y * view.y;
            d += n.z * view.z;
            if (d < 0) continue;
            o.d = d;
            o.z = (a.y + b.y + c.y) / 3 + 10000;
            o.v1 = to_image(a.x, a.z, kRaster, kRaster);
            o.v2 = to_image(b.x, b.z, kRaster, kRaster);
            o.v3 = to_image(c.x, c.z, kRaster, kRaster);
            // sample rows its bounding box reaches (fill_triangle's own test)
            const float fymin = fminf(o.v1.y, fminf(o.v2.y, o.v3.y));
            const float fymax = fmaxf(o.v1.y, fmaxf(o.v2.y, o.v3.y));
            const int ymin = int(fymin), ymax = int(fymax + 0.5);
            if (ymin >= kRaster || ymax < 0) continue;
            const int gy0 = ymin <= 0 ? 0 : (ymin + kStride - 1) / kStride * kStride;
            const int gy1 = ymax < kRaster - 1 ? ymax : kRaster - 1;
            if (gy0 > gy1) continue;
            o.rlo = gy0 / kStride;
            o.rhi = gy1 / kStride + 1;
        }
    }
    // phase 2, over bands of sample rows holding about equal numbers of
    // facets: every band takes its facets in mesh order, so each sample
    // sees MonkeyGL's z-buffer sequence
    int band[17];
    {
        long hist[kBox] = {}, total = 0;
        for (size_t f = 0; f < nf; ++f)
            for (int r = sf[f].rlo; r < sf[f].rhi; ++r) ++hist[r];
        for (int r = 0; r < kBox; ++r) total += hist[r];
        band[0] = 0;
        long acc = 0;
        int b = 1;
        for (int r = 0; r < kBox && b < nthreads; ++r) {
            acc += hist[r];
            if (acc * nthreads >= total * b) band[b++] = r + 1;
        }
        for (; b <= nthreads; ++b) band[b] = kBox;
    }
#pragma omp parallel num_threads(nthreads)
    {
        const int t = omp_get_thread_num();
        const int blo = t < nthreads ? band[t] : kBox, bhi = t < nthreads ? band[t + 1] : kBox;
        RowSpan span;
        for (size_t f = 0; f < nf && blo < bhi; ++f) {
            const Shaded &o = sf[f];
            if (o.rhi <= blo || o.rlo >= bhi) continue;
            fill_triangle(*R, o.d, o.z, o.v1, o.v2, o.v3, span, blo, bhi);
        }
    }
    // VRImageLayer::MergeOrientationBox: RGBA(0.902, 0.902, 0.302) * diffuse
    // + 0.05, each step clamped to [0, 1], truncated to 8 bits
    const float cr = 0.902f, cg = 0.902f, cb = 0.302f;
    auto trim = [](float v) { return v < 0 ? 0.0f : (v > 1 ? 1.0f : v); };
    for (int j = 0; j < kBox; ++j) {
        const int y = height - kBox + j;
        for (int i = 0; i < kBox; ++i) {
            const float diffuse = R->img[j * kBox + i];
            if (!(diffuse > 0)) continue;
            const int x = width - kBox + i;
            const float r = trim(trim(cr * diffuse) + 0.05f);
            const float g = trim(trim(cg * diffuse) + 0.05f);
            const float b = trim(trim(cb * diffuse) + 0.05f);
            uint8_t *p = rgb + 3 * ((size_t)y * width + x);
            p[0] = (uint8_t)int(r * 255);
            p[1] = (uint8_t)int(g * 255);
            p[2] = (uint8_t)int(b * 255);
        }
    }
    return MK_OK;
}

extern "C" int mk_draw_line_rgb(uint8_t *rgb, int width, int height, float x0, float y0, float x1, float y1,
                                int line_width, const float color[3]) {
    if (!rgb || !color || width <= 0 || height <= 0 || line_width < 0) {
        set_err("mk_draw_line_rgb: bad arguments");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const uint8_t r = (uint8_t)int(color[0] * 255), g = (uint8_t)int(color[1] * 255),
                  b = (uint8_t)int(color[2] * 255);
    draw_line(x0, y0, x1, y1, line_width, [&](int x, int y) {
        if (x < 0 || x >= width || y < 0 || y >= height) return;
        uint8_t *p = rgb + 3 * ((size_t)y * width + x);
        p[0] = r;
        p[1] = g;
        p[2] = b;
    });
    return MK_OK;
}

// ---------------------------------------------------------------------------
// Text annotations.  MonkeyGL draws VR annotations from 8-bit glyph masks of
// three font sizes (core/AnnotationUtils.cpp:42-376) with
// AnnotationUtils::Textout2Image (core/AnnotationUtils.cpp:419-458).  The
// masks are not part of this library: a glyph file (format below) supplies
// them, and the drawing follows Textout2Image:
//   - the text is taken one byte at a time; a byte without a glyph counts as
//     a glyph of width -1 and height -1 (nothing drawn, the pen moves back one
//     pixel), as MonkeyGL's map lookup of an unknown character gives;
//   - right / centred text starts the total width (sum of the widths, the
//     height of the last glyph) / half of it (integer division) to the left;
//   - a glyph pixel with mask m > 0 inside the image becomes m * colour in
//     each channel, converted to 8 bits by truncation;
//   - nothing is drawn into images of width or height below 10.
// Glyph file: "MKGLYPH1", uint32 count, then per glyph: uint8 font size
// (0 small, 1 middle, 2 big), uint8 key length, the key bytes (the
// character), uint16 width, uint16 height, width * height mask bytes.
struct mk_font_s {
    struct Glyph {
        int w = -1, h = -1;
        std::vector<uint8_t> mask;
    };
    std::unordered_map<std::string, Glyph> glyphs[3];
};

namespace {

const mk_font_s::Glyph &font_glyph(const mk_font_s *f, int size, char c) {
    static const mk_font_s::Glyph unknown;
    if (size < 0 || size > 2) return unknown;
    auto it = f->glyphs[size].find(std::string(1, c));
    return it == f->glyphs[size].end() ? unknown : it->second;
}

// float -> 8 bits as an x86 build of MonkeyGL's assignment converts it
// (truncation to a 32-bit integer, then its low byte)
inline uint8_t to_u8(float v) { return (uint8_t)(int32_t)v; }

}  // namespace

extern "C" int mk_font_load(const char *path, mk_font *out) {
    if (!path || !out) {
        set_err("mk_font_load: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        set_err(std::string("mk_font_load: cannot open ") + path);
        return MK_ERR_INVALID_ARGUMENT;
    }
    std::unique_ptr<mk_font_s> f(new mk_font_s());
    char magic[8];
    uint32_t n = 0;
    bool ok = fread(magic, 1, 8, fp) == 8 && memcmp(magic, "MKGLYPH1", 8) == 0 && fread(&n, 4, 1, fp) == 1 &&
              n <= 4096;
    for (uint32_t i = 0; ok && i < n; ++i) {
        uint8_t size = 0, klen = 0;
        uint16_t w = 0, h = 0;
        char key[256];
        ok = fread(&size, 1, 1, fp) == 1 && fread(&klen, 1, 1, fp) == 1 && size <= 2 && klen > 0 &&
             fread(key, 1, klen, fp) == klen && fread(&w, 2, 1, fp) == 1 && fread(&h, 2, 1, fp) == 1;
        if (!ok) break;
        mk_font_s::Glyph g;
        g.w = w;
        g.h = h;
        g.mask.resize((size_t)w * h);
        ok = g.mask.empty() || fread(g.mask.data(), 1, g.mask.size(), fp) == g.mask.size();
        if (ok) f->glyphs[size][std::string(key, klen)] = std::move(g);
    }
    fclose(fp);
    if (!ok) {
        set_err(std::string("mk_font_load: malformed glyph file ") + path);
        return MK_ERR_INVALID_ARGUMENT;
    }
    *out = f.release();
    return MK_OK;
}

extern "C" int mk_font_destroy(mk_font font) {
    if (!font) return MK_ERR_INVALID_ARGUMENT;
    delete font;
    return MK_OK;
}

extern "C" int mk_text_size(mk_font font, const char *text, int font_size, int *width, int *height) {
    if (!font || !text || !width || !height) {
        set_err("mk_text_size: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    // AnnotationUtils::GetSize (core/AnnotationUtils.cpp:460-470)
    int w = 0, h = 0;
    for (const char *c = text; *c; ++c) {
        const mk_font_s::Glyph &g = font_glyph(font, font_size, *c);
        w += g.w;
        h = g.h;
    }
    *width = w;
    *height = h;
    return MK_OK;
}

extern "C" int mk_draw_text_rgb(mk_font font, uint8_t *rgb, int width, int height, const char *text, int x, int y,
                                int font_size, int format, const float color[3]) {
    if (!font || !rgb || !text || !color || width < 10 || height < 10 || format < 0 || format > 2) {
        set_err("mk_draw_text_rgb: bad arguments (image of at least 10x10, format 0..2)");
        return MK_ERR_INVALID_ARGUMENT;
    }
    int x0 = x;
    if (format != 0) {                                 // AnnotationFormatRight = 1, Center = 2
        int w = 0, h = 0;
        mk_text_size(font, text, font_size, &w, &h);
        x0 -= format == 2 ? w / 2 : w;
    }
    for (const char *c = text; *c; ++c) {
        const mk_font_s::Glyph &g = font_glyph(font, font_size, *c);
        for (int yy = y; yy < y + g.h; ++yy) {
            if (yy < 0 || yy >= height) continue;
            for (int xx = x0; xx < x0 + g.w; ++xx) {
                if (xx < 0 || xx >= width) continue;
                const uint8_t m = g.mask[(size_t)(yy - y) * g.w + (xx - x0)];
                if (m == 0) continue;
                uint8_t *p = rgb + 3 * ((size_t)yy * width + xx);
                p[0] = to_u8(m * color[0]);
                p[1] = to_u8(m * color[1]);
                p[2] = to_u8(m * color[2]);
            }
        }
        x0 += g.w;
    }
    return MK_OK;
}
