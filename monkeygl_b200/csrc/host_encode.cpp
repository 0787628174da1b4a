// host_encode.cpp -- PNG + Base64 encoding of finished images, the output
// form of MonkeyGL's GetVRData_pngString / GetPlaneData_pngString
// (core/HelloMonkey.cpp:212-259, 333-413: fpng, then Base64).
//
// The image is written as one 8-bit PNG (colour type 2 for RGB, 6 for RGBA,
// filter 0 on every row) whose zlib stream is compressed in parallel: the
// rows are cut into bands of at least 32 rows (at most 64 bands), every band
// is deflated on its own (level 1, no dictionary shared with other bands)
// and ended with a full flush, the last one with the final block; the bands'
// streams are concatenated behind one zlib header and the Adler-32 of the
// whole is combined from theirs.  The band count depends on the image only,
// so the bytes are the same on every machine.  The decoded pixels are the
// image's; the compressed bytes differ from fpng's.
#include <omp.h>
#include <stdint.h>
#include <string.h>
#include <zlib.h>

#include <string>
#include <vector>

#include "host_encode.h"
#include "mk_internal.h"

namespace mk {

namespace {

constexpr int kMaxBands = 64;
constexpr int kMinBandRows = 32;

int band_count(int h) {
    int k = h / kMinBandRows;
    return k < 1 ? 1 : (k > kMaxBands ? kMaxBands : k);
}

void put_be32(std::vector<uint8_t> &v, uint32_t x) {
    v.push_back(x >> 24);
    v.push_back((x >> 16) & 0xff);
    v.push_back((x >> 8) & 0xff);
    v.push_back(x & 0xff);
}

void put_chunk(std::vector<uint8_t> &png, const char *type, const uint8_t *data, size_t n) {
    put_be32(png, (uint32_t)n);
    const size_t start = png.size();
    png.insert(png.end(), type, type + 4);
    if (n) png.insert(png.end(), data, data + n);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, png.data() + start, (uInt)(png.size() - start));
    put_be32(png, (uint32_t)crc);
}

}  // namespace

std::vector<uint8_t> encode_png(const uint8_t *pixels, int w, int h, int channels) {
    std::vector<uint8_t> png;
    if (!pixels || w <= 0 || h <= 0 || (channels != 3 && channels != 4)) return png;
    const size_t row = (size_t)w * channels;
    const int K = band_count(h);
    std::vector<std::vector<uint8_t>> z(K);
    std::vector<uLong> adler(K), raw_len(K);
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : ok)
    for (int k = 0; k < K; ++k) {
        const int y0 = (int)((long long)h * k / K), y1 = (int)((long long)h * (k + 1) / K);
        std::vector<uint8_t> raw((row + 1) * (size_t)(y1 - y0));
        for (int y = y0; y < y1; ++y) {
            uint8_t *r = &raw[(size_t)(y - y0) * (row + 1)];
            r[0] = 0;
            memcpy(r + 1, pixels + (size_t)y * row, row);
        }
        z_stream s;
        memset(&s, 0, sizeof(s));
        if (deflateInit2(&s, 1, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY) != Z_OK) {
            ok = false;
            continue;
        }
        z[k].resize(deflateBound(&s, (uLong)raw.size()) + 16);
        s.next_in = raw.data();
        s.avail_in = (uInt)raw.size();
        s.next_out = z[k].data();
        s.avail_out = (uInt)z[k].size();
        const int rc = deflate(&s, k == K - 1 ? Z_FINISH : Z_FULL_FLUSH);
        const bool done = k == K - 1 ? rc == Z_STREAM_END : (rc == Z_OK && s.avail_in == 0);
        z[k].resize(z[k].size() - s.avail_out);
        deflateEnd(&s);
        adler[k] = adler32(adler32(0L, Z_NULL, 0), raw.data(), (uInt)raw.size());
        raw_len[k] = (uLong)raw.size();
        ok = ok && done;
    }
    if (!ok) return png;
    size_t zlen = 2 + 4;
    for (int k = 0; k < K; ++k) zlen += z[k].size();
    std::vector<uint8_t> zs;
    zs.reserve(zlen);
    zs.push_back(0x78);                  // deflate, 32 KiB window
    zs.push_back(0x01);                  // no dictionary, fastest level; (0x7801 % 31 == 0)
    uLong a = adler[0];
    for (int k = 0; k < K; ++k) {
        zs.insert(zs.end(), z[k].begin(), z[k].end());
        if (k > 0) a = adler32_combine(a, adler[k], (z_off_t)raw_len[k]);
    }
    put_be32(zs, (uint32_t)a);
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    png.reserve(zs.size() + 64);
    png.insert(png.end(), sig, sig + 8);
    uint8_t ihdr[13];
    const uint32_t be[2] = {(uint32_t)w, (uint32_t)h};
    for (int i = 0; i < 2; ++i) {
        ihdr[4 * i] = be[i] >> 24;
        ihdr[4 * i + 1] = (be[i] >> 16) & 0xff;
        ihdr[4 * i + 2] = (be[i] >> 8) & 0xff;
        ihdr[4 * i + 3] = be[i] & 0xff;
    }
    ihdr[8] = 8;
    ihdr[9] = channels == 3 ? 2 : 6;
    ihdr[10] = ihdr[11] = ihdr[12] = 0;
    put_chunk(png, "IHDR", ihdr, 13);
    put_chunk(png, "IDAT", zs.data(), zs.size());
    put_chunk(png, "IEND", nullptr, 0);
    return png;
}

size_t base64_encode(const uint8_t *data, size_t n, char *out) {
    static const char tbl[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    size_t o = 0, i = 0;
    for (; i + 2 < n; i += 3) {
        const uint32_t v = (data[i] << 16) | (data[i + 1] << 8) | data[i + 2];
        out[o++] = tbl[v >> 18];
        out[o++] = tbl[(v >> 12) & 63];
        out[o++] = tbl[(v >> 6) & 63];
        out[o++] = tbl[v & 63];
    }
    if (i < n) {
        uint32_t v = data[i] << 16;
        if (i + 1 < n) v |= data[i + 1] << 8;
        out[o++] = tbl[v >> 18];
        out[o++] = tbl[(v >> 12) & 63];
        out[o++] = i + 1 < n ? tbl[(v >> 6) & 63] : '=';
        out[o++] = '=';
    }
    return o;
}

std::string base64_string(const uint8_t *data, size_t n) {
    std::string s(((n + 2) / 3) * 4, '\0');
    base64_encode(data, n, &s[0]);
    return s;
}

size_t encoded_capacity(int w, int h, int channels) {
    if (w <= 0 || h <= 0 || (channels != 3 && channels != 4)) return 0;
    const size_t raw = ((size_t)w * channels + 1) * h;
    // deflateBound per band (stored blocks in the worst case) plus a flush
    // marker per band, zlib header/trailer and the PNG chunks
    const size_t zb = raw + (raw >> 12) + (raw >> 14) + (raw >> 25) + 64 * (size_t)(kMaxBands + 1);
    const size_t png = zb + 8 + 25 + 12 + 12 + 64;
    return ((png + 2) / 3) * 4 + 1;
}

}  // namespace mk

extern "C" int mk_encoded_capacity(int width, int height, int channels, size_t *bytes) {
    if (!bytes) {
        mk::set_last_error("mk_encoded_capacity: null argument");
        return MK_ERR_INVALID_ARGUMENT;
    }
    *bytes = mk::encoded_capacity(width, height, channels);
    if (*bytes == 0) {
        mk::set_last_error("mk_encoded_capacity: bad image size or channel count (3 or 4)");
        return MK_ERR_INVALID_ARGUMENT;
    }
    return MK_OK;
}

extern "C" int mk_encode_png_base64(const uint8_t *pixels, int width, int height, int channels, char *out,
                                    size_t capacity, size_t *length) {
    if (!pixels || !out || !length || width <= 0 || height <= 0 || (channels != 3 && channels != 4)) {
        mk::set_last_error("mk_encode_png_base64: bad arguments");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const std::vector<uint8_t> png = mk::encode_png(pixels, width, height, channels);
    if (png.empty()) {
        mk::set_last_error("mk_encode_png_base64: compression failed");
        return MK_ERR_OUT_OF_MEMORY;
    }
    const size_t need = ((png.size() + 2) / 3) * 4;
    if (need + 1 > capacity) {
        mk::set_last_error("mk_encode_png_base64: output buffer too small (see mk_encoded_capacity)");
        return MK_ERR_INVALID_ARGUMENT;
    }
    const size_t n = mk::base64_encode(png.data(), png.size(), out);
    out[n] = '\0';
    *length = n;
    return MK_OK;
}
