// host_encode.h -- PNG + Base64 encoding of finished images (host_encode.cpp).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace mk {

// 8-bit PNG of a w x h image with 3 (RGB) or 4 (RGBA) channels, rows
// compressed in parallel bands; empty on failure.
std::vector<uint8_t> encode_png(const uint8_t *pixels, int w, int h, int channels);
// Base64 of n bytes into out (4 * ceil(n / 3) characters, no terminator);
// returns the characters written.
size_t base64_encode(const uint8_t *data, size_t n, char *out);
std::string base64_string(const uint8_t *data, size_t n);
// Bytes that always hold the Base64 PNG of a w x h image and its NUL.
size_t encoded_capacity(int w, int h, int channels);

}  // namespace mk
