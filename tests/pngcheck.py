"""PNG + Base64 decoding for the tests (zlib and the PNG chunk layout, no
imaging library): the inverse of mk_encode_png_base64 for 8-bit RGB/RGBA
images with filter 0 on every row."""
import base64
import zlib

import numpy as np


def decode_png_base64(text):
    """(H, W, C) uint8 of a Base64 PNG; checks the chunk CRCs and the zlib
    stream (its Adler-32 included)."""
    b = base64.b64decode(text, validate=True)
    assert b[:8] == b"\x89PNG\r\n\x1a\n", "PNG signature"
    i, idat, hdr = 8, b"", None
    while i < len(b):
        n = int.from_bytes(b[i:i + 4], "big")
        t, d = b[i + 4:i + 8], b[i + 8:i + 8 + n]
        assert zlib.crc32(t + d) == int.from_bytes(b[i + 8 + n:i + 12 + n], "big"), f"CRC of {t!r}"
        if t == b"IHDR":
            hdr = d
        elif t == b"IDAT":
            idat += d
        i += 12 + n
    w, h = int.from_bytes(hdr[:4], "big"), int.from_bytes(hdr[4:8], "big")
    assert hdr[8] == 8 and hdr[9] in (2, 6)
    ch = 3 if hdr[9] == 2 else 4
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, w * ch + 1)
    assert (raw[:, 0] == 0).all(), "row filters"
    return raw[:, 1:].reshape(h, w, ch)
