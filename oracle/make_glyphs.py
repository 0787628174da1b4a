"""TEST INFRASTRUCTURE / build step: extract MonkeyGL's annotation glyph
masks into a glyph file for the library's text drawing (mk_font_load).

MonkeyGL keeps its glyphs as data inside core/AnnotationUtils.cpp; this
repository does not carry them.  The script asks MonkeyGL's own host
library, built from its unmodified sources (oracle/_ref/libmkref_host.so,
`make -C oracle ref-host`), for the glyph of every printable ASCII
character at each of its three font sizes (mkrh_glyph in
ref_host_capture.cpp: AnnotationUtils::GetSize and a Textout2Image call in
white on black) and writes them in the format include/monkeygl_b200.h
describes:

    python oracle/make_glyphs.py oracle/_ref/libmkref_host.so oracle/_ref/resources/annotation_glyphs.bin
"""
import ctypes as C
import struct
import sys
from pathlib import Path


def main(lib_path, out_path):
    L = C.CDLL(str(lib_path))
    L.mkrh_glyph.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    buf = (C.c_ubyte * (256 * 256))()
    wh = (C.c_int * 2)()
    glyphs = []
    for size in (0, 1, 2):
        for code in range(0x20, 0x7f):
            key = bytes([code])
            if L.mkrh_glyph(key, size, buf, len(buf), wh) != 1:
                continue
            w, h = wh[0], wh[1]
            glyphs.append((size, key, w, h, bytes(buf[: w * h])))
    out = Path(out_path)
    out.parent.mkdir(parents=True, exist_ok=True)
    with open(out, "wb") as f:
        f.write(b"MKGLYPH1")
        f.write(struct.pack("<I", len(glyphs)))
        for size, key, w, h, mask in glyphs:
            f.write(struct.pack("<BB", size, len(key)))
            f.write(key)
            f.write(struct.pack("<HH", w, h))
            f.write(mask)
    print(f"{out}: {len(glyphs)} glyphs")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
