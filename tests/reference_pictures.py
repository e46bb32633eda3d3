"""Codestreams decoded by the reference's own CPU decoder for the golden picture digests.

Each entry names a codestream (a committed fixture of tests/golden/, or a seeded recipe of
the project's writer whose SHA-256 is recorded so a changed writer is caught), the
reference OutputFormat, the reference's DecodeJobConfig::mDwtDecodeTopLevel (-1 = full
resolution; otherwise `levels - top` resolution levels are discarded,
decoder/core/src/decoderconcrete.cpp:715-721), and whether the reference's 5/3 column-end
arithmetic (bmi_cpu_dwt_decoder.cpp:3364-3398) is part of the picture (J2K_FLAG_REF_COMPAT).

tests/golden/make_golden.py decodes them with oracle/_ref/libref_cpu.so (built from the
reference tree) and writes tests/golden/reference_pictures.json; the tests compare the
oracle (CPU) and the device path (GPU) with those digests.

Only single-tile pictures and pictures whose tiles are all full-size are listed: the
reference's decoder writes run-to-run different values into partial edge tiles and
segfaults on 1920x1080 pictures with 512x512 tiles, so no such picture can pin anything.
"""
import hashlib
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

FMT_32BITS_ARGB, FMT_48BITS_RGB, FMT_24BITS_RGB, FMT_32BITS_4COMPONENTS = 0, 1, 2, 3


def _file(name):
    def make():
        with open(os.path.join(GOLDEN, name), "rb") as f:
            return f.read()
    return make


def _c2():
    from jpeg2000_decoder_b200 import synth
    return synth.c2_stream(2)


def _c3_full_tiles():
    """C3's coding parameters (9/7 + ICT, 512x512 tiles, 3 layers at 0.5/1/2 bpp) on the
    first C3 frame cropped to its 3 x 2 full tiles."""
    from jpeg2000_decoder_b200 import native, synth
    frame = synth.video_frames(3, n=1)[0][:, :1024, :1536]
    return native.encode(np.ascontiguousarray(frame), 8, **synth.C3_PARAMS)


def _rgb12(reversible):
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fields_and_edges(21, 256, 256)
    img = (img.astype(np.uint32) * 16 + np.random.default_rng(21).integers(0, 16, img.shape)).astype(np.uint16)
    if reversible:
        return native.encode(img, 12, reversible=1, levels=5)
    return native.encode(img, 12, **synth.C2_PARAMS)


def _gray97():
    from jpeg2000_decoder_b200 import native, synth
    return native.encode(synth.fields_and_edges(22, 256, 256)[:1], 8, **synth.C2_PARAMS)


# name: (stream maker, format, top level, reference 5/3 column-end arithmetic)
PICTURES = {
    "c1_gray_53": (_file("c1_gray_53.j2k"), FMT_32BITS_4COMPONENTS, -1, True),
    "c1_gray_53_top3": (_file("c1_gray_53.j2k"), FMT_32BITS_4COMPONENTS, 3, True),
    "rgb256_53_rct": (_file("rgb256_53_rct.j2k"), FMT_24BITS_RGB, -1, True),
    "rgb256_97_1bpp": (_file("rgb256_97_1bpp.j2k"), FMT_24BITS_RGB, -1, False),
    "rgb256_97_1bpp_argb32": (_file("rgb256_97_1bpp.j2k"), FMT_32BITS_ARGB, -1, False),
    "c2_rgb2048_97_1bpp": (_c2, FMT_24BITS_RGB, -1, False),
    "c2_rgb2048_97_1bpp_top3": (_c2, FMT_24BITS_RGB, 3, False),
    "c3params_rgb1536x1024_97_tiles512_3layers": (_c3_full_tiles, FMT_24BITS_RGB, -1, False),
    "rgb256_12bit_97": (lambda: _rgb12(False), FMT_48BITS_RGB, -1, False),
    "rgb256_12bit_53_rct": (lambda: _rgb12(True), FMT_48BITS_RGB, -1, True),
    "gray256_97": (_gray97, FMT_32BITS_4COMPONENTS, -1, False),
}

_cache = {}


def stream(name):
    if name not in _cache:
        _cache[name] = PICTURES[name][0]()
    return _cache[name]


def sha(data):
    return hashlib.sha256(bytes(data)).hexdigest()


def row_digests(out, height):
    rows = np.frombuffer(bytes(out), np.uint8).reshape(height, -1)
    return [hashlib.sha256(r.tobytes()).hexdigest()[:16] for r in rows]


def discard_of(levels, top):
    """Resolution levels discarded for the reference's mDwtDecodeTopLevel."""
    return 0 if top < 0 or top >= levels else levels - top
