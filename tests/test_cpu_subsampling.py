"""Sub-sampled components (SIZ XRsiz / YRsiz) and the JP2 colour specification, on the CPU.

Component c of a sub-sampled picture lives on its own grid (T.800 B.2-B.3: the tile's
reference-grid bounds divided by XRsiz / YRsiz, rounded up); packed pictures show each
component's nearest-left sample, i.e. sub-sampled components are replicated.  The
reference detects the 4:2:0 / 4:2:2 / vertical-only layouts (decoder/codec/src/
dec_jp2.cpp:488-523) and builds their code-block geometry (dec_init.cpp:86-88, :700-702),
but its CPU DWT and MCT never read XRsiz / YRsiz, so its sub-sampled pictures are wrong
(chroma errors up to 255 on the streams below): these are pinned by lossless identity,
by OpenJPEG's decode of the same streams, and by the device matching the oracle.
"""
import io

import numpy as np
import pytest

import oracle_util

LAYOUTS = [("420", (1, 2, 2), (1, 2, 2)), ("422", (1, 2, 2), (1, 1, 1)), ("440", (1, 1, 1), (1, 2, 2))]


def subsampled_stream(kind, reversible=1, tiles=0, levels=3, h=136, w=200, seed=31, depth=8):
    from jpeg2000_decoder_b200 import native, synth
    sx, sy = dict((k, (a, b)) for k, a, b in LAYOUTS)[kind]
    img = synth.fields_and_edges(seed, h, w)
    if depth > 8:
        img = (img.astype(np.uint32) << (depth - 8)).astype(np.uint16)
    cs = native.encode(img, depth, reversible=reversible, levels=levels, use_mct=0, sub_x=list(sx), sub_y=list(sy),
                       tile_w=tiles, tile_h=tiles, guard_bits=0 if reversible else 1)
    planes = [img[c][::sy[c], ::sx[c]] for c in range(3)]
    return cs, img, planes, sx, sy


def replicated(planes, sx, sy, h, w):
    return [np.repeat(np.repeat(p, b, 0), a, 1)[:h, :w] for p, a, b in zip(planes, sx, sy)]


def components_from_coef(plan, coef):
    """Each component's reconstructed samples on its own grid, from the oracle's buffer."""
    I = plan.info
    out = [np.zeros((I.comp_h[c], I.comp_w[c]), np.int64) for c in range(I.ncomp)]
    for tc in plan.tilecomps():
        reg = coef[tc.coef_off:tc.coef_off + tc.w * tc.h].reshape(tc.h, tc.w)
        out[tc.comp][tc.y0:tc.y0 + tc.h, tc.x0:tc.x0 + tc.w] = reg
    return out


@pytest.mark.parametrize("kind", [k for k, _, _ in LAYOUTS])
@pytest.mark.parametrize("tiles", [0, 64])
def test_subsampled_lossless_components_and_replicated_output(pkg, kind, tiles):
    from jpeg2000_decoder_b200 import native
    cs, img, planes, sx, sy = subsampled_stream(kind, tiles=tiles)
    plan = native.Plan(cs)
    I = plan.info
    assert list(I.sub_x[:3]) == list(sx) and list(I.sub_y[:3]) == list(sy)
    for c in range(3):
        assert (I.comp_h[c], I.comp_w[c]) == planes[c].shape
    rc, out, coef = oracle_util.oracle_decode(plan, native.FMT_24BITS_3COMPONENTS)
    assert rc == 0
    comps = components_from_coef(plan, coef)
    for c in range(3):
        assert np.array_equal(comps[c] + 128, planes[c]), c  # 5/3: the un-shifted component is exact
    px = out.reshape(I.height, I.width, 3)
    want = replicated(planes, sx, sy, I.height, I.width)
    for c in range(3):
        assert np.array_equal(px[:, :, 2 - c], want[c]), c  # component c in byte 2 - c


@pytest.mark.parametrize("kind", [k for k, _, _ in LAYOUTS])
def test_subsampled_streams_match_openjpeg(pkg, kind):
    """OpenJPEG (Pillow) decodes the same streams, replicating the chroma and converting
    YCbCr to RGB; the same conversion of our packed components gives the same bytes."""
    from PIL import Image
    from jpeg2000_decoder_b200 import native
    for rev in (1, 0):
        cs, img, planes, sx, sy = subsampled_stream(kind, reversible=rev)
        plan = native.Plan(cs)
        I = plan.info
        rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_24BITS_3COMPONENTS)
        assert rc == 0
        px = out.reshape(I.height, I.width, 3)
        ycc = Image.merge("YCbCr", [Image.fromarray(np.ascontiguousarray(px[:, :, 2 - c])) for c in range(3)])
        ours = np.array(ycc.convert("RGB")).astype(int)
        theirs = np.array(Image.open(io.BytesIO(cs)).convert("RGB")).astype(int)
        d = np.abs(ours - theirs).max()
        # 9/7: components within 2 of OpenJPEG's (its float lifting and rounding against the
        # reference's (int) truncation), which the YCbCr -> RGB conversion scales by up to
        # 1 + 1.772 before its own rounding
        assert d <= (0 if rev else 6), (kind, rev, d)


def test_subsampled_reduced_resolution_and_12bit(pkg):
    from jpeg2000_decoder_b200 import native
    cs, img, planes, sx, sy = subsampled_stream("420", levels=4, depth=12, h=160, w=256)
    full = native.Plan(cs)
    rc, _, coef = oracle_util.oracle_decode(full, native.FMT_48BITS_3COMPONENTS)
    assert rc == 0
    comps = components_from_coef(full, coef)
    for c in range(3):
        assert np.array_equal(comps[c] + 2048, planes[c])
    half = native.Plan(cs, discard_levels=1)
    I = half.info
    assert (I.width, I.height) == (128, 80)
    assert (I.comp_w[1], I.comp_h[1]) == (64, 40)
    rc, out, _ = oracle_util.oracle_decode(half, native.FMT_48BITS_3COMPONENTS)
    assert rc == 0 and out.size == 128 * 80 * 6


def test_mct_over_unequally_sampled_components_is_refused(pkg):
    """The inverse RCT / ICT combines components sample by sample (T.800 G.1): a stream
    that asks for it over differently sampled components is refused, not decoded wrongly."""
    from jpeg2000_decoder_b200 import native
    cs, *_ = subsampled_stream("420")
    data = bytearray(cs)
    cod = data.index(b"\xff\x52")
    data[cod + 8] = 1  # COD: SGcod multiple component transform
    with pytest.raises(native.J2kError) as e:
        native.Plan(bytes(data))
    assert e.value.code == native.J2K_ERR_UNSUPPORTED


def _jp2(codestream, colr_enum=None, colr_method=1):
    """A minimal JP2 file around a codestream (T.800 I.5): signature, file type, header
    (image header + colour specification), contiguous codestream."""
    import struct

    def box(t, payload):
        return struct.pack(">I", 8 + len(payload)) + t + payload
    ihdr = box(b"ihdr", struct.pack(">IIHBBBB", 1, 1, 3, 7, 7, 0, 0))
    parts = [ihdr]
    if colr_enum is not None:
        body = bytes([colr_method, 0, 0]) + (struct.pack(">I", colr_enum) if colr_method == 1 else b"\0\0\0\0")
        parts.append(box(b"colr", body))
    return (box(b"jP  ", b"\r\n\x87\n") + box(b"ftyp", b"jp2 \0\0\0\0jp2 ") + box(b"jp2h", b"".join(parts)) +
            box(b"jp2c", codestream))


def test_jp2_colour_box_and_formats(pkg):
    """JP2 header boxes: the colour specification is read (refused for an enumerated
    colour space other than sRGB / greyscale / sYCC, as the reference refuses it), and
    the picture decodes exactly as its bare codestream."""
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fields_and_edges(41, 64, 96)
    cs = native.encode(img, 8, reversible=1, levels=3)
    bare = oracle_util.oracle_decode(native.Plan(cs), native.FMT_24BITS_RGB)[1]
    for enum in (16, 18, None):
        wrapped = oracle_util.oracle_decode(native.Plan(_jp2(cs, enum)), native.FMT_24BITS_RGB)[1]
        assert np.array_equal(bare, wrapped)
    with pytest.raises(native.J2kError) as e:
        native.Plan(_jp2(cs, 12))  # CMYK
    assert e.value.code == native.J2K_ERR_UNSUPPORTED
    native.Plan(_jp2(cs, 12, colr_method=2))  # an ICC profile is not checked
    with pytest.raises(native.J2kError):
        native.Plan(_jp2(cs, 16)[:-len(cs) - 8] + b"\0\0\0\x08jp2x")  # no codestream box


def test_reference_api_reports_the_picture_format(pkg):
    """BMI::Decoder::PreDecode's mFormat follows the reference's rules (dec_jp2.cpp:488-523):
    the component sampling picks 4:2:0 / 4:2:2 / vertical-only, and three equally sampled
    components are RGB or YUV444 by the JP2 colour space (16 sRGB, 18 sYCC), else by the
    COD transform flag."""
    import ctypes
    from jpeg2000_decoder_b200 import native, synth
    RAW, RGB, YUV444, YUV422, YUV420, BAYERGRB, COMPONENT4 = range(7)
    f = native.lib().bmi_decoder_predecode_format

    def fmt(cs):
        a, m = ctypes.c_int(-1), ctypes.c_int(-1)
        assert f(cs, len(cs), ctypes.byref(a), ctypes.byref(m)) == 0
        return a.value, m.value
    for kind, want in (("420", YUV420), ("422", YUV422), ("440", BAYERGRB)):
        assert fmt(subsampled_stream(kind)[0]) == (want, 0)
        assert fmt(subsampled_stream(kind, reversible=0)[0]) == (want, 1)
    img = synth.fields_and_edges(43, 64, 64)
    rgb = native.encode(img, 8, reversible=1, levels=2)
    plain = native.encode(img, 8, reversible=1, levels=2, use_mct=0)
    assert fmt(rgb)[0] == RGB and fmt(plain)[0] == YUV444
    assert fmt(_jp2(plain, 16))[0] == RGB and fmt(_jp2(rgb, 18))[0] == YUV444
    assert fmt(native.encode(img[:1], 8, reversible=1, levels=2))[0] == RAW
    four = np.concatenate([img, img[:1]])
    assert fmt(native.encode(four, 8, reversible=1, levels=2, use_mct=0))[0] == COMPONENT4
