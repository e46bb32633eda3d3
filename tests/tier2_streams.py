"""Codestreams that exercise the Tier-2 front end beyond the benchmark configurations.

* `marker_cases()`: the project encoder with SOP / EPH markers, packed packet headers
  (PPM in the main header, PPT in tile-part headers), several tile-parts per tile (in tile
  order or interleaved across tiles) and progression volumes (POC in the main header or in
  the first tile-part header of each tile).  All are lossless, so every case must decode to
  its source picture.
* `splice_tiles()`: a codestream whose tiles carry their own COD / QCD in the first
  tile-part header (T.800 A.4.2: tile-part COD/QCD override the main header's for that
  tile), assembled from two encodings of one picture with different coding parameters
  and the same tile grid, transform and component transform.
"""
import struct

import numpy as np

H, W = 96, 128


def source():
    from jpeg2000_decoder_b200 import synth
    return synth.fields_and_edges(41, H, W)


def marker_cases():
    """(name, encoder keywords, OpenJPEG 2.5.4 agrees) for the lossless marker variants."""
    from jpeg2000_decoder_b200 import native
    L, NL = 3, 3
    sop, eph, ppm, ppt = native.ENC_SOP, native.ENC_EPH, native.ENC_PPM, native.ENC_PPT
    return [
        ("sop", dict(markers=sop), True),
        ("eph", dict(markers=eph), True),
        ("sop_eph", dict(markers=sop | eph), True),
        ("ppm", dict(markers=ppm), True),
        ("ppm_sop_eph", dict(markers=ppm | sop | eph), True),
        ("ppt", dict(markers=ppt), True),
        ("ppt_eph_3parts", dict(markers=ppt | eph, tile_parts=3), True),
        ("ppm_3parts", dict(markers=ppm, tile_parts=3), True),
        # T.800 A.7.4: Nppm counts the headers of the next tile-part in codestream order;
        # OpenJPEG 2.5.4 reads this arrangement in tile order instead and does not agree
        ("ppm_3parts_interleaved", dict(markers=ppm, tile_parts=3, interleave_tile_parts=1), False),
        ("4parts_interleaved", dict(tile_parts=4, interleave_tile_parts=1), True),
        ("poc_main", dict(poc=[(0, 0, 1, L + 1, 3, 0), (0, 0, NL, 2, 3, 1), (0, 0, NL, L + 1, 3, 2)]), True),
        ("poc_tile", dict(poc=[(0, 0, 2, L + 1, 3, 4), (0, 0, NL, L + 1, 2, 1), (0, 2, NL, L + 1, 3, 0)],
                          poc_in_tiles=1), True),
        ("poc_tile_ppt_sop_2parts", dict(poc=[(1, 0, NL, L + 1, 3, 2), (0, 0, NL, 1, 3, 0)], poc_in_tiles=1,
                                         markers=ppt | sop, tile_parts=2), True),
    ]


BASE = dict(reversible=1, levels=3, num_layers=3, layer_bpp=[0.5, 1.5, 0], tile_w=64, tile_h=32, cbw_exp=4, cbh_exp=4)


def encode_case(kw, img=None):
    from jpeg2000_decoder_b200 import native
    p = dict(BASE)
    p.update(kw)
    return native.encode(source() if img is None else img, 8, **p)


def _segments(cs, start):
    """Marker segments from `start` up to the first SOT: [(marker, offset, total length)]."""
    out, i = [], start
    while True:
        m = struct.unpack(">H", cs[i:i + 2])[0]
        if m == 0xFF90:
            return out, i
        n = struct.unpack(">H", cs[i + 2:i + 4])[0]
        out.append((m, i, 2 + n))
        i += 2 + n


def _tile_parts(cs, first_sot):
    """[(tile index, header markers bytes, body bytes)] in codestream order."""
    parts, i = [], first_sot
    while struct.unpack(">H", cs[i:i + 2])[0] == 0xFF90:
        isot, psot = struct.unpack(">HI", cs[i + 4:i + 10])
        j = i + 12
        while struct.unpack(">H", cs[j:j + 2])[0] != 0xFF93:
            j += 2 + struct.unpack(">H", cs[j + 2:j + 4])[0]
        parts.append((isot, cs[i + 12:j], cs[j + 2:i + psot]))
        i += psot
    return parts


def splice_tiles(cs_a, cs_b, take_b):
    """Main header of `cs_a`; the tiles t with take_b(t) come from `cs_b` with cs_b's COD
    and QCD written into their first tile-part header."""
    segs_a, sot_a = _segments(cs_a, 2)
    segs_b, sot_b = _segments(cs_b, 2)
    cod_qcd_b = b"".join(cs_b[o:o + n] for m, o, n in segs_b if m in (0xFF52, 0xFF5C))
    parts_a, parts_b = _tile_parts(cs_a, sot_a), _tile_parts(cs_b, sot_b)
    out = bytearray(cs_a[:sot_a])
    for (ta, ma, ba), (tb, mb, bb) in zip(parts_a, parts_b):
        assert ta == tb
        t, markers, body = (tb, cod_qcd_b + mb, bb) if take_b(ta) else (ta, ma, ba)
        out += struct.pack(">HHHIBB", 0xFF90, 10, t, 12 + len(markers) + 2 + len(body), 0, 1)
        out += markers + b"\xff\x93" + body
    out += b"\xff\xd9"
    return bytes(out)


def splice_cases():
    """(name, codestream, lossless) for tile-header coding overrides."""
    img = source()
    a = encode_case(dict(progression=0), img)
    b = encode_case(dict(progression=2, levels=2, num_layers=1, layer_bpp=[0], cbw_exp=5, cbh_exp=3,
                         markers=2, mode=3), img)  # RPCL, 2 levels, 32x8 blocks, EPH, BYPASS+RESET
    c = encode_case(dict(progression=1, levels=4, num_layers=2, layer_bpp=[1.0, 0], tile_w=64, tile_h=32,
                         cbw_exp=3, cbh_exp=5), img)
    return [("a_with_b_odd_tiles", splice_tiles(a, b, lambda t: t % 2 == 1)),
            ("b_with_a_even_tiles", splice_tiles(b, a, lambda t: t % 2 == 0)),
            ("a_with_c_first_row", splice_tiles(a, c, lambda t: t < W // 64))]


def transform_mismatch_stream():
    """A 5/3 stream with one tile switched to 9/7 by its tile header (refused: the device
    path runs one wavelet per image)."""
    img = source()
    a = encode_case(dict(), img)
    b = encode_case(dict(reversible=0, num_layers=1, layer_bpp=[0]), img)
    return splice_tiles(a, b, lambda t: t == 1)


def as_rgb(out, h=H, w=W):
    """24-bit output (B, G, R byte order) as (3, h, w) uint16 planes."""
    return np.ascontiguousarray(out.reshape(h, w, 3)[:, :, ::-1].transpose(2, 0, 1)).astype(np.uint16)


def random_cases(seed, n):
    """(keywords, bit depth, height, width) of `n` seeded lossless encoder configurations:
    levels 0-4, code-block sizes 4..64, 1-5 layers, mode switches (CAUSAL included), all
    progressions, tiles
    of any multiple of 2^levels (the coarsest LL band may start on an odd coordinate),
    SOP / EPH, PPM or PPT, tile-parts (interleaved or not) and POC volumes covering every
    packet."""
    import random
    from jpeg2000_decoder_b200 import native
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        L = rng.randint(0, 4)
        h, w = rng.randint(17, 120), rng.randint(17, 150)
        depth = rng.choice([8, 12])
        NL = rng.randint(1, 5)
        bpp = sorted(rng.uniform(0.3, 6) for _ in range(NL - 1)) + [0]
        kw = dict(reversible=1, levels=L, num_layers=NL, layer_bpp=bpp, cbw_exp=rng.randint(2, 6),
                  cbh_exp=rng.randint(2, 6),
                  mode=rng.choice([0, 1, 2, 3, 4, 0x08, 0x0B, 0x20, 0x2C, 0x33, 0x37, 0x2F]),
                  progression=rng.randrange(5))
        kw["cbh_exp"] = min(kw["cbh_exp"], 12 - kw["cbw_exp"])
        if rng.random() < 0.6:
            t = 1 << L
            kw["tile_w"] = t * rng.randint(max(1, 16 // t), max(2, 64 // t))
            kw["tile_h"] = t * rng.randint(max(1, 16 // t), max(2, 64 // t))
        m = (native.ENC_SOP if rng.random() < 0.4 else 0) | (native.ENC_EPH if rng.random() < 0.4 else 0)
        r = rng.random()
        m |= native.ENC_PPM if r < 0.25 else (native.ENC_PPT if r < 0.5 else 0)
        kw["markers"] = m
        if rng.random() < 0.5:
            kw["tile_parts"] = rng.randint(2, 5)
            kw["interleave_tile_parts"] = rng.randrange(2)
        if rng.random() < 0.4:
            vols = [(0, 0, rng.randint(1, NL), rng.randint(1, L + 1), rng.randint(1, 3), rng.randrange(5)),
                    (0, 0, NL, L + 1, 3, rng.randrange(5))]
            if rng.random() < 0.5:
                vols.insert(1, (rng.randint(0, L), 0, NL, L + 1, 3, rng.randrange(5)))
            kw["poc"] = vols
            kw["poc_in_tiles"] = rng.randrange(2)
        out.append((kw, depth, h, w))
    return out


def random_case_stream(seed, i, kw, depth, h, w):
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fractal_rgb(seed * 1000 + i, h, w, bitdepth=depth)
    return img, native.encode(img, depth, **kw)


def rgb_of(out, depth, h, w):
    """Packed 24-bit (8-bit pictures) or 48-bit (12-bit pictures) output as (3, h, w)."""
    if depth == 8:
        return out.reshape(h, w, 3)[:, :, ::-1].transpose(2, 0, 1).astype(np.uint16)
    return out.view(np.uint16).reshape(h, w, 3)[:, :, ::-1].transpose(2, 0, 1) >> 4
