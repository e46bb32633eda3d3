"""Host Tier-2 front end on streams beyond the benchmark configurations (CPU only).

Every stream is planned by the library (j2k_plan_create) and decoded by the oracle from that
plan; the checks are the lossless identity with the source picture, or, for the 9/7
fixture written by OpenJPEG, agreement with OpenJPEG's own decode within one level.
Covered: several precincts per resolution under all five progression orders (T.800
B.12.1.1-B.12.1.5), precinct-limited code-block sizes, POC volumes in the main and tile-part
headers, PPM / PPT packed packet headers, SOP / EPH markers, tile-parts (also interleaved
across tiles), tile-part COD / QCD overriding the main header, and the T.800 magnitude bit
count for 9/7 bands with two guard bits (E.1.1.1).
"""
import io
import json
import os

import numpy as np
import pytest

import oracle_util
import tier2_streams as ts
from conftest import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "tier2")


@pytest.fixture(scope="module")
def pkg():
    from conftest import load_package
    return load_package()


def _manifest():
    with open(os.path.join(FIX, "manifest.json")) as f:
        return json.load(f)


def _oracle_rgb(cs, h, w):
    from jpeg2000_decoder_b200 import native
    plan = native.Plan(cs)
    rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_24BITS_RGB)
    assert rc == 0
    return out.reshape(h, w, 3)[:, :, ::-1]


@pytest.mark.parametrize("name", sorted(_manifest()["streams"]))
def test_openjpeg_precinct_fixtures(pkg, name):
    man = _manifest()
    exp = np.load(os.path.join(FIX, "expected.npz"))
    spec = man["streams"][name]
    with open(os.path.join(FIX, name), "rb") as f:
        cs = f.read()
    rgb = _oracle_rgb(cs, man["height"], man["width"]).astype(int)
    want = exp[spec["expect"]].astype(int)
    tol = spec.get("tolerance", 0)
    assert np.abs(rgb - want).max() <= tol, name


@pytest.mark.parametrize("case", ts.marker_cases(), ids=lambda c: c[0])
def test_marker_variants_lossless(pkg, case):
    name, kw, openjpeg_agrees = case
    cs = ts.encode_case(kw)
    src = ts.source()
    rgb = _oracle_rgb(cs, ts.H, ts.W)
    assert np.array_equal(rgb.transpose(2, 0, 1), src), name
    if openjpeg_agrees:  # the stream itself is valid: an independent decoder reads it
        Image = pytest.importorskip("PIL.Image")
        ref = np.asarray(Image.open(io.BytesIO(cs)).convert("RGB"))
        assert np.array_equal(ref.transpose(2, 0, 1), src), name


@pytest.mark.parametrize("case", ts.splice_cases(), ids=lambda c: c[0])
def test_tile_header_coding_overrides(pkg, case):
    name, cs = case
    rgb = _oracle_rgb(cs, ts.H, ts.W)
    assert np.array_equal(rgb.transpose(2, 0, 1), ts.source()), name
    Image = pytest.importorskip("PIL.Image")
    ref = np.asarray(Image.open(io.BytesIO(cs)).convert("RGB"))
    assert np.array_equal(ref.transpose(2, 0, 1), ts.source()), name


def test_refusals(pkg):
    """A tile that switches the wavelet, POC with a broken length, signed samples, PPM and PPT
    together."""
    from jpeg2000_decoder_b200 import native
    with pytest.raises(native.J2kError) as e:
        native.Plan(ts.transform_mismatch_stream())
    assert e.value.code == native.J2K_ERR_UNSUPPORTED
    cs = bytearray(ts.encode_case(dict(poc=[(0, 0, 3, 4, 3, 0)])))
    i = cs.find(b"\xff\x5f")
    cs[i + 3] += 1  # Lpoc no longer a whole number of entries
    with pytest.raises(native.J2kError):
        native.Plan(bytes(cs))
    signed = bytearray(ts.encode_case(dict()))
    i = signed.find(b"\xff\x51") + 40  # Ssiz of component 0
    signed[i] |= 0x80
    with pytest.raises(native.J2kError) as e:
        native.Plan(bytes(signed))
    assert e.value.code == native.J2K_ERR_UNSUPPORTED
    ppm = ts.encode_case(dict(markers=native.ENC_PPM))
    ppt = ts.encode_case(dict(markers=native.ENC_PPT))
    segs, sot = ts._segments(ppm, 2)
    with pytest.raises(native.J2kError):
        native.Plan(ppm[:sot] + ppt[ts._segments(ppt, 2)[1]:])


def test_cinema_profile_poc_and_tile_parts(pkg):
    """OpenJPEG's 2K digital-cinema profile: CPRL, precincts, 32x32 blocks, two guard
    bits, a POC in the first tile-part header, TLM and one tile-part per resolution."""
    Image = pytest.importorskip("PIL.Image")
    from jpeg2000_decoder_b200 import native, synth
    src = np.ascontiguousarray(np.moveaxis(synth.fields_and_edges(12, 1080, 2048).astype(np.uint8), 0, -1))
    f = io.BytesIO()
    Image.fromarray(src, "RGB").save(f, "JPEG2000", no_jp2=True, cinema_mode="cinema2k-24")
    cs = f.getvalue()
    assert b"\xff\x5f" in cs  # POC present
    plan = native.Plan(cs)
    assert plan.info.progression == 4 and plan.info.guard_bits == 2
    rgb = _oracle_rgb(cs, 1080, 2048).astype(int)
    ref = np.asarray(Image.open(io.BytesIO(cs)).convert("RGB")).astype(int)
    assert np.abs(rgb - ref).max() <= 1


def test_large_plans_threaded_copy_and_concurrency(pkg):
    """A plan of more than 4 MB of coded bytes copies them on several threads and recycles
    its buffer; plans made concurrently from several threads are identical, and the picture
    decodes to its source."""
    import ctypes
    import hashlib
    from concurrent.futures import ThreadPoolExecutor
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fractal_rgb(7, 768, 1536, bitdepth=12)
    cs = native.encode(img, 12, reversible=1, levels=5, cbw_exp=5, cbh_exp=5, num_layers=4,
                       layer_bpp=[1, 3, 6, 0], progression=2, mode=3)
    assert len(cs) > (4 << 20)

    def digest(_):
        p = native.Plan(cs)
        h = hashlib.sha1(ctypes.string_at(native.lib().j2k_plan_bytes(p.h), p.info.coded_bytes))
        h.update(bytes(p.cblks()))
        h.update(ctypes.string_at(native.lib().j2k_plan_seglens(p.h), 4 * p.info.num_segs))
        return h.hexdigest()

    with ThreadPoolExecutor(8) as ex:
        digests = list(ex.map(digest, range(16)))
    assert len(set(digests)) == 1
    plan = native.Plan(cs)
    rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_48BITS_RGB)
    assert rc == 0
    rgb = out.view(np.uint16).reshape(768, 1536, 3)[:, :, ::-1].transpose(2, 0, 1) >> 4
    assert np.array_equal(rgb, img)


def test_mutated_streams_are_planned_or_refused(pkg):
    """Seeded corruptions (bytes flipped in the headers or anywhere, truncations, runs
    inserted or deleted) of the Tier-2 variant streams: every call returns a plan or an
    error code, never an exception through the C ABI or a crash, and a tenth of the plans
    also go through the oracle's decode."""
    import random
    from jpeg2000_decoder_b200 import native
    seeds = []
    for name in sorted(os.listdir(FIX)):
        if name.endswith(".j2k"):
            with open(os.path.join(FIX, name), "rb") as f:
                seeds.append(f.read())
    seeds += [ts.encode_case(kw) for _, kw, _ in ts.marker_cases()]
    seeds += [cs for _, cs in ts.splice_cases()]
    rng = random.Random(1234)
    planned = refused = 0
    for _ in range(1500):
        cs = bytearray(rng.choice(seeds))
        kind = rng.randrange(4)
        if kind == 0:
            for _ in range(rng.randint(1, 4)):
                cs[rng.randrange(min(len(cs), 400))] = rng.randrange(256)
        elif kind == 1:
            for _ in range(rng.randint(1, 16)):
                cs[rng.randrange(len(cs))] = rng.randrange(256)
        elif kind == 2:
            cs = cs[: rng.randrange(2, len(cs))]
        else:
            j = rng.randrange(len(cs))
            if rng.random() < 0.5:
                cs[j:j] = bytes(rng.randrange(256) for _ in range(rng.randint(1, 8)))
            else:
                del cs[j:j + rng.randint(1, 8)]
        try:
            plan = native.Plan(bytes(cs))
        except native.J2kError:
            refused += 1
            continue
        planned += 1
        if rng.random() < 0.1 and plan.info.coef_elems < (1 << 24):
            oracle_util.oracle_decode(plan, native.FMT_NONE)
    assert planned > 0 and refused > 0


def test_randomized_encoder_roundtrips(pkg):
    """120 seeded lossless configurations (levels, block sizes, layers, mode switches,
    progressions, tilings, SOP/EPH, PPM/PPT, tile-parts, POC) decode to their sources."""
    from jpeg2000_decoder_b200 import native
    for i, (kw, depth, h, w) in enumerate(ts.random_cases(2024, 120)):
        img, cs = ts.random_case_stream(2024, i, kw, depth, h, w)
        plan = native.Plan(cs)
        fmt = native.FMT_24BITS_RGB if depth == 8 else native.FMT_48BITS_RGB
        rc, out, _ = oracle_util.oracle_decode(plan, fmt)
        assert rc == 0, (i, kw)
        assert np.array_equal(ts.rgb_of(out, depth, h, w), img), (i, kw)


def test_image_and_tile_origins(pkg):
    """Image and tile-grid origins other than (0, 0): the picture is the grid from the image
    origin, reduced resolutions have T.800's ceil(Xsiz / 2^d) - ceil(XOsiz / 2^d) columns, and
    an origin that makes a synthesised resolution start on an odd coordinate is refused."""
    from jpeg2000_decoder_b200 import native
    with open(os.path.join(FIX, "ojp_offset32x16_tileorigin16x8_lrcp.j2k"), "rb") as f:
        cs = f.read()
    man = _manifest()
    for d in (0, 1, 2, 3):
        plan = native.Plan(cs, discard_levels=d)
        W, H = man["width"] + 32, man["height"] + 16  # Xsiz, Ysiz
        assert (plan.info.width, plan.info.height) == (-(-W // 2 ** d) - (-(-32 // 2 ** d)),
                                                         -(-H // 2 ** d) - (-(-16 // 2 ** d)))
        rc, _, _ = oracle_util.oracle_decode(plan, native.FMT_24BITS_RGB)
        assert rc == 0
    Image = pytest.importorskip("PIL.Image")
    src = np.load(os.path.join(FIX, "expected.npz"))["source"]
    f = io.BytesIO()
    Image.fromarray(src, "RGB").save(f, "JPEG2000", no_jp2=True, offset=(33, 16), tile_offset=(16, 8),
                                     tile_size=(64, 48), num_resolutions=4)
    with pytest.raises(native.J2kError) as e:
        native.Plan(f.getvalue())
    assert e.value.code == native.J2K_ERR_UNSUPPORTED


def test_threaded_tiles_give_identical_plans(pkg):
    """The Tier-2 of a multi-tile picture spread over several host threads
    (j2k_plan_create_mt) gives the same plan as one thread, at full and reduced resolution."""
    import ctypes
    import hashlib
    from jpeg2000_decoder_b200 import native

    def digest(cs, threads, discard):
        p = native.Plan(cs, discard_levels=discard, threads=threads)
        I = p.info
        h = hashlib.sha1(bytes(I))
        h.update(ctypes.string_at(native.lib().j2k_plan_bytes(p.h), I.coded_bytes))
        h.update(bytes(p.cblks()))
        h.update(ctypes.string_at(native.lib().j2k_plan_seglens(p.h), 4 * I.num_segs))
        h.update(ctypes.string_at(native.lib().j2k_plan_tilecomps(p.h), I.num_tilecomps * ctypes.sizeof(native.TileComp)))
        return h.hexdigest()

    streams = [ts.encode_case(kw) for _, kw, _ in ts.marker_cases()] + [cs for _, cs in ts.splice_cases()]
    streams += [ts.random_case_stream(77, i, *c)[1] for i, c in enumerate(ts.random_cases(77, 20))]
    for cs in streams:
        for discard in (0, 1):
            want = digest(cs, 1, discard)
            for threads in (2, 5):
                assert digest(cs, threads, discard) == want


@pytest.mark.parametrize("mode", [0x08, 0x09, 0x0E, 0x28, 0x2F])
def test_causal_mode_streams(pkg, mode):
    """CAUSAL (T.800 D.7), alone and with the other mode switches: OpenJPEG decodes the
    encoder's stream to its source (the contexts are the standard's), and so does the
    oracle from the library's plan."""
    from jpeg2000_decoder_b200 import native
    img = ts.source()
    cs = native.encode(img, 8, reversible=1, levels=3, cbw_exp=4, cbh_exp=5, mode=mode, num_layers=2,
                       layer_bpp=[1.0, 0])
    assert np.array_equal(_oracle_rgb(cs, ts.H, ts.W).transpose(2, 0, 1), img)
    Image = pytest.importorskip("PIL.Image")
    ref = np.asarray(Image.open(io.BytesIO(cs)).convert("RGB"))
    assert np.array_equal(ref.transpose(2, 0, 1), img)


def test_plain_c_caller_of_the_c_abi(pkg):
    """A C99 program including every public header, linked against the library, plans a
    codestream through the C ABI (one and three threads give the same plan), sees the
    error codes, and gets J2K_ERR_NODEVICE (or a context, on a GPU host) for a device
    context."""
    import shutil
    import subprocess
    from jpeg2000_decoder_b200 import native
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no C compiler")
    out_dir = os.path.join(ROOT, "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "c_abi_consumer")
    lib_dir = os.path.dirname(native.LIB_PATH)
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_abi_consumer.c"), "-L", lib_dir, "-l:" + os.path.basename(native.LIB_PATH),
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    name = os.path.join(ROOT, "tests", "golden", "rgb300x200_97_tiles_3layers.j2k")
    r = subprocess.run([exe, name], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    w, h, ncomp, cblks, coded, ctx_rc = (int(x) for x in r.stdout.split())
    plan = native.Plan(open(name, "rb").read())
    assert (w, h, ncomp, cblks, coded) == (plan.info.width, plan.info.height, plan.info.ncomp,
                                           plan.info.num_cblks, plan.info.coded_bytes)
    assert ctx_rc in (native.J2K_OK, native.J2K_ERR_NODEVICE)


def test_plan_builder_under_sanitizers(pkg):
    """The plan builder built with AddressSanitizer + UndefinedBehaviorSanitizer plans or
    refuses 1500 seeded corruptions of the Tier-2 variant streams without a report."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    out_dir = os.path.join(ROOT, "_build", "asan")
    seed_dir = os.path.join(out_dir, "seeds")
    os.makedirs(seed_dir, exist_ok=True)
    streams = []
    for name in sorted(os.listdir(FIX)):
        if name.endswith(".j2k"):
            with open(os.path.join(FIX, name), "rb") as f:
                streams.append(f.read())
    streams += [ts.encode_case(kw) for _, kw, _ in ts.marker_cases()]
    streams += [ts.random_case_stream(99, i, *c)[1] for i, c in enumerate(ts.random_cases(99, 12))]
    for i, cs in enumerate(streams):
        with open(os.path.join(seed_dir, "s%03d.j2k" % i), "wb") as f:
            f.write(cs)
    csrc = os.path.join(ROOT, "jpeg2000-decoder_b200", "csrc")
    exe = os.path.join(out_dir, "asan_plan_fuzz")
    srcs = [os.path.join(ROOT, "tests", "asan_plan_fuzz.cpp"), os.path.join(csrc, "codestream.cpp"),
            os.path.join(csrc, "plan_api.cpp")]
    deps = srcs + [os.path.join(csrc, "codestream.h"), os.path.join(csrc, "plan.h"),
                   os.path.join(ROOT, "include", "j2k_gpu.h")]
    if not os.path.exists(exe) or os.path.getmtime(exe) < max(os.path.getmtime(d) for d in deps):
        build = subprocess.run([gxx, "-O1", "-g", "-std=c++17", "-pthread", "-fsanitize=address,undefined",
                                "-fno-omit-frame-pointer", "-I", os.path.join(ROOT, "include"), "-I", csrc] + srcs +
                               ["-o", exe], capture_output=True, text=True)
        if build.returncode != 0 and "sanitize" in build.stderr:
            pytest.skip("no sanitizer runtime")
        assert build.returncode == 0, build.stderr[-2000:]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe, seed_dir, "7", "1500"], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and "planned" in r.stdout, (r.stdout + r.stderr)[-3000:]


@pytest.mark.parametrize("depth", [1, 2, 15, 16])
def test_bit_depth_extremes_lossless(pkg, depth):
    """1, 2, 15 and 16-bit lossless pictures (with and without BYPASS+RESET) decode to
    their sources through the plan and the oracle."""
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fractal_rgb(3, 70, 90, bitdepth=depth)
    for mode in (0, 3):
        cs = native.encode(img, depth, reversible=1, levels=3, mode=mode)
        rc, out, _ = oracle_util.oracle_decode(native.Plan(cs), native.FMT_48BITS_RGB)
        assert rc == 0
        rgb = out.view(np.uint16).reshape(70, 90, 3)[:, :, ::-1].transpose(2, 0, 1) >> (16 - depth)
        assert np.array_equal(rgb, img), (depth, mode)


@pytest.mark.parametrize("kw", [dict(), dict(tile_size=(64, 48), num_resolutions=4),
                                dict(precinct_size=(32, 32), codeblock_size=(16, 16), progression="PCRL",
                                     num_resolutions=4),
                                dict(precinct_size=(16, 16), codeblock_size=(8, 8), progression="RPCL",
                                     tile_size=(64, 64), num_resolutions=3)],
                         ids=["one_tile", "tiles", "precincts_pcrl", "precincts_rpcl_tiles"])
def test_openjpeg_16bit_gray_identical(pkg, kw):
    """16-bit grayscale 5/3 streams written by OpenJPEG: the plan + oracle reconstruct the
    same integers as OpenJPEG's own decoder (checked against its decode rather than the
    source, which OpenJPEG's writer does not reproduce exactly for every tiling)."""
    Image = pytest.importorskip("PIL.Image")
    import warnings
    from jpeg2000_decoder_b200 import native, synth
    g = synth.fractal_rgb(5, 90, 120, bitdepth=16)[0].astype(np.uint16)
    f = io.BytesIO()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", DeprecationWarning)
        Image.fromarray(g, "I;16").save(f, "JPEG2000", no_jp2=True, **kw)
    cs = f.getvalue()
    ref = np.asarray(Image.open(io.BytesIO(cs))).astype(np.int64)
    plan = native.Plan(cs)
    I = plan.info
    assert (I.bitdepth, I.ncomp, I.reversible) == (16, 1, 1)
    rc, _, comp = oracle_util.oracle_decode(plan, native.FMT_NONE)
    assert rc == 0
    img = np.zeros((I.height, I.width), np.int64)
    for tc in plan.tilecomps():
        img[tc.y0:tc.y0 + tc.h, tc.x0:tc.x0 + tc.w] = comp[tc.coef_off:tc.coef_off + tc.w * tc.h].reshape(tc.h, tc.w)
    assert np.array_equal(img + (1 << 15), ref)


@pytest.mark.parametrize("kw", [dict(quality_layers=[8], quality_mode="rates"),
                                dict(quality_layers=[3], quality_mode="rates", tile_size=(64, 64), num_resolutions=4),
                                dict()], ids=["rate8", "rate3_tiles", "near_lossless"])
def test_openjpeg_16bit_gray_97_within_two(pkg, kw):
    """16-bit grayscale 9/7 streams written by OpenJPEG (two guard bits): the oracle's float
    reconstruction, rounded, is within 2 of OpenJPEG's decode out of 65535 (the two 9/7
    implementations order their float operations differently)."""
    Image = pytest.importorskip("PIL.Image")
    import warnings
    from jpeg2000_decoder_b200 import native, synth
    g = synth.fractal_rgb(5, 90, 120, bitdepth=16)[0].astype(np.uint16)
    f = io.BytesIO()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", DeprecationWarning)
        Image.fromarray(g, "I;16").save(f, "JPEG2000", no_jp2=True, irreversible=True, **kw)
    cs = f.getvalue()
    ref = np.asarray(Image.open(io.BytesIO(cs))).astype(np.int64)
    plan = native.Plan(cs)
    I = plan.info
    rc, _, comp = oracle_util.oracle_decode(plan, native.FMT_NONE)
    assert rc == 0 and I.reversible == 0
    img = np.zeros((I.height, I.width), np.float64)
    for tc in plan.tilecomps():
        img[tc.y0:tc.y0 + tc.h, tc.x0:tc.x0 + tc.w] = \
            comp.view(np.float32)[tc.coef_off:tc.coef_off + tc.w * tc.h].reshape(tc.h, tc.w)
    ours = np.clip(np.floor(img + 0.5) + (1 << 15), 0, 65535).astype(np.int64)
    assert np.abs(ours - ref).max() <= 2


@pytest.mark.parametrize("kw", [dict(), dict(tile_size=(64, 48), precinct_size=(32, 32), codeblock_size=(16, 16),
                                             progression="CPRL", num_resolutions=4)], ids=["one_tile", "tiles_cprl"])
def test_openjpeg_rgba_four_components(pkg, kw):
    """4-component (RGBA) streams written by OpenJPEG decode exactly into both 32-bit packed
    formats, component c in byte 3 - c (the layout of the reference's 4-component merge)."""
    Image = pytest.importorskip("PIL.Image")
    from jpeg2000_decoder_b200 import native, synth
    rgb = np.moveaxis(synth.fields_and_edges(8, 70, 90).astype(np.uint8), 0, -1)
    a = synth.fractal_rgb(9, 70, 90, bitdepth=8)[0].astype(np.uint8)
    rgba = np.ascontiguousarray(np.dstack([rgb, a]))
    f = io.BytesIO()
    Image.fromarray(rgba, "RGBA").save(f, "JPEG2000", no_jp2=True, **kw)
    plan = native.Plan(f.getvalue())
    assert plan.info.ncomp == 4
    for fmt in (native.FMT_32BITS_ARGB, native.FMT_32BITS_4COMPONENTS):
        rc, out, _ = oracle_util.oracle_decode(plan, fmt)
        assert rc == 0
        assert np.array_equal(out.reshape(70, 90, 4)[:, :, ::-1], rgba)
