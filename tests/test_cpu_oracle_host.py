"""CPU-only tests: the oracle pinned to the reference's own Tier-1 (golden digests), the
lossless and mode-switch round trips, the host Tier-2 front end, the C-ABI exports and the
replica sharding used by multi-GPU runs.  No compute call touches a GPU here."""
import ctypes
import hashlib
import io
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle_util
from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def _read(name):
    with open(os.path.join(GOLDEN, name), "rb") as f:
        return f.read()


@pytest.mark.parametrize("name", [k for k, v in json.load(open(os.path.join(GOLDEN, "golden.json"))).items()
                                  if "reference_t1_sha256_16" in v])
def test_oracle_t1_matches_reference_golden(pkg, name):
    """Every code-block decoded by the oracle equals the reference's decode_code_block."""
    from jpeg2000_decoder_b200 import native
    g = _golden()[name]
    plan = native.Plan(_read(name))
    assert plan.info.num_cblks == g["blocks"]
    for i, want in enumerate(g["reference_t1_sha256_16"]):
        rc, out = oracle_util.oracle_block(plan, i)
        assert rc == 0
        assert hashlib.sha256(out.tobytes()).hexdigest()[:16] == want, (name, i)


def test_oracle_t1_matches_live_reference(pkg):
    """When the reference's Tier-1 is built here, compare it live on fresh streams."""
    if oracle_util.ref_t1() is None:
        pytest.skip("reference Tier-1 build (oracle/_ref) not present")
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fields_and_edges(21, 192, 160)
    streams = [native.encode(img, 8, **synth.C2_PARAMS),
               native.encode(img, 8, reversible=1, levels=4, cbw_exp=5, cbh_exp=5),
               native.encode(img[:1], 8, reversible=0, levels=3, cbw_exp=4, cbh_exp=6, layer_bpp=[0])]
    for cs in streams:
        plan = native.Plan(cs)
        for i in range(plan.info.num_cblks):
            a = oracle_util.oracle_block(plan, i)
            b = oracle_util.reference_block(plan, i)
            assert a[0] == 0 and b[0] == 0
            assert np.array_equal(a[1], b[1]), i


def test_c1_lossless_identity(pkg):
    from jpeg2000_decoder_b200 import native, synth
    src = synth.sinusoid_gray(1)
    cs = _read("c1_gray_53.j2k")
    assert cs == synth.c1_stream(1)  # the fixture is reproducible from its seed
    plan = native.Plan(cs)
    rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_32BITS_4COMPONENTS)
    assert rc == 0
    gray = out.reshape(512, 512, 4)[:, :, 3]
    assert np.array_equal(gray, src[0])


def test_ref_compat_reproduces_reference_bottom_rows(pkg):
    """With the reference's column-end arithmetic the bottom 2^L - 1 rows differ (L = 5)."""
    from jpeg2000_decoder_b200 import native, synth
    src = synth.sinusoid_gray(1)[0]
    plan = native.Plan(_read("c1_gray_53.j2k"))
    rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_32BITS_4COMPONENTS, ref_compat=1)
    gray = out.reshape(512, 512, 4)[:, :, 3]
    bad_rows = np.nonzero((gray != src).any(axis=1))[0]
    assert bad_rows.min() == 512 - 31 and len(bad_rows) == 31


@pytest.mark.parametrize("mode", [0x00, 0x01, 0x02, 0x03, 0x04, 0x07, 0x20, 0x23])
def test_mode_switch_lossless_roundtrip(pkg, mode):
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fractal_rgb(31 + mode, 72, 136)
    cs = native.encode(img, 12, **dict(synth.C4_PARAMS, mode=mode))
    plan = native.Plan(cs)
    rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_48BITS_RGB)
    assert rc == 0
    rgb = out.view(np.uint16).reshape(72, 136, 3)[:, :, ::-1].transpose(2, 0, 1) >> 4
    assert np.array_equal(rgb, img)


def test_encoder_streams_decode_with_openjpeg(pkg):
    """Independent cross-check of the test encoder: OpenJPEG (via Pillow) decodes it."""
    PIL = pytest.importorskip("PIL.Image")
    from jpeg2000_decoder_b200 import synth
    src = synth.sinusoid_gray(1)[0]
    dec = np.array(PIL.open(io.BytesIO(_read("c1_gray_53.j2k"))))
    assert np.array_equal(dec, src)
    rgb = np.array(PIL.open(io.BytesIO(_read("rgb256_53_rct.j2k")))).transpose(2, 0, 1)
    assert np.array_equal(rgb, synth.fields_and_edges(11, 256, 256))


def test_97_oracle_vs_fp64_and_openjpeg(pkg):
    """FP32 reference arithmetic vs an FP64 synthesis of the same Tier-1 output."""
    from jpeg2000_decoder_b200 import native
    plan = native.Plan(_read("rgb256_97_1bpp.j2k"))
    rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_24BITS_RGB)
    assert rc == 0
    rgb = out.reshape(256, 256, 3)[:, :, ::-1].transpose(2, 0, 1)
    ref64 = oracle_util.fp64_decode(plan)
    psnr, maxabs = oracle_util.psnr_maxabs(rgb, ref64, 8)
    # (int) truncation of the reference costs < 1 LSB; its plane-0 rule can add a few LSB
    assert psnr > 45 and maxabs <= 8


def test_plan_geometry_and_tiers(pkg):
    from jpeg2000_decoder_b200 import native
    plan = native.Plan(_read("rgb300x200_97_tiles_3layers.j2k"))
    I = plan.info
    assert (I.width, I.height, I.ncomp, I.levels, I.layers) == (300, 200, 3, 5, 3)
    assert I.ntiles_x * I.ntiles_y == 6 and I.num_tilecomps == 18
    tcs = plan.tilecomps()
    assert sum(t.w * t.h for t in tcs) == I.coef_elems == 300 * 200 * 3
    for cb in plan.cblks():
        assert 1 <= cb.w <= 64 and 1 <= cb.h <= 64 and cb.out_off + (cb.h - 1) * cb.out_stride + cb.w <= I.coef_elems
    # fewer layers decode fewer passes; reduced resolution shrinks the output
    few = native.Plan(_read("rgb300x200_97_tiles_3layers.j2k"), max_layers=1)
    assert sum(c.num_passes for c in few.cblks()) < sum(c.num_passes for c in plan.cblks())
    small = native.Plan(_read("rgb300x200_97_tiles_3layers.j2k"), discard_levels=2)
    assert (small.info.width, small.info.height) == (75, 50)


def test_parser_rejects_or_survives_corrupt_input(pkg):
    from jpeg2000_decoder_b200 import native
    cs = bytearray(_read("rgb256_97_1bpp.j2k"))
    with pytest.raises(native.J2kError):
        native.Plan(b"\x00\x01\x02\x03")
    with pytest.raises(native.J2kError):
        native.Plan(bytes(cs[:40]))  # main header cut
    # a truncated tile body plans (missing packets are empty) and decodes without error
    plan = native.Plan(bytes(cs[: len(cs) // 2]))
    rc, out, _ = oracle_util.oracle_decode(plan, native.FMT_24BITS_RGB)
    assert out.size == 256 * 256 * 3
    # random corruption of packet bodies: the oracle must stay in bounds
    rng = np.random.default_rng(0)
    for _ in range(5):
        bad = bytearray(cs)
        for pos in rng.integers(len(cs) // 4, len(cs), 20):
            bad[pos] = int(rng.integers(0, 256))
        try:
            plan = native.Plan(bytes(bad))
        except native.J2kError:
            continue
        oracle_util.oracle_decode(plan, native.FMT_24BITS_RGB)


def _declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:BMI::Status|int|void|size_t|const char \*|const [a-z0-9_]+ \*)\s*\**\s*"
                             r"([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_c_abi_library_exports_every_declared_symbol(pkg):
    from jpeg2000_decoder_b200 import native
    lib = native.lib()
    declared = _declared_functions()
    assert {"j2k_gpu_batch_launch", "BMI_dec", "bmi_decoder_decode", "j2k_plan_create"} <= declared
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True).stdout
    assert "_ZN3BMI7Decoder3GetEv" in out and "_ZN3BMI7Decoder9TerminateEv" in out


def test_no_cpu_fallback_without_device(pkg):
    from jpeg2000_decoder_b200 import native
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(native.J2kError) as e:
        native.GpuContext()
    assert e.value.code == native.J2K_ERR_NODEVICE
    # the reference-facing C API reports failure instead of decoding on the CPU
    assert native.lib().bmi_decoder_init(1, 1) != 0
    with pytest.raises(native.J2kError) as e:
        native.Server()
    assert e.value.code == native.J2K_ERR_NODEVICE


def test_noalloc_idwt_refuses_inconsistent_resolution_tables(pkg):
    """The allocation-free inverse DWT checks a hand-built tile-component description
    before it enqueues anything: resolutions that do not nest inside the tile-component (a
    full resolution other than the tile size, a level larger than the next finer one, or
    not half of it) return J2K_ERR_ARG.  No device is touched, so this runs on the CPU."""
    import ctypes
    from jpeg2000_decoder_b200 import native
    fn = native.lib().j2k_gpu_tile_idwt_noalloc

    def tc_with(res_w, res_h, w=64, h=48):
        tc = native.TileComp()
        tc.w, tc.h, tc.levels = w, h, len(res_w) - 1
        for r, (a, b) in enumerate(zip(res_w, res_h)):
            tc.res_w[r], tc.res_h[r] = a, b
        return tc

    bad_tables = [([16, 32, 65], [12, 24, 48]),    # full resolution wider than the tile-component
                  ([16, 32, 64], [12, 24, 4096]),  # full resolution taller than the caller's buffer
                  ([40, 32, 64], [12, 24, 48]),    # a coarser level wider than the next finer one
                  ([16, 20, 64], [12, 24, 48]),    # a level that is not half of the next one
                  ([-1, 32, 64], [12, 24, 48])]    # negative size
    for res_w, res_h in bad_tables:
        tc = tc_with(res_w, res_h)
        rc = fn(ctypes.byref(tc), 1, 0, ctypes.c_void_p(16), ctypes.c_void_p(16), 64, None)
        assert rc == native.J2K_ERR_ARG, (res_w, res_h, rc)
