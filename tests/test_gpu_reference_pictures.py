"""The device path against pictures decoded by the reference's own CPU decoder.

Same bars as tests/test_cpu_reference_pictures.py, through the C ABI on the GPU:
  * 5/3 and RCT: bit-exact with J2K_FLAG_REF_COMPAT; the T.800 default differs only in
    the bottom 2^L - 1 rows of each tile (the reference's column-end arithmetic);
  * 9/7 + ICT (FP32 on the device): within 1 LSB of the reference's samples.  A digest
    match proves 0 LSB; otherwise the prebuilt reference library (oracle/_ref, shipped with
    the repository) decodes the picture again and the largest difference must be <= 1.
PSNR and max-abs of the lossy pictures against the FP64 9/7 synthesis are printed.
"""
import json
import os
import sys

import numpy as np
import pytest

import oracle_util
import reference_pictures as rp
from conftest import ROOT
from test_cpu_reference_pictures import (NINE_SEVEN_LSB, REF_JSON, bottom_rows, compare_with_reference,
                                         random_reference_config)

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_cpu_runner  # noqa: E402


def _golden():
    with open(REF_JSON) as f:
        return json.load(f)


def _device_decode(ctx, plan, fmt, flags):
    ctx.begin()
    slot = ctx.add(plan, fmt, flags)
    ctx.launch()
    assert ctx.sync() == 0
    rc, bad = ctx.status(slot)
    assert rc == 0 and bad == 0
    return ctx.output(slot)


def _plan(name, g):
    from jpeg2000_decoder_b200 import native
    cs = rp.stream(name)
    assert rp.sha(cs) == g["stream_sha256"], "%s: codestream differs from the one the reference decoded" % name
    levels = native.Plan(cs).info.levels
    return cs, native.Plan(cs, discard_levels=rp.discard_of(levels, g["top_level"]))


@pytest.mark.parametrize("name", sorted(_golden()))
def test_device_matches_reference_picture(gpu_ctx, name):
    from jpeg2000_decoder_b200 import native
    g = _golden()[name]
    cs, plan = _plan(name, g)
    flags = native.FLAG_REF_COMPAT if g["ref_compat"] else 0
    out = _device_decode(gpu_ctx, plan, g["format"], flags)
    if not g["reversible"] and plan.info.levels:
        ps, mx = oracle_util.psnr_maxabs(_unpack(out, g, plan), oracle_util.fp64_decode(plan), plan.info.bitdepth)
        print("%s: PSNR %.2f dB, max-abs %.2f vs FP64 9/7" % (name, ps, mx))
    if rp.sha(out) == g["output_sha256"]:
        return
    assert not g["reversible"], "%s: 5/3 picture differs from the reference's" % name
    if not ref_cpu_runner.available():
        pytest.fail("%s differs from the reference digest and no reference library is here to count LSBs" % name)
    r = ref_cpu_runner.decode([cs], g["format"], threads=1, top_level=g["top_level"], timeout=300)
    assert r["ok"], r["error"]
    d = compare_with_reference(out, r["outputs"][0], g["format"], False)
    assert d <= NINE_SEVEN_LSB


def _unpack(out, g, plan):
    """(ncomp, H, W) samples at the component bit depth from a packed picture."""
    I = plan.info
    fmt = g["format"]
    if fmt == 3:  # one component in the last byte of each 32-bit pixel, 8-bit container
        return out.reshape(I.height, I.width, 4)[:, :, 3][None].astype(np.float64) * (1 << max(0, I.bitdepth - 8))
    wide = fmt == 1  # 16-bit container, B, G, R
    px = (np.frombuffer(out.tobytes(), np.uint16) if wide else out).reshape(I.height, I.width, -1)
    v = px[:, :, [2, 1, 0]].transpose(2, 0, 1).astype(np.float64)  # B, G, R(, A) in memory for formats 0, 1, 2
    return v / (1 << (16 - I.bitdepth)) if wide else v


@pytest.mark.parametrize("name", sorted(k for k, v in _golden().items() if v["reversible"]))
def test_device_t800_differs_only_in_reference_defect_rows(gpu_ctx, name):
    g = _golden()[name]
    _, plan = _plan(name, g)
    out = _device_decode(gpu_ctx, plan, g["format"], 0)
    got = rp.row_digests(out, g["height"])
    bad = [y for y, (a, b) in enumerate(zip(got, g["row_sha256_16"])) if a != b]
    L = plan.tilecomps()[0].levels
    th = plan.info.tile_h if plan.info.ntiles_y > 1 else g["height"]
    allowed = {y for y in range(g["height"]) if y % th >= th - bottom_rows(L)}
    assert bad and set(bad) <= allowed, (name, bad[:8])


def test_device_matches_live_reference_on_random_configurations(gpu_ctx):
    """Seeded random configurations inside the reference's valid domain, decoded by the
    prebuilt reference library on the host and by the device path."""
    if not ref_cpu_runner.available():
        pytest.skip("the reference's CPU decoder (oracle/_ref/libref_cpu.so) is not present")
    from jpeg2000_decoder_b200 import native
    worst = 0
    for seed in range(800, 824):
        cs, fmt, rev = random_reference_config(seed)
        r = ref_cpu_runner.decode([cs], fmt, threads=1, timeout=120)  # single-worker engine: its workers race
        assert r["ok"], (seed, r["error"])
        out = _device_decode(gpu_ctx, native.Plan(cs), fmt, native.FLAG_REF_COMPAT if rev else 0)
        worst = max(worst, compare_with_reference(out, r["outputs"][0], fmt, rev))
    print("device vs live reference, 24 random configurations: max |d| =", worst)
