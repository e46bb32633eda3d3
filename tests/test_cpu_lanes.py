"""The one-block-per-lane Tier-1 machine (csrc/t1_lanes.cuh), built for the host from the
same source the device kernel compiles, against the reference's Tier-1 digests and the
oracle, block by block.  The device kernel around it (cooperative rewrite, queue) is
covered by the GPU parity tests (test_lane_form_mode_switches_shapes_and_refills and the
t1_form 3 cases)."""
import ctypes
import hashlib
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle_util
from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def lanes(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("lanes") / "liblanes_host.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-o", so, os.path.join(ROOT, "tests", "lanes_host.cpp")],
                   check=True)
    lib = ctypes.CDLL(so)
    lib.lanes_host_steps.restype = ctypes.c_ulonglong
    return lib


def _blocks(lib, plan):
    """(index, status, raw samples) of every block the lane form takes."""
    cbs = plan.cblks()
    for i in range(plan.info.num_cblks):
        cb = cbs[i]
        out = np.zeros(cb.w * cb.h, np.int32)
        rc = lib.lanes_host_block(ctypes.byref(cb), plan.bytes_ptr(), plan.seglens_ptr(),
                                  out.ctypes.data_as(ctypes.c_void_p))
        if rc != -1:
            yield i, rc, out


def _check_against_oracle(lib, cs):
    from jpeg2000_decoder_b200 import native
    plan = native.Plan(cs)
    n = 0
    for i, rc, out in _blocks(lib, plan):
        orc, want = oracle_util.oracle_block(plan, i)
        assert rc == orc and np.array_equal(out, want), ("block", i)
        n += 1
    return n


@pytest.mark.parametrize("name", [k for k, v in json.load(open(os.path.join(GOLDEN, "golden.json"))).items()
                                  if "reference_t1_sha256_16" in v])
def test_lanes_match_reference_golden(pkg, lanes, name):
    """Every code-block of the fixtures equals the reference's decode_code_block output."""
    from jpeg2000_decoder_b200 import native
    g = json.load(open(os.path.join(GOLDEN, "golden.json")))[name]
    with open(os.path.join(GOLDEN, name), "rb") as f:
        plan = native.Plan(f.read())
    seen = 0
    for i, rc, out in _blocks(lanes, plan):
        assert rc == 0
        assert hashlib.sha256(out.tobytes()).hexdigest()[:16] == g["reference_t1_sha256_16"][i], (name, i)
        seen += 1
    assert seen == g["blocks"]


def test_lanes_mode_switches_and_shapes(pkg, lanes):
    """Context reset, per-pass termination, segmentation symbols, stripe-causal contexts,
    predictable termination and their combinations; code-blocks from 4x64 to 64x64; 5/3
    and 9/7; the oracle's blocks bit for bit."""
    from jpeg2000_decoder_b200 import native, synth
    img = synth.fractal_rgb(13, 96, 160, bitdepth=12)
    for mode in (0x02, 0x04, 0x08, 0x10, 0x20, 0x06, 0x2E, 0x3E):
        cs = native.encode(img, 12, reversible=1, levels=4, cbw_exp=5, cbh_exp=5, num_layers=3, layer_bpp=[1, 3, 0],
                           mode=mode)
        assert _check_against_oracle(lanes, cs) > 0, mode
    img8 = synth.fractal_rgb(14, 70, 133)
    for cw, ch in ((6, 4), (4, 6), (3, 3), (6, 2), (2, 6), (5, 6), (2, 2)):
        cs = native.encode(img8, 8, reversible=0, levels=3, cbw_exp=cw, cbh_exp=ch, num_layers=2, layer_bpp=[1, 4],
                           mode=0x08 if cw == 3 else 0)
        assert _check_against_oracle(lanes, cs) > 0, (cw, ch)


def test_lanes_benchmark_parameters_and_random_configurations(pkg, lanes):
    """A 1080p frame with the video configuration's parameters (9/7, 512x512 tiles, three
    layers), the lossless 2048x2048 configuration's first blocks, and seeded random encoder
    configurations; bypass blocks are left to the warp forms and skipped here."""
    from jpeg2000_decoder_b200 import native, synth
    import tier2_streams as ts
    assert _check_against_oracle(lanes, native.encode(synth.fields_and_edges(3, 1080, 1920), 8,
                                                      **synth.C3_PARAMS)) > 1900
    assert _check_against_oracle(lanes, synth.c1_stream(1)) > 0
    for i, (kw, depth, h, w) in enumerate(ts.random_cases(2025, 24)):
        _, cs = ts.random_case_stream(2025, i, kw, depth, h, w)
        _check_against_oracle(lanes, cs)
