"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Run where the reference tree is available (its root as the argument or in
J2K_REFERENCE_DIR); it builds oracle/_ref/libref_t1.so (oracle/build_ref.sh) and
oracle/_ref/libref_cpu.so (oracle/build_ref_cpu.sh) from that tree:

    python tests/golden/make_golden.py <reference root>

golden.json: for each fixture codestream (the project's writer; the OpenJPEG-written
streams of tier2/ that use no mode switch), the SHA-256 of the reference's Tier-1
(decode_code_block, bmi_block_decoder.cpp:589-853) output for every code-block.

reference_pictures.json: for each picture of tests/reference_pictures.py, the reference's
whole CPU decoder (BMI::Decoder: Tier-2, Tier-1, dequantisation, inverse DWT, inverse
MCT, DC shift, pack) decodes the codestream; the SHA-256 of the packed output (and, for
5/3 pictures, of each output row) is recorded with the codestream's own SHA-256.

The GPU box has no reference tree; the tests compare the oracle and the device path with
these digests (and with the prebuilt oracle/_ref libraries where they travelled along).
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)
sys.path.insert(0, TESTS)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from conftest import load_package  # noqa: E402

load_package()
from jpeg2000_decoder_b200 import build, native, synth  # noqa: E402
import oracle_util  # noqa: E402
import ref_cpu_runner  # noqa: E402
import reference_pictures as rp  # noqa: E402


def fixtures():
    yield "c1_gray_53.j2k", synth.c1_stream(1)
    img = synth.fields_and_edges(11, 256, 256)
    yield "rgb256_97_1bpp.j2k", native.encode(img, 8, **synth.C2_PARAMS)
    yield "rgb256_53_rct.j2k", native.encode(img, 8, reversible=1, levels=5)
    yield "rgb300x200_97_tiles_3layers.j2k", native.encode(synth.fields_and_edges(12, 200, 300), 8,
                                                           **dict(synth.C3_PARAMS, tile_w=128, tile_h=128))
    # mode switches: beyond the reference (it asserts on BYPASS); pinned by lossless identity
    yield "rgb12_53_bypass_reset.j2k", native.encode(synth.fractal_rgb(13, 96, 160), 12, **synth.C4_PARAMS)


def t1_entry(cs):
    plan = native.Plan(cs)
    entry = {"bytes": len(cs), "blocks": plan.info.num_cblks, "reversible": plan.info.reversible,
             "cbstyle": plan.info.cbstyle}
    if plan.info.cbstyle & 0x3F == 0:  # the reference's live Tier-1 implements no mode switch
        digests = []
        for i in range(plan.info.num_cblks):
            rc, out = oracle_util.reference_block(plan, i)
            assert rc == 0, (i, rc)
            digests.append(hashlib.sha256(out.tobytes()).hexdigest()[:16])
        entry["reference_t1_sha256_16"] = digests
    return entry


def pictures():
    meta = {}
    for name, (_, fmt, top, compat) in rp.PICTURES.items():
        cs = rp.stream(name)
        r = ref_cpu_runner.decode([cs], fmt, threads=1, top_level=top, timeout=300)
        if not r["ok"]:
            raise SystemExit("%s: %s" % (name, r["error"]))
        out = r["outputs"][0]
        w, h = r["sizes"][0]
        plan = native.Plan(cs, discard_levels=rp.discard_of(native.Plan(cs).info.levels, top))
        assert (plan.info.width, plan.info.height) == (w, h), (name, w, h)
        entry = {"stream_sha256": rp.sha(cs), "format": fmt, "top_level": top, "ref_compat": compat, "width": w,
                 "height": h, "reversible": plan.info.reversible, "output_sha256": rp.sha(out)}
        if plan.info.reversible:
            entry["row_sha256_16"] = rp.row_digests(out, h)
        meta[name] = entry
        print(name, w, h, entry["output_sha256"][:16])
    return meta


def main():
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("J2K_REFERENCE_DIR")
    if not reference:
        raise SystemExit("usage: make_golden.py <reference root> (or set J2K_REFERENCE_DIR)")
    build.build_library()
    build.build_oracle(reference=reference)
    if oracle_util.ref_t1() is None or not ref_cpu_runner.available():
        raise SystemExit("reference libraries not built: needs the reference tree")
    meta = {}
    for name, cs in fixtures():
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(cs)
        meta[name] = t1_entry(cs)
        print(name, meta[name]["bytes"], meta[name]["blocks"])
    tier2 = os.path.join(HERE, "tier2")
    for fn in sorted(os.listdir(tier2)):
        if fn.endswith(".j2k"):
            with open(os.path.join(tier2, fn), "rb") as f:
                e = t1_entry(f.read())
            if "reference_t1_sha256_16" in e:
                meta["tier2/" + fn] = e
                print("tier2/" + fn, e["bytes"], e["blocks"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)
    with open(os.path.join(HERE, "reference_pictures.json"), "w") as f:
        json.dump(pictures(), f, indent=1)


if __name__ == "__main__":
    main()
