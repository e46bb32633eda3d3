"""Generate the golden fixtures of tests/golden/.

Run in a container that has the reference tree (it builds oracle/_ref/libref_t1.so from
/root/reference via oracle/build_ref.sh).  For each fixture codestream written by the
project's encoder, the reference's own Tier-1 (decode_code_block) decodes every
code-block and the SHA-256 of its raw int32 output is recorded.  The GPU box has no
reference tree; the tests compare the oracle and the GPU path against these digests.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from conftest import load_package  # noqa: E402

load_package()
from jpeg2000_decoder_b200 import build, native, synth  # noqa: E402
import oracle_util  # noqa: E402


def fixtures():
    yield "c1_gray_53.j2k", synth.c1_stream(1)
    img = synth.fields_and_edges(11, 256, 256)
    yield "rgb256_97_1bpp.j2k", native.encode(img, 8, **synth.C2_PARAMS)
    yield "rgb256_53_rct.j2k", native.encode(img, 8, reversible=1, levels=5)
    yield "rgb300x200_97_tiles_3layers.j2k", native.encode(synth.fields_and_edges(12, 200, 300), 8,
                                                           **dict(synth.C3_PARAMS, tile_w=128, tile_h=128))
    # mode switches: beyond the reference (it asserts on BYPASS); pinned by lossless identity
    yield "rgb12_53_bypass_reset.j2k", native.encode(synth.fractal_rgb(13, 96, 160), 12, **synth.C4_PARAMS)


def main():
    build.build_library()
    build.build_oracle()
    if oracle_util.ref_t1() is None:
        raise SystemExit("reference Tier-1 not built: needs the reference tree")
    meta = {}
    for name, cs in fixtures():
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(cs)
        plan = native.Plan(cs)
        entry = {"bytes": len(cs), "blocks": plan.info.num_cblks, "reversible": plan.info.reversible,
                 "cbstyle": plan.info.cbstyle}
        if plan.info.cbstyle & 0x07 == 0:
            digests = []
            for i in range(plan.info.num_cblks):
                rc, out = oracle_util.reference_block(plan, i)
                assert rc == 0, (name, i, rc)
                digests.append(hashlib.sha256(out.tobytes()).hexdigest()[:16])
            entry["reference_t1_sha256_16"] = digests
        meta[name] = entry
        print(name, entry["bytes"], entry["blocks"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
