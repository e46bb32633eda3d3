"""Generate the Tier-2 fixtures of tests/golden/tier2/ with an independent encoder.

OpenJPEG (the copy inside Pillow, `PIL.features.version("jpg_2000")`) writes small
codestreams that exercise what the project's own writer does not: several precincts per
resolution under every progression order, precinct-limited code-block sizes, partial tiles,
image and tile-grid origins other than (0, 0), and 9/7 quantisation with two guard bits.
The lossless ones must decode to the source picture; for the 9/7 one OpenJPEG's own
decoded picture is stored as the expected output (floating-point 9/7 implementations
differ by at most one level after rounding).

    python tests/golden/tier2/make_tier2.py
"""
import io
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from conftest import load_package  # noqa: E402

load_package()
from jpeg2000_decoder_b200 import synth  # noqa: E402

PROGRESSIONS = ["LRCP", "RLCP", "RPCL", "PCRL", "CPRL"]
H, W = 60, 80


def source():
    return np.ascontiguousarray(np.moveaxis(synth.fields_and_edges(31, H, W).astype(np.uint8), 0, -1))


def main():
    from PIL import Image, features
    src = source()
    pil = Image.fromarray(src, "RGB")
    manifest = {"openjpeg": features.version("jpg_2000"), "height": H, "width": W, "streams": {}}
    expected = {"source": src}

    def save(name, **kw):
        f = io.BytesIO()
        pil.save(f, "JPEG2000", no_jp2=True, **kw)
        with open(os.path.join(HERE, name), "wb") as g:
            g.write(f.getvalue())
        return f.getvalue()

    for prog in PROGRESSIONS:
        name = "ojp_%s_prec16_cb8_tiles.j2k" % prog.lower()
        save(name, progression=prog, precinct_size=(16, 16), codeblock_size=(8, 8), num_resolutions=4,
             quality_layers=[30, 10, 0], quality_mode="rates", tile_size=(64, 48))
        manifest["streams"][name] = {"expect": "source", "progression": prog}
    for name, kw in [("ojp_offset32x16_tileorigin16x8_lrcp.j2k",
                      dict(offset=(32, 16), tile_offset=(16, 8), tile_size=(64, 48), num_resolutions=4)),
                     ("ojp_offset48x24_tileorigin40x20_pcrl.j2k",
                      dict(offset=(48, 24), tile_offset=(40, 20), tile_size=(32, 32), num_resolutions=3,
                           progression="PCRL"))]:
        save(name, precinct_size=(16, 16), codeblock_size=(8, 8), quality_layers=[30, 10, 0],
             quality_mode="rates", **kw)
        manifest["streams"][name] = {"expect": "source", "origin": list(kw["offset"])}
    name = "ojp_cprl_97_guard2.j2k"
    cs = save(name, progression="CPRL", precinct_size=(32, 32), codeblock_size=(16, 16), num_resolutions=4,
              quality_layers=[12, 4], quality_mode="rates", irreversible=True, tile_size=(64, 48))
    expected["ojp_cprl_97_guard2"] = np.asarray(Image.open(io.BytesIO(cs)).convert("RGB"))
    manifest["streams"][name] = {"expect": "ojp_cprl_97_guard2", "tolerance": 1}
    np.savez_compressed(os.path.join(HERE, "expected.npz"), **expected)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
