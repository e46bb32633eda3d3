"""Decode one benchmark workload a few times through the C ABI (profiling driver).

    python jpeg2000-decoder_b200/profile_decode.py --workload c2 --repeat 2 [--quick] [--frames N] [--t1-form F]

Each repeat is one batch decode (Tier-1, DWT levels, output stage) of the whole workload;
run it under ncu with -s/-c to capture a chosen launch of a chosen kernel.
"""
import argparse
import importlib.util
import os
import sys

PKG = os.path.dirname(os.path.abspath(__file__))


def _load():
    name = "jpeg2000_decoder_b200"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(PKG, "__init__.py"),
                                                      submodule_search_locations=[PKG])
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--frames", type=int, default=0, help="decode only the first N pictures of the workload")
    ap.add_argument("--t1-form", type=int, default=0, help="Tier-1 kernel form: 0 auto, 1 compact, 2 unrolled")
    a = ap.parse_args()
    _load()
    from jpeg2000_decoder_b200 import native, synth
    cfg, streams, fmt = synth.workload(a.workload, a.quick)
    if a.frames > 0:
        streams = streams[:a.frames]
    ctx = native.GpuContext()
    ctx.set_tuning(t1_form=a.t1_form)
    plans = [native.Plan(s) for s in streams]
    for it in range(a.repeat):
        ctx.begin()
        for p in plans:
            ctx.add(p, fmt)
        ctx.launch()
        rc = ctx.sync()
        if rc != 0:
            raise SystemExit("decode failed: %d" % rc)
        print(a.workload, it, ctx.timing(), "launches", ctx.launches())


if __name__ == "__main__":
    main()
