"""Seeded synthetic images and codestreams for the five benchmark configurations.

No public dataset is involved: every image is generated from a seed with the shapes,
value ranges and content statistics of the configuration it stands in for, and encoded
by the project's own Part-1 writer (csrc/encoder).

C1  512x512 8-bit gray, sum of 8 random sinusoids (periods 8-256 px) + N(0, 8^2);
    reversible 5/3, 5 levels, 64x64 blocks, 1 tile, 1 layer, LRCP, no mode switches.
C2  2048x2048 RGB 8-bit, smooth fields + random rectangles (contrast 20-200) + N(0, 4^2);
    9/7 + ICT, expounded quantisation, G = 1, 5 levels, 64x64 blocks, 1 layer, ~1.0 bpp.
C3  64 frames 1920x1080 RGB 8-bit: one seeded picture shifted 0-3 px per frame + fresh
    N(0, 3^2); 9/7 + ICT, 512x512 tiles, 5 levels, 64x64 blocks, 3 layers ~0.5/1/2 bpp.
C4  16 x 4096x2160 RGB 12-bit 1/f^2 fractal noise in [0, 4095]; 5/3 + RCT, 6 levels,
    32x32 blocks, 8 layers, RPCL, BYPASS + RESET.
C5  request mix: sizes uniform over {256^2, 512^2, 1024^2, 1920x1080, 4096x2160}, half
    8-bit lossless 5/3 + RCT, half 8/12-bit 9/7 + ICT at 0.5-2 bpp, 64x64 blocks.
"""
import hashlib
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import native

CACHE = os.environ.get("J2K_BENCH_CACHE", "/tmp/j2k_bench_cache")


def sinusoid_gray(seed, h=512, w=512, sigma=8.0):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    img = np.zeros((h, w))
    for _ in range(8):
        px, py = rng.uniform(8, 256, 2)
        ph = rng.uniform(0, 2 * np.pi)
        a = rng.uniform(8, 24)
        img += a * np.sin(2 * np.pi * (xx / px + yy / py) + ph)
    img += 128 + rng.normal(0, sigma, (h, w))
    return np.clip(np.rint(img), 0, 255).astype(np.uint16)[None]


def fields_and_edges(seed, h, w, sigma=4.0, nrect=60):
    """Smooth colour fields plus piecewise-constant rectangles and Gaussian noise."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    out = np.empty((3, h, w), np.float32)
    for c in range(3):
        f = np.full((h, w), 128.0, np.float32)
        for _ in range(4):
            kx, ky = rng.uniform(0.5, 3.0, 2) * 2 * np.pi / np.array([w, h])
            f += rng.uniform(10, 40) * np.sin(kx * xx + ky * yy + rng.uniform(0, 2 * np.pi)).astype(np.float32)
        out[c] = f
    for _ in range(nrect):
        x0, y0 = rng.integers(0, w), rng.integers(0, h)
        rw, rh = rng.integers(w // 40 + 1, w // 4 + 2), rng.integers(h // 40 + 1, h // 4 + 2)
        contrast = rng.uniform(20, 200) * rng.choice([-1, 1])
        tint = rng.uniform(0.5, 1.0, 3)
        for c in range(3):
            out[c, y0:y0 + rh, x0:x0 + rw] += np.float32(contrast * tint[c])
    out += rng.normal(0, sigma, out.shape).astype(np.float32)
    return np.clip(np.rint(out), 0, 255).astype(np.uint16)


def fractal_rgb(seed, h, w, bitdepth=12):
    """1/f^2 power-spectrum noise per component, scaled to the full sample range."""
    rng = np.random.default_rng(seed)
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    f2 = fx * fx + fy * fy
    f2[0, 0] = 1.0
    amp = (1.0 / np.sqrt(f2)).astype(np.float32)  # power ~ 1/f^2, amplitude ~ 1/f
    out = np.empty((3, h, w), np.uint16)
    top = (1 << bitdepth) - 1
    for c in range(3):
        spec = (rng.normal(size=f2.shape) + 1j * rng.normal(size=f2.shape)).astype(np.complex64) * amp
        spec[0, 0] = 0
        img = np.fft.irfft2(spec, s=(h, w)).astype(np.float32)
        lo, hi = np.percentile(img, [0.5, 99.5])
        img = (img - lo) / max(hi - lo, 1e-6) * top
        out[c] = np.clip(np.rint(img), 0, top).astype(np.uint16)
    return out


def video_frames(seed, n=64, h=1080, w=1920, sigma=3.0):
    base = fields_and_edges(seed, h + 200, w + 200, sigma=0.0).astype(np.float32)
    rng = np.random.default_rng(seed + 1)
    frames = []
    ox = oy = 0
    for _ in range(n):
        ox = min(ox + int(rng.integers(0, 4)), 199)
        oy = min(oy + int(rng.integers(0, 4)), 199)
        f = base[:, oy:oy + h, ox:ox + w] + rng.normal(0, sigma, (3, h, w)).astype(np.float32)
        frames.append(np.clip(np.rint(f), 0, 255).astype(np.uint16))
    return frames


# ------------------------------------------------------------------ codestreams -------
C1_PARAMS = dict(reversible=1, levels=5, cbw_exp=6, cbh_exp=6, num_layers=1, layer_bpp=[0], progression=0)
C2_PARAMS = dict(reversible=0, levels=5, cbw_exp=6, cbh_exp=6, num_layers=1, layer_bpp=[1.0], progression=0,
                 guard_bits=1)
C3_PARAMS = dict(reversible=0, levels=5, cbw_exp=6, cbh_exp=6, tile_w=512, tile_h=512, num_layers=3,
                 layer_bpp=[0.5, 1.0, 2.0], progression=0, guard_bits=1)
C4_PARAMS = dict(reversible=1, levels=6, cbw_exp=5, cbh_exp=5, num_layers=8,
                 layer_bpp=[0.5, 1, 2, 3, 4, 6, 8, 0], progression=2, mode=0x03)


def c1_stream(seed=1):
    return native.encode(sinusoid_gray(seed), 8, **C1_PARAMS)


def c2_stream(seed=2, size=2048):
    return native.encode(fields_and_edges(seed, size, size), 8, **C2_PARAMS)


def c3_streams(seed=3, n=64, h=1080, w=1920, workers=None):
    frames = video_frames(seed, n, h, w)
    with ThreadPoolExecutor(max_workers=workers or 4) as ex:
        return list(ex.map(lambda f: native.encode(f, 8, **C3_PARAMS), frames))


def c4_streams(seed=4, n=16, h=2160, w=4096, workers=None):
    def one(i):
        return native.encode(fractal_rgb(seed * 1000 + i, h, w), 12, **C4_PARAMS)
    with ThreadPoolExecutor(max_workers=workers or 4) as ex:
        return list(ex.map(one, range(n)))


C5_SIZES = [(256, 256), (512, 512), (1024, 1024), (1080, 1920), (2160, 4096)]


def c5_request(seed):
    """One request of the serving mix: (codestream, pixels)."""
    rng = np.random.default_rng(seed)
    h, w = C5_SIZES[int(rng.integers(0, len(C5_SIZES)))]
    if rng.random() < 0.5:
        img = fields_and_edges(seed, h, w, nrect=max(4, (h * w) >> 16))
        cs = native.encode(img, 8, reversible=1, levels=5, cbw_exp=6, cbh_exp=6, num_layers=1, layer_bpp=[0])
    else:
        depth = 8 if rng.random() < 0.5 else 12
        img = fields_and_edges(seed, h, w, nrect=max(4, (h * w) >> 16))
        if depth == 12:
            img = (img.astype(np.uint32) * 16 + rng.integers(0, 16, img.shape)).astype(np.uint16)
        bpp = float(rng.uniform(0.5, 2.0))
        cs = native.encode(img, depth, reversible=0, levels=5, cbw_exp=6, cbh_exp=6, num_layers=1, layer_bpp=[bpp],
                           guard_bits=1)
    return cs, h * w


def c5_format(cs):
    """Packed RGB output format of a serving request: 24-bit for 8-bit pictures, 48-bit above."""
    plan = native.Plan(cs)
    return native.FMT_24BITS_RGB if plan.info.bitdepth <= 8 else native.FMT_48BITS_RGB


def c5_pool(n_distinct=48, seed=5, workers=None):
    """Distinct serving requests (codestreams) from per-request seeds."""
    with ThreadPoolExecutor(max_workers=workers or 4) as ex:
        return [cs for cs, _ in ex.map(c5_request, [seed * 100000 + i for i in range(n_distinct)])]


# ------------------------------------------------------------------ workloads ---------
def _cached(key, make):
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, hashlib.sha1(key.encode()).hexdigest() + ".npz")
    if os.path.exists(path):
        d = np.load(path, allow_pickle=False)
        return [bytes(d["s%d" % i]) for i in range(int(d["n"]))]
    streams = make()
    # several processes (one per GPU) may build the same workload at once: each writes its
    # own file and renames it into place, so a reader never sees a partly written cache
    tmp = "%s.%d.tmp.npz" % (path[:-4], os.getpid())
    np.savez(tmp, n=len(streams), **{"s%d" % i: np.frombuffer(s, np.uint8) for i, s in enumerate(streams)})
    os.replace(tmp, path)
    return streams


def workload(name, quick=False):
    """(config dict, list of codestreams, output format)."""
    if name == "c3":
        nd = 4 if quick else 16
        reps = 1 if quick else 4
        distinct = _cached("c3-v1-%d" % nd, lambda: c3_streams(3, n=nd, workers=os.cpu_count()))
        streams = [distinct[i % nd] for i in range(nd * reps)]
        cfg = {"workload": "C3 batched video-frame decode", "frames": len(streams), "distinct_frames": nd,
               "size": "1920x1080", "components": 3, "bitdepth": 8, "wavelet": "9/7+ICT", "tiles": "512x512",
               "levels": 5, "codeblock": "64x64", "layers": 3, "layer_bpp": [0.5, 1.0, 2.0]}
        return cfg, streams, native.FMT_24BITS_RGB
    if name == "c2":
        streams = _cached("c2-v1", lambda: [c2_stream(2)])
        cfg = {"workload": "C2 single 2048x2048 RGB 9/7+ICT ~1 bpp", "frames": 1, "size": "2048x2048",
               "components": 3, "bitdepth": 8, "wavelet": "9/7+ICT", "levels": 5, "codeblock": "64x64",
               "layers": 1}
        return cfg, streams, native.FMT_24BITS_RGB
    if name == "c4":
        n = 2 if quick else 16
        nd = min(n, 4)
        distinct = _cached("c4-v1-%d" % nd, lambda: c4_streams(4, n=nd, workers=os.cpu_count()))
        streams = [distinct[i % nd] for i in range(n)]
        cfg = {"workload": "C4 batched 12-bit lossless", "frames": n, "distinct_frames": nd, "size": "4096x2160",
               "components": 3, "bitdepth": 12, "wavelet": "5/3+RCT", "levels": 6, "codeblock": "32x32",
               "layers": 8, "progression": "RPCL", "mode": "BYPASS+RESET"}
        return cfg, streams, native.FMT_48BITS_RGB
    if name == "c1":
        streams = _cached("c1-v1", lambda: [c1_stream(1)])
        cfg = {"workload": "C1 512x512 gray 5/3 lossless", "frames": 1, "size": "512x512", "components": 1,
               "bitdepth": 8, "wavelet": "5/3", "levels": 5, "codeblock": "64x64", "layers": 1}
        return cfg, streams, native.FMT_32BITS_4COMPONENTS
    if name == "c5":
        nd = 12 if quick else 48
        streams = _cached("c5-v1-%d" % nd, lambda: c5_pool(nd, workers=os.cpu_count()))
        cfg = {"workload": "C5 serving stream", "distinct_requests": nd,
               "sizes": ["256x256", "512x512", "1024x1024", "1920x1080", "4096x2160"],
               "mix": "half 8-bit 5/3+RCT lossless, half 8/12-bit 9/7+ICT at 0.5-2 bpp", "codeblock": "64x64"}
        return cfg, streams, None
    raise SystemExit("unknown workload " + name)
