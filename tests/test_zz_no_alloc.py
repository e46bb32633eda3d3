"""The allocation-free inverse DWT entry point (j2k_gpu_tile_idwt_noalloc).

It serves callers that cannot call cudaMalloc — code running during CUDA stream capture,
real-time callbacks, or hosts that own every device buffer — by keeping its intermediate
levels in a static device array.  Here the caller's input and output buffers come from
torch (the test may allocate; the entry point must not), and its result must equal what
the regular batched path reconstructs, bit for bit (the tolerance of every parity test
here), on two calls in a row (the second call finds the first call's data in the shared
array).  Collected last so that a failure here cannot hide the other tests.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _read(name):
    with open(os.path.join(GOLDEN, name), "rb") as f:
        return f.read()


@pytest.mark.parametrize("name,flags", [("rgb300x200_97_tiles_3layers.j2k", 0), ("c1_gray_53.j2k", 0),
                                        ("c1_gray_53.j2k", 1), ("rgb12_53_bypass_reset.j2k", 0)])
def test_noalloc_idwt_matches_batched_path(pkg, name, flags):
    import torch
    from jpeg2000_decoder_b200 import native
    torch.cuda.init()
    plan = native.Plan(_read(name))
    ctx = native.GpuContext()
    try:
        ctx.begin()
        ctx.add(plan, native.FMT_NONE, flags)
        ctx.launch()
        assert ctx.sync() == 0
        t1 = ctx.coefficients(0, 0)     # Tier-1 output, Mallat layout per tile-component
        ref = ctx.coefficients(0, 1)    # reconstructed tile-components of the batched path
    finally:
        ctx.close()
    dt = torch.int32 if plan.info.reversible else torch.float32
    stream = torch.cuda.Stream()
    L = native.lib()
    for call in range(2):
        for tc in plan.tilecomps():
            n = tc.w * tc.h
            src = torch.from_numpy(np.ascontiguousarray(t1[tc.coef_off:tc.coef_off + n])).to("cuda")
            out = torch.full((tc.h, tc.w), -7, dtype=dt, device="cuda")
            rc = L.j2k_gpu_tile_idwt_noalloc(ctypes.byref(tc), plan.info.reversible, flags,
                                             ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(out.data_ptr()), tc.w,
                                             ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0, rc
            stream.synchronize()
            got = out.cpu().numpy().reshape(-1)
            want = ref[tc.coef_off:tc.coef_off + n]
            assert np.array_equal(got.view(np.int32), want.view(np.int32)), (call, tc.tile, tc.comp)


def test_noalloc_rejects_oversized_tiles(pkg):
    from jpeg2000_decoder_b200 import native
    tc = native.TileComp()  # 8192x8192, 2 levels: the 4096x4096 level needs 2 x 64 MiB of scratch
    tc.w, tc.h, tc.levels = 8192, 8192, 2
    for r, (w, h) in enumerate([(2048, 2048), (4096, 4096), (8192, 8192)]):
        tc.res_w[r], tc.res_h[r] = w, h
    rc = native.lib().j2k_gpu_tile_idwt_noalloc(ctypes.byref(tc), 1, 0, ctypes.c_void_p(1), ctypes.c_void_p(1), 8192,
                                                None)
    assert rc == -3  # J2K_ERR_UNSUPPORTED: beyond the static scratch array
