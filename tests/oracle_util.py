"""Test-side access to the oracle: the C restatement (oracle/liboracle.so), the reference's
own Tier-1 (oracle/_ref/libref_t1.so, when built) and an FP64 9/7 + ICT synthesis in numpy
that anchors the float path's error budget."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "liboracle.so")
REF_T1 = os.path.join(ROOT, "oracle", "_ref", "libref_t1.so")

_orc = None
_ref = None


def orc():
    global _orc
    if _orc is None:
        _orc = ctypes.CDLL(ORACLE)
    return _orc


def ref_t1():
    """The reference's decode_code_block, or None when its build is absent."""
    global _ref
    if _ref is None and os.path.exists(REF_T1):
        _ref = ctypes.CDLL(REF_T1)
    return _ref


def _ptr(arr):
    return ctypes.c_void_p(ctypes.addressof(arr))


def oracle_decode(plan, fmt, ref_compat=0):
    I = plan.info
    from jpeg2000_decoder_b200 import native
    nbytes = plan.output_bytes(fmt) if fmt != native.FMT_NONE else 0
    out = np.zeros(max(1, nbytes), np.uint8)
    coef = np.zeros(max(1, I.coef_elems), np.int32)
    rc = orc().oracle_decode(ctypes.byref(I), _ptr(plan.cblks()), I.num_cblks, plan.bytes_ptr(), plan.seglens_ptr(),
                             _ptr(plan.tilecomps()), I.num_tilecomps, ref_compat, fmt if nbytes else 0,
                             out.ctypes.data_as(ctypes.c_void_p) if nbytes else None,
                             coef.ctypes.data_as(ctypes.c_void_p))
    return rc, out[:nbytes], coef


def oracle_t1_coefficients(plan):
    I = plan.info
    coef = np.zeros(max(1, I.coef_elems), np.int32)
    status = np.zeros(max(1, I.num_cblks), np.int32)
    bad = orc().oracle_t1_place(_ptr(plan.cblks()), I.num_cblks, plan.bytes_ptr(), plan.seglens_ptr(),
                                coef.ctypes.data_as(ctypes.c_void_p), status.ctypes.data_as(ctypes.c_void_p))
    return bad, coef


def oracle_block(plan, i):
    cb = plan.cblks()[i]
    out = np.zeros(cb.w * cb.h, np.int32)
    rc = orc().oracle_t1_block(ctypes.byref(cb), plan.bytes_ptr(), plan.seglens_ptr(),
                               out.ctypes.data_as(ctypes.c_void_p))
    return rc, out


def reference_block(plan, i):
    lib = ref_t1()
    cb = plan.cblks()[i]
    out = np.zeros(cb.w * cb.h, np.int32)
    numbps = (cb.mb << 11) if (cb.flags & 0x40) else cb.mb
    rc = lib.ref_t1_block(cb.w, cb.h, cb.missing, cb.num_passes, numbps, cb.band,
                          ctypes.c_void_p(plan.bytes_ptr().value + cb.data_off), cb.data_len,
                          out.ctypes.data_as(ctypes.c_void_p))
    return rc, out


# ------------------------------------------------------------ FP64 9/7 synthesis ------
# Standard T.800 dequantisation and synthesis in float64 from the same integer Tier-1
# output: the error budget of the FP32 path is stated against this.
K = 1.230174104914001
LIFT = [(0.443506852043971, 0), (0.882911075530934, 1), (-0.052980118572961, 0), (-1.586134342059924, 1)]


def _inv97_axis(a, nlow, axis):
    a = np.moveaxis(a, axis, 0)
    n = a.shape[0]
    if n == 1:
        return np.moveaxis(a.copy(), 0, axis)
    y = np.empty_like(a)
    y[0::2] = a[:nlow] * K
    y[1::2] = a[nlow:] / K
    idx = np.arange(n)
    left = np.abs(idx - 1)
    right = idx + 1
    right[right >= n] = 2 * (n - 1) - right[right >= n]
    for c, par in LIFT:
        sel = idx[par::2]
        y[sel] = y[sel] - c * (y[left[sel]] + y[right[sel]])
    return np.moveaxis(y, 0, axis)


def _signmag(v):
    v = v.astype(np.int64)
    mag = v & 0x7FFFFFFF
    return np.where(v & 0x80000000, -mag, mag)


def fp64_decode(plan):
    """(ncomp, H, W) float64 component samples + DC shift, before MCT clamp/rounding."""
    I = plan.info
    coef = np.zeros(max(1, I.coef_elems), np.float64)
    for i, cb in enumerate(plan.cblks()):
        rc, raw = oracle_block(plan, i)
        q = _signmag(raw).reshape(cb.h, cb.w).astype(np.float64)
        eps, mu = cb.spqcd >> 11, cb.spqcd & 0x7FF
        gain_b = 0 if cb.band == 0 else (2 if cb.band == 3 else 1)
        delta = 2.0 ** (I.bitdepth + gain_b - eps) * (1.0 + mu / 2048.0)
        for y in range(cb.h):
            o = cb.out_off + y * cb.out_stride
            coef[o:o + cb.w] = q[y] * delta
    comps = np.zeros((I.ncomp, I.height, I.width))
    for tc in plan.tilecomps():
        reg = coef[tc.coef_off:tc.coef_off + tc.w * tc.h].reshape(tc.h, tc.w).copy()
        for r in range(1, tc.levels + 1):
            rw, rh, lw, lh = tc.res_w[r], tc.res_h[r], tc.res_w[r - 1], tc.res_h[r - 1]
            sub = _inv97_axis(reg[:rh, :rw], lw, 1)
            reg[:rh, :rw] = _inv97_axis(sub, lh, 0)
        comps[tc.comp, tc.y0:tc.y0 + tc.h, tc.x0:tc.x0 + tc.w] = reg
    dc = float(1 << (I.bitdepth - 1))
    if I.ncomp >= 3 and I.mct:
        y, u, v = comps[0], comps[1], comps[2]
        return np.stack([y + 1.402 * v, y - 0.34413 * u - 0.71414 * v, y + 1.772 * u]) + dc
    return comps + dc


def psnr_maxabs(decoded, reference, bitdepth):
    ref = np.clip(reference, 0, (1 << bitdepth) - 1)
    d = decoded.astype(np.float64) - ref
    mse = float(np.mean(d * d))
    peak = float((1 << bitdepth) - 1)
    return (10 * np.log10(peak * peak / mse) if mse > 0 else float("inf")), float(np.max(np.abs(d)))
