"""FP64 T.800 9/7 dequantisation and synthesis: the yardstick for the FP32 path's error.

Standard dequantisation (Delta_b = 2^(R_b - eps_b) (1 + mu_b / 2^11), T.800 E.1.1.1) and the
standard 1D_SR lifting with K scaling (T.800 F.3.8) in float64, applied to the Tier-1
sample values of a plan's code-blocks; DC level shift and the irreversible colour
transform (T.800 G.3) in float64 too, before any clamp or rounding.  The caller supplies
each block's Tier-1 values (in the units the plan's step parameters refer to): the tests
take them from the oracle, bench.py from the device's own Tier-1 output.
"""
import numpy as np

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


def synthesize(plan, raw_values):
    """(ncomp, H, W) float64 component samples + DC shift (+ ICT), before clamp/rounding.
    raw_values(i, cb) -> (cb.h, cb.w) float64 Tier-1 values of code-block i."""
    I = plan.info
    coef = np.zeros(max(1, I.coef_elems), np.float64)
    for i, cb in enumerate(plan.cblks()):
        q = raw_values(i, cb)
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
