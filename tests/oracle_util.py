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
from fp64_97 import psnr_maxabs, synthesize  # noqa: E402,F401


def fp64_decode(plan):
    """(ncomp, H, W) float64 T.800 synthesis (+ DC shift, + ICT) from the oracle's Tier-1."""
    def raw_values(i, cb):
        rc, raw = oracle_block(plan, i)
        return _signmag(raw).reshape(cb.h, cb.w).astype(np.float64)
    return synthesize(plan, raw_values)


def _signmag(v):
    v = v.astype(np.int64)
    mag = v & 0x7FFFFFFF
    return np.where(v & 0x80000000, -mag, mag)
