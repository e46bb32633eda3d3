"""ctypes bindings of the in-tree native libraries.

libj2k_b200.so: the C ABI of include/j2k_gpu.h (host Tier-2 plans + the sm_100a decode
path) and the reference-facing C entry points (BMI_dec_* of include/bmi_jp2dec.h and the
bmi_decoder_* binding of BMI::Decoder).  libj2kenc.so: the test codestream writer.
The product path has no fallback: loading fails loudly when a library is missing.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("J2K_B200_LIB") or os.path.join(PKG, "libj2k_b200.so")
ENC_PATH = os.path.join(PKG, "libj2kenc.so")

# OutputFormat (reference codec_datatype.h)
FMT_32BITS_ARGB = 0
FMT_48BITS_RGB = 1
FMT_24BITS_RGB = 2
FMT_32BITS_4COMPONENTS = 3
FMT_64BITS_4COMPONENTS = 4
FMT_48BITS_3COMPONENTS = 5
FMT_24BITS_3COMPONENTS = 6
FMT_NONE = 7
FMT_64BITS_ARGB = 8
FMT_BYTES = {0: 4, 1: 6, 2: 3, 3: 4, 4: 8, 5: 6, 6: 3, 8: 8}

FLAG_REF_COMPAT = 1
FLAG_KEEP_COMPONENTS = 2

J2K_OK = 0
J2K_ERR_ARG = -1
J2K_ERR_PARSE = -2
J2K_ERR_NODEVICE = -9
J2K_ERR_DECODE = -7
J2K_ERR_TIMEOUT = -6
J2K_ERR_NOMEM = -5
J2K_ERR_STATE = -8
J2K_ERR_UNSUPPORTED = -3


class J2kError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__("%s failed: %d (%s)" % (what, code, status_string(code)))


class ImageInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "width", "height", "ncomp", "bitdepth", "is_signed", "tile_w", "tile_h", "ntiles_x", "ntiles_y",
        "levels", "reversible", "mct", "layers", "progression", "cbw", "cbh", "cbstyle", "guard_bits",
        "num_cblks", "num_tilecomps", "num_segs")] + [("coded_bytes", ctypes.c_uint64), ("coef_elems", ctypes.c_uint64),
                                                       ("origin_x", ctypes.c_int32), ("origin_y", ctypes.c_int32)] + [
        (n, ctypes.c_int32 * 4) for n in ("sub_x", "sub_y", "comp_x0", "comp_y0", "comp_w", "comp_h")]


class CodeBlock(ctypes.Structure):
    _fields_ = [("data_off", ctypes.c_uint32), ("data_len", ctypes.c_uint32), ("out_off", ctypes.c_uint64),
                ("out_stride", ctypes.c_uint32), ("seg_off", ctypes.c_uint32), ("gain", ctypes.c_float),
                ("w", ctypes.c_uint16), ("h", ctypes.c_uint16), ("num_passes", ctypes.c_uint8),
                ("missing", ctypes.c_uint8), ("band", ctypes.c_uint8), ("mb", ctypes.c_uint8),
                ("flags", ctypes.c_uint8), ("nseg", ctypes.c_uint8), ("spqcd", ctypes.c_uint16)]


class TileComp(ctypes.Structure):
    _fields_ = [("coef_off", ctypes.c_uint64), ("x0", ctypes.c_int32), ("y0", ctypes.c_int32),
                ("w", ctypes.c_int32), ("h", ctypes.c_int32), ("levels", ctypes.c_int32),
                ("comp", ctypes.c_int32), ("tile", ctypes.c_int32),
                ("res_w", ctypes.c_int32 * 11), ("res_h", ctypes.c_int32 * 11)]


class Tuning(ctypes.Structure):
    _fields_ = [("t1_warps_per_cta", ctypes.c_int), ("dwt_tile", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("t1_form", ctypes.c_int), ("t1_latency_waves", ctypes.c_int), ("dwt_coarse", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("mem_budget", ctypes.c_size_t), ("pipeline_depth", ctypes.c_int),
                ("max_batch_images", ctypes.c_int), ("max_batch_pixels", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("mean_batch_images", ctypes.c_double), ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("busy_s", ctypes.c_double), ("pixels", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("gpu_ms", ctypes.c_double), ("stage_ms", ctypes.c_double),
                ("enqueue_ms", ctypes.c_double), ("pool_growths", ctypes.c_uint64), ("pinned_allocs", ctypes.c_uint64)]


class EncParams(ctypes.Structure):
    _fields_ = [("reversible", ctypes.c_int), ("levels", ctypes.c_int), ("cbw_exp", ctypes.c_int),
                ("cbh_exp", ctypes.c_int), ("tile_w", ctypes.c_int), ("tile_h", ctypes.c_int),
                ("num_layers", ctypes.c_int), ("layer_bpp", ctypes.c_double * 32), ("progression", ctypes.c_int),
                ("mode", ctypes.c_int), ("use_mct", ctypes.c_int), ("guard_bits", ctypes.c_int),
                ("base_step", ctypes.c_double), ("num_threads", ctypes.c_int), ("markers", ctypes.c_int),
                ("tile_parts", ctypes.c_int), ("interleave_tile_parts", ctypes.c_int), ("num_poc", ctypes.c_int),
                ("poc", (ctypes.c_int * 6) * 8), ("poc_in_tiles", ctypes.c_int),
                ("sub_x", ctypes.c_int * 4), ("sub_y", ctypes.c_int * 4)]

ENC_SOP, ENC_EPH, ENC_PPM, ENC_PPT = 1, 2, 4, 8


assert ctypes.sizeof(CodeBlock) == 40

_lib = None
_enc = None

# every symbol include/j2k_gpu.h, include/bmi_jp2dec.h and include/bmi_decoder_c.h declare
EXPORTS = [
    "j2k_plan_create", "j2k_plan_create_mt", "j2k_plan_destroy", "j2k_plan_info", "j2k_plan_cblks", "j2k_plan_seglens",
    "j2k_plan_bytes", "j2k_plan_tilecomps", "j2k_output_bytes", "j2k_status_string",
    "j2k_gpu_ctx_create", "j2k_gpu_ctx_destroy", "j2k_gpu_mem_usage", "j2k_gpu_batch_begin",
    "j2k_gpu_batch_add", "j2k_gpu_batch_footprint", "j2k_gpu_batch_launch", "j2k_gpu_batch_stage", "j2k_gpu_batch_run", "j2k_gpu_batch_sync",
    "j2k_gpu_image_status", "j2k_gpu_output_device", "j2k_gpu_output_copy", "j2k_gpu_output_copy_async",
    "j2k_gpu_component_copy",
    "j2k_gpu_coefficients_copy", "j2k_gpu_last_timing", "j2k_gpu_last_launches", "j2k_gpu_set_tuning",
    "j2k_gpu_get_tuning", "j2k_gpu_autotune", "j2k_gpu_decode", "j2k_gpu_tile_idwt_noalloc",
    "j2k_server_create", "j2k_server_destroy", "j2k_server_submit", "j2k_server_wait", "j2k_server_result",
    "j2k_server_latency_us",
    "j2k_server_release", "j2k_server_drain", "j2k_server_stats_get", "j2k_server_stats_reset",
    "BMI_dec_info", "BMI_dec_init", "BMI_dec_isr", "BMI_dec", "BMI_dec_thumbnail", "BMI_dec_exit",
    "bmi_decoder_init", "bmi_decoder_set_job", "bmi_decoder_decode", "bmi_decoder_predecode",
    "bmi_decoder_predecode_format",
    "bmi_decoder_status", "bmi_decoder_result", "bmi_decoder_thumbnail", "bmi_decoder_component_int",
    "bmi_decoder_component_float", "bmi_decoder_release", "bmi_decoder_terminate",
]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("native library %s is missing: run jpeg2000-decoder_b200/build.py" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        vp, i, u64, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_size_t
        L.j2k_plan_create.argtypes = [ctypes.c_char_p, sz, i, i, ctypes.c_uint, ctypes.POINTER(vp)]
        L.j2k_plan_create_mt.argtypes = [ctypes.c_char_p, sz, i, i, ctypes.c_uint, i, ctypes.POINTER(vp)]
        L.j2k_plan_destroy.argtypes = [vp]
        L.j2k_plan_destroy.restype = None
        L.j2k_plan_info.argtypes = [vp, ctypes.POINTER(ImageInfo)]
        for f in ("j2k_plan_cblks", "j2k_plan_seglens", "j2k_plan_bytes", "j2k_plan_tilecomps"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = vp
        L.j2k_output_bytes.argtypes = [ctypes.POINTER(ImageInfo), i]
        L.j2k_output_bytes.restype = sz
        L.j2k_status_string.argtypes = [i]
        L.j2k_status_string.restype = ctypes.c_char_p
        L.j2k_gpu_ctx_create.argtypes = [i, sz, ctypes.POINTER(vp)]
        L.j2k_gpu_ctx_destroy.argtypes = [vp]
        L.j2k_gpu_ctx_destroy.restype = None
        L.j2k_gpu_mem_usage.argtypes = [vp, ctypes.POINTER(sz), ctypes.POINTER(sz)]
        L.j2k_gpu_batch_begin.argtypes = [vp]
        L.j2k_gpu_batch_add.argtypes = [vp, vp, i, i, ctypes.POINTER(i)]
        L.j2k_gpu_batch_footprint.argtypes = [vp, ctypes.POINTER(sz)]
        L.j2k_gpu_batch_launch.argtypes = [vp, vp]
        L.j2k_gpu_batch_stage.argtypes = [vp, vp]
        L.j2k_gpu_batch_run.argtypes = [vp, vp]
        L.j2k_gpu_batch_sync.argtypes = [vp, i]
        L.j2k_gpu_image_status.argtypes = [vp, i, ctypes.POINTER(i)]
        L.j2k_gpu_output_device.argtypes = [vp, i, ctypes.POINTER(vp), ctypes.POINTER(sz)]
        L.j2k_gpu_output_copy.argtypes = [vp, i, vp, sz]
        L.j2k_gpu_output_copy_async.argtypes = [vp, i, vp, sz]
        L.j2k_gpu_component_copy.argtypes = [vp, i, i, vp, sz]
        L.j2k_gpu_coefficients_copy.argtypes = [vp, i, i, vp, sz]
        f = ctypes.POINTER(ctypes.c_float)
        L.j2k_gpu_last_timing.argtypes = [vp, f, f, f, f]
        L.j2k_gpu_last_launches.argtypes = [vp, ctypes.POINTER(i)]
        L.j2k_gpu_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.j2k_gpu_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.j2k_gpu_autotune.argtypes = [vp, vp, i, ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_float)]
        L.j2k_gpu_decode.argtypes = [vp, ctypes.c_char_p, sz, i, i, vp, sz]
        L.j2k_gpu_tile_idwt_noalloc.argtypes = [ctypes.POINTER(TileComp), i, i, vp, vp, i, vp]
        L.j2k_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.j2k_server_destroy.argtypes = [vp]
        L.j2k_server_destroy.restype = None
        L.j2k_server_submit.argtypes = [vp, ctypes.c_char_p, sz, i, i]
        L.j2k_server_submit.restype = ctypes.c_int64
        L.j2k_server_wait.argtypes = [vp, ctypes.c_int64, vp, sz, ctypes.POINTER(sz), i]
        L.j2k_server_result.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(vp), ctypes.POINTER(sz), i]
        L.j2k_server_latency_us.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]
        L.j2k_server_release.argtypes = [vp, ctypes.c_int64]
        L.j2k_server_drain.argtypes = [vp]
        L.j2k_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.j2k_server_stats_reset.argtypes = [vp]
        L.bmi_decoder_init.argtypes = [i, i]
        L.bmi_decoder_set_job.argtypes = [i, i, ctypes.c_uint, i]
        L.bmi_decoder_set_job.restype = None
        L.bmi_decoder_decode.argtypes = [ctypes.c_char_p, i, ctypes.POINTER(ctypes.c_double)]
        L.bmi_decoder_predecode.argtypes = [ctypes.c_char_p, i] + [ctypes.POINTER(i)] * 5
        L.bmi_decoder_status.argtypes = [i]
        L.bmi_decoder_result.argtypes = [i, ctypes.POINTER(i)]
        L.bmi_decoder_result.restype = vp
        L.bmi_decoder_thumbnail.argtypes = [i, ctypes.POINTER(i)]
        L.bmi_decoder_thumbnail.restype = vp
        L.bmi_decoder_component_int.argtypes = [i, i, ctypes.POINTER(i)]
        L.bmi_decoder_component_int.restype = vp
        L.bmi_decoder_component_float.argtypes = [i, i, ctypes.POINTER(i)]
        L.bmi_decoder_component_float.restype = vp
        L.bmi_decoder_release.argtypes = [i]
        L.bmi_decoder_release.restype = None
        L.bmi_decoder_terminate.restype = None
        _lib = L
    return _lib


def status_string(code):
    try:
        return lib().j2k_status_string(int(code)).decode()
    except Exception:  # noqa: BLE001 - message helper only
        return "?"


def enc():
    global _enc
    if _enc is None:
        if not os.path.exists(ENC_PATH):
            raise RuntimeError("encoder library %s is missing: run jpeg2000-decoder_b200/build.py" % ENC_PATH)
        E = ctypes.CDLL(ENC_PATH)
        E.j2kenc_default_params.argtypes = [ctypes.POINTER(EncParams)]
        E.j2kenc_default_params.restype = None
        E.j2kenc_encode.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(EncParams), ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)),
                                    ctypes.POINTER(ctypes.c_size_t)]
        E.j2kenc_free.argtypes = [ctypes.c_void_p]
        E.j2kenc_free.restype = None
        _enc = E
    return _enc


def encode(planes, bitdepth, **kw):
    """Encode a (ncomp, H, W) uint16 array; keyword names follow j2kenc_params."""
    E = enc()
    p = EncParams()
    E.j2kenc_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if k == "layer_bpp":
            for n, x in enumerate(v):
                p.layer_bpp[n] = float(x)
        elif k in ("sub_x", "sub_y"):  # per-component sub-sampling factors
            arr = getattr(p, k)
            for n, x in enumerate(v):
                arr[n] = int(x)
        elif k == "poc":  # list of (RS, CS, LYE, RE, CE, progression)
            p.num_poc = len(v)
            for n, e in enumerate(v):
                for j, x in enumerate(e):
                    p.poc[n][j] = int(x)
        else:
            setattr(p, k, v)
    a = np.ascontiguousarray(planes, dtype=np.uint16)
    if a.ndim == 2:
        a = a[None]
    c, h, w = a.shape
    out = ctypes.POINTER(ctypes.c_uint8)()
    n = ctypes.c_size_t()
    rc = E.j2kenc_encode(a.ctypes.data_as(ctypes.c_void_p), w, h, c, bitdepth, ctypes.byref(p), ctypes.byref(out),
                         ctypes.byref(n))
    if rc != 0:
        raise ValueError("j2kenc_encode failed: %d" % rc)
    try:
        return ctypes.string_at(out, n.value)
    finally:
        E.j2kenc_free(out)


class Plan:
    """Host Tier-2 result of one codestream (j2k_plan_*)."""

    def __init__(self, codestream, discard_levels=0, max_layers=0, ignore_components=0, threads=1):
        self._cs = bytes(codestream)
        self.h = ctypes.c_void_p()
        rc = lib().j2k_plan_create_mt(self._cs, len(self._cs), discard_levels, max_layers, ignore_components,
                                      threads, ctypes.byref(self.h))
        if rc != J2K_OK:
            raise J2kError(rc, "j2k_plan_create")
        self.info = ImageInfo()
        lib().j2k_plan_info(self.h, ctypes.byref(self.info))

    def close(self):
        if self.h:
            lib().j2k_plan_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def cblks(self):
        n = self.info.num_cblks
        if n == 0:
            return (CodeBlock * 0)()
        return (CodeBlock * n).from_address(lib().j2k_plan_cblks(self.h))

    def tilecomps(self):
        return (TileComp * self.info.num_tilecomps).from_address(lib().j2k_plan_tilecomps(self.h))

    def bytes_ptr(self):
        return ctypes.c_void_p(lib().j2k_plan_bytes(self.h))

    def seglens_ptr(self):
        return ctypes.c_void_p(lib().j2k_plan_seglens(self.h))

    def output_bytes(self, fmt):
        return lib().j2k_output_bytes(ctypes.byref(self.info), fmt)


class GpuContext:
    """j2k_gpu context: batches of plans decoded by the sm_100a kernels."""

    def __init__(self, device=0, mem_budget=0):
        self.h = ctypes.c_void_p()
        rc = lib().j2k_gpu_ctx_create(device, mem_budget, ctypes.byref(self.h))
        if rc != J2K_OK:
            raise J2kError(rc, "j2k_gpu_ctx_create")
        self.plans = []

    def close(self):
        if self.h:
            lib().j2k_gpu_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def _ck(self, rc, what):
        if rc != J2K_OK:
            raise J2kError(rc, what)

    def begin(self):
        self.plans = []
        self._ck(lib().j2k_gpu_batch_begin(self.h), "batch_begin")

    def add(self, plan, fmt=FMT_NONE, flags=0):
        slot = ctypes.c_int()
        self._ck(lib().j2k_gpu_batch_add(self.h, plan.h, fmt, flags, ctypes.byref(slot)), "batch_add")
        self.plans.append((plan, fmt))
        return slot.value

    def footprint(self):
        n = ctypes.c_size_t()
        self._ck(lib().j2k_gpu_batch_footprint(self.h, ctypes.byref(n)), "batch_footprint")
        return n.value

    def launch(self, stream=None):
        self._ck(lib().j2k_gpu_batch_launch(self.h, stream), "batch_launch")

    def stage(self, stream=None):
        self._ck(lib().j2k_gpu_batch_stage(self.h, stream), "batch_stage")

    def run(self, stream=None):
        self._ck(lib().j2k_gpu_batch_run(self.h, stream), "batch_run")

    def sync(self, timeout_ms=-1):
        return lib().j2k_gpu_batch_sync(self.h, timeout_ms)

    def status(self, slot):
        bad = ctypes.c_int()
        rc = lib().j2k_gpu_image_status(self.h, slot, ctypes.byref(bad))
        return rc, bad.value

    def output_device(self, slot):
        p = ctypes.c_void_p()
        n = ctypes.c_size_t()
        self._ck(lib().j2k_gpu_output_device(self.h, slot, ctypes.byref(p), ctypes.byref(n)), "output_device")
        return p.value, n.value

    def output(self, slot):
        plan, fmt = self.plans[slot]
        n = plan.output_bytes(fmt)
        out = np.empty(n, np.uint8)
        self._ck(lib().j2k_gpu_output_copy(self.h, slot, out.ctypes.data_as(ctypes.c_void_p), n), "output_copy")
        return out

    def output_async(self, slot, ptr, nbytes):
        """Enqueue the copy of a slot's output to host address `ptr` (pinned) behind the
        decode; the next sync() covers it.  The buffer must outlive that sync."""
        self._ck(lib().j2k_gpu_output_copy_async(self.h, slot, ctypes.c_void_p(ptr), nbytes), "output_copy_async")

    def component(self, slot, comp):
        plan, _ = self.plans[slot]
        I = plan.info
        dt = np.int32 if I.reversible else np.float32
        out = np.empty((I.height, I.width), dt)
        self._ck(lib().j2k_gpu_component_copy(self.h, slot, comp, out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
                 "component_copy")
        return out

    def coefficients(self, slot, stage):
        plan, _ = self.plans[slot]
        I = plan.info
        dt = np.int32 if I.reversible else np.float32
        out = np.empty(max(1, I.coef_elems), dt)
        self._ck(lib().j2k_gpu_coefficients_copy(self.h, slot, stage, out.ctypes.data_as(ctypes.c_void_p),
                                                 out.nbytes), "coefficients_copy")
        return out

    def timing(self):
        v = [ctypes.c_float() for _ in range(4)]
        self._ck(lib().j2k_gpu_last_timing(self.h, *[ctypes.byref(x) for x in v]), "last_timing")
        return dict(t1_ms=v[0].value, dwt_ms=v[1].value, h2d_ms=v[2].value, total_ms=v[3].value)

    def launches(self):
        n = ctypes.c_int()
        self._ck(lib().j2k_gpu_last_launches(self.h, ctypes.byref(n)), "last_launches")
        return n.value

    def set_tuning(self, t1_warps_per_cta=0, dwt_tile=0, use_graph=0, t1_form=0, t1_latency_waves=0, dwt_coarse=0):
        t = Tuning(t1_warps_per_cta, dwt_tile, use_graph, t1_form, t1_latency_waves, dwt_coarse)
        self._ck(lib().j2k_gpu_set_tuning(self.h, ctypes.byref(t)), "set_tuning")

    def get_tuning(self):
        t = Tuning()
        self._ck(lib().j2k_gpu_get_tuning(self.h, ctypes.byref(t)), "get_tuning")
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def autotune(self, iters=2, stream=None):
        """Time the staged batch under each Tier-1 form / CTA width; the auto form then uses
        the winner for batches of this size.  Returns (winner tuning dict, Tier-1 ms)."""
        t, ms = Tuning(), ctypes.c_float()
        self._ck(lib().j2k_gpu_autotune(self.h, stream, iters, ctypes.byref(t), ctypes.byref(ms)), "autotune")
        return {k: getattr(t, k) for k, _ in Tuning._fields_}, ms.value

    def mem_usage(self):
        r, b = ctypes.c_size_t(), ctypes.c_size_t()
        self._ck(lib().j2k_gpu_mem_usage(self.h, ctypes.byref(r), ctypes.byref(b)), "mem_usage")
        return r.value, b.value

    def decode(self, codestream, fmt, flags=0):
        """One image, host in / host out."""
        plan = Plan(codestream)
        self.begin()
        slot = self.add(plan, fmt, flags)
        self.launch()
        self._ck(self.sync(), "batch_sync")
        out = self.output(slot) if fmt != FMT_NONE else None
        rc, bad = self.status(slot)
        return out, rc, bad, plan


class Server:
    """Continuous-batching decode service (include/j2k_server.h): submit codestreams as they
    arrive, wait for each result; pending requests are merged into shared launches."""

    def __init__(self, device=0, mem_budget=0, pipeline_depth=2, max_batch_images=0, max_batch_pixels=0):
        cfg = ServerConfig(device, mem_budget, pipeline_depth, max_batch_images, max_batch_pixels)
        h = ctypes.c_void_p()
        rc = lib().j2k_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != J2K_OK:
            raise J2kError(rc, "server_create")
        self.h = h

    def submit(self, codestream, fmt, flags=0):
        rid = lib().j2k_server_submit(self.h, codestream, len(codestream), fmt, flags)
        if rid < 0:
            raise J2kError(int(rid), "server_submit")
        return rid

    def wait(self, rid, out=None, timeout_ms=-1):
        """Returns (status, bytes); copies the output into `out` (a uint8 numpy array)."""
        n = ctypes.c_size_t()
        ptr = out.ctypes.data_as(ctypes.c_void_p) if out is not None else None
        cap = out.nbytes if out is not None else 0
        rc = lib().j2k_server_wait(self.h, rid, ptr, cap, ctypes.byref(n), timeout_ms)
        return rc, n.value

    def result(self, rid):
        rc, n = self.wait(rid)
        if rc != J2K_OK:
            raise J2kError(rc, "server request %d" % rid)
        out = np.empty(n, np.uint8)
        rc, _ = self.wait(rid, out)
        if rc != J2K_OK:
            raise J2kError(rc, "server request %d" % rid)
        return out

    def view(self, rid, timeout_ms=-1):
        """(status, zero-copy uint8 view of the output, valid until release)."""
        ptr, n = ctypes.c_void_p(), ctypes.c_size_t()
        rc = lib().j2k_server_result(self.h, rid, ctypes.byref(ptr), ctypes.byref(n), timeout_ms)
        if rc != J2K_OK or not ptr.value or not n.value:
            return rc, None
        return rc, np.ctypeslib.as_array((ctypes.c_uint8 * n.value).from_address(ptr.value))

    def latency_us(self, rid):
        v = ctypes.c_double()
        rc = lib().j2k_server_latency_us(self.h, rid, ctypes.byref(v))
        if rc != J2K_OK:
            raise J2kError(rc, "server_latency")
        return v.value

    def release(self, rid):
        lib().j2k_server_release(self.h, rid)

    def drain(self):
        lib().j2k_server_drain(self.h)

    def stats(self):
        st = ServerStats()
        lib().j2k_server_stats_get(self.h, ctypes.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def reset_stats(self):
        lib().j2k_server_stats_reset(self.h)

    def close(self):
        if self.h:
            lib().j2k_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
