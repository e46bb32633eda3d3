"""Throughput benchmark of the B200 JPEG 2000 Part-1 decode path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3|c2|c4|c1|c5] [--impl ours|reference]
    python bench.py --workload c3 --frames 16 --decode-repeat 2 [--t1-form 1]   (profiling mode)

Default workload (metric: Mpixel/s decoded, batched): the batched video-frame decode —
64 frames of 1920x1080 RGB 8-bit, 9/7 + ICT, 512x512 tiles, 5 levels, 64x64 code-blocks,
3 quality layers (~0.5/1/2 bpp), decoded at full layers; all code-blocks of all frames in
one Tier-1 launch, all tile-components in shared DWT level launches.  Inputs are seeded
synthetic frames encoded by the project's writer (no dataset); 16 distinct frames are
encoded and each appears 4 times in the batch (identical decode work per copy).

One step = one decode of the whole batch.  `value` times steps with the coded bytes and
work lists resident in HBM (CUDA events on the launch stream, L2 flushed between steps);
`e2e` times the public C-ABI path from host memory: host Tier-2 of every frame,
pinned H2D, decode, D2H of every decoded picture into pinned host buffers, with two contexts
alternating so one step's host work overlaps the previous step's decode.  `--workload c5` runs the serving stream
through the continuous-batching service instead (see run_serve).  Multi-GPU runs are replicas (each rank
decodes its own copy of the batch; images are independent, no collective on the data path).
"""
import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))


def load_package():
    name = "jpeg2000_decoder_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "jpeg2000-decoder_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()
from jpeg2000_decoder_b200 import native, synth  # noqa: E402

METRIC = "Mpixel/s decoded (batched+served vs plain GPU path); p50/p99 decode latency"


def workload(name, quick=False):
    return synth.workload(name, quick)


def parse_all(streams, pool):
    return list(pool.map(native.Plan, streams))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = "/tmp/j2k_clocks_%d.csv" % os.getpid()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except OSError:
            return None
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 3 + i and "Active" in r[3 + i]
                          and "Not" not in r[3 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


T1_FORMS = {1: "compact (one block per warp)", 2: "unrolled (one block per warp)", 3: "lanes (one block per lane)"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic():
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# ------------------------------------------------------------------ replicas ----------
def max_over_ranks(seconds_or_ms, dist, device="cuda"):
    """The slowest rank's time (the job's time): replicas decode independent copies and
    meet only here, so the job finishes when the last one does."""
    if not dist:
        return float(seconds_or_ms)
    import torch
    t = torch.tensor([float(seconds_or_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, world, steps, total_time_s):
    """Whole-job units per second: every rank processed `units_per_rank` per step."""
    return units_per_rank * world * steps / total_time_s


# ------------------------------------------------------------------ CPU baselines -------
def host_cores():
    """Host threads this process may run on (its CPU affinity), else the machine's count."""
    try:
        return len(os.sched_getaffinity(0)) or 1
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def reference_sample(name, streams):
    """Codestreams of this workload that the reference's own decoder takes, and what they are.

    C1, C2 and the serving requests are single-tile pictures it decodes (bit-exact against
    ours, tests/test_cpu_reference_pictures.py).  It segfaults on C3's frames (their partial
    512x512 edge tiles), so C3 is sampled by the same coding parameters on the 3 x 2 full
    tiles of C3 frames.  Its Tier-1 has no BYPASS / RESET (bmi_mq_decoder.cpp:206-210), so C4
    has no reference sample."""
    if name == "c3":
        frames = synth.video_frames(3, n=4)
        cs = [native.encode(np.ascontiguousarray(f[:, :1024, :1536]), 8, **synth.C3_PARAMS) for f in frames]
        return cs, ("C3 coding parameters (9/7+ICT, 512x512 tiles, 3 layers) on the 3x2 full tiles (1536x1024) of "
                    "4 C3 frames; the reference's decoder segfaults on C3's partial edge tiles")
    if name in ("c1", "c2"):
        return list(streams[:1]), "the workload's picture"
    if name == "c5":
        return list(streams), "the %d distinct requests of the serving pool" % len(streams)
    return None, "no reference sample: the reference's Tier-1 implements no BYPASS / RESET"


def reference_cpu(name, streams, fmt, steps, warmup, workers=None, step_seconds=1.0, per_process=20):
    """The reference's own CPU decoder (BMI::Decoder built from its sources into
    oracle/_ref/libref_cpu.so; oracle/ref_cpu_runner.py runs it in child processes) on the
    workload's reference sample, on every host core.

    The reference engine's worker threads race: with several workers per engine it stops
    after a few dozen decodes (a picture whose status never leaves PARSING, or a segfault),
    while single-worker engines decode reliably.  So the host's cores each run their own
    single-worker engine process (EnginConfig::mThreadNum = 1), each decoding one sample
    picture over and over (pictures assigned round-robin), at most `per_process` timed
    decodes per process after one untimed decode of its own; each decode is timed inside
    its process as the wall clock of Decode() + GetResult() (the reference's Tier-2
    included).  One step = `passes` decodes per process, as many as fill about
    `step_seconds`; a step lasts as long as its slowest process.  None when the library
    or a sample is missing."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_cpu_runner
    if not ref_cpu_runner.available():
        return None
    cs, what = reference_sample(name, streams)
    if not cs:
        return None
    workers = workers or host_cores()
    fmts = [fmt if fmt is not None else synth.c5_format(c) for c in cs]

    def timed(i, n):
        """n timed decodes of sample picture i on a single-worker engine: ms each, size."""
        out, size = [], None
        while len(out) < n:
            k = min(per_process, n - len(out))
            r = ref_cpu_runner.decode([cs[i]], fmts[i], threads=1, reps=k + 1, timeout=600, time_only=True)
            if not r["ok"]:
                raise RuntimeError(r["error"])
            out += r["ms"][0][1:]
            size = r["sizes"][0]
        return out, size

    try:
        one_ms = max(timed(i, 1)[0][0] for i in range(len(cs)))
        passes = max(1, int(round(step_seconds * 1e3 / max(one_ms, 1e-3))))
        n = (warmup + steps) * passes
        with ThreadPoolExecutor(max_workers=workers) as ex:
            runs = list(ex.map(lambda w: timed(w % len(cs), n), range(workers)))
    except RuntimeError as e:
        return {"error": str(e)}
    step_ms = [max(sum(ms[(warmup + k) * passes:(warmup + k + 1) * passes]) for ms, _ in runs) for k in range(steps)]
    px = sum(w * h for _, (w, h) in runs) * passes * steps
    total_s = sum(step_ms) / 1e3
    return {"value": px / total_s / 1e6, "unit": "Mpixel/s", "cores": workers, "kind": "reference",
            "sample": "%s; %d single-worker reference engines (one per host core) each decoding %d pictures per "
                      "step, %d timed steps after %d warm-up steps, %.1f s" % (
                          what, workers, passes, steps, warmup, total_s),
            "ms_per_step": total_s * 1e3 / steps}


def cpu_decode_sample(streams, fmt, budget_s=15.0, threads=None):
    """The CPU restatement of the reference's path (oracle/liboracle.so) on a bounded sample
    of the workload: one picture per host thread at a time (host Tier-2 of each picture
    inside the timed loop); `cores` is the number of threads that had a picture."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from jpeg2000_decoder_b200 import build
    build.build_oracle()
    import oracle_util
    threads = threads or host_cores()
    sample = list(streams[:max(1, min(len(streams), threads))])
    used = min(len(sample), threads)

    def one(cs):
        p = native.Plan(cs)
        f = fmt if fmt is not None else (native.FMT_24BITS_RGB if p.info.bitdepth <= 8 else native.FMT_48BITS_RGB)
        oracle_util.oracle_decode(p, f)
        return p.info.width * p.info.height

    orc = oracle_util.orc()
    orc.oracle_decisions.restype = ctypes.c_ulonglong
    with ThreadPoolExecutor(max_workers=used) as ex:
        d0 = orc.oracle_decisions()
        t0 = time.perf_counter()
        px = 0
        rounds = 0
        while True:
            px += sum(ex.map(one, sample))
            rounds += 1
            if time.perf_counter() - t0 > budget_s or rounds >= 8:
                break
        dt = time.perf_counter() - t0
        decisions_per_px = (orc.oracle_decisions() - d0) / max(1, px)
    cpu_decode_sample.decisions_per_px = decisions_per_px
    return {"value": px / dt / 1e6, "unit": "Mpixel/s", "cores": used, "kind": "port",
            "sample": "%d picture decodes (%d distinct, host Tier-2 included) in %.1f s on %d threads" % (
                rounds * len(sample), len(sample), dt, used)}


cpu_decode_sample.decisions_per_px = None


def cpu_baseline(name, streams, fmt, steps=10, warmup=2, port_budget=8.0):
    """The reference where it decodes the workload, else the CPU restatement; the port's
    figure rides along, so the reader can scale one by the other."""
    ref = reference_cpu(name, streams, fmt, steps, warmup, step_seconds=1.0)
    port = cpu_decode_sample(streams, fmt, budget_s=port_budget)
    if ref and "error" not in ref:
        out = dict(ref)
        out["port"] = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in port.items()}
        return out
    out = dict(port)
    if ref:
        out["reference_error"] = ref["error"]
    return out


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    cfg, streams, fmt = workload(args.workload, args.quick)
    base = reference_cpu(args.workload, streams, fmt, args.steps, args.warmup)
    if not base or "error" in base:
        port = [cpu_decode_sample(streams, fmt, budget_s=1.0) for _ in range(args.warmup)]
        port = [cpu_decode_sample(streams, fmt, budget_s=5.0) for _ in range(args.steps)]
        reason = base["error"] if base else reference_sample(args.workload, streams)[1]
        base = dict(port[-1], value=float(np.median([p["value"] for p in port])), reference_unavailable=reason)
    value = base["value"]
    line = {"metric": METRIC, "value": round(value, 3), "unit": "Mpixel/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/int32", "data": "synthetic (seeded, project encoder)", "config": cfg, "impl": "reference",
            "cpu_baseline": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in base.items()},
            "e2e": {"value": round(value, 3), "unit": "Mpixel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------ GPU arm -----------
def fp64_check(ctx, plans, fmt, frames=2, fmts=None):
    """PSNR and max-abs of the device's packed 9/7 pictures against an FP64 T.800
    synthesis (tests/fp64_97.py) of the device's own Tier-1 values, on the first `frames`
    pictures of the batch.  Each block's Tier-1 values are its stage-0 coefficients divided
    by the block's gain (exact to float32 rounding, ~1e-7 relative), so the comparison
    measures the FP32 dequantisation, lifting, ICT and (int) truncation only."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import fp64_97
    worst_psnr, worst_abs = float("inf"), 0.0
    for n, p in enumerate(plans[:frames]):
        if fmts is not None:
            fmt = fmts[n]
        ctx.begin()
        slot = ctx.add(p, fmt)  # the benched path: last level fused with the ICT and pack
        ctx.launch()
        assert ctx.sync() == 0
        coef = ctx.coefficients(slot, 0).astype(np.float64)
        out = ctx.output(slot)

        def raw(i, cb, coef=coef):
            v = np.empty((cb.h, cb.w))
            for y in range(cb.h):
                o = cb.out_off + y * cb.out_stride
                v[y] = coef[o:o + cb.w] / cb.gain
            return v
        want = fp64_97.synthesize(p, raw)
        I = p.info
        if fmt == native.FMT_24BITS_RGB:
            got = out.reshape(I.height, I.width, 3)[:, :, [2, 1, 0]].transpose(2, 0, 1)
        elif fmt == native.FMT_48BITS_RGB:
            got = out.view(np.uint16).reshape(I.height, I.width, 3)[:, :, [2, 1, 0]].transpose(2, 0, 1) >> (
                16 - I.bitdepth)
        else:
            return None
        ps, mx = fp64_97.psnr_maxabs(got, want, I.bitdepth)
        worst_psnr, worst_abs = min(worst_psnr, ps), max(worst_abs, mx)
    return {"pictures": min(frames, len(plans)), "psnr_db_min": round(worst_psnr, 2), "max_abs": round(worst_abs, 3),
            "against": "FP64 T.800 dequantisation + 9/7 synthesis + ICT of the same Tier-1 values, before rounding"}


def build_workloads_once(items, rank, dist):
    """Rank 0 encodes the workloads ((name, quick) pairs) into the cache while the other
    ranks wait, so N ranks do not all encode the same pictures at once."""
    if dist:
        if rank == 0:
            for name, quick in items:
                workload(name, quick)
        dist.barrier()


def run_gpu(args, rank, world, dist):
    import torch
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    build_workloads_once([(args.workload, args.quick)] +
                         ([("c5", False)] if args.workload != "c5" and not args.no_serving else []), rank, dist)
    cfg, streams, fmt = workload(args.workload, args.quick)
    pool = ThreadPoolExecutor(max_workers=os.cpu_count())
    plans = parse_all(streams, pool)
    pixels = sum(p.info.width * p.info.height for p in plans)
    ctx = native.GpuContext(dev)
    stream = torch.cuda.Stream()  # a real stream handle: the decode and the events share it
    sp = ctypes.c_void_p(stream.cuda_stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")  # 256 MB > L2

    # ---- device-resident decode (value)
    ctx.begin()
    for p in plans:
        ctx.add(p, fmt)
    ctx.stage(sp)
    tuned = None
    if not args.no_autotune:
        tuned, _ = ctx.autotune(2, sp)
    ctx.set_tuning(use_graph=0 if args.no_graph else 1)
    for _ in range(args.warmup):
        ctx.run(sp)
        assert ctx.sync() == 0
    launches_per_step = ctx.launches()
    bad = sum(ctx.status(i)[1] for i in range(len(plans)))
    times, t1s, dwts = [], [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.run(sp)
            e1.record(stream)
            assert ctx.sync() == 0
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            tm = ctx.timing()
            t1s.append(tm["t1_ms"])
            dwts.append(tm["dwt_ms"])
    torch.cuda.synchronize()
    step_ms = float(np.mean(times))
    total_ms = float(np.sum(times))
    total_ms = max_over_ranks(total_ms, dist)
    value = replica_throughput(pixels, world, args.steps, total_ms / 1e3) / 1e6

    ctx.set_tuning(use_graph=0)  # the batches below are decoded once each: nothing to replay
    # ---- plain per-image GPU path: one image per launch sequence
    plain_ms = []
    uniq = plans[: min(len(plans), 16)]
    for it in range(2):
        t0 = time.perf_counter()
        for p in uniq:
            ctx.begin()
            ctx.add(p, fmt)
            ctx.launch(sp)
            assert ctx.sync() == 0
        if it:
            plain_ms.append((time.perf_counter() - t0) * 1e3)
    plain = sum(p.info.width * p.info.height for p in uniq) / (plain_ms[0] / 1e3) / 1e6

    # ---- end to end through the C ABI with host buffers.  Each step: host Tier-2 of every
    # codestream, stage (pinned) + H2D, decode, D2H of every picture into pinned host
    # buffers (enqueued behind the decode, so they overlap the host's next step).  Two
    # contexts alternate, so the host work of one step overlaps the device decode of the
    # previous one, as a decoding service would run; the time is the wall clock from the
    # first step's parse to the last step's pictures on the host.  (The library starts a
    # step whose Tier-1 fills the GPU after the previous step's decode; smaller ones overlap.)
    import torch
    ctx2 = native.GpuContext(dev)
    ctxs = [ctx, ctx2]
    e2e_streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    e2e_sp = [ctypes.c_void_p(x.cuda_stream) for x in e2e_streams]
    outs = [[torch.empty(p.output_bytes(fmt), dtype=torch.uint8).pin_memory() for p in plans] for _ in range(2)]
    h2d = sum(p.info.coded_bytes for p in plans)
    d2h = sum(o.numel() for o in outs[0])

    host_ms = {"parse": 0.0, "stage_launch": 0.0, "wait": 0.0}

    def e2e_run(nsteps):
        pending = None
        for it in range(nsteps):
            k = it % 2
            t0 = time.perf_counter()
            ps = parse_all(streams, pool)
            t1 = time.perf_counter()
            ctxs[k].begin()
            for p in ps:
                ctxs[k].add(p, fmt)
            ctxs[k].launch(e2e_sp[k])
            for i, o in enumerate(outs[k]):
                ctxs[k].output_async(i, o.data_ptr(), o.numel())
            t2 = time.perf_counter()
            if pending is not None:
                assert ctxs[pending].sync() == 0
            t3 = time.perf_counter()
            host_ms["parse"] += (t1 - t0) * 1e3
            host_ms["stage_launch"] += (t2 - t1) * 1e3
            host_ms["wait"] += (t3 - t2) * 1e3
            pending = k
        assert ctxs[pending].sync() == 0

    e2e_run(2)  # warm: both contexts' pools and pinned buffers at size
    # at least 20 steps: the first step's host Tier-2 and staging and the last step's D2H are
    # not overlapped (about 8 ms each on C3), so over 10 steps they add ~1.6 ms to a step
    n_e2e = max(20, args.steps)
    for key in host_ms:
        host_ms[key] = 0.0
    t0 = time.perf_counter()
    e2e_run(n_e2e)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist)
    e2e = replica_throughput(pixels, world, n_e2e, e2e_s) / 1e6
    e2e_ms = [e2e_s * 1e3 / n_e2e]
    ctx2.close()

    # ---- PSNR / max-abs of the FP32 9/7 path against an FP64 synthesis of the same Tier-1
    # (rank 0 only: it is reported once, and the FP64 synthesis is host work the other ranks'
    # processes would repeat on the same cores)
    fp64 = (fp64_check(ctx, plans, fmt) if rank == 0 and not plans[0].info.reversible and not args.no_fp64
            else None)

    # ---- a shortened serving stream (C5 mix) through the continuous-batching service
    serving = None
    if args.workload != "c5" and not args.no_serving:
        _, spool, _ = workload("c5", False)  # the full pool of 48 distinct seeded requests
        # three warm-up passes: the device pools and the pinned output arena reach their
        # steady-state sizes before the timed pass
        m = serve_measure(dev, spool, args.serving_requests, args.depth, args.batch_mpix, 0.0, 3, 5 + rank, dist)
        _, serving = serving_summary(m, world)
        serving["stream"] = "C5 mix: %d requests drawn from %d distinct seeded requests" % (
            args.serving_requests, len(spool))

    if rank != 0:
        return
    # ---- roofline of the dominant kernel (Tier-1) and of the DWT + MCT stage
    t1_ms = float(np.mean(t1s))
    dwt_ms = float(np.mean(dwts))
    samples = sum(p.info.coef_elems for p in plans)
    coded = sum(p.info.coded_bytes for p in plans)
    out_bytes = d2h
    peak, peak_kind = measured_peaks()
    t1_bytes = coded + 4 * samples
    dwt_bytes = 4 * samples + out_bytes
    tr = profile_traffic().get(args.workload, {})
    dominant = "t1" if t1_ms >= dwt_ms else "dwt"
    roof_t1 = {"bound": "hbm", "achieved": round(t1_bytes / (t1_ms / 1e3) / 1e9, 2), "peak": peak, "unit": "GB/s",
               "frac": round(t1_bytes / (t1_ms / 1e3) / 1e9 / peak, 4), "traffic": tr.get("t1_bytes_per_launch"),
               "kernel": "t1_kernel", "peak_source": peak_kind, "algorithmic_bytes": t1_bytes,
               "ms_per_launch": round(t1_ms, 4), "note": "serial MQ decode: issue/latency bound, not HBM bound"}
    roof_dwt = {"bound": "hbm", "achieved": round(dwt_bytes / (dwt_ms / 1e3) / 1e9, 2), "peak": peak, "unit": "GB/s",
                "frac": round(dwt_bytes / (dwt_ms / 1e3) / 1e9 / peak, 4), "traffic": tr.get("dwt_bytes_per_step"),
                "kernel": "dwt_level_kernel + output_kernel", "peak_source": peak_kind,
                "algorithmic_bytes": dwt_bytes, "ms_per_step": round(dwt_ms, 4)}
    base = cpu_baseline(args.workload, streams, fmt, port_budget=args.cpu_budget)
    dpp = cpu_decode_sample.decisions_per_px
    if dpp:
        # Tier-1 work rate: decisions of the standard decoding process (MQ symbols incl. run
        # and uniform ones, raw bits; counted by the CPU restatement on the sample, whose
        # pictures are those of the batch) and compressed bytes per second of Tier-1 time
        roof_t1["decisions_per_s"] = round(dpp * pixels / (t1_ms / 1e3), 1)
        roof_t1["decisions_per_px"] = round(dpp, 3)
    roof_t1["compressed_bytes_per_s"] = round(coded / (t1_ms / 1e3), 1)
    clocks = clk.summary()
    # Tier-1 is bound by instruction issue: its own roofline is warp instructions issued per
    # second (live decisions/s x the warp instructions per decision of the profiled compact
    # form) against 4 issue slots per SM per cycle at the sampled SM clock
    roof_t1_issue = None
    ipd = tr.get("t1_warp_inst_per_decision")
    if dpp and ipd and tuned and tuned["t1_form"] == 1 and clocks.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        peak_issue = sms * 4 * clocks["sm_mhz"] * 1e6
        achieved = dpp * pixels / (t1_ms / 1e3) * ipd
        roof_t1_issue = {"bound": "issue", "achieved": round(achieved / 1e9, 1), "peak": round(peak_issue / 1e9, 1),
                         "unit": "Gwarp-inst/s", "frac": round(achieved / peak_issue, 4),
                         "warp_inst_per_decision": ipd, "kernel": "t1_kernel_compact",
                         "source": "profiles/traffic.json (ncu instruction count of the same kernel)"}
    cfg = dict(cfg)
    cfg.update({"parallelism": "replicas x%d" % world, "l2": "flushed between steps (256 MB write)",
                "bad_blocks": bad, "cuda_graph": not args.no_graph,
                "autotuned_t1": ({"form": T1_FORMS.get(tuned["t1_form"], "auto"),
                                  "warps_per_cta": tuned["t1_warps_per_cta"]} if tuned else None),
                "autotuned_dwt": ({"coarse_levels": "one shared-memory kernel" if tuned["dwt_coarse"] == 1
                                   else "one launch per level",
                                   "candidates": ["coarse levels (<= 64 a side) in one kernel",
                                                  "one launch per level"]} if tuned else None)})
    line = {"metric": METRIC, "value": round(value, 2), "unit": "Mpixel/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(step_ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (9/7) / int32 (5/3)", "data": "synthetic (seeded, project encoder)",
            "config": cfg,
            "e2e": {"value": round(e2e, 2), "unit": "Mpixel/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": round(float(np.median(e2e_ms)), 3),
                    "steps": n_e2e,
                    "includes": "per step: host Tier-2 of every codestream, staging + H2D, decode, D2H of every "
                                "picture into pinned host buffers; two contexts alternate so one step's host "
                                "work overlaps the previous step's decode (wall clock over the steps, pipeline "
                                "fill and drain included)",
                    "host_ms_per_step": {k: round(v / n_e2e, 3) for k, v in host_ms.items()}},
            "plain_gpu_path": {"value": round(plain, 2), "unit": "Mpixel/s", "images": len(uniq),
                               "what": "one image per launch sequence, host buffers"},
            "speedup_vs_plain": round(e2e / plain, 2),
            "speedup_vs_plain_note": "e2e / plain_gpu_path: both host buffer to host buffer, wall clock",
            "roofline": roof_t1 if dominant == "t1" else roof_dwt,
            "roofline_dwt": roof_dwt, "roofline_t1": roof_t1, "roofline_t1_issue": roof_t1_issue,
            "stage_ms": {"t1": round(t1_ms, 4), "dwt_mct": round(dwt_ms, 4)},
            "cpu_baseline": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in base.items()},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks}
    if fp64:
        line["config"]["fp64_check"] = fp64
    if serving:
        line["serving"] = serving
    print(json.dumps(line))


# ------------------------------------------------------------------ serving (C5) -------
def serve_measure(dev, pool, n_req, depth, batch_mpix, rate=0.0, warmup=1, seed=5, dist=None, sampler=None):
    """Requests of mixed size / depth / wavelet through the continuous-batching service.

    Phase 1 (throughput): the whole request stream is submitted at once from several
    threads while client threads take and release each result; Mpixel/s over that wall time
    (codestreams in host memory, packed pixels back in host memory: an end-to-end figure).
    Phase 2 (latency): Poisson arrivals at `rate` requests/s (default 70 % of the phase-1
    request rate); p50 / p99 are submit-to-result times.  The plain path decodes the same
    stream one request per launch sequence on one context, also host buffer to host buffer,
    so plain and served are measured the same way."""
    import threading

    import torch
    fmts = [synth.c5_format(cs) for cs in pool]
    px_of = [native.Plan(cs).info.width * native.Plan(cs).info.height for cs in pool]
    rng = np.random.default_rng(seed)
    order = [int(i) for i in rng.integers(0, len(pool), n_req)]
    total_px = sum(px_of[i] for i in order)

    # ---- plain path: one request per launch sequence
    ctx = native.GpuContext(dev)
    for i in range(len(pool)):
        ctx.decode(pool[i], fmts[i])
    n_plain = min(n_req, 4 * len(pool))
    t0 = time.perf_counter()
    for i in order[:n_plain]:
        _, rc, _, _ = ctx.decode(pool[i], fmts[i])
        assert rc == native.J2K_OK
    plain_s = time.perf_counter() - t0
    plain = sum(px_of[i] for i in order[:n_plain]) / plain_s / 1e6
    ctx.close()

    srv = native.Server(device=dev, pipeline_depth=depth, max_batch_pixels=int(batch_mpix * 2 ** 20))

    def serve_pass(idx, when=None):
        """Submit idx (at times `when` after the start, else at once) from 8 threads while 4
        client threads take each result (zero-copy view) in submission order and release
        it.  Returns (wall seconds, failed requests)."""
        ids = [None] * len(idx)
        ready = [threading.Event() for _ in idx]
        failed = [0]
        t_start = time.perf_counter()

        def submitter(k, nthreads):
            for j in range(k, len(idx), nthreads):
                if when is not None:
                    dt = t_start + when[j] - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                ids[j] = srv.submit(pool[idx[j]], fmts[idx[j]])
                ready[j].set()

        def client(k, nthreads):
            for j in range(k, len(idx), nthreads):
                ready[j].wait()
                rc, view = srv.view(ids[j])
                if rc != native.J2K_OK or view is None:
                    failed[0] += 1
                srv.release(ids[j])

        th = [threading.Thread(target=submitter, args=(k, 8)) for k in range(8)]
        th += [threading.Thread(target=client, args=(k, 4)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        return time.perf_counter() - t_start, failed[0]

    # ---- warm-up: the device pools and pinned buffers grow to their steady-state sizes
    for _ in range(max(3, warmup)):
        serve_pass(order)

    # ---- phase 1: saturation
    srv.reset_stats()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.__enter__()
    sat_s, bad = serve_pass(order)
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__()
    st1 = srv.stats()
    sat_s = max_over_ranks(sat_s, dist)

    # ---- phase 2: Poisson arrivals
    rate = rate or 0.7 * n_req / sat_s
    gaps = rng.exponential(1.0 / rate, n_req)
    when = np.cumsum(gaps) - gaps[0]
    srv.reset_stats()
    poisson_s, bad2 = serve_pass(order, when)
    st2 = srv.stats()
    srv.close()
    return {"order": order, "fmts": fmts, "total_px": total_px, "sat_s": sat_s, "bad": bad + bad2, "plain": plain,
            "n_plain": n_plain, "st1": st1, "st2": st2, "rate": rate, "poisson_s": poisson_s}


def serving_summary(m, world):
    n_req = len(m["order"])
    value = replica_throughput(m["total_px"], world, 1, m["sat_s"]) / 1e6
    st1, st2 = m["st1"], m["st2"]
    return value, {
        "saturation": {"mpix_s": round(value, 2), "requests_s": round(n_req / m["sat_s"], 1),
                       "gpu_busy_ms": round(st1["gpu_ms"], 2), "wall_ms": round(m["sat_s"] * 1e3, 2),
                       "host_stage_ms": round(st1["stage_ms"], 2), "host_enqueue_ms": round(st1["enqueue_ms"], 2),
                       "pool_growths": st1["pool_growths"], "pinned_allocs": st1["pinned_allocs"],
                       "batches": st1["batches"], "mean_batch_images": round(st1["mean_batch_images"], 2),
                       "p50_ms": round(st1["p50_us"] / 1e3, 3), "p99_ms": round(st1["p99_us"] / 1e3, 3)},
        "poisson": {"rate_rps": round(m["rate"], 1),
                    "offered_mpix_s": round(m["rate"] * m["total_px"] / n_req / 1e6, 1),
                    "achieved_mpix_s": round(m["total_px"] / m["poisson_s"] / 1e6, 2),
                    "p50_ms": round(st2["p50_us"] / 1e3, 3), "p99_ms": round(st2["p99_us"] / 1e3, 3),
                    "max_ms": round(st2["max_us"] / 1e3, 3), "batches": st2["batches"],
                    "mean_batch_images": round(st2["mean_batch_images"], 2)},
        "plain_gpu_path": {"mpix_s": round(m["plain"], 2), "requests": m["n_plain"],
                           "what": "one request per launch sequence, host buffer to host buffer"},
        "served_vs_plain": round(value / m["plain"], 2), "requests": n_req, "bad_requests": m["bad"]}


def run_serve(args, rank, world, dist):
    """C5: the serving stream (serve_measure) as the bench line."""
    import torch
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    build_workloads_once([("c5", args.quick)], rank, dist)
    cfg, pool, _ = workload("c5", args.quick)
    n_req = args.requests or (200 if args.quick else 2000)
    clk = ClockSampler(dev)
    m = serve_measure(dev, pool, n_req, args.depth, args.batch_mpix, args.rate, args.warmup, 5 + rank, dist, clk)
    if rank != 0:
        return
    value, serving = serving_summary(m, world)
    # FP64 error of the pool's 9/7 requests: the four of them with the fewest pixels that
    # cover both bit depths
    irr = sorted((native.Plan(cs) for cs in pool if not native.Plan(cs).info.reversible),
                 key=lambda p: p.info.width * p.info.height)
    pick = [p for p in irr if p.info.bitdepth == 8][:2] + [p for p in irr if p.info.bitdepth > 8][:2]
    fctx = native.GpuContext(dev)
    fp64 = fp64_check(fctx, pick, None, frames=len(pick),
                      fmts=[native.FMT_24BITS_RGB if p.info.bitdepth <= 8 else native.FMT_48BITS_RGB for p in pick])
    fctx.close()
    if fp64:
        fp64["requests"] = ["%dx%d %d-bit" % (p.info.width, p.info.height, p.info.bitdepth) for p in pick]
    base = cpu_baseline("c5", pool, None, port_budget=args.cpu_budget)
    order, fmts = m["order"], m["fmts"]
    h2d = sum(len(pool[i]) for i in order)
    cfg = dict(cfg)
    cfg.update({"requests": n_req, "pipeline_depth": args.depth, "batch_mpix_cap": args.batch_mpix,
                "parallelism": "replicas x%d" % world, "bad_requests": m["bad"],
                "l2": "inputs differ per request; no flush", "fp64_check": fp64})
    line = {"metric": METRIC, "value": round(value, 2), "unit": "Mpixel/s", "n_gpus": world, "steps": 1,
            "warmup": args.warmup, "ms_per_step": round(m["sat_s"] * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (9/7) / int32 (5/3)",
            "data": "synthetic (seeded requests, project encoder)", "config": cfg,
            "e2e": {"value": round(value, 2), "unit": "Mpixel/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(sum(native.Plan(pool[i]).output_bytes(fmts[i]) for i in order)),
                    "includes": "submit (host Tier-2) + merged batches + D2H of every request, wall clock"},
            "serving": serving,
            "plain_gpu_path": {"value": serving["plain_gpu_path"]["mpix_s"], "unit": "Mpixel/s",
                               "requests": m["n_plain"], "what": "one request per launch sequence, host buffers"},
            "speedup_vs_plain": serving["served_vs_plain"],
            "cpu_baseline": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in base.items()},
            "gpu_launches": int(m["st1"]["launches"]),
            "clocks": clk.summary()}
    print(json.dumps(line))


def run_decode_repeat(args):
    """Profiling mode: decode the workload (or its first --frames pictures) --decode-repeat
    times, one batch decode each, printing the stage times; no bench line.  Run it under
    ncu with -s / -c to capture a chosen launch of a chosen kernel."""
    import torch
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    cfg, streams, fmt = workload(args.workload, args.quick)
    if args.frames > 0:
        streams = streams[:args.frames]
    ctx = native.GpuContext(dev)
    ctx.set_tuning(t1_form=args.t1_form, dwt_coarse=args.dwt_coarse)
    plans = [native.Plan(s) for s in streams]
    for it in range(args.decode_repeat):
        ctx.begin()
        for p in plans:
            ctx.add(p, fmt)
        ctx.launch()
        rc = ctx.sync()
        if rc != 0:
            raise SystemExit("decode failed: %d" % rc)
        print(args.workload, it, ctx.timing(), "launches", ctx.launches(), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c3", choices=["c3", "c2", "c4", "c1", "c5"])
    ap.add_argument("--requests", type=int, default=0, help="c5: requests in the stream (default 2000)")
    ap.add_argument("--rate", type=float, default=0.0, help="c5: Poisson arrival rate, requests/s")
    ap.add_argument("--depth", type=int, default=2, help="c5: batches in flight")
    ap.add_argument("--batch-mpix", type=float, default=128, help="c5: pixel cap of one batch (Mpixel)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quick", action="store_true", help="small batch for smoke runs")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-autotune", action="store_true", help="skip the Tier-1 shape autotuner")
    ap.add_argument("--no-graph", action="store_true", help="enqueue launches instead of replaying a CUDA graph")
    ap.add_argument("--no-serving", action="store_true", help="skip the shortened serving stream of the default line")
    ap.add_argument("--serving-requests", type=int, default=960, help="requests of the shortened serving stream")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 error check")
    ap.add_argument("--decode-repeat", type=int, default=0,
                    help="profiling mode: decode the workload this many times, print stage times, no bench line")
    ap.add_argument("--frames", type=int, default=0, help="profiling mode: only the first N pictures")
    ap.add_argument("--t1-form", type=int, default=0, help="profiling mode: Tier-1 form 0 auto, 1 compact, 2 unrolled, 3 lanes")
    ap.add_argument("--dwt-coarse", type=int, default=0,
                    help="profiling mode: coarse DWT levels 0 auto, 1 fused into one kernel, 2 one launch per level")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.decode_repeat:
        run_decode_repeat(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        if args.workload == "c5":
            run_serve(args, rank, world, dist)
        else:
            run_gpu(args, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
