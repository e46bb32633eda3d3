"""Run the reference's own CPU decoder (oracle/_ref/libref_cpu.so) in a child process.

TEST AND BASELINE INFRASTRUCTURE ONLY.  The reference engine is a process-wide singleton
that segfaults on pictures with partial edge tiles (decoder/core/src/decoderconcrete.cpp
worker path; observed on every 1920x1080 picture with 512x512 tiles), so every use goes
through a child process with a time limit: a crash or a hang there costs the caller one
failed call, never its own process.

    decode(streams, fmt, threads=..., top_level=-1, reps=1, timeout=...) -> dict
        {"ok": bool, "error": str, "threads": n, "outputs": [bytes per stream] (first rep),
         "sizes": [(w, h)], "ms": [[ms per rep] per stream], "status": [BMI::Status per stream]}

Run as a script it is that child: it reads a request (pickle) from stdin and writes the
reply to the file named in the request.
"""
import os
import pickle
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_cpu.so")


def available():
    return os.path.exists(LIB)


def decode(streams, fmt, threads=None, top_level=-1, reps=1, timeout=120.0, time_only=False):
    """Decode each codestream `reps` times with the reference (status 0 = READY)."""
    if not available():
        return {"ok": False, "error": "reference library not built (oracle/build_ref_cpu.sh)"}
    threads = threads or os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "reply.pkl")
        req = {"streams": [bytes(s) for s in streams], "fmt": int(fmt), "threads": int(threads),
               "top_level": int(top_level), "reps": int(reps), "reply": out, "time_only": bool(time_only)}
        try:
            # cwd: the reference writes its debug log (jp2codecLog.txt) into the working directory
            p = subprocess.run([sys.executable, os.path.abspath(__file__)], input=pickle.dumps(req),
                               stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout, cwd=td)
        except subprocess.TimeoutExpired:
            return {"ok": False, "error": "reference decoder did not finish within %.0f s" % timeout}
        if p.returncode != 0 or not os.path.exists(out):
            tail = (p.stderr or b"").decode(errors="replace").strip().splitlines()[-1:]
            return {"ok": False, "error": "reference decoder exited with %d %s" % (p.returncode, " ".join(tail))}
        with open(out, "rb") as f:
            reply = pickle.load(f)
    reply["ok"] = all(s == 0 for s in reply["status"])
    reply["error"] = "" if reply["ok"] else "reference status %s" % reply["status"]
    return reply


def _child():
    import ctypes
    req = pickle.loads(sys.stdin.buffer.read())
    lib = ctypes.CDLL(LIB)
    n = lib.ref_cpu_init(req["threads"])
    reply = {"threads": n, "outputs": [], "sizes": [], "ms": [], "status": []}
    cap = 0
    buf = None
    for cs in req["streams"]:
        need = 64 << 20
        if need > cap:
            cap = need
            buf = ctypes.create_string_buffer(cap)
        w, h, nb, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        times = []
        st = 0
        out = b""
        for r in range(req["reps"]):
            st = lib.ref_cpu_decode(cs, len(cs), req["fmt"], req["top_level"], buf, ctypes.c_long(cap), ctypes.byref(w),
                                    ctypes.byref(h), ctypes.byref(nb), ctypes.byref(ms))
            times.append(ms.value)
            if st != 0:
                break
            if r == 0 and not req["time_only"]:
                out = buf.raw[:nb.value]
        reply["outputs"].append(out)
        reply["sizes"].append((w.value, h.value))
        reply["ms"].append(times)
        reply["status"].append(int(st))
    with open(req["reply"], "wb") as f:
        pickle.dump(reply, f)
    sys.stdout.flush()
    os._exit(0)  # the reference engine's worker threads are never joined: skip exit-time teardown


if __name__ == "__main__":
    _child()
