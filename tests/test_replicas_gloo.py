"""The multi-GPU path of bench.py on CPU: two gloo ranks (world size 2) run the replica
reduction exactly as the GPU ranks do (barrier, MAX of the per-rank times, whole-job
throughput), and the reference arm prints only on rank 0."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    dist.barrier()
    t = bench.max_over_ranks(1.0 + rank, dist, device="cpu")  # rank 1 is the slower replica
    v = bench.replica_throughput(10.0, world, 3, t)
    q.put((rank, t, v))
    dist.destroy_process_group()


def test_replica_reduction_world_size_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, v in got:
        assert t == 2.0                      # both ranks see the slowest rank's time
        assert v == pytest.approx(10.0 * 2 * 3 / 2.0)


def test_reference_arm_prints_on_rank_zero_only(tmp_path):
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c1",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env["RANK"] = "0"
    env["LOCAL_RANK"] = "0"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c1",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    # the reference's own decoder when its library is built here, else the CPU restatement
    have_ref = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so"))
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == ("reference" if have_ref else "port")
