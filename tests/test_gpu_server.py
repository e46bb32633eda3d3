"""The continuous-batching service (include/j2k_server.h) on the GPU.

Requests of different sizes, bit depths and wavelets are submitted from several threads
while earlier batches run, so they are merged into shared launches; every result must be
bit-identical to the same codestream decoded alone (tolerance 0: the batch shares launches
but not arithmetic), and the oracle checks the decode of one of them."""
import threading

import numpy as np
import pytest

import oracle_util

pytestmark = pytest.mark.gpu


def _mix():
    from jpeg2000_decoder_b200 import native, synth
    out = []
    rng = np.random.default_rng(11)
    for i, (h, w) in enumerate([(256, 256), (512, 512), (1024, 1024), (1080, 1920), (256, 256), (512, 512)]):
        img = synth.fields_and_edges(100 + i, h, w, nrect=8)
        if i % 3 == 0:
            cs = native.encode(img, 8, reversible=1, levels=5, cbw_exp=6, cbh_exp=6, num_layers=1, layer_bpp=[0])
            fmt = native.FMT_24BITS_RGB
        elif i % 3 == 1:
            cs = native.encode(img, 8, reversible=0, levels=5, cbw_exp=6, cbh_exp=6, num_layers=1,
                               layer_bpp=[float(rng.uniform(0.5, 2.0))], guard_bits=1)
            fmt = native.FMT_24BITS_RGB
        else:
            img12 = (img.astype(np.uint32) * 16 + rng.integers(0, 16, img.shape)).astype(np.uint16)
            cs = native.encode(img12, 12, reversible=0, levels=5, cbw_exp=6, cbh_exp=6, num_layers=1,
                               layer_bpp=[1.0], guard_bits=1)
            fmt = native.FMT_48BITS_RGB
        out.append((cs, fmt))
    return out


def test_served_results_equal_alone(pkg):
    from jpeg2000_decoder_b200 import native
    mix = _mix()
    alone = []
    ctx = native.GpuContext()
    try:
        for cs, fmt in mix:
            o, rc, bad, plan = ctx.decode(cs, fmt)
            assert rc == native.J2K_OK and bad == 0
            alone.append(o.copy())
        # the oracle agrees with the lone decode of the 12-bit 9/7 request
        cs, fmt = mix[2]
        plan = native.Plan(cs)
        orc, oout, _ = oracle_util.oracle_decode(plan, fmt)
        assert orc == 0 and np.array_equal(alone[2], oout)
    finally:
        ctx.close()

    srv = native.Server(pipeline_depth=2)
    try:
        reqs = list(range(len(mix))) * 4  # 24 requests, each codestream four times
        ids = [None] * len(reqs)

        def submitter(k):
            for j in range(k, len(reqs), 3):
                cs, fmt = mix[reqs[j]]
                ids[j] = srv.submit(cs, fmt)

        th = [threading.Thread(target=submitter, args=(k,)) for k in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for j, rid in enumerate(ids):
            got = srv.result(rid)
            assert np.array_equal(got, alone[reqs[j]]), "request %d differs from its lone decode" % j
            rc, view = srv.view(rid)
            assert rc == native.J2K_OK and np.array_equal(view, got)
            assert srv.latency_us(rid) > 0
            srv.release(rid)
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["batches"] <= len(reqs)
        print("server: %d batches for %d requests, p50 %.0f us, p99 %.0f us" % (
            st["batches"], len(reqs), st["p50_us"], st["p99_us"]))
    finally:
        srv.close()


def test_server_rejects_bad_input_and_keeps_serving(pkg):
    from jpeg2000_decoder_b200 import native
    cs, fmt = _mix()[0]
    srv = native.Server()
    try:
        with pytest.raises(native.J2kError) as e:
            srv.submit(b"\xff\x4f\xff\x51" + b"\x00" * 10, fmt)
        assert e.value.code == native.J2K_ERR_PARSE
        rid = srv.submit(cs, fmt)
        assert srv.result(rid).nbytes == 256 * 256 * 3
    finally:
        srv.close()


def test_server_memory_budget_splits_batches(pkg):
    """A budget that holds about one large picture per slot forces one picture per batch."""
    from jpeg2000_decoder_b200 import native
    mix = _mix()
    cs, fmt = mix[3]  # 1920x1080
    plan = native.Plan(cs)
    per = plan.info.coef_elems * 12 + plan.info.coded_bytes + (8 << 20)
    srv = native.Server(mem_budget=int(per * 1.5) * 2, pipeline_depth=2)
    try:
        ids = [srv.submit(cs, fmt) for _ in range(6)]
        outs = [srv.result(i) for i in ids]
        assert all(np.array_equal(o, outs[0]) for o in outs)
        assert srv.stats()["mean_batch_images"] <= 1.0 + 1e-9
    finally:
        srv.close()
