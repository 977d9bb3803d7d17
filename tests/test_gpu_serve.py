"""Serving: continuous batching of frames from concurrent streams.

Every frame served in a mix of streams (different sizes, bit depths, film
grain on some) must come out sample for sample as the same frame filtered
alone through the per-frame path; admission under a small memory budget
(evicting idle streams), a frame that cannot fit at all, and a malformed
frame must each fail or wait alone without disturbing the others.
"""
import threading

import numpy as np
import pytest

from rav2d_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import os

    from rav2d_b200 import gpu

    os.environ.setdefault("R2G_TUNE_CACHE", "/tmp/r2g-autotune-test.txt")
    c = gpu.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def solo():
    """A second context for the frames filtered alone (a context with a
    server attached is driven only through the server)."""
    from rav2d_b200 import gpu

    c = gpu.Context(0)
    yield c
    c.close()


STREAMS = [
    (640, 360, 8, True),
    (1280, 720, 10, False),
    (352, 288, 10, True),
    (1920, 1080, 8, True),
    (128, 128, 10, False),
    (640, 360, 10, True),
]


def _stream_frames(k, n):
    w, h, bd, g = STREAMS[k]
    return [synth.make_frame(w, h, bd, 0x5E4E0000 + 64 * k + i, chain="full", grain=g) for i in range(n)]


def _alone(solo, sf):
    from rav2d_b200 import gpu

    if sf.fgd is not None:
        return gpu.filter_frame(solo, sf, grain=True)
    f = gpu.filter_frame(solo, sf)
    return f, f


def _same(a, b, sf, what):
    for pl in range(3):
        h, w = sf.height >> (pl > 0), sf.width >> (pl > 0)
        assert np.array_equal(a[pl][:h, :w], b[pl][:h, :w]), f"{what}: plane {pl} differs"


def test_serving_mix_equals_alone(ctx, solo):
    from rav2d_b200 import gpu

    per_stream = [_stream_frames(k, 3) for k in range(len(STREAMS))]
    srv = gpu.Server(ctx, mem_budget=8 << 30, max_batch=16)
    try:
        ids = []
        lock = threading.Lock()

        def producer(k):
            for sf in per_stream[k]:
                dst = [np.zeros_like(p) for p in sf.planes]
                ref = [np.zeros_like(p) for p in sf.planes]
                rid = srv.submit(k, sf, sf.planes, dst, ref)
                with lock:
                    ids.append((rid, sf, dst, ref))

        ths = [threading.Thread(target=producer, args=(k,)) for k in range(len(STREAMS))]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        batch_sizes = []
        for rid, sf, dst, ref in ids:
            rc, res = srv.wait(rid, 120000)
            assert rc == 0 and res.status == 0, (rc, res.status)
            batch_sizes.append(res.batch_frames)
        st = srv.stats()
        assert st["completed"] == len(ids) and st["failed"] == 0
        for rid, sf, dst, ref in ids:
            want_f, want_disp = _alone(solo, sf)
            _same(ref, want_f, sf, f"filtered {sf.width}x{sf.height}/{sf.bitdepth}")
            _same(dst, want_disp, sf, f"display {sf.width}x{sf.height}/{sf.bitdepth}")
        assert max(batch_sizes) > 1  # frames of different streams shared a batch
    finally:
        srv.close()


def test_serving_budget_evicts_idle_streams(ctx, solo):
    from rav2d_b200 import gpu

    # room for about two 640x360 frames: streams must take turns
    sfs = [synth.make_frame(640, 360, 10, 0x5E4E1000 + i, chain="full", grain=False) for i in range(4)]
    one = 5 * sum(p.nbytes for p in sfs[0].planes) + 2 * 40 * 1024 + sfs[0].masks.nbytes + sfs[0].lr.nbytes
    srv = gpu.Server(ctx, mem_budget=2 * one, max_batch=8, frames_per_stream=1)
    try:
        reqs = []
        for rep in range(2):
            for k, sf in enumerate(sfs):
                dst = [np.zeros_like(p) for p in sf.planes]
                reqs.append((srv.submit(k, sf, sf.planes, dst), sf, dst))
        for rid, sf, dst in reqs:
            rc, res = srv.wait(rid, 120000)
            assert rc == 0 and res.status == 0
            _same(dst, _alone(solo, sf)[1], sf, "under budget pressure")
        st = srv.stats()
        assert st["evictions"] > 0
        assert st["resident_bytes"] <= 2 * one
    finally:
        srv.close()


def test_serving_rejects_alone(ctx, solo):
    from rav2d_b200 import gpu

    good = synth.make_frame(320, 192, 8, 0x5E4E2000, chain="full", grain=True)
    big = synth.make_frame(1280, 720, 10, 0x5E4E2001, chain="db")
    bad = synth.make_frame(320, 192, 8, 0x5E4E2002, chain="full")
    bad.fp.layout = 0  # 4:0:0 is not served: rejected at admission
    budget = 4 << 20  # the 720p 10-bit frame needs about 16 MB
    srv = gpu.Server(ctx, mem_budget=budget, max_batch=8)
    try:
        outs = {}
        for name, k, sf in (("good", 0, good), ("big", 1, big), ("bad", 2, bad)):
            dst = [np.zeros_like(p) for p in sf.planes]
            outs[name] = (srv.submit(k, sf, sf.planes, dst), sf, dst)
        rc, res = srv.wait(outs["big"][0], 60000)
        assert rc == 0 and res.status == abi.R2G_E_OOM
        rc, res = srv.wait(outs["bad"][0], 60000)
        assert rc == 0 and res.status == abi.R2G_E_INVALID
        rid, sf, dst = outs["good"]
        rc, res = srv.wait(rid, 60000)
        assert rc == 0 and res.status == 0
        _same(dst, _alone(solo, sf)[1], sf, "good frame beside rejected ones")
        # an id that was never issued, and a released one
        assert srv.wait(10 ** 9, 0)[0] == abi.R2G_E_INVALID
        assert srv.wait(rid, 0)[0] == abi.R2G_E_INVALID
    finally:
        srv.close()


def test_serving_poll_and_close_stream(ctx):
    from rav2d_b200 import gpu

    sf = synth.make_frame(640, 360, 10, 0x5E4E3000, chain="full", grain=True)
    srv = gpu.Server(ctx, mem_budget=1 << 30)
    try:
        dst = [np.zeros_like(p) for p in sf.planes]
        rid = srv.submit(7, sf, sf.planes, dst)
        rc, _ = srv.wait(rid, 0)
        assert rc in (0, abi.R2G_E_NOTREADY)
        if rc == abi.R2G_E_NOTREADY:
            rc, res = srv.wait(rid, 60000)
            assert rc == 0 and res.status == 0
        assert srv.close_stream(7) == 0
        # the worker frees the stream's frames once idle
        import time

        for _ in range(200):
            if srv.stats()["resident_bytes"] == 0:
                break
            time.sleep(0.01)
        assert srv.stats()["resident_bytes"] == 0
    finally:
        srv.close()
