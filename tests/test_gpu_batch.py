"""Batched mode: one persistent launch per stage over many frames.

A batch mixes frame sizes, bit depths, filter chains and film grain; every
frame of it must come out sample for sample the same as the per-frame path
(itself byte-exact against the oracle), and a frame's output must not depend
on what else is in its batch.  Successive batches alternate the two staging
slots and grow them, which these tests cover too.
"""
import numpy as np
import pytest

from rav2d_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import os

    from rav2d_b200 import gpu

    os.environ.setdefault("R2G_TUNE_CACHE", "/tmp/r2g-autotune-test.txt")
    c = gpu.Context(0)
    yield c
    c.close()


def _frames(specs):
    out = []
    for i, (w, h, bd, chain, grain) in enumerate(specs):
        out.append(synth.make_frame(w, h, bd, 0xBA7C0000 + i, chain=chain, grain=grain))
    return out


def _per_frame(ctx, sf, grain):
    from rav2d_b200 import gpu

    return gpu.filter_frame(ctx, sf, grain=grain)


def _batch(ctx, sfs):
    frames = []
    for sf in sfs:
        fr = ctx.frame(sf.width, sf.height, sf.bitdepth)
        fr.upload(sf.planes)
        frames.append(fr)
    t = ctx.batch_submit(list(zip(frames, sfs)))
    assert ctx.wait(t, 60000) == 0
    outs = []
    for fr, sf in zip(frames, sfs):
        f = fr.download(sf.planes, 0)
        g = fr.download(sf.planes, 1) if sf.fgd is not None else None
        outs.append((f, g))
        fr.free()
    return outs


def _same(a, b, sf, what):
    for pl in range(3):
        h, w = sf.height >> (pl > 0), sf.width >> (pl > 0)
        assert np.array_equal(a[pl][:h, :w], b[pl][:h, :w]), f"{what}: plane {pl} differs"


MIX = [
    (640, 360, 8, "full", True),
    (352, 288, 10, "db_cdef", True),
    (1280, 720, 10, "full", True),
    (128, 128, 8, "db", False),
    (1920, 1080, 10, "full", True),
    (72, 40, 10, "full", False),
    (640, 360, 10, "full", True),
]


def test_batch_matches_per_frame(ctx):
    sfs = _frames(MIX)
    got = _batch(ctx, sfs)
    for sf, (f, g) in zip(sfs, got):
        if sf.fgd is not None:
            wf, wg = _per_frame(ctx, sf, True)
            _same(g, wg, sf, f"grain {sf.width}x{sf.height}/{sf.bitdepth}")
        else:
            wf = _per_frame(ctx, sf, False)
        _same(f, wf, sf, f"filter {sf.width}x{sf.height}/{sf.bitdepth}")


def test_batch_alone_equals_in_mix(ctx):
    sfs = _frames(MIX)
    mixed = _batch(ctx, sfs)
    # the same frames one per batch (alternating slots), then reversed
    for i, sf in enumerate(sfs):
        (f, g), = _batch(ctx, [sf])
        _same(f, mixed[i][0], sf, "alone vs mix (filter)")
        if g is not None:
            _same(g, mixed[i][1], sf, "alone vs mix (grain)")
    rev = _batch(ctx, sfs[::-1])
    for (f, g), (mf, mg), sf in zip(rev[::-1], mixed, sfs):
        _same(f, mf, sf, "reversed batch (filter)")
        if g is not None:
            _same(g, mg, sf, "reversed batch (grain)")


def test_batch_grows_and_reports_grid(ctx):
    small = _frames([(64, 64, 8, "db", False)])
    _batch(ctx, small)
    # many small frames grow the batch's staging slots; the 1080p and 4K
    # frames of the same call run through the per-frame pipeline
    big = _frames([(1920, 1080, 10, "full", True)] * 2 + [(3840, 2160, 8, "full", True)] +
                  [(640, 360, 10, "full", True)] * 24)
    got = _batch(ctx, big)
    for k in (2, 26):
        wf, wg = _per_frame(ctx, big[k], True)
        _same(got[k][0], wf, big[k], f"frame {k} after growth (filter)")
        _same(got[k][1], wg, big[k], f"frame {k} after growth (grain)")
    sms, cfg = ctx.batch_config()
    assert sms > 0 and all(v >= 0 for v in cfg.values())  # 0: one CTA per work item


def test_batch_oracle_spot_check(ctx, oracle):
    sf = synth.make_frame(320, 192, 10, 0xBA7C1000, chain="full", grain=True)
    (f, g), = _batch(ctx, [sf])
    want = oracle.filter_frame(sf)
    _same(f, want, sf, "batch vs oracle (filter)")
    _same(g, oracle.apply_grain(sf, want), sf, "batch vs oracle (grain)")


@pytest.mark.parametrize("rows", [16, 32])
def test_batch_lr_tile_shape(tmp_path, monkeypatch, rows):
    """The loop-restoration tile shape (luma rows per work item) the autotuner
    may pick gives the same output as the per-frame path (32 rows): a tune
    cache that pins the shape forces it for a mixed batch."""
    import torch

    from rav2d_b200 import gpu

    name = torch.cuda.get_device_name(0)
    cache = tmp_path / "tune.txt"
    lines = []
    for cls in range(3):
        for k in range(4):
            lines.append(f"{name}|{cls}|{k}|1|{rows if k == 2 else 0}")
    cache.write_text("\n".join(lines) + "\n")
    monkeypatch.setenv("R2G_TUNE_CACHE", str(cache))
    c = gpu.Context(0)
    try:
        sfs = _frames([(640, 360, 10, "full", True), (1280, 720, 8, "full", False), (200, 136, 10, "full", False),
                       (1920, 1080, 10, "full", True)])
        got = _batch(c, sfs)
        assert c.batch_tile_rows()["loop_restoration"] == rows
        for (f, g), sf in zip(got, sfs):
            wf = _per_frame(c, sf, sf.fgd is not None)
            if sf.fgd is not None:
                wf, wg = wf
                _same(g, wg, sf, f"lr rows {rows} (grain)")
            _same(f, wf, sf, f"lr rows {rows} (filter)")
    finally:
        c.close()
