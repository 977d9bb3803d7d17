"""The per-frame and batch entry points reject what they cannot run, with a
status code and a message, and leave the context usable.

The reference's filters are infallible (its decoder never hands them a
frame they cannot take); the C ABI instead validates on the host and returns
R2G_E_INVALID (unsupported layout, sizes, parameters, call order), R2G_E_OOM
(the context's device-memory budget), R2G_E_NOTREADY / R2G_E_TIMEOUT (bounded
waits).  Every case here is decided on the host or by a timed wait on an
event; none makes a kernel fail.
"""
import ctypes as C

import pytest

from rav2d_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from rav2d_b200 import gpu as g

    return g


@pytest.fixture()
def ctx(gpu):
    c = gpu.Context(0)
    yield c
    c.close()


def _code(excinfo):
    return excinfo.value.code


def test_frame_alloc_rejects_bad_geometry(gpu, ctx):
    for w, h, bd in ((100, 64, 10), (64, 62, 10), (64, 64, 12), (0, 64, 8)):
        with pytest.raises(gpu.R2gError) as e:
            ctx.frame(w, h, bd)
        assert _code(e) == abi.R2G_E_INVALID, (w, h, bd)
    ctx.frame(64, 64, 8).free()  # the context still works


def test_budget_exhaustion(gpu):
    c = gpu.Context(0, mem_budget=8 << 20)
    try:
        with pytest.raises(gpu.R2gError) as e:
            c.frame(1920, 1080, 10)  # about 35 MB of planes and side-info
        assert _code(e) == abi.R2G_E_OOM
        c.frame(64, 64, 10).free()  # a frame within the budget still fits
    finally:
        c.close()


def _filter_rc(gpu, ctx, fr, sf, fp=None, lr=None):
    side = abi.side_info(sf.masks, sf.lr if lr is None else lr)
    return gpu.lib().r2g_frame_filter(ctx.h, fr.h, C.byref(sf.fp if fp is None else fp), C.byref(side), sf.inloop)


def test_filter_rejects_unsupported_frames(gpu, ctx):
    sf = synth.make_frame(128, 128, 10, 0xE0A1, chain="full")
    fr = ctx.frame(128, 128, 10)
    try:
        fr.upload(sf.planes)
        cases = []
        for field, value, words in (("layout", 3, "4:2:0"), ("sb128", 1, "superblocks"), ("width", 120, "match"),
                                    ("bitdepth", 8, "match")):
            fp = type(sf.fp).from_buffer_copy(sf.fp)
            setattr(fp, field, value)
            cases.append((fp, None, words))
        fp = type(sf.fp).from_buffer_copy(sf.fp)
        fp.restoration_unit_size[0] = 4
        cases.append((fp, None, "unit size"))
        lr = sf.lr.copy()
        lr["lr"]["restoration_type"][0, 1, 0] = abi.RESTORE_PC_WIENER
        cases.append((None, lr, "PC-Wiener"))
        for fp, lr, words in cases:
            rc = _filter_rc(gpu, ctx, fr, sf, fp, lr)
            assert rc == abi.R2G_E_INVALID, words
            assert words in gpu.lib().r2g_last_error(ctx.h).decode()
        # the unchanged frame still filters
        assert _filter_rc(gpu, ctx, fr, sf) == 0
        ctx.sync()
    finally:
        fr.free()


def test_call_order_and_grain_ranges(gpu, ctx):
    sf = synth.make_frame(128, 64, 10, 0xE0A2, chain="db", grain=True)
    fr = ctx.frame(128, 64, 10)
    try:
        fr.upload(sf.planes)
        with pytest.raises(gpu.R2gError) as e:  # nothing filtered yet
            fr.download(sf.planes, 0)
        assert _code(e) == abi.R2G_E_INVALID
        with pytest.raises(gpu.R2gError) as e:  # grain needs a filtered frame
            fr.grain(sf.fgd, sf.grain_seed)
        assert _code(e) == abi.R2G_E_INVALID
        fr.filter(sf)
        # the ranges the reference's parser admits (obu.rs:272-325)
        for field, value in (("ar_coeff_lag", 4), ("block_size", 2), ("scaling_shift", 12), ("ar_coeff_shift", 5),
                             ("ar_coeff_shift", 10), ("grain_scale_shift", 4), ("grain_scale_shift", -1),
                             ("num_points", (15, 0, 0)), ("num_points", (8, -1, 0)), ("num_points", (8, 0, 99))):
            fgd = type(sf.fgd).from_buffer_copy(sf.fgd)
            if field == "num_points":
                for i, v in enumerate(value):
                    fgd.num_points[i] = v
            else:
                setattr(fgd, field, value)
            with pytest.raises(gpu.R2gError) as e:
                fr.grain(fgd, sf.grain_seed)
            assert _code(e) == abi.R2G_E_INVALID, field
        with pytest.raises(gpu.R2gError) as e:
            fr.grain(sf.fgd, 0x10000)  # seeds are 16-bit
        assert _code(e) == abi.R2G_E_INVALID
        with pytest.raises(gpu.R2gError) as e:  # no grained copy yet
            fr.download(sf.planes, 1)
        assert _code(e) == abi.R2G_E_INVALID
        fr.grain(sf.fgd, sf.grain_seed)
        fr.download(sf.planes, 1)
    finally:
        fr.free()


def test_bounded_waits(gpu, ctx):
    """A batch of sixteen 4K frames runs for milliseconds: a zero-timeout wait
    right after the submit reports not-ready, a 1 ms wait times out, an
    unbounded wait completes it, and the spent ticket is then unknown."""
    sf = synth.make_frame(3840, 2160, 10, 0xE0A3, chain="full")
    frames = []
    try:
        for _ in range(16):
            fr = ctx.frame(3840, 2160, 10)
            fr.upload(sf.planes)
            fr.stage(sf)
            frames.append(fr)
        ctx.sync()
        items = [(fr, sf) for fr in frames]
        ctx.batch_submit(items, staged=True)  # first batch: tunes and builds the graph
        assert ctx.wait(ctx.batch_submit(items, staged=True), -1) == 0
        t = ctx.batch_submit(items, staged=True)
        assert ctx.wait(t, 0) == abi.R2G_E_NOTREADY
        assert ctx.wait(t, 1) == abi.R2G_E_TIMEOUT
        assert ctx.wait(t, -1) == 0
        assert ctx.wait(t, 0) == abi.R2G_E_INVALID
        ctx.sync()
    finally:
        for fr in frames:
            fr.free()
