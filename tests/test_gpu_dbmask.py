"""Deblock edge masks built on the device from block records
(R2gSideInfo.db_masks) against the oracle's decode-order walk over the same
create_db_mask calls (lf_mask.rs:399-503, decode.rs:7869-7912, contexts reset
as decode.rs:207 does), and whole-frame parity with records instead of
masks."""
import numpy as np
import pytest

from rav2d_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from rav2d_b200 import gpu

    c = gpu.Context(0)
    yield c
    c.close()


def _frame(w, h, bd, seed, *, tiles=(0,), seg=False, chain="full"):
    sf = synth.make_frame(w, h, bd, seed, chain=chain, lossless=seg)
    rng = np.random.default_rng(seed + 17)
    blocks, hdr = synth.make_db_blocks(rng, w, h, seg_ids=8 if seg else 1, tile_cols=tiles)
    sf.use_db_blocks(blocks, hdr, garbage_rng=rng)
    return sf


MASK_CASES = [
    # (w, h, tile column starts in 4x4 units, segments + lossless, seed)
    (64, 64, (0,), False, 1),
    (72, 40, (0,), False, 2),
    (640, 360, (0,), True, 3),
    (1280, 720, (0, 128), False, 4),
    (1920, 1080, (0, 192, 320), True, 5),
    (3840, 2160, (0, 320, 640), False, 6),
]


@pytest.mark.parametrize("w,h,tiles,seg,seed", MASK_CASES)
def test_device_masks_match_decode_walk(ctx, oracle, w, h, tiles, seg, seed):
    from rav2d_b200 import gpu

    sf = _frame(w, h, 10, seed, tiles=tiles, seg=seg)
    want = oracle.build_db_masks(sf)
    f = gpu.Frame(ctx, w, h, 10)
    try:
        f.stage(sf)
        got = f.read_masks()
    finally:
        f.free()
    for k in ("filter_y", "filter_uv"):
        if not np.array_equal(got[k], want[k]):
            idx = np.argwhere(got[k] != want[k])[0]
            raise AssertionError(f"{k} differs at {tuple(idx)}: gpu={got[k][tuple(idx)]} ref={want[k][tuple(idx)]}")
    # every other field is uploaded as given
    for k in abi.AV2_FILTER_DTYPE.names:
        if k not in ("filter_y", "filter_uv"):
            assert np.array_equal(got[k], sf.masks[k]), k


@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("w,h,seed", [(640, 360, 11), (1920, 1080, 12)])
def test_frame_parity_with_block_records(ctx, oracle, w, h, bd, seed):
    from rav2d_b200 import gpu

    sf = _frame(w, h, bd, seed, tiles=(0, 64), seg=True)
    want = oracle.filter_frame(sf)  # walks the records itself
    got = gpu.filter_frame(ctx, sf)
    for pl, (g, wnt) in enumerate(zip(got, want)):
        hh, ww = h >> (pl > 0), w >> (pl > 0)
        assert np.array_equal(g[:hh, :ww], wnt[:hh, :ww]), f"plane {pl}"


def test_bad_record_is_reported_once(ctx):
    from rav2d_b200 import gpu

    sf = _frame(256, 256, 8, 21, chain="db")
    blocks = sf.meta["db_blocks"].copy()
    blocks[0]["bs"] = 40  # no such block size
    sf.use_db_blocks(blocks, sf.meta["db_hdr"])
    f = gpu.Frame(ctx, 256, 256, 8)
    try:
        f.stage(sf)
        with pytest.raises(gpu.R2gError) as e:
            ctx.sync()
        assert "block records" in str(e.value)
        ctx.sync()  # the count was reported and cleared
    finally:
        f.free()


def test_record_header_checks(ctx):
    from rav2d_b200 import gpu

    sf = _frame(256, 256, 8, 22, chain="db")
    f = gpu.Frame(ctx, 256, 256, 8)
    try:
        for bad in ({"tile_cols": (0, 0)}, {"tile_cols": (0, 400)}, {"tile_rows": ()}):
            hdr = dict(sf.meta["db_hdr"], **bad)
            sf.use_db_blocks(sf.meta["db_blocks"], hdr)
            with pytest.raises(gpu.R2gError):
                f.stage(sf)
    finally:
        f.free()


def test_no_records_gives_empty_masks(ctx):
    from rav2d_b200 import gpu

    sf = _frame(128, 128, 8, 23, chain="db")
    sf.use_db_blocks(np.zeros(0, abi.DB_BLOCK_DTYPE), sf.meta["db_hdr"], garbage_rng=np.random.default_rng(0))
    f = gpu.Frame(ctx, 128, 128, 8)
    try:
        f.stage(sf)
        got = f.read_masks()
    finally:
        f.free()
    assert not got["filter_y"].any() and not got["filter_uv"].any()
