"""The oracle's decode-order walk over a frame's create_db_mask calls
(decode.rs:7869-7912 with the contexts of decode.rs:207), checked on frames
whose masks follow from the reference's mask builders by hand, and the
block-record generator's invariants."""
import numpy as np

from rav2d_b200 import abi, synth

BS_8X8, BS_16X16 = 24, 18


def _sf(w, h, blocks, **hdr):
    sf = synth.make_frame(w, h, 8, 1, chain="db")
    h2 = {"sub_pu": 0, "tip_frame_mode": 0, "tip_subpel_filter": 0, "tip_refine_mv": 0, "tile_cols": (0,),
          "tile_rows": (0,)}
    h2.update(hdr)
    sf.use_db_blocks(np.array(blocks, abi.DB_BLOCK_DTYPE), h2)
    return sf


def _grid(w4, h4, step, bs, chroma=False):
    return [(x, y, bs, abi.DBB_INTRA | (abi.DBB_CHROMA if chroma else 0), 0, 0, 0, 0, -1, -1)
            for y in range(0, h4, step) for x in range(0, w4, step)]


def test_uniform_8x8_intra_grid(oracle):
    """8x8 intra blocks, 8x8 transforms (TX_PART_TBL[Bs8x8][None] = Tx8x8,
    log2 width 1): every outer edge is level min(1, 1) = 1, or min(1, 3) at
    the frame's left / top (the reset context); no inner edges."""
    sf = _sf(64, 64, _grid(16, 16, 2, BS_8X8))
    m = oracle.build_db_masks(sf)["filter_y"][0]
    for d in (0, 1):
        for pos in range(16):
            want = 0xffff if pos % 2 == 0 else 0
            assert m[d][pos][1][0] == want, (d, pos)
            assert m[d][pos][0][0] == 0 and m[d][pos][2][0] == 0 and m[d][pos][3][0] == 0


def test_left_context_is_the_neighbours_level(oracle):
    """A 16x16 block (Tx16x16: level 2) right of an 8x8 column (level 1):
    the shared edge takes min(2, 1) = 1, the 16x16's own inner rows none."""
    blocks = [(0, 0, BS_8X8, abi.DBB_INTRA, 0, 0, 0, 0, -1, -1),
              (0, 2, BS_8X8, abi.DBB_INTRA, 0, 0, 0, 0, -1, -1),
              (2, 0, BS_16X16, abi.DBB_INTRA, 0, 0, 0, 0, -1, -1)]
    sf = _sf(64, 64, blocks)
    m = oracle.build_db_masks(sf)["filter_y"][0]
    assert m[0][2][1][0] & 0b1111 == 0b1111  # rows 0..3 of column 2 at level 1
    assert m[0][2][2][0] & 0b1111 == 0
    assert m[1][0][2][0] & 0b111100 == 0b111100  # the 16x16's top edge: min(2, reset 3)


def test_tile_column_resets_the_left_context(oracle):
    """At a tile column start the left context is the reset value 3, so the
    edge keeps the block's own level even though the block to its left has a
    lower one."""
    blocks = [(x, 0, BS_8X8, abi.DBB_INTRA, 0, 0, 0, 0, -1, -1) for x in range(0, 64, 2)] + \
             [(x, 0, BS_16X16, abi.DBB_INTRA, 0, 0, 0, 0, -1, -1) for x in range(64, 128, 4)]
    no_tiles = oracle.build_db_masks(_sf(512, 64, blocks))["filter_y"]
    tiles = oracle.build_db_masks(_sf(512, 64, blocks, tile_cols=(0, 64)))["filter_y"]
    assert no_tiles[1][0][0][1][0] & 1 and not no_tiles[1][0][0][2][0] & 1  # SB256 1, column 0: min(2, 1)
    assert tiles[1][0][0][2][0] & 1 and not tiles[1][0][0][1][0] & 1          # reset: min(2, 3)


def test_generator_tiles_the_frame():
    """Luma records cover every 4x4 of the frame exactly once, chroma records
    every chroma 4x4 (bs sizes from BLOCK_DIMENSIONS)."""
    bd = synth._c_table("BLOCK_DIMENSIONS", np.int32)
    for w, h, seed in ((72, 40, 1), (640, 360, 2), (1920, 1080, 3)):
        b, _ = synth.make_db_blocks(np.random.default_rng(seed), w, h, tile_cols=(0, 64) if w > 512 else (0,))
        bw4, bh4 = w // 4, h // 4
        for chroma in (False, True):
            cov = np.zeros((bh4, bw4), np.int32)
            sel = b[(b["flags"] & abi.DBB_CHROMA) != 0] if chroma else b[(b["flags"] & abi.DBB_CHROMA) == 0]
            for r in sel:
                ww, hh = bd[r["bs"]][:2]
                cov[r["by"]:r["by"] + hh, r["bx"]:r["bx"] + ww] += 1
            if chroma:
                cov = cov[::2, ::2]
            assert (cov == 1).all(), (w, h, chroma)
