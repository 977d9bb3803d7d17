"""Frames with several tile rows through the oracle: init_start_of_tile_row
(decode.rs:99-120) marks each tile row's first superblock row, and only loop
restoration reads it (lr_sbrow_apply, looprestoration.rs:2401-2548: the
superblock row's stripe is split at the tile row's top edge into an 8-row
stripe that reads the rows below it in place and a first stripe of the tile
row that reads four saved deblocked rows above it).  Deblocking and CDEF take
no tile-row input (their start_of_tile_row / sbrow_start arguments are
unused, deblock.rs:791, :2154, cdef.rs:746-750)."""
import copy

import numpy as np
import pytest

from rav2d_b200 import abi, synth


def _with_tile_rows(sf, starts_sb):
    out = copy.copy(sf)
    fp = abi.FrameParams()
    C = __import__("ctypes")
    C.memmove(C.byref(fp), C.byref(sf.fp), C.sizeof(fp))
    fp.tile_rows = len(starts_sb) - 1
    for i, v in enumerate(starts_sb):
        fp.tile_row_start_sb[i] = v
    out.fp = fp
    return out


@pytest.mark.parametrize("bd", [8, 10])
def test_tile_rows_change_only_loop_restoration_near_the_split(oracle, bd):
    sf = synth.make_frame(256, 320, bd, 40 + bd)  # 5 superblock rows
    one = oracle.filter_frame(sf)
    two = oracle.filter_frame(_with_tile_rows(sf, [0, 2, 5]))  # tile row 1 starts at luma row 128
    for pl, (a, b) in enumerate(zip(one, two)):
        ss = pl > 0
        diff = np.nonzero((a != b).any(axis=1))[0]
        if len(diff):
            split = 128 >> ss
            # the 8-row stripe above the split and the first stripe below it,
            # with the filters' reach (at most 6 rows) on either side
            assert diff.min() >= split - (8 >> ss) - 6 and diff.max() < split + (64 >> ss) + 6, (pl, diff)
    assert any((a != b).any() for a, b in zip(one, two)), "the split changed nothing"


def test_tile_rows_do_not_touch_deblock_or_cdef(oracle):
    sf = synth.make_frame(256, 320, 10, 50)
    inloop = abi.INLOOP_DEBLOCK | abi.INLOOP_CDEF | abi.INLOOP_CCSO
    one = oracle.filter_frame(sf, inloop=inloop)
    three = oracle.filter_frame(_with_tile_rows(sf, [0, 1, 3, 5]), inloop=inloop)
    for a, b in zip(one, three):
        assert np.array_equal(a, b)


def test_zero_tile_rows_is_one(oracle):
    sf = synth.make_frame(128, 192, 8, 51)
    assert all(np.array_equal(a, b)
               for a, b in zip(oracle.filter_frame(sf), oracle.filter_frame(_with_tile_rows(sf, [0, 3]))))
