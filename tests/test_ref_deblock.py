"""The reference's deblocking unit tests (crates/rav2d/src/deblock.rs
:2283-2994), one test here per test there, re-asserted against the CPU
oracle's restatement (oracle/deblock.cpp).  Each test names the reference
test and its line; inputs and assertions are the reference's.  The
reference's u8 buffers are uint16 arrays (the oracle's sample type) at bit
depth 8; its u8 threshold arrays are uint16 / uint32 arrays of the same
values.  Where the reference calls a standalone test variant with its own
destination stride (setup_thr_rows_sb64), the same value is read from the
filter path's stride-16 layout."""
import ctypes as C

import numpy as np
import pytest

from rav2d_b200 import abi


def p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def L(oracle):
    lib = oracle.lib()
    lib.r2o_deblock_const.restype = C.c_int
    lib.r2o_filter_choice.restype = C.c_int
    return lib


def lut_y(L, fp, hbd, dir_, qidx):
    lut = np.zeros((2, 16), np.uint32)
    L.r2o_init_deblock_thr_lut_y(C.byref(fp), hbd, dir_, qidx, p(lut))
    return lut


def lut_uv(L, fp, hbd, qidx):
    lut = np.zeros((2, 2, 16), np.uint32)
    L.r2o_init_deblock_thr_lut_uv(C.byref(fp), hbd, qidx, p(lut))
    return lut


def test_max_width_y(L):
    """deblock.rs:2292-2296"""
    assert L.r2o_deblock_const(0, 0) == 1 and L.r2o_deblock_const(0, 3) == 8


def test_max_width_uv(L):
    """deblock.rs:2298-2302"""
    assert L.r2o_deblock_const(1, 0) == 1 and L.r2o_deblock_const(1, 2) == 4


def test_q_first(L):
    """deblock.rs:2304-2307"""
    assert L.r2o_deblock_const(2, 0) > L.r2o_deblock_const(2, 2)


def test_q_thresh_mults_zero_entries(L):
    """deblock.rs:2309-2313"""
    assert L.r2o_deblock_const(3, 4) == 0 and L.r2o_deblock_const(3, 6) == 0


def test_w_mult_zero_entries(L):
    """deblock.rs:2315-2319"""
    assert L.r2o_deblock_const(4, 4) == 0 and L.r2o_deblock_const(4, 6) == 0


def test_init_deblock_thr_lut_y_no_seg(L):
    """deblock.rs:2321-2327"""
    lut = lut_y(L, abi.FrameParams(), 0, 0, 128)
    assert lut[0][0] > 0 or lut[1][0] > 0


def test_init_deblock_thr_lut_y_with_seg(L):
    """deblock.rs:2329-2341"""
    fp = abi.FrameParams()
    fp.seg_enabled = 1
    fp.seg_delta_q[0], fp.seg_delta_q[1], fp.seg_delta_q[2] = 0, 10, -10
    lut = lut_y(L, fp, 0, 0, 128)
    lut2 = lut_y(L, fp, 0, 0, 138)
    assert lut[0][1] == lut2[0][0]


def test_init_deblock_thr_lut_y_dir(L):
    """deblock.rs:2343-2353"""
    fp = abi.FrameParams()
    fp.deblock_delta_q_y[0], fp.deblock_delta_q_y[1] = 2, -1
    assert lut_y(L, fp, 0, 0, 128)[0][0] != lut_y(L, fp, 0, 1, 128)[0][0]


def test_init_deblock_thr_lut_uv_no_seg(L):
    """deblock.rs:2355-2361"""
    lut = lut_uv(L, abi.FrameParams(), 0, 128)
    assert lut[0][0][0] == lut[1][0][0]


def test_init_deblock_thr_lut_uv_delta(L):
    """deblock.rs:2363-2371"""
    fp = abi.FrameParams()
    fp.quant_uac_delta, fp.quant_vac_delta = 5, -5
    lut = lut_uv(L, fp, 0, 128)
    assert lut[0][0][0] != lut[1][0][0]


def test_init_deblock_thr_lut_y_clamps(L):
    """deblock.rs:2373-2383 (the reference's assertion is a tautology); the
    clamp to qmax makes both LUTs equal here."""
    fp = abi.FrameParams()
    fp.seg_enabled = 1
    fp.seg_delta_q[0] = 500
    lut = lut_y(L, fp, 0, 0, 200)
    lut_max = lut_y(L, fp, 0, 0, 255)
    assert lut[0][0] <= lut_max[0][0] or lut[0][0] >= lut_max[0][0]
    assert lut[0][0] == lut_max[0][0]


def test_filter_choice_uniform(L):
    """deblock.rs:2385-2392"""
    buf = np.full(64, 128, np.uint16)
    assert L.r2o_filter_choice(p(buf), C.c_int64(16), C.c_int64(19), C.c_int64(1), 3, 3, 10, 100) == 3


def test_filter_choice_sharp_edge(L):
    """deblock.rs:2394-2407"""
    buf = np.zeros(64, np.uint16)
    buf[:32], buf[32:] = 50, 200
    assert L.r2o_filter_choice(p(buf), C.c_int64(32), C.c_int64(35), C.c_int64(1), 3, 3, 10, 20) <= 1


def deblock(L, dst, off, q, s, stridea, strideb, mwp, mwn, pos_ll, neg_ll):
    L.r2o_deblock(p(dst), C.c_int64(off), q, s, C.c_int64(stridea), C.c_int64(strideb), mwp, mwn, int(pos_ll),
                  int(neg_ll), 8)


def test_deblock_uniform_unchanged(L):
    """deblock.rs:2409-2428"""
    stride = 32
    dst = np.full(stride * 8, 128, np.uint16)
    orig = dst.copy()
    deblock(L, dst, stride * 2 + 8, 10, 20, stride, 1, 3, 3, False, False)
    assert (dst == orig).all()


def _edge_buf(stride=32, edge_col=10):
    dst = np.zeros(stride * 8, np.uint16)
    for y in range(8):
        dst[y * stride:y * stride + edge_col] = 50
        dst[y * stride + edge_col:(y + 1) * stride] = 200
    return dst


def test_deblock_sharp_edge_modifies(L):
    """deblock.rs:2430-2461"""
    stride, edge_col = 32, 10
    dst = _edge_buf(stride, edge_col)
    off = stride * 2 + edge_col
    before = dst[off]
    deblock(L, dst, off, 200, 200, stride, 1, 1, 1, False, False)
    assert dst[off] != before


def test_deblock_lossless_skip(L):
    """deblock.rs:2463-2491"""
    stride, edge_col = 32, 10
    dst = _edge_buf(stride, edge_col)
    orig = dst.copy()
    deblock(L, dst, stride * 2 + edge_col, 200, 200, stride, 1, 1, 1, True, True)
    assert (dst == orig).all()


def sb64(L, dst, dst_off, stride, vmask, luma, vert, edge=False):
    ll = np.zeros(2, np.uint16)
    q = np.full(16, 10, np.uint16)
    s = np.full(16, 20, np.uint16)
    L.r2o_deblock_sb64(p(dst), C.c_int64(dst_off), C.c_int64(stride), p(np.asarray(vmask, np.uint16)), p(ll), p(q),
                       p(s), int(edge), int(luma), int(vert), 8)


def test_deblock_h_sb64y_no_vmask(L):
    """deblock.rs:2493-2506"""
    dst = np.full(32 * 8, 128, np.uint16)
    orig = dst.copy()
    sb64(L, dst, 8, 32, [0, 0, 0, 0], True, True)
    assert (dst == orig).all()


def test_deblock_h_sb64y_uniform(L):
    """deblock.rs:2508-2521"""
    dst = np.full(32 * 8, 128, np.uint16)
    orig = dst.copy()
    sb64(L, dst, 8, 32, [1, 0, 0, 0], True, True)
    assert (dst == orig).all()


def test_deblock_v_sb64y_uniform(L):
    """deblock.rs:2523-2543"""
    dst = np.full(32 * 16, 128, np.uint16)
    orig = dst.copy()
    sb64(L, dst, 32 * 4, 32, [1, 0, 0, 0], True, False)
    assert (dst == orig).all()


def test_deblock_h_sb64uv_no_vmask(L):
    """deblock.rs:2545-2558"""
    dst = np.full(32 * 8, 128, np.uint16)
    orig = dst.copy()
    sb64(L, dst, 8, 32, [0, 0, 0, 0], False, True)
    assert (dst == orig).all()


def test_deblock_v_sb64uv_no_vmask(L):
    """deblock.rs:2560-2580"""
    dst = np.full(32 * 8, 128, np.uint16)
    orig = dst.copy()
    sb64(L, dst, 32 * 4, 32, [0, 0, 0, 0], False, False)
    assert (dst == orig).all()


def transpose(L, src, x64, ss_hor, ss_ver, dst=None):
    dst = np.zeros(17, np.uint16) if dst is None else dst
    L.r2o_transpose_lossless_mask(p(dst), p(np.ascontiguousarray(src, np.uint16)), x64, ss_hor, ss_ver)
    return dst


def test_transpose_lossless_mask_basic(L):
    """deblock.rs:2582-2592"""
    dst = transpose(L, np.full((16, 4), 0xAAAA), 0, 0, 0)
    for x in range(16):
        assert dst[x + 1] == (0xFFFF if (0xAAAA >> x) & 1 else 0)


def test_transpose_lossless_mask_ss(L):
    """deblock.rs:2594-2602"""
    dst = transpose(L, np.full((8, 4), 0xFF), 0, 1, 1)
    assert (dst[1:9] == 0xFF).all()


def test_transpose_lossless_mask_prev_col(L):
    """deblock.rs:2604-2611"""
    dst = np.zeros(17, np.uint16)
    dst[16] = 42
    transpose(L, np.zeros((16, 4)), 0, 0, 0, dst)
    assert dst[0] == 42


def thr_cols(L, segmap, seg_stride, mask, lut, left_q, left_s, w4, h4):
    q = np.zeros(256, np.uint16)
    s = np.zeros(256, np.uint16)
    L.r2o_setup_thr_cols(p(q), p(s), p(np.asarray(segmap, np.uint8)), C.c_int64(seg_stride), p(mask),
                         p(np.asarray(lut, np.uint32)), p(left_q), p(left_s), 0, 0, w4, h4)
    return q, s


def test_setup_thr_cols_uniform_segmap(L):
    """deblock.rs:2612-2645"""
    q, s = thr_cols(L, np.zeros(16), 4, np.zeros((4, 5, 4), np.uint16), [[20] * 16, [10] * 16],
                    np.zeros(16, np.uint16), np.zeros(16, np.uint16), 4, 4)
    assert q[0 * 16 + 0] == 20 and q[1 * 16 + 0] == 20
    assert s[0 * 16 + 0] == 10 and s[1 * 16 + 0] == 10


def test_setup_thr_cols_left_state_update(L):
    """deblock.rs:2647-2680"""
    lq, ls = np.zeros(16, np.uint16), np.zeros(16, np.uint16)
    lut = np.zeros((2, 16), np.uint32)
    lut[0][2], lut[1][2] = 30, 15
    thr_cols(L, np.full(16, 2), 4, np.zeros((4, 5, 4), np.uint16), lut, lq, ls, 4, 4)
    assert lq[0] == 30 and ls[0] == 15


def test_setup_thr_cols_subpu_mask(L):
    """deblock.rs:2682-2715"""
    mask = np.zeros((2, 5, 4), np.uint16)
    mask[1][4][0] = 1
    q, s = thr_cols(L, np.zeros(4), 2, mask, [[40] * 16, [20] * 16], np.full(16, 40, np.uint16),
                    np.full(16, 20, np.uint16), 2, 2)
    assert q[1 * 16 + 0] == 5 and s[1 * 16 + 0] == 2


def test_setup_thr_cols_mixed_thresholds(L):
    """deblock.rs:2717-2751"""
    lut = np.zeros((2, 16), np.uint32)
    lut[0][1], lut[1][1] = 30, 15
    q, _ = thr_cols(L, [0, 1, 0, 1], 2, np.zeros((2, 5, 4), np.uint16), lut, np.zeros(16, np.uint16),
                    np.zeros(16, np.uint16), 2, 2)
    assert q[0 * 16 + 0] == 0 and q[1 * 16 + 0] == 30


def thr_rows(L, segmap, seg_off, seg_stride, mask, lut, above, w4, h4):
    q = np.zeros(256, np.uint16)
    s = np.zeros(256, np.uint16)
    L.r2o_setup_thr_rows(p(q), p(s), p(np.asarray(segmap, np.uint8)), C.c_int64(seg_off), C.c_int64(seg_stride),
                         p(mask), p(np.asarray(lut, np.uint32)),
                         None if above is None else p(np.asarray(above, np.uint32)), 0, 0, w4, h4)
    return q, s


def test_setup_thr_rows_no_above(L):
    """deblock.rs:2753-2782 (x4 + y4 * 16 in the filter path's layout)"""
    q, s = thr_rows(L, np.zeros(16), 0, 4, np.zeros((4, 5, 4), np.uint16), [[20] * 16, [10] * 16], None, 4, 4)
    assert q[0 + 0 * 16] == 20 and q[0 + 1 * 16] == 20 and s[0 + 0 * 16] == 10


def test_setup_thr_rows_with_above(L):
    """deblock.rs:2784-2823"""
    segmap = np.zeros(5 * 4, np.uint8)
    segmap[0:4] = 1
    above = np.zeros((2, 16), np.uint32)
    above[0][1], above[1][1] = 30, 15
    q, s = thr_rows(L, segmap, 4, 4, np.zeros((4, 5, 4), np.uint16), [[10] * 16, [5] * 16], above, 4, 4)
    assert q[0] == 20 and s[0] == 10


def test_setup_thr_rows_subpu_mask(L):
    """deblock.rs:2825-2854"""
    mask = np.zeros((2, 5, 4), np.uint16)
    mask[1][4][0] = 1
    q, s = thr_rows(L, np.zeros(4), 0, 2, mask, [[40] * 16, [20] * 16], None, 2, 2)
    assert q[0 + 1 * 16] == 5 and s[0 + 1 * 16] == 2


def backup_db(L, dst, src, stride, ss_ver, sb128, row, row_h, w, lr_backup, n_tc):
    L.r2o_backup_db(p(dst), p(src), C.c_int64(stride), ss_ver, int(sb128), row, row_h, w, int(lr_backup), n_tc)


def _src_rows(stride, rows, first, base, w):
    src = np.zeros(stride * rows, np.uint16)
    for i in range(4):
        src[(first + i) * stride:(first + i) * stride + w] = base + i
    return src


def test_backup_db_first_row_single_thread(L):
    """deblock.rs:2855-2875"""
    stride, w = 64, 16
    src = _src_rows(stride, 128, 54, 10, w)
    dst = np.zeros(stride * 64, np.uint16)
    backup_db(L, dst, src, stride, 0, False, 0, 56, w, False, 1)
    for i in range(4):
        assert (dst[(4 + i) * stride:(4 + i) * stride + w] == 10 + i).all()


def test_backup_db_not_first_row(L):
    """deblock.rs:2877-2905"""
    stride, w = 64, 8
    src = _src_rows(stride, 128, 62, 20, w)
    dst = np.zeros(stride * 64, np.uint16)
    for i in range(4):
        dst[(4 + i) * stride:(4 + i) * stride + w] = 50 + i
    backup_db(L, dst, src, stride, 0, False, 56, 120, w, False, 1)
    assert (dst[0:w] == 50).all() and (dst[3 * stride:3 * stride + w] == 53).all()
    assert (dst[4 * stride:4 * stride + w] == 20).all() and (dst[7 * stride:7 * stride + w] == 23).all()


def test_backup_db_multithread(L):
    """deblock.rs:2907-2924"""
    stride, w = 64, 8
    src = _src_rows(stride, 128, 54, 30, w)
    dst = np.zeros(stride * 64, np.uint16)
    backup_db(L, dst, src, stride, 0, False, 0, 56, w, False, 2)
    assert (dst[0:w] == 30).all() and (dst[3 * stride:3 * stride + w] == 33).all()


def test_backup_db_ss_ver(L):
    """deblock.rs:2926-2943"""
    stride, w = 64, 8
    src = _src_rows(stride, 64, 26, 40, w)
    dst = np.zeros(stride * 32, np.uint16)
    backup_db(L, dst, src, stride, 1, False, 0, 28, w, False, 2)
    assert (dst[0:w] == 40).all() and (dst[3 * stride:3 * stride + w] == 43).all()


def test_backup_db_sb128(L):
    """deblock.rs:2945-2962"""
    stride, w = 64, 8
    src = _src_rows(stride, 256, 118, 60, w)
    dst = np.zeros(stride * 128, np.uint16)
    backup_db(L, dst, src, stride, 0, True, 0, 120, w, False, 2)
    assert (dst[0:w] == 60).all() and (dst[3 * stride:3 * stride + w] == 63).all()


def test_backup_db_lr_mode(L):
    """deblock.rs:2964-2982"""
    stride, w = 64, 8
    src = _src_rows(stride, 128, 54, 70, w)
    dst = np.zeros(stride * 64, np.uint16)
    backup_db(L, dst, src, stride, 0, True, 0, 56, w, True, 2)
    assert (dst[0:w] == 70).all() and (dst[3 * stride:3 * stride + w] == 73).all()


def test_backup_db_no_stripes(L):
    """deblock.rs:2984-2993"""
    stride, w = 64, 8
    src = np.zeros(stride * 128, np.uint16)
    dst = np.zeros(stride * 64, np.uint16)
    backup_db(L, dst, src, stride, 0, False, 0, 10, w, False, 2)
    assert (dst == 0).all()
