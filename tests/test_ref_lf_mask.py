"""The reference's deblock mask-builder unit tests (crates/rav2d/src/
lf_mask.rs:504-952), one test here per test there, re-asserted against the
CPU oracle's restatement (oracle/lf_mask.cpp, oracle/deblock.cpp).  Each
test names the reference test and its line; inputs and assertions are the
reference's.  Masks are [2][64][5][4] uint16 arrays (direction, position
across, level, 16-bit segment along); a single position's masks are [5][4]."""
import ctypes as C

import numpy as np
import pytest

from rav2d_b200 import abi

TXP_NONE, TXP_H5, TXP_V5 = 0, 6, 7
BS_8X8, I420 = 24, 1


def p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def L(oracle):
    lib = oracle.lib()
    lib.r2o_mask_inner_edges_v.argtypes = [C.c_void_p, C.c_uint64] + [C.c_int] * 5
    lib.r2o_mask_inner_edges_h.argtypes = [C.c_void_p, C.c_uint64] + [C.c_int] * 5
    lib.r2o_deblock_quant_thr.restype = C.c_uint32
    lib.r2o_deblock_side_thr.restype = C.c_uint32
    return lib


def masks2():
    return np.zeros((2, 64, 5, 4), np.uint16)


def test_av2_filter_default(L):
    """lf_mask.rs:508-513"""
    f = np.zeros(1, abi.AV2_FILTER_DTYPE)
    f["qidx"][0][0] = 7
    L.r2o_av2_filter_default(p(f))
    assert f["cdef_idx"][0][0] == -1
    assert f["qidx"][0][0] == 0


def test_av2_restoration_default(L):
    """lf_mask.rs:515-519"""
    r = np.ones(1, abi.AV2_RESTORATION_DTYPE)
    L.r2o_av2_restoration_default(p(r))
    assert r["lr"]["restoration_type"][0][0][0] == 0


def test_mask_outer_edge_l_basic(L):
    """lf_mask.rs:521-530"""
    m = np.zeros((5, 4), np.uint16)
    lv = np.full(4, 2, np.uint8)
    L.r2o_mask_outer_edge_l(p(m), 0, 4, 1, p(lv))
    assert m[1][0] == 0b1111
    assert (lv == 1).all()


def test_mask_outer_edge_l_min_level(L):
    """lf_mask.rs:532-542"""
    m = np.zeros((5, 4), np.uint16)
    lv = np.full(2, 1, np.uint8)
    L.r2o_mask_outer_edge_l(p(m), 0, 2, 3, p(lv))
    assert m[1][0] == 0b11 and m[3][0] == 0
    assert (lv == 3).all()


def test_mask_outer_edge_l_crosses_segment(L):
    """lf_mask.rs:544-553"""
    m = np.zeros((5, 4), np.uint16)
    lv = np.full(4, 2, np.uint8)
    L.r2o_mask_outer_edge_l(p(m), 14, 4, 2, p(lv))
    assert m[2][0] & (1 << 14) and m[2][0] & (1 << 15)
    assert m[2][1] & 1 and m[2][1] & 2


def test_mask_outer_edge_t_basic(L):
    """lf_mask.rs:555-564"""
    m = np.zeros((5, 4), np.uint16)
    a = np.full(4, 3, np.uint8)
    L.r2o_mask_outer_edge_t(p(m), 0, 4, 2, p(a))
    assert m[2][0] == 0b1111
    assert (a == 2).all()


def test_mask_outer_edge_t_min_level(L):
    """lf_mask.rs:566-572"""
    m = np.zeros((5, 4), np.uint16)
    a = np.zeros(3, np.uint8)
    L.r2o_mask_outer_edge_t(p(m), 0, 3, 2, p(a))
    assert m[0][0] == 0b111


def test_mask_inner_edges_v_basic(L):
    """lf_mask.rs:574-583"""
    m = masks2()
    L.r2o_mask_inner_edges_v(p(m), 0x0001_0001_0001_0001, 0, 8, 1, 4, 4)
    assert list(m[0][4][1]) == [1, 1, 1, 1]


def test_mask_inner_edges_v_zero_inner(L):
    """lf_mask.rs:585-596"""
    m = masks2()
    L.r2o_mask_inner_edges_v(p(m), 0, 0, 8, 1, 4, 4)
    assert (m[0] == 0).all()


def test_mask_inner_edges_h_basic(L):
    """lf_mask.rs:598-607"""
    m = masks2()
    L.r2o_mask_inner_edges_h(p(m), 0x0003_0003_0003_0003, 0, 8, 2, 4, 4)
    assert list(m[1][4][2]) == [3, 3, 3, 3]


def test_mask_inner_edges_h_zero_inner(L):
    """lf_mask.rs:609-620"""
    m = masks2()
    L.r2o_mask_inner_edges_h(p(m), 0, 0, 8, 1, 4, 4)
    assert (m[1] == 0).all()


def test_mask_inner_edges_h_multiple_steps(L):
    """lf_mask.rs:622-631"""
    m = masks2()
    L.r2o_mask_inner_edges_h(p(m), 0xFF, 0, 16, 1, 2, 4)
    for idx in (2, 6, 10, 14):
        assert m[1][idx][1][0] != 0


DIM_8X8 = np.array([2, 2, 1, 1], np.int32)  # lf_mask.rs:633-644 (w, h, lw, lh)
DIM_4X4 = np.array([1, 1, 0, 0], np.int32)  # lf_mask.rs:646-657


def edges_part(L, m, by4, bx4, w4, h4, part, dim, a, lv):
    L.r2o_mask_edges_part(p(m), by4, bx4, w4, h4, part, p(dim), 3, 3, p(a), p(lv))


def test_mask_edges_part_none_no_inner(L):
    """lf_mask.rs:659-680"""
    m = masks2()
    edges_part(L, m, 0, 0, 2, 2, TXP_NONE, DIM_8X8, np.zeros(2, np.uint8), np.zeros(2, np.uint8))
    assert m[0][0][0][0] != 0 and m[1][0][0][0] != 0


def test_mask_edges_part_none_with_inner(L):
    """lf_mask.rs:682-703"""
    m = masks2()
    edges_part(L, m, 0, 0, 4, 4, TXP_NONE, DIM_4X4, np.zeros(4, np.uint8), np.zeros(4, np.uint8))
    assert m[0][1][0][0] != 0 and m[1][1][0][0] != 0


def test_mask_edges_part_h5(L):
    """lf_mask.rs:705-726"""
    m = masks2()
    edges_part(L, m, 0, 0, 4, 8, TXP_H5, DIM_8X8, np.zeros(4, np.uint8), np.zeros(8, np.uint8))
    assert m[1][0][0][0] != 0 and m[0][0][0][0] != 0


def test_mask_edges_part_v5(L):
    """lf_mask.rs:728-749"""
    m = masks2()
    edges_part(L, m, 0, 0, 8, 4, TXP_V5, DIM_8X8, np.zeros(8, np.uint8), np.zeros(4, np.uint8))
    assert m[0][0][0][0] != 0 and m[1][0][0][0] != 0


def test_mask_edges_part_updates_context(L):
    """lf_mask.rs:751-774"""
    m = masks2()
    a, lv = np.zeros(2, np.uint8), np.zeros(2, np.uint8)
    edges_part(L, m, 0, 0, 2, 2, TXP_NONE, DIM_8X8, a, lv)
    assert list(a) == [1, 1] and list(lv) == [1, 1]


def subpu(L, w4, h4, hsz, vsz, ds):
    m = masks2()
    L.r2o_mask_subpu_edges(p(m), 0, 0, w4, h4, 1, 1, hsz, vsz, ds)
    return m


def test_mask_subpu_edges_hsz_only(L):
    """lf_mask.rs:776-788"""
    m = subpu(L, 8, 4, 4, 0, 15)
    assert m[0][4][1][0] != 0
    assert (m[1] == 0).all()


def test_mask_subpu_edges_vsz_only(L):
    """lf_mask.rs:790-802"""
    m = subpu(L, 4, 8, 0, 4, 15)
    assert m[1][4][1][0] != 0
    assert (m[0] == 0).all()


def test_mask_subpu_edges_both(L):
    """lf_mask.rs:804-810"""
    m = subpu(L, 8, 8, 4, 4, 0)
    assert m[0][4][1][0] != 0 and m[1][4][1][0] != 0


def test_mask_subpu_edges_ds_mask_sets_noskip(L):
    """lf_mask.rs:812-817"""
    assert subpu(L, 8, 4, 4, 0, 15)[0][4][4][0] != 0


def test_mask_subpu_edges_no_ds_mask(L):
    """lf_mask.rs:819-824"""
    assert subpu(L, 8, 4, 4, 0, 0)[0][4][4][0] == 0


def test_deblock_quant_thr_8bit(L):
    """lf_mask.rs:826-831"""
    assert L.r2o_deblock_quant_thr(0, 128) > 0
    assert L.r2o_deblock_quant_thr(0, 0) == (64 + 4) >> 9


def test_deblock_quant_thr_10bit(L):
    """lf_mask.rs:833-837"""
    assert L.r2o_deblock_quant_thr(1, 200) > 0


def test_deblock_quant_thr_clamps(L):
    """lf_mask.rs:839-847"""
    assert L.r2o_deblock_quant_thr(0, -10) == L.r2o_deblock_quant_thr(0, 0)
    assert L.r2o_deblock_quant_thr(0, 9999) == L.r2o_deblock_quant_thr(0, 255)


def test_deblock_side_thr_8bit(L):
    """lf_mask.rs:849-853 (a tautology there); the value is in range."""
    assert 0 <= L.r2o_deblock_side_thr(0, 128) < 1 << 16


def test_deblock_side_thr_10bit(L):
    """lf_mask.rs:855-859 (evaluated only there); the value is in range."""
    assert 0 <= L.r2o_deblock_side_thr(1, 200) < 1 << 16


def test_deblock_side_thr_clamps(L):
    """lf_mask.rs:861-866"""
    assert L.r2o_deblock_side_thr(0, -10) == L.r2o_deblock_side_thr(0, 0)


def transpose(L, src, x64, ss_hor, ss_ver, dst):
    L.r2o_transpose_lossless_mask(p(dst), p(np.ascontiguousarray(src, np.uint16)), x64, ss_hor, ss_ver)


def test_transpose_lossless_mask_identity(L):
    """lf_mask.rs:868-876"""
    dst = np.zeros(17, np.uint16)
    transpose(L, np.zeros((16, 4)), 0, 0, 0, dst)
    assert (dst[1:17] == 0).all()


def test_transpose_lossless_mask_single_bit(L):
    """lf_mask.rs:878-885"""
    src = np.zeros((16, 4), np.uint16)
    src[3][0] = 1 << 5
    dst = np.zeros(17, np.uint16)
    transpose(L, src, 0, 0, 0, dst)
    assert dst[5 + 1] & (1 << 3) == 1 << 3


def test_transpose_lossless_mask_ss(L):
    """lf_mask.rs:887-896"""
    src = np.zeros((16, 4), np.uint16)
    src[0][0] = 0xFF
    dst = np.zeros(17, np.uint16)
    transpose(L, src, 0, 1, 1, dst)
    assert all(dst[x + 1] & 1 == 1 for x in range(8))


def test_transpose_lossless_mask_prev_column(L):
    """lf_mask.rs:898-905"""
    dst = np.zeros(17, np.uint16)
    dst[16] = 0xABCD
    transpose(L, np.zeros((16, 4)), 0, 0, 0, dst)
    assert dst[0] == 0xABCD


def test_create_db_mask_intra_block(L):
    """lf_mask.rs:907-951: an 8x8 intra block with a residual marks edges."""
    m = masks2()
    blk = np.array([BS_8X8, 1, 0, 0, 0, 0, 0, -1, 0, 0, 0], np.int32)
    hdr = np.zeros(12, np.int32)  # FrameHeader / SequenceHeader defaults
    a, lv = np.zeros(64, np.uint8), np.zeros(64, np.uint8)
    L.r2o_create_db_mask(p(m), p(blk), BS_8X8, 0, 0, 64, 64, I420, 0, p(a), p(lv), p(hdr))
    assert (m != 0).any()
