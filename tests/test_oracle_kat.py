"""Pin the CPU oracle to the reference: every exact-value assertion of the
reference's own unit tests for the filter path, re-asserted against the
oracle's restatement (test names cite the reference test they mirror)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def p(a):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- tables
def test_table_sizes_and_digests():
    """gdf_tables.rs:2640-2656 table sizes; the FNV digests recorded in the
    generated header match the committed data."""
    hdr = open(os.path.join(ROOT, "rav2d_b200", "csrc", "av2_tables.h")).read()
    digests = dict((m.group(1), (int(m.group(2)), int(m.group(3), 16)))
                   for m in re.finditer(r"X\((\w+), (\d+), 0x([0-9a-f]+)ULL\)", hdr))
    assert digests["GDF_ALPHA"][0] == 3168
    assert digests["GDF_WEIGHT"][0] == 9504
    assert digests["GDF_INTRA_ERROR"][0] == 24576
    assert digests["GDF_INTER_ERROR"][0] == 30000
    assert digests["GAUSSIAN_SEQUENCE"][0] == 2048
    assert digests["PC_WIENER_LUT_TO_CLASS"][0] == 4096
    for name, (n, h) in digests.items():
        m = re.search(r"R2G_TABLE\(\w+, " + name + r"\)[\[\]\d]* = \{(.*?)\};", hdr, re.S)
        vals = [int(v) for v in re.findall(r"-?\d+", m.group(1))]
        assert len(vals) == n
        acc = 0xCBF29CE484222325
        for v in vals:
            for b in (v & 0xFFFFFFFF).to_bytes(4, "little"):
                acc = ((acc ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
        assert acc == h, name


# ---------------------------------------------------------------- deblock
def test_deblock_quant_thr_zero(oracle):
    # lf_mask.rs:827-831
    assert oracle.lib().r2o_deblock_quant_thr(0, 0) == (64 + 4) >> 9


def test_dq_lookup(oracle):
    L = oracle.lib()
    assert L.r2o_dq_lookup(0) == 64
    assert L.r2o_dq_lookup(1) == 40
    assert L.r2o_dq_lookup(25) == 80
    assert L.r2o_dq_lookup(300) == L.r2o_dq_lookup(255)


def test_filter_choice_uniform(oracle):
    # deblock.rs:2386-2392
    buf = np.full(64, 128, np.uint16)
    assert oracle.lib().r2o_filter_choice(p(buf), 16, 19, 1, 3, 3, 10, 100) == 3


def test_filter_choice_sharp_edge(oracle):
    # deblock.rs:2395-2406
    buf = np.zeros(64, np.uint16)
    buf[:32] = 50
    buf[32:] = 200
    assert oracle.lib().r2o_filter_choice(p(buf), 32, 35, 1, 3, 3, 10, 20) <= 1


def test_deblock_uniform_unchanged(oracle):
    # deblock.rs:2408-2427
    stride = 32
    dst = np.full(stride * 8, 128, np.uint16)
    orig = dst.copy()
    oracle.lib().r2o_deblock(p(dst), stride * 2 + 8, 10, 20, stride, 1, 3, 3, 0, 0, 8)
    assert (dst == orig).all()


def _setup_thr_cols(oracle, segmap, mask, lut, left_q, left_s, w4, h4):
    q = np.zeros(256, np.uint16)
    s = np.zeros(256, np.uint16)
    oracle.lib().r2o_setup_thr_cols(p(q), p(s), p(segmap), C.c_int64(w4), p(mask), p(lut), p(left_q), p(left_s),
                                    0, 0, w4, h4)
    return q, s


def test_setup_thr_cols_uniform_segmap(oracle):
    # deblock.rs:2613-2646: prev 0 | cur 20 -> 20; (20+20+1)>>1 -> 20
    lut = np.array([[20] * 16, [10] * 16], np.uint32)
    q, s = _setup_thr_cols(oracle, np.zeros(16, np.uint8), np.zeros((4, 5, 4), np.uint16), lut,
                           np.zeros(16, np.uint16), np.zeros(16, np.uint16), 4, 4)
    assert q[0 * 16 + 0] == 20 and q[1 * 16 + 0] == 20
    assert s[0] == 10 and s[16] == 10


def test_setup_thr_cols_left_state_update(oracle):
    # deblock.rs:2648-2680
    lut = np.zeros((2, 16), np.uint32)
    lut[0, 2], lut[1, 2] = 30, 15
    lq, ls = np.zeros(16, np.uint16), np.zeros(16, np.uint16)
    _setup_thr_cols(oracle, np.full(16, 2, np.uint8), np.zeros((4, 5, 4), np.uint16), lut, lq, ls, 4, 4)
    assert lq[0] == 30 and ls[0] == 15


def test_setup_thr_cols_subpu_mask(oracle):
    # deblock.rs:2682-2720: subpu bit -> threshold >> 3 (40 -> 5, 20 -> 2)
    mask = np.zeros((2, 5, 4), np.uint16)
    mask[0, 4, 0] = 0b10  # x4 = 0, y4 = 1
    lut = np.array([[40] * 16, [20] * 16], np.uint32)
    q, s = _setup_thr_cols(oracle, np.zeros(4, np.uint8), mask, lut, np.full(16, 40, np.uint16),
                           np.full(16, 20, np.uint16), 2, 2)
    assert q[0 + 1] == 5 and s[0 + 1] == 2


def test_backup_db_first_row_single_thread(oracle):
    # deblock.rs:2856-2875
    stride, w = 64, 16
    src = np.zeros(stride * 128, np.uint16)
    for i in range(4):
        src[(54 + i) * stride:(54 + i) * stride + w] = 10 + i
    dst = np.zeros(stride * 64, np.uint16)
    oracle.lib().r2o_backup_db(p(dst), p(src), C.c_int64(stride), 0, 0, 0, 56, w, 0, 1)
    for i in range(4):
        assert (dst[(4 + i) * stride:(4 + i) * stride + w] == 10 + i).all()


def test_backup_db_not_first_row(oracle):
    # deblock.rs:2877-2900
    stride, w = 64, 8
    src = np.zeros(stride * 128, np.uint16)
    for i in range(4):
        src[(62 + i) * stride:(62 + i) * stride + w] = 20 + i
    dst = np.zeros(stride * 64, np.uint16)
    for i in range(4):
        dst[(4 + i) * stride:(4 + i) * stride + w] = 50 + i
    oracle.lib().r2o_backup_db(p(dst), p(src), C.c_int64(stride), 0, 0, 56, 120, w, 0, 1)
    assert (dst[0:w] == 50).all() and (dst[3 * stride:3 * stride + w] == 53).all()
    assert (dst[4 * stride:4 * stride + w] == 20).all() and (dst[7 * stride:7 * stride + w] == 23).all()


# ---------------------------------------------------------------- cdef
def test_adjust_strength(oracle):
    # cdef.rs:1286-1310
    L = oracle.lib()
    assert L.r2o_adjust_strength(100, 0) == 0
    assert L.r2o_adjust_strength(100, 32) == (100 * 4 + 8) >> 4
    assert L.r2o_adjust_strength(100, 1 << 18) > L.r2o_adjust_strength(100, 64)
    a, b, c = (L.r2o_adjust_strength(100, v) for v in (64, 256, 4096))
    assert a <= b <= c


def test_constrain(oracle):
    # cdef.rs:1213-1240
    L = oracle.lib()
    assert L.r2o_constrain(5, 0, 1) == 0
    assert L.r2o_constrain(0, 10, 1) == 0
    assert L.r2o_constrain(3, 10, 1) == 3
    assert L.r2o_constrain(-3, 10, 1) == -3


def test_cdef_find_dir(oracle):
    # cdef.rs:1242-1265: a non-flat block yields dir in 0..8 with var > 0;
    # a flat block has var 0.
    L = oracle.lib()
    img = np.array([[(x * 16) for x in range(8)] for _ in range(8)], np.uint16).ravel()
    var = C.c_uint32(0)
    d = L.r2o_cdef_find_dir(p(img), 8, C.byref(var), 8)
    assert 0 <= d < 8 and var.value > 0
    flat = np.full(64, 128, np.uint16)
    L.r2o_cdef_find_dir(p(flat), 8, C.byref(var), 8)
    assert var.value == 0


# ---------------------------------------------------------------- ccso
def test_ccso_score_boundary(oracle):
    # ccso.rs:400-405 and :283-285
    L = oracle.lib()
    assert L.r2o_ccso_score(10, 10, 0) == 1
    assert L.r2o_ccso_score(-10, 10, 0) == 1
    assert L.r2o_ccso_score(11, 10, 0) == 2
    assert L.r2o_ccso_score(-11, 10, 0) == 0
    assert L.r2o_ccso_score(-5, 10, 0) == 1
    assert L.r2o_ccso_score(11, 10, 1) == 1


@pytest.mark.parametrize("bo_only", [True, False])
def test_ccso_prep(oracle, bo_only):
    # ccso.rs:289-356: flat 128 input, band = 128 >> (8 - 4) = 8
    src = np.full(16 * 16, 128, np.uint16)
    left = np.full((16, 2), 128, np.uint16)
    top = np.full(32, 128, np.uint16)
    bottom = np.full(32, 128, np.uint16)
    dst = np.zeros(64, np.uint8)
    oracle.lib().r2o_ccso_prep(p(dst), 8, p(src), C.c_int64(16), C.c_int64(0), p(left), p(top), C.c_int64(2),
                               p(bottom), C.c_int64(2), 4, 0, 10, 0, int(bo_only), 15, 8, 8, 0, 0, 8)
    if bo_only:
        assert (dst == 128 >> 4).all()
    else:
        assert ((dst & 0x1F) == 8).all()


def test_ccso_add(oracle):
    # ccso.rs:358-376 -> 133; :378-398 skip mask leaves 128
    lut = np.array([0, 5, -5, 10, -10, 15, -15, 20], np.int8)
    dst = np.full(16, 128, np.uint16)
    idx = np.zeros(16, np.uint8)
    offs = np.full(8, 0x21, np.uint8)
    ll = np.zeros((1, 4), np.uint16)
    oracle.lib().r2o_ccso_add(p(dst), C.c_int64(4), p(idx), 4, p(offs), p(lut), 4, 4, p(ll), 8)
    assert dst[0] == 133
    dst = np.full(16, 128, np.uint16)
    ll = np.full((1, 4), 0xFFFF, np.uint16)
    oracle.lib().r2o_ccso_add(p(dst), C.c_int64(4), p(idx), 4, p(np.zeros(8, np.uint8)),
                              p(np.full(8, 10, np.int8)), 4, 4, p(ll), 8)
    assert (dst == 128).all()


# ---------------------------------------------------------------- LR
def test_get_qval_given_tskip_zero(oracle):
    # looprestoration.rs:2581-2584
    assert oracle.lib().r2o_get_qval_given_tskip(0, 0, 0, 0) == 255 * -547
    L = oracle.lib()
    assert L.r2o_get_qval_given_tskip(64, 300, 1, 0) != L.r2o_get_qval_given_tskip(64, 300, 1, 2)


def _row_luma(oracle, src, o, src_o, stride, w, edges, ss_hor, ss_ver, flt, n=32):
    dst = np.zeros(n, np.uint16)
    oracle.lib().r2o_backup_row_luma(p(dst), o, p(src), C.c_int64(src_o), C.c_int64(stride), w, edges, ss_hor,
                                     ss_ver, flt)
    return dst


def test_backup_row_luma(oracle):
    # looprestoration.rs:2709-2775
    stride = 32
    src = np.zeros(stride * 2 + 16, np.uint16)
    src[4:20] = 100
    src[4 + stride:20 + stride] = 200
    d = _row_luma(oracle, src, 4, 4, stride, 8, 0, 1, 1, 0)
    assert d[4] == (100 + 200 + 100 + 200) >> 2
    d = _row_luma(oracle, src, 4, 4, stride, 8, 0, 0, 1, 1)
    assert (d[4:12] == 150).all()
    d = _row_luma(oracle, src, 4, 4, stride, 8, 0, 0, 1, 2)
    assert (d[4:12] == 100).all()
    src = np.full(stride * 2 + 16, 80, np.uint16)
    d = _row_luma(oracle, src, 6, 6, stride, 8, 1 | 2, 0, 1, 2)
    assert (d[2:18] == 80).all()


def _flat_unit(w=8, h=8, stride=16):
    p_ = np.full(stride * (h + 8), 128, np.uint16)
    left = np.full((h + 8, 6), 128, np.uint16)
    lpf = np.full(stride * 8, 128, np.uint16)
    ll = np.zeros((h // 4 + 2, 4), np.uint16)
    return p_, left, lpf, ll


def test_ns_wiener_single_y_identity(oracle):
    # looprestoration.rs:2959-3010: zero taps on flat 128 -> 128
    w = h = 8
    stride = 16
    buf, left, lpf, ll = _flat_unit(w, h, stride)
    filt = np.zeros(16, np.int8)
    oracle.lib().r2o_ns_wiener_single_y(p(buf), C.c_int64(0), C.c_int64(stride), p(left), p(lpf), C.c_int64(0),
                                        p(lpf), C.c_int64(0), w, h, p(filt), 15, p(ll), 8)
    assert (buf.reshape(-1, stride)[:h, :w] == 128).all()


@pytest.mark.parametrize("pretrained", [False, True])
def test_wiener_multi_identity(oracle, pretrained):
    # looprestoration.rs:3105-3185 (user and pretrained identity)
    w = h = 8
    stride = 16
    buf, left, lpf, ll = _flat_unit(w, h, stride)
    lut = np.zeros(256, np.uint8)
    noskip = np.zeros(66, np.uint16)
    fu = np.zeros((1, 18), np.int8)
    fp_ = np.zeros((1, 13), np.int16)
    fp_[0, 12] = 128
    oracle.lib().r2o_wiener_multi(p(buf), C.c_int64(0), C.c_int64(stride), p(left), p(lpf), C.c_int64(0), p(lpf),
                                  C.c_int64(0), w, h, None if pretrained else p(fu), p(fp_) if pretrained else None,
                                  p(lut), p(noskip), 32, 15, p(ll), 8)
    assert (buf.reshape(-1, stride)[:h, :w] == 128).all()


# ---------------------------------------------------------------- film grain
def test_round2(oracle):
    # filmgrain.rs:966-977
    L = oracle.lib()
    assert L.r2o_round2(10, 1) == 5
    assert L.r2o_round2(11, 1) == 6
    assert L.r2o_round2(7, 2) == 2
    assert L.r2o_round2(-10, 1) == -5


def test_random_number(oracle):
    # filmgrain.rs:943-964: deterministic LFSR, varying outputs
    L = oracle.lib()
    st = C.c_uint32(1)
    vals = [L.r2o_get_random_number(4, C.byref(st)) for _ in range(32)]
    assert any(v != vals[0] for v in vals)
    st2 = C.c_uint32(1)
    assert vals == [L.r2o_get_random_number(4, C.byref(st2)) for _ in range(32)]
    st = C.c_uint32(0)
    assert L.r2o_get_random_number(11, C.byref(st)) == 0


def _scaling(oracle, bitdepth, pts):
    sc = np.full(1 << bitdepth, 0xFF, np.uint8)
    a = np.array(pts, np.uint8).reshape(-1, 2) if pts else np.zeros((0, 2), np.uint8)
    oracle.lib().r2o_generate_scaling(bitdepth, p(np.ascontiguousarray(a)), len(pts), p(sc))
    return sc


def test_generate_scaling_hbd(oracle):
    # filmgrain.rs:1296-1342
    assert (_scaling(oracle, 10, []) == 0).all()
    s = _scaling(oracle, 10, [[128, 200]])
    assert s[0] == 200 and s[511] == 200 and s[512] == 200 and s[1023] == 200
    s = _scaling(oracle, 10, [[0, 0], [255, 255]])
    assert s[0] == 0 and s[1023] == 255 and 120 < s[512] < 140
    s = _scaling(oracle, 10, [[0, 0], [100, 100]])
    assert (np.diff(s[:400].astype(int)) >= 0).all()
    s = _scaling(oracle, 10, [[0, 10], [128, 200]])
    assert s[1] > 0 and s[2] > 0 and s[3] > 0


def test_generate_scaling_8bpc(oracle):
    # filmgrain.rs:1240-1294 (8-bit LUT: flat ends, linear middle)
    s = _scaling(oracle, 8, [[0, 0], [255, 255]])
    assert s[0] == 0 and s[255] == 255 and 120 < s[128] < 136
    s = _scaling(oracle, 8, [[64, 50]])
    assert (s == 50).all()
