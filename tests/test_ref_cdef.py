"""The reference's CDEF unit tests (crates/rav2d/src/cdef.rs:1183-1550), one
test here per test there, re-asserted against the CPU oracle's restatement
(oracle/cdef.cpp).  Each test names the reference test and its line; inputs
and assertions are the reference's.  The reference's 8-bit entry points
(cdef_find_dir, cdef_padding_8bpc, cdef_filter_block_8bpc) are the oracle's
functions at bit depth 8 on uint16-held samples."""
import ctypes as C

import numpy as np
import pytest

HAVE_LEFT, HAVE_RIGHT, HAVE_TOP, HAVE_BOTTOM = 1, 2, 4, 8
ALL = HAVE_TOP | HAVE_BOTTOM | HAVE_LEFT | HAVE_RIGHT
I16_MIN = -32768


def p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def L(oracle):
    lib = oracle.lib()
    for n in ("r2o_constrain", "r2o_adjust_strength", "r2o_cdef_pri_tap", "r2o_cdef_apply_constrain",
              "r2o_cdef_find_dir"):
        getattr(lib, n).restype = C.c_int
    return lib


def find_dir(L, img, stride=8, bd=8):
    var = C.c_uint32(0)
    d = L.r2o_cdef_find_dir(p(img), C.c_int64(stride), C.byref(var), bd)
    return d, var.value


def filter_block(L, dst, stride, dst_off, left, top, top_off, bottom, bottom_off, pri, sec, dir_, damping, w, h,
                 edges, bd=8):
    L.r2o_cdef_filter_block(p(dst), C.c_int64(stride), C.c_int64(dst_off), p(left), p(top), C.c_int64(top_off),
                            p(bottom), C.c_int64(bottom_off), pri, sec, dir_, damping, w, h, edges, bd)


def padding(L, tmp, tmp_stride, src, src_stride, src_off, left, top, top_off, bottom, bottom_off, w, h, edges):
    L.r2o_cdef_padding(p(tmp), tmp_stride, p(src), C.c_int64(src_stride), C.c_int64(src_off), p(left), p(top),
                       C.c_int64(top_off), p(bottom), C.c_int64(bottom_off), w, h, edges)


def test_constrain_zero_diff(L):
    """cdef.rs:1187-1190"""
    assert L.r2o_constrain(0, 10, 1) == 0


def test_constrain_small_diff(L):
    """cdef.rs:1192-1197"""
    r = L.r2o_constrain(3, 10, 1)
    assert 0 < r <= 3


def test_constrain_negative_diff(L):
    """cdef.rs:1199-1203"""
    assert L.r2o_constrain(-5, 10, 1) < 0


def test_constrain_large_diff_clamped(L):
    """cdef.rs:1205-1209"""
    assert L.r2o_constrain(100, 10, 1) <= 10


def test_constrain_zero_threshold(L):
    """cdef.rs:1211-1214"""
    assert L.r2o_constrain(5, 0, 1) == 0


def test_fill_basic(L):
    """cdef.rs:1216-1227"""
    buf = np.zeros(24, np.int16)
    L.r2o_cdef_fill(p(buf), C.c_int64(6), 4, 3)
    for y in range(3):
        for x in range(4):
            assert buf[y * 6 + x] == I16_MIN
        assert buf[y * 6 + 4] == 0 and buf[y * 6 + 5] == 0


def test_cdef_find_dir_uniform(L):
    """cdef.rs:1229-1236"""
    d, var = find_dir(L, np.full(64, 128, np.uint16))
    assert 0 <= d < 8
    assert var == 0


def test_cdef_find_dir_vertical(L):
    """cdef.rs:1238-1250"""
    img = np.array([[64 if x < 4 else 192 for x in range(8)] for y in range(8)], np.uint16).ravel()
    d, var = find_dir(L, img)
    assert 0 <= d < 8 and var > 0


def test_cdef_find_dir_horizontal(L):
    """cdef.rs:1252-1264"""
    img = np.array([[64 if y < 4 else 192 for x in range(8)] for y in range(8)], np.uint16).ravel()
    d, var = find_dir(L, img)
    assert 0 <= d < 8 and var > 0


def test_cdef_pri_tap(L):
    """cdef.rs:1266-1272"""
    assert [L.r2o_cdef_pri_tap(s) for s in (4, 3, 2, 1)] == [4, 3, 4, 3]


def test_cdef_apply_constrain_zero(L):
    """cdef.rs:1274-1277"""
    assert L.r2o_cdef_apply_constrain(100, 100, 100, 10, 1, 4) == 0


def test_cdef_apply_constrain_symmetric(L):
    """cdef.rs:1279-1283"""
    assert L.r2o_cdef_apply_constrain(100, 105, 95, 10, 1, 4) == 0


def test_adjust_strength_zero_var(L):
    """cdef.rs:1285-1288"""
    assert L.r2o_adjust_strength(100, 0) == 0


def test_adjust_strength_low_var(L):
    """cdef.rs:1290-1294"""
    assert L.r2o_adjust_strength(100, 32) == (100 * 4 + 8) >> 4


def test_adjust_strength_high_var(L):
    """cdef.rs:1296-1300"""
    assert L.r2o_adjust_strength(100, 1 << 18) > L.r2o_adjust_strength(100, 64)


def test_adjust_strength_monotonic(L):
    """cdef.rs:1302-1310"""
    a, b, c = (L.r2o_adjust_strength(100, v) for v in (64, 256, 4096))
    assert a <= b <= c


def test_cdef_padding_all_edges(L):
    """cdef.rs:1312-1339"""
    src = np.full(16 * 16, 100, np.uint16)
    left = np.tile(np.array([50, 60], np.uint16), 8)
    top = np.full(64, 200, np.uint16)
    bottom = np.full(64, 150, np.uint16)
    tmp = np.zeros(12 * 20, np.int16)
    padding(L, tmp, 12, src, 16, 2, left, top, 2, bottom, 2, 8, 8, ALL)
    o = 2 * 12 + 2
    assert tmp[o] == 100 and tmp[o - 1] == 60 and tmp[o - 2] == 50


def test_cdef_padding_no_edges(L):
    """cdef.rs:1341-1356"""
    src = np.full(16 * 16, 100, np.uint16)
    left = np.zeros(16, np.uint16)
    top = np.zeros(32, np.uint16)
    bottom = np.zeros(32, np.uint16)
    tmp = np.zeros(12 * 20, np.int16)
    padding(L, tmp, 12, src, 16, 0, left, top, 0, bottom, 0, 8, 8, 0)
    o = 2 * 12 + 2
    assert tmp[o] == 100 and tmp[o - 1] == I16_MIN and tmp[o - 12] == I16_MIN


def cdef_bufs(val, stride, w, h):
    """make_cdef_test_bufs (cdef.rs:1358-1369)."""
    return (np.full(stride * (h + 4), val, np.uint16), np.full(2 * h, val, np.uint16),
            np.full(stride * 2 + w + 4, val, np.uint16), np.full(stride * 2 + w + 4, val, np.uint16))


def test_cdef_filter_block_uniform(L):
    """cdef.rs:1371-1392"""
    stride = 16
    dst, left, top, bottom = cdef_bufs(128, stride, 8, 8)
    dst_off = stride + 2
    filter_block(L, dst, stride, dst_off, left, top, 2, bottom, 2, 8, 4, 0, 6, 8, 8, ALL)
    for y in range(8):
        assert (dst[dst_off + y * stride:dst_off + y * stride + 8] == 128).all()


def test_cdef_filter_block_pri_only(L):
    """cdef.rs:1394-1413"""
    stride = 16
    dst_off = stride + 2
    dst = np.full(stride * 12, 128, np.uint16)
    dst[dst_off + 3 * stride + 3] = 120
    left = np.full(16, 128, np.uint16)
    top = np.full(stride * 2 + 12, 128, np.uint16)
    bottom = np.full(stride * 2 + 12, 128, np.uint16)
    filter_block(L, dst, stride, dst_off, left, top, 2, bottom, 2, 8, 0, 0, 6, 8, 8, ALL)
    assert dst[dst_off + 3 * stride + 3] != 120


def test_cdef_filter_block_sec_only(L):
    """cdef.rs:1415-1434"""
    stride = 16
    dst_off = stride + 2
    dst = np.full(stride * 12, 128, np.uint16)
    dst[dst_off + 3 * stride + 3] = 120
    left = np.full(16, 128, np.uint16)
    top = np.full(stride * 2 + 12, 128, np.uint16)
    bottom = np.full(stride * 2 + 12, 128, np.uint16)
    filter_block(L, dst, stride, dst_off, left, top, 2, bottom, 2, 0, 4, 0, 6, 8, 8, ALL)
    assert dst[dst_off + 3 * stride + 3] != 120


def test_cdef_filter_block_pri_sec_combined(L):
    """cdef.rs:1436-1475"""
    stride = 16
    dst_off = stride + 2
    dst = np.zeros(stride * 12, np.uint16)
    for y in range(8):
        for x in range(8):
            dst[dst_off + y * stride + x] = (y * 20 + x * 10) & 0xFF
    left = np.array([[(y * 20 - 20) & 0xFF, (y * 20 - 10) & 0xFF] for y in range(8)], np.uint16).ravel()
    top = np.zeros(stride * 2 + 12, np.uint16)
    bottom = np.zeros(stride * 2 + 12, np.uint16)
    for x in range(12):
        top[x] = top[stride + x] = (x * 10) & 0xFF
        bottom[x] = (8 * 20 + x * 10) & 0xFF
        bottom[stride + x] = (9 * 20 + x * 10) & 0xFF
    orig = dst.copy()
    filter_block(L, dst, stride, dst_off, left, top, 2, bottom, 2, 8, 4, 3, 6, 8, 8, ALL)
    blk = lambda a: np.array([a[dst_off + y * stride:dst_off + y * stride + 8] for y in range(8)])  # noqa: E731
    assert (blk(dst) != blk(orig)).any()


def test_cdef_filter_block_no_edges(L):
    """cdef.rs:1477-1490"""
    stride = 16
    dst_off = stride + 2
    dst, left, top, bottom = cdef_bufs(128, stride, 8, 8)
    filter_block(L, dst, stride, dst_off, left, top, 2, bottom, 2, 8, 4, 0, 6, 8, 8, 0)
    for y in range(8):
        assert (dst[dst_off + y * stride:dst_off + y * stride + 8] == 128).all()


def test_backup2lines_plane_positive_stride(L):
    """cdef.rs:1492-1505"""
    stride = 16
    src = np.array([(y * 16 + x) & 0xFF for y in range(8) for x in range(16)], np.uint16)
    dst = np.zeros(2 * stride, np.uint16)
    L.r2o_backup2lines_plane(p(dst), C.c_int64(0), p(src), C.c_int64(0), C.c_int64(stride), 8)
    assert (dst[0:16] == src[6 * 16:7 * 16]).all()
    assert (dst[16:32] == src[7 * 16:8 * 16]).all()


def test_backup2lines_plane_i420_chroma(L):
    """cdef.rs:1507-1518"""
    stride = 8
    src = np.arange(4 * stride, dtype=np.uint16)
    dst = np.zeros(2 * stride, np.uint16)
    L.r2o_backup2lines_plane(p(dst), C.c_int64(0), p(src), C.c_int64(0), C.c_int64(stride), 4)
    assert (dst[0:8] == src[16:24]).all()
    assert (dst[8:16] == src[24:32]).all()


def test_backup2x8_plane(L):
    """cdef.rs:1520-1535"""
    stride = 16
    src = np.array([(y * 16 + x) & 0xFF for y in range(8) for x in range(16)], np.uint16)
    dst = np.zeros(16, np.uint16)
    L.r2o_backup2x8_plane(p(dst), p(src), C.c_int64(0), C.c_int64(stride), C.c_int64(6), 8)
    for y in range(8):
        assert dst[2 * y] == src[y * 16 + 4] and dst[2 * y + 1] == src[y * 16 + 5]


def test_backup2x8_plane_chroma_4rows(L):
    """cdef.rs:1537-1549"""
    stride = 8
    src = np.arange(1, 4 * stride + 1, dtype=np.uint16)
    dst = np.zeros(16, np.uint16)
    L.r2o_backup2x8_plane(p(dst), p(src), C.c_int64(0), C.c_int64(stride), C.c_int64(4), 4)
    assert list(dst[0:2]) == [3, 4]
    assert list(dst[2:4]) == [11, 12]
