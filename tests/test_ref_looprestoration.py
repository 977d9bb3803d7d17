"""The reference's loop-restoration unit tests (crates/rav2d/src/
looprestoration.rs:2550-3362), one test here per test there, re-asserted
against the CPU oracle's restatement (oracle/lr.cpp).  Each test names the
reference test and its line; inputs and assertions are the reference's.  The
reference's u8 buffers are uint16 arrays here (the oracle's sample type) with
bit depth 8; [P; 6] left borders are (n, 6) arrays."""
import ctypes as C

import numpy as np
import pytest

LEFT, RIGHT, TOP, BOTTOM = 1, 2, 4, 8
ALL = TOP | BOTTOM | LEFT | RIGHT
U16P = C.POINTER(C.c_uint16)


def p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def L(oracle):
    lib = oracle.lib()
    lib.r2o_lr_const.restype = C.c_int
    lib.r2o_get_qval_given_tskip.restype = C.c_int
    lib.r2o_get_class_lut_idx.restype = C.c_int
    return lib


def row_ptrs(rows):
    """The reference's &[&[P]]: an array of row pointers (rows kept alive by
    the caller)."""
    arr = (U16P * len(rows))()
    for i, r in enumerate(rows):
        arr[i] = r.ctypes.data_as(U16P)
    return arr


def const(L, which, i, k=0):
    return L.r2o_lr_const(which, i, k)


def pair(L, which, i):
    return [const(L, which, i, 0), const(L, which, i, 1)]


def test_pc_wiener_normalizer(L):
    """looprestoration.rs:2554-2557"""
    assert const(L, 0, 3) == 7


def test_get_qval_given_tskip_8bpc(L):
    """looprestoration.rs:2559-2563"""
    assert L.r2o_get_qval_given_tskip(16, 100, 0, 0) != 0


def test_get_qval_given_tskip_all_modes(L):
    """looprestoration.rs:2565-2571 (the reference only evaluates all four
    modes); the values are also distinct per mode here."""
    vals = [L.r2o_get_qval_given_tskip(32, 200, i, 0) for i in range(4)]
    assert len(set(vals)) == 4


def test_get_qval_given_tskip_10bpc(L):
    """looprestoration.rs:2573-2578"""
    assert L.r2o_get_qval_given_tskip(64, 300, 1, 0) != L.r2o_get_qval_given_tskip(64, 300, 1, 2)


def test_get_qval_given_tskip_zero(L):
    """looprestoration.rs:2580-2584: 255 * MODE_OFFSETS[0]"""
    assert L.r2o_get_qval_given_tskip(0, 0, 0, 0) == 255 * const(L, 7, 0)
    assert const(L, 7, 0) == -547


def test_lr_edge_flags(L):
    """looprestoration.rs:2586-2592"""
    assert [const(L, 6, i) for i in range(4)] == [1, 2, 4, 8]


def backup_row(L, dst, o, src, src_o, left, left_off, w, edge_len, edges):
    L.r2o_backup_row(p(dst), o, p(src), C.c_int64(src_o), p(left), left_off, w, edge_len, edges)


def test_backup_row_no_edges(L):
    """looprestoration.rs:2594-2604"""
    src = np.full(32, 10, np.uint16)
    left = np.zeros(32, np.uint16)
    dst = np.zeros(32, np.uint16)
    o = 6
    backup_row(L, dst, o, src, 0, left, 0, 16, 6, 0)
    assert (dst[0:o] == 10).all()
    assert (dst[o:o + 16] == src[0:16]).all()
    assert (dst[o + 16:o + 22] == src[15]).all()


def test_backup_row_both_edges(L):
    """looprestoration.rs:2606-2626"""
    src = np.full(32, 50, np.uint16)
    src[0], src[15] = 10, 90
    left = np.full(16, 20, np.uint16)
    dst = np.zeros(32, np.uint16)
    o = 6
    backup_row(L, dst, o, src, 0, left, 6, 16, 6, LEFT | RIGHT)
    assert (dst[o:o + 16] == src[0:16]).all()
    assert (dst[0:o] == 20).all() and (dst[o + 16:o + 22] == 50).all()


def test_backup_row_lpf_no_edges(L):
    """looprestoration.rs:2628-2637"""
    src = np.full(32, 42, np.uint16)
    dst = np.zeros(32, np.uint16)
    o = 6
    L.r2o_backup_row_lpf(p(dst), o, p(src), C.c_int64(0), 16, 6, 0)
    assert (dst[0:o] == 42).all()
    assert (dst[o:o + 16] == src[0:16]).all()
    assert (dst[o + 16:o + 22] == src[15]).all()


def gradient_row(L, rows, row_off, col_off, w, shift):
    dst = np.zeros((16, 4), np.uint16)
    L.r2o_compute_gradient_row(p(dst), row_ptrs(rows), row_off, col_off, w, shift)
    return dst


def test_compute_gradient_row_flat(L):
    """looprestoration.rs:2639-2650"""
    row = np.full(32, 128, np.uint16)
    dst = gradient_row(L, [row] * 5, 2, 2, 4, 0)
    assert (dst[:3] == 0).all()


def test_compute_gradient_row_edge(L):
    """looprestoration.rs:2652-2660"""
    flat, bright = np.full(32, 100, np.uint16), np.full(32, 200, np.uint16)
    dst = gradient_row(L, [flat, bright, flat, bright, flat], 2, 2, 4, 0)
    assert dst[0][0] > 0


def gdf_add(L, pix, err, ll):
    L.r2o_gdf_add(p(pix), C.c_int64(8), p(err), 8, 8, 8, 16, p(ll), 8)


def test_gdf_add_basic(L):
    """looprestoration.rs:2662-2669"""
    pix = np.full(64, 128, np.uint16)
    gdf_add(L, pix, np.full(64, 10, np.int8), np.zeros((2, 4), np.uint16))
    assert pix[0] > 128


def test_gdf_add_skip_mask(L):
    """looprestoration.rs:2671-2678"""
    pix = np.full(64, 128, np.uint16)
    gdf_add(L, pix, np.full(64, 10, np.int8), np.full((2, 4), 0xFFFF, np.uint16))
    assert (pix == 128).all()


def test_gdf_add_negative_err(L):
    """looprestoration.rs:2680-2687"""
    pix = np.full(64, 128, np.uint16)
    gdf_add(L, pix, np.full(64, -10, np.int8), np.zeros((2, 4), np.uint16))
    assert pix[0] < 128


def test_get_class_lut_idx_flat(L):
    """looprestoration.rs:2689-2696 (the reference only evaluates it); the
    index is a valid PC_WIENER_LUT_TO_CLASS position."""
    rows = [np.full(64, 128, np.uint16) for _ in range(16)]
    noskip = np.full(16, 0xFFFF, np.uint16)
    idx = L.r2o_get_class_lut_idx(row_ptrs(rows), 6, 0, p(noskip), 32, 1, 1, 8, 0)
    assert 0 <= idx < 4096


def row_luma(L, dst, o, src, src_o, stride, w, edges, ss_hor, ss_ver, flt):
    L.r2o_backup_row_luma(p(dst), o, p(src), C.c_int64(src_o), C.c_int64(stride), w, edges, ss_hor, ss_ver, flt)


def test_backup_row_luma_no_ss_ver(L):
    """looprestoration.rs:2698-2706"""
    src = np.full(64, 42, np.uint16)
    dst = np.zeros(32, np.uint16)
    o = 6
    row_luma(L, dst, o, src, 0, 16, 16, 0, 0, 0, 0)
    assert (dst[o:o + 16] == src[0:16]).all()
    assert (dst[o - 4:o] == 42).all()


def _luma_src(stride=32):
    src = np.zeros(stride * 2 + 16, np.uint16)
    src[4:20] = 100
    src[4 + stride:20 + stride] = 200
    return src


def test_backup_row_luma_box_filter(L):
    """looprestoration.rs:2708-2720"""
    dst = np.zeros(32, np.uint16)
    row_luma(L, dst, 4, _luma_src(), 4, 32, 8, 0, 1, 1, 0)
    assert dst[4] == (100 + 200 + 100 + 200) >> 2


def test_backup_row_luma_vert_avg(L):
    """looprestoration.rs:2722-2736"""
    dst = np.zeros(32, np.uint16)
    row_luma(L, dst, 4, _luma_src(), 4, 32, 8, 0, 0, 1, 1)
    assert (dst[4:12] == 150).all()


def test_backup_row_luma_copy(L):
    """looprestoration.rs:2738-2752"""
    dst = np.zeros(32, np.uint16)
    row_luma(L, dst, 4, _luma_src(), 4, 32, 8, 0, 0, 1, 2)
    assert (dst[4:12] == 100).all()


def test_backup_row_luma_edges(L):
    """looprestoration.rs:2754-2775"""
    stride = 32
    src = np.full(stride * 2 + 16, 80, np.uint16)
    dst = np.zeros(32, np.uint16)
    o = 6
    row_luma(L, dst, o, src, 6, stride, 8, LEFT | RIGHT, 0, 1, 2)
    assert (dst[o:o + 8] == 80).all()
    assert (dst[o - 4:o] == 80).all()
    assert (dst[o + 8:o + 12] == 80).all()


def single_y(L, pix, p_off, stride, left, lpf, lpf_bottom, w, h, filt, edges, ll):
    L.r2o_ns_wiener_single_y(p(pix), C.c_int64(p_off), C.c_int64(stride), p(left), p(lpf), C.c_int64(4),
                             p(lpf_bottom), C.c_int64(4), w, h, p(filt), edges, p(ll), 8)


def test_ns_wiener_single_y_identity(L):
    """looprestoration.rs:2777-2820"""
    stride, h, w = 16, 8, 8
    p_off = stride + 4
    pix = np.full(stride * (h + 8), 128, np.uint16)
    left = np.full((h + 4, 6), 128, np.uint16)
    lpf = np.full(stride * 4 + 8, 128, np.uint16)
    lpf_bottom = np.full(stride * 2 + 8, 128, np.uint16)
    ll = np.zeros(((h >> 2) + 1, 4), np.uint16)
    single_y(L, pix, p_off, stride, left, lpf, lpf_bottom, w, h, np.zeros(16, np.int8), ALL, ll)
    for y in range(h):
        assert (pix[p_off + y * stride:p_off + y * stride + w] == 128).all()


def test_ns_wiener_single_y_skip_mask(L):
    """looprestoration.rs:2822-2862"""
    stride, h, w = 16, 8, 8
    p_off = stride + 4
    pix = np.full(stride * (h + 8), 100, np.uint16)
    pix[p_off + 3 * stride + 3] = 80
    orig = pix.copy()
    left = np.full((h + 4, 6), 100, np.uint16)
    lpf = np.full(stride * 4 + 8, 100, np.uint16)
    lpf_bottom = np.full(stride * 2 + 8, 100, np.uint16)
    ll = np.full(((h >> 2) + 1, 4), 0xFFFF, np.uint16)
    single_y(L, pix, p_off, stride, left, lpf, lpf_bottom, w, h, np.full(16, 4, np.int8), ALL, ll)
    for y in range(h):
        r = slice(p_off + y * stride, p_off + y * stride + w)
        assert (pix[r] == orig[r]).all()


def test_ns_wiener_single_y_filters_noise(L):
    """looprestoration.rs:2864-2899"""
    stride, h, w = 16, 8, 8
    p_off = stride + 4
    pix = np.full(stride * (h + 8), 128, np.uint16)
    pix[p_off + 4 * stride + 4] = 110
    left = np.full((h + 4, 6), 128, np.uint16)
    lpf = np.full(stride * 4 + 8, 128, np.uint16)
    lpf_bottom = np.full(stride * 2 + 8, 128, np.uint16)
    filt = np.array([8, 6, 4, 3, 2, 2, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0], np.int8)
    ll = np.zeros(((h >> 2) + 1, 4), np.uint16)
    single_y(L, pix, p_off, stride, left, lpf, lpf_bottom, w, h, filt, ALL, ll)
    assert 110 < pix[p_off + 4 * stride + 4] < 128


def test_wiener_ns_config_y_table(L):
    """looprestoration.rs:2901-2906"""
    assert const(L, 1, -1) == 16
    assert pair(L, 1, 0) == [1, 0] and pair(L, 1, 15) == [3, -3]


def test_wiener_ns_config_uv(L):
    """looprestoration.rs:2908-2912"""
    assert const(L, 2, -1) == 6 and const(L, 3, -1) == 12


def test_pc_wiener_config(L):
    """looprestoration.rs:2914-2919"""
    assert const(L, 4, -1) == 12
    assert pair(L, 4, 0) == [1, 0] and pair(L, 4, 11) == [0, 3]


def multi_data(h, stride):
    """make_wiener_multi_test_data (looprestoration.rs:2921-2956)."""
    p_off = stride + 4
    pix = np.full(stride * (h + 8), 128, np.uint16)
    left = np.full((h + 8, 6), 128, np.uint16)
    lpf = np.full(stride * 6 + 8, 128, np.uint16)
    lpf_bottom = np.full(stride * 4 + 8, 128, np.uint16)
    ll = np.zeros(((h >> 2) + 1, 4), np.uint16)
    noskip = np.full((h >> 2) + 1, 0xFFFF, np.uint16)
    return pix, p_off, left, lpf, 4, lpf_bottom, 4, ll, noskip


def multi(L, pix, p_off, stride, left, lpf, lpf_off, lpf_bottom, lpf_bottom_off, w, h, fu, fpt, lut, noskip, ll):
    L.r2o_wiener_multi(p(pix), C.c_int64(p_off), C.c_int64(stride), p(left), p(lpf), C.c_int64(lpf_off),
                       p(lpf_bottom), C.c_int64(lpf_bottom_off), w, h, None if fu is None else p(fu),
                       None if fpt is None else p(fpt), p(lut), p(noskip), 32, ALL, p(ll), 8)


def test_wiener_multi_user_identity(L):
    """looprestoration.rs:2958-2994 (ns_wiener_multi)"""
    w = h = 8
    stride = 16
    pix, p_off, left, lpf, lo, lpb, lbo, ll, noskip = multi_data(h, stride)
    multi(L, pix, p_off, stride, left, lpf, lo, lpb, lbo, w, h, np.zeros((1, 18), np.int8), None,
          np.zeros(256, np.uint8), noskip, ll)
    for y in range(h):
        assert (pix[p_off + y * stride:p_off + y * stride + w] == 128).all()


def test_wiener_multi_pretrained_identity(L):
    """looprestoration.rs:2996-3033 (pc_wiener)"""
    w = h = 8
    stride = 16
    pix, p_off, left, lpf, lo, lpb, lbo, ll, noskip = multi_data(h, stride)
    fpt = np.zeros((1, 13), np.int16)
    fpt[0][12] = 128
    multi(L, pix, p_off, stride, left, lpf, lo, lpb, lbo, w, h, None, fpt, np.zeros(256, np.uint8), noskip, ll)
    for y in range(h):
        assert (pix[p_off + y * stride:p_off + y * stride + w] == 128).all()


def test_wiener_multi_skip_mask(L):
    """looprestoration.rs:3035-3079"""
    w = h = 8
    stride = 16
    pix, p_off, left, lpf, lo, lpb, lbo, _, noskip = multi_data(h, stride)
    pix[:] = 100
    ll = np.full(((h >> 2) + 1, 4), 0xFFFF, np.uint16)
    multi(L, pix, p_off, stride, left, lpf, lo, lpb, lbo, w, h, np.full((1, 18), 127, np.int8), None,
          np.zeros(256, np.uint8), noskip, ll)
    for y in range(h):
        assert (pix[p_off + y * stride:p_off + y * stride + w] == 100).all()


def single_uv(L, pix, p_off, stride, left, lpf, lpf_bottom, w, h, filt, luma, luma_off, lstride, luma_top, lt_off,
              luma_bottom, lb_off, ss_hor, ss_ver, ds, ll):
    L.r2o_ns_wiener_single_uv(p(pix), C.c_int64(p_off), C.c_int64(stride), p(left), p(lpf), C.c_int64(4),
                              p(lpf_bottom), C.c_int64(4), w, h, p(filt), p(luma), C.c_int64(luma_off),
                              C.c_int64(lstride), p(luma_top), C.c_int64(lt_off), p(luma_bottom), C.c_int64(lb_off),
                              ss_hor, ss_ver, ds, ALL, p(ll), 8)


def _uv_case(val, h, stride, lstride, luma_rows):
    pix = np.full(stride * (h + 6), val, np.uint16)
    left = np.full((h + 4, 6), val, np.uint16)
    lpf = np.full(stride * 4 + 8, val, np.uint16)
    lpf_bottom = np.full(stride * 4 + 8, val, np.uint16)
    luma = np.full(lstride * luma_rows, val, np.uint16)
    luma_top = np.full(lstride * 4 + 8, val, np.uint16)
    luma_bottom = np.full(lstride * 4 + 8, val, np.uint16)
    return pix, left, lpf, lpf_bottom, luma, luma_top, luma_bottom


def test_ns_wiener_single_uv_identity(L):
    """looprestoration.rs:3081-3132"""
    w = h = 8
    stride, lstride = 16, 32
    p_off = stride + 4
    pix, left, lpf, lpb, luma, lt, lb = _uv_case(128, h, stride, lstride, h * 2 + 12)
    single_uv(L, pix, p_off, stride, left, lpf, lpb, w, h, np.zeros(18, np.int8), luma, 4 * lstride + 8, lstride,
              lt, 8, lb, 8, 1, 1, 2, np.zeros(((h >> 2) + 1, 4), np.uint16))
    for y in range(h):
        assert (pix[p_off + y * stride:p_off + y * stride + w] == 128).all()


def test_ns_wiener_single_uv_no_subsample(L):
    """looprestoration.rs:3134-3185"""
    w = h = 8
    stride, lstride = 16, 16
    p_off = stride + 4
    pix, left, lpf, lpb, luma, lt, lb = _uv_case(128, h, stride, lstride, h + 12)
    single_uv(L, pix, p_off, stride, left, lpf, lpb, w, h, np.zeros(18, np.int8), luma, 4 * lstride + 4, lstride,
              lt, 4, lb, 4, 0, 0, 2, np.zeros(((h >> 2) + 1, 4), np.uint16))
    for y in range(h):
        assert (pix[p_off + y * stride:p_off + y * stride + w] == 128).all()


def test_ns_wiener_single_uv_skip_mask(L):
    """looprestoration.rs:3187-3238"""
    w = h = 8
    stride, lstride = 16, 16
    p_off = stride + 4
    pix, left, lpf, lpb, luma, lt, lb = _uv_case(100, h, stride, lstride, h + 12)
    single_uv(L, pix, p_off, stride, left, lpf, lpb, w, h, np.full(18, 127, np.int8), luma, 4 * lstride + 4,
              lstride, lt, 4, lb, 4, 0, 0, 2, np.full(((h >> 2) + 1, 4), 0xFFFF, np.uint16))
    for y in range(h):
        assert (pix[p_off + y * stride:p_off + y * stride + w] == 100).all()


def test_gdf_coords(L):
    """looprestoration.rs:3240-3245"""
    assert const(L, 5, -1) == 18
    assert pair(L, 5, 0) == [6, 0] and pair(L, 5, 17) == [0, 1]


def gdf_prep(L, ref_dst_idx):
    w = h = 8
    stride = 24
    p_off = 6 * stride + 6
    pix = np.full(stride * (h + 14), 128, np.uint16)
    left = np.full((h + 8, 6), 128, np.uint16)
    lpf = np.full(stride * 8 + 8, 128, np.uint16)
    lpf_bottom = np.full(stride * 4 + 8, 128, np.uint16)
    dst = np.full(h * w, 99, np.int8)
    L.r2o_gdf_prep(p(dst), w, p(pix), C.c_int64(p_off), C.c_int64(stride), p(left), p(lpf), C.c_int64(6),
                   p(lpf_bottom), C.c_int64(6), w, h, ref_dst_idx, 0, ALL, 8)
    return dst


def test_gdf_prep_uniform(L):
    """looprestoration.rs:3247-3284 (the reference only reads every output);
    every output is written, and a flat block gives one error value (all 18
    differences and 4 gradient features are 0, so every pixel indexes the
    same error entry)."""
    dst = gdf_prep(L, 0)
    assert (dst == dst[0]).all()


def test_gdf_prep_inter(L):
    """looprestoration.rs:3286-3323 (inter table, ref_dst_idx 1); as above."""
    dst = gdf_prep(L, 1)
    assert (dst == dst[0]).all()


def test_backup_nxu_3_pixels(L):
    """looprestoration.rs:3325-3335"""
    src = np.arange(32, dtype=np.uint16)
    dst = np.zeros((4, 6), np.uint16)
    L.r2o_backup_nxu(p(dst), C.c_int64(4), p(src), C.c_int64(32), C.c_int64(5), C.c_int64(8), 4, C.c_int64(3))
    assert (dst[0][3:6] == src[2:5]).all()
    assert (dst[1][3:6] == src[10:13]).all()
    assert (dst[2][3:6] == src[18:21]).all()
    assert (dst[3][3:6] == src[26:29]).all()


def test_backup_nxu_6_pixels(L):
    """looprestoration.rs:3337-3345"""
    src = np.arange(24, dtype=np.uint16)
    dst = np.zeros((2, 6), np.uint16)
    L.r2o_backup_nxu(p(dst), C.c_int64(2), p(src), C.c_int64(24), C.c_int64(6), C.c_int64(8), 2, C.c_int64(6))
    assert list(dst[0]) == [0, 1, 2, 3, 4, 5]
    assert list(dst[1]) == [8, 9, 10, 11, 12, 13]


def test_copy_n_lines(L):
    """looprestoration.rs:3347-3353"""
    src = np.arange(30, dtype=np.uint16)
    dst = np.zeros(30, np.uint16)
    L.r2o_copy_n_lines(p(dst), C.c_int64(30), p(src), C.c_int64(30), C.c_int64(10), C.c_int64(3))
    assert (dst == src).all()


def test_copy_n_lines_single_row(L):
    """looprestoration.rs:3355-3361"""
    src = np.array([1, 2, 3, 4, 5], np.uint16)
    dst = np.zeros(5, np.uint16)
    L.r2o_copy_n_lines(p(dst), C.c_int64(5), p(src), C.c_int64(5), C.c_int64(5), C.c_int64(1))
    assert list(dst) == [1, 2, 3, 4, 5]
