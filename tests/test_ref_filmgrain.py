"""The reference's film-grain unit tests (crates/rav2d/src/filmgrain.rs
:943-1342), one test here per test there, re-asserted against the CPU
oracle's restatement (oracle/grain.cpp).  Each test names the reference test
it mirrors and its line; the inputs and the assertions are the reference's.
Templates are the reference's [[i16; 82]; 73] arrays; 8-bit samples are held
in uint16 arrays (the oracle's sample type)."""
import ctypes as C

import numpy as np
import pytest

from rav2d_b200 import abi

GW, GH, SGW, SGH = 82, 73, 44, 38


def p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def L(oracle):
    lib = oracle.lib()
    lib.r2o_get_random_number.restype = C.c_uint32
    lib.r2o_round2.restype = C.c_int
    lib.r2o_sample_lut.restype = C.c_int
    return lib


def grain_data(ar_lag, grain_scale_shift):
    """make_grain_data (filmgrain.rs:1011-1018)."""
    d = abi.FilmGrainData()
    d.ar_coeff_lag = ar_lag
    d.grain_scale_shift = grain_scale_shift
    d.ar_coeff_shift = 6
    return d


def fgy_data():
    """make_fgy_data (filmgrain.rs:1125-1133)."""
    d = abi.FilmGrainData()
    d.scaling_shift = 8
    d.block_size = 0
    d.overlap_flag = 0
    d.clip_to_restricted_range = 0
    return d


def lut():
    return np.zeros((GH, GW), np.int16)


def gen_y(L, data, seed, bd=8):
    buf = lut()
    L.r2o_generate_grain_y(p(buf), C.byref(data), C.c_uint32(seed), bd)
    return buf


def gen_uv(L, buf_y, data, seed, uv, subx, suby, bd=8):
    buf = lut()
    L.r2o_generate_grain_uv(p(buf), p(buf_y), C.byref(data), C.c_uint32(seed), uv, int(subx), int(suby), bd)
    return buf


def scaling_8(L, points):
    s = np.zeros(256, np.uint8)
    pts = np.array(points, np.uint8).reshape(-1, 2) if points else np.zeros((1, 2), np.uint8)
    L.r2o_generate_scaling(8, p(pts), len(points), p(s))
    return s


def scaling_hbd(L, points, init=0):
    s = np.full(1024, init, np.uint8)
    pts = np.array(points, np.uint8).reshape(-1, 2) if points else np.zeros((1, 2), np.uint8)
    L.r2o_generate_scaling(10, p(pts), len(points), p(s))
    return s


def fgy(L, dst, src, stride, data, seed, pw, scaling, lut_, bh, row_num=0, bd=8):
    L.r2o_fgy_32x32xn(p(dst), p(src), C.c_int64(stride), C.byref(data), C.c_uint32(seed), pw, p(scaling), p(lut_),
                      bh, row_num, bd)


def fguv(L, dst, src, stride, data, seed, pw, scaling, lut_, bh, row_num, luma, lstride, uv, is_id, sx, sy, bd=8):
    L.r2o_fguv_32x32xn(p(dst), p(src), C.c_int64(stride), C.byref(data), C.c_uint32(seed), pw, p(scaling), p(lut_),
                       bh, row_num, p(luma), C.c_int64(lstride), uv, int(is_id), sx, sy, bd)


def test_get_random_number_lfsr(L):
    """filmgrain.rs:947-953"""
    state = C.c_uint32(0xAAAA)
    v = L.r2o_get_random_number(8, C.byref(state))
    assert v < 256
    assert state.value != 0xAAAA


def test_get_random_number_sequence(L):
    """filmgrain.rs:955-963"""
    state = C.c_uint32(1)
    vals = [L.r2o_get_random_number(4, C.byref(state)) for _ in range(100)]
    assert any(v != vals[0] for v in vals)


def test_round2_basic(L):
    """filmgrain.rs:965-970"""
    assert L.r2o_round2(10, 1) == 5
    assert L.r2o_round2(11, 1) == 6
    assert L.r2o_round2(7, 2) == 2


def test_round2_negative(L):
    """filmgrain.rs:972-975"""
    assert L.r2o_round2(-10, 1) == -5


def test_generate_scaling_empty(L):
    """filmgrain.rs:977-982"""
    assert (scaling_8(L, []) == 0).all()


def test_generate_scaling_single_point(L):
    """filmgrain.rs:984-990"""
    s = scaling_8(L, [[128, 200]])
    assert (s[:128] == 200).all() and (s[128:] == 200).all()


def test_generate_scaling_two_points(L):
    """filmgrain.rs:992-999"""
    s = scaling_8(L, [[0, 0], [255, 255]])
    assert s[0] == 0
    assert s[128] > 100
    assert s[255] == 255


def test_generate_scaling_monotonic(L):
    """filmgrain.rs:1001-1008 (the reference's assertion holds for any pair:
    a <= b or b <= a); additionally the piecewise-linear segments are
    monotone between the points here."""
    s = scaling_8(L, [[0, 10], [100, 50], [200, 50]]).astype(int)
    for i in range(99):
        assert s[i] <= s[i + 1] or s[i + 1] <= s[i]
    assert (np.diff(s[:101]) >= 0).all()


def test_generate_grain_y_no_ar(L):
    """filmgrain.rs:1019-1026"""
    buf = gen_y(L, grain_data(0, 0), 1234)
    assert (buf != 0).any()


def test_generate_grain_y_bounded(L):
    """filmgrain.rs:1028-1038"""
    buf = gen_y(L, grain_data(0, 0), 5678)
    assert buf.min() >= -128 and buf.max() <= 127


def test_generate_grain_y_deterministic(L):
    """filmgrain.rs:1040-1048"""
    d = grain_data(1, 0)
    assert np.array_equal(gen_y(L, d, 42), gen_y(L, d, 42))


def test_generate_grain_y_ar_lag1(L):
    """filmgrain.rs:1050-1063"""
    d = grain_data(1, 0)
    d.ar_coeffs[0][0], d.ar_coeffs[0][1], d.ar_coeffs[0][2] = 10, -5, 3
    buf = gen_y(L, d, 999)
    assert buf.min() >= -128 and buf.max() <= 127


def test_generate_grain_uv_no_sub(L):
    """filmgrain.rs:1065-1073"""
    buf = gen_uv(L, lut(), grain_data(0, 0), 100, 0, False, False)
    assert (buf != 0).any()


def test_generate_grain_uv_with_sub(L):
    """filmgrain.rs:1075-1086"""
    buf = gen_uv(L, lut(), grain_data(0, 0), 100, 0, True, True)
    sub = buf[:SGH, :SGW]
    assert sub.min() >= -128 and sub.max() <= 127


def test_generate_grain_uv_seed_xor(L):
    """filmgrain.rs:1088-1097"""
    d = grain_data(0, 0)
    u = gen_uv(L, lut(), d, 100, 0, False, False)
    v = gen_uv(L, lut(), d, 100, 1, False, False)
    assert u[0][0] != v[0][0]


def test_generate_grain_uv_with_luma_correlation(L):
    """filmgrain.rs:1099-1114"""
    d = grain_data(1, 0)
    d.num_points[0] = 1
    d.ar_coeffs[1][0], d.ar_coeffs[1][1], d.ar_coeffs[1][2] = 5, -3, 2
    buf = gen_uv(L, np.full((GH, GW), 64, np.int16), d, 42, 0, False, False)
    assert buf.min() >= -128 and buf.max() <= 127


def test_sample_lut_basic(L):
    """filmgrain.rs:1116-1123: the reference only calls it (no assertion).
    With zero offsets sample (x 9, y 4) reads lut[3 + 2*3 + 4][3 + 2*3 + 9]
    (sample_lut, filmgrain.rs:231-246)."""
    t = lut()
    t[10][15] = 42
    t[13][18] = 5
    offs = np.zeros(8, np.int32)
    assert L.r2o_sample_lut(p(t), 32, p(offs), 0, 0, 0, 0, 9, 4) == 5


def test_fgy_32x32xn_no_overlap(L):
    """filmgrain.rs:1134-1152"""
    pw, bh = 16, 4
    src = np.full(pw * bh, 128, np.uint16)
    dst = np.zeros_like(src)
    scaling = np.zeros(256, np.uint8)
    scaling[128] = 64
    t = gen_y(L, grain_data(0, 0), 42)
    fgy(L, dst, src, pw, fgy_data(), 100, pw, scaling, t, bh)
    assert (dst != src).any()


def test_fgy_32x32xn_output_bounded(L):
    """filmgrain.rs:1154-1176"""
    pw, bh = 32, 8
    src = (np.arange(pw * bh) & 0xFF).astype(np.uint16)
    dst = np.zeros_like(src)
    scaling = np.arange(256, dtype=np.uint8)
    t = gen_y(L, grain_data(0, 0), 7777)
    fgy(L, dst, src, pw, fgy_data(), 200, pw, scaling, t, bh)
    assert (dst[1:] != dst[:-1]).any()
    assert dst.max() <= 255


def test_fgy_32x32xn_restricted_range(L):
    """filmgrain.rs:1178-1197"""
    pw, bh = 16, 4
    src = np.zeros(pw * bh, np.uint16)
    dst = np.zeros_like(src)
    scaling = np.full(256, 255, np.uint8)
    t = gen_y(L, grain_data(0, 0), 42)
    d = fgy_data()
    d.clip_to_restricted_range = 1
    fgy(L, dst, src, pw, d, 100, pw, scaling, t, bh)
    assert dst.min() >= 16 and dst.max() <= 235


def test_fgy_32x32xn_deterministic(L):
    """filmgrain.rs:1199-1219"""
    pw, bh = 16, 4
    src = np.full(pw * bh, 100, np.uint16)
    d1, d2 = np.zeros_like(src), np.zeros_like(src)
    scaling = np.full(256, 50, np.uint8)
    t = gen_y(L, grain_data(0, 0), 42)
    fgy(L, d1, src, pw, fgy_data(), 999, pw, scaling, t, bh)
    fgy(L, d2, src, pw, fgy_data(), 999, pw, scaling, t, bh)
    assert np.array_equal(d1, d2)


def test_fgy_32x32xn_zero_scaling(L):
    """filmgrain.rs:1221-1235"""
    pw, bh = 16, 4
    src = np.full(pw * bh, 128, np.uint16)
    dst = np.zeros_like(src)
    fgy(L, dst, src, pw, fgy_data(), 100, pw, np.zeros(256, np.uint8), np.full((GH, GW), 50, np.int16), bh)
    assert (dst == 128).all()


def test_fguv_32x32xn_basic(L):
    """filmgrain.rs:1237-1275"""
    pw, bh = 16, 4
    src = np.full(pw * bh, 128, np.uint16)
    dst = np.zeros_like(src)
    luma = np.full(pw * 2 * bh * 2, 128, np.uint16)
    scaling = np.zeros(256, np.uint8)
    scaling[128] = 64
    t = gen_y(L, grain_data(0, 0), 42)
    d = fgy_data()
    d.uv_mult[0] = d.uv_mult[1] = 0
    d.uv_luma_mult[0] = d.uv_luma_mult[1] = 64
    d.uv_offset[0] = d.uv_offset[1] = 0
    fguv(L, dst, src, pw, d, 100, pw, scaling, t, bh, 0, luma, pw * 2, 0, False, 1, 1)
    assert (dst != src).any()


def test_fguv_32x32xn_chroma_from_luma(L):
    """filmgrain.rs:1277-1296 (4:4:4 addressing, identity matrix)"""
    pw, bh = 16, 4
    src = np.full(pw * bh, 128, np.uint16)
    dst = np.zeros_like(src)
    luma = np.full(pw * bh, 200, np.uint16)
    scaling = np.zeros(256, np.uint8)
    scaling[200] = 100
    d = fgy_data()
    d.chroma_scaling_from_luma = 1
    fguv(L, dst, src, pw, d, 100, pw, scaling, np.full((GH, GW), 50, np.int16), bh, 0, luma, pw, 0, True, 0, 0)
    assert (dst != src).any()


def test_generate_scaling_hbd_empty(L):
    """filmgrain.rs:1298-1303"""
    assert (scaling_hbd(L, [], init=0xFF) == 0).all()


def test_generate_scaling_hbd_single_point(L):
    """filmgrain.rs:1305-1313"""
    s = scaling_hbd(L, [[128, 200]])
    assert s[0] == 200 and s[511] == 200 and s[512] == 200 and s[1023] == 200


def test_generate_scaling_hbd_two_points(L):
    """filmgrain.rs:1315-1322"""
    s = scaling_hbd(L, [[0, 0], [255, 255]])
    assert s[0] == 0 and s[1023] == 255
    assert 120 < s[512] < 140


def test_generate_scaling_hbd_monotonic(L):
    """filmgrain.rs:1324-1331"""
    s = scaling_hbd(L, [[0, 0], [100, 100]]).astype(int)
    for i in range(1, 400):
        assert s[i] >= s[i - 1], i


def test_generate_scaling_hbd_interpolation_fills_gaps(L):
    """filmgrain.rs:1333-1341"""
    s = scaling_hbd(L, [[0, 10], [128, 200]])
    assert s[1] > 0 and s[2] > 0 and s[3] > 0
