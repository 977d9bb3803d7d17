"""The reference's CCSO unit tests (crates/rav2d/src/ccso.rs:255-407), one
test here per test there, re-asserted against the CPU oracle's restatement
(oracle/cdef.cpp: ccso_score, ccso_prep, ccso_add).  The reference's 8-bit
entry points are the oracle's functions at bit depth 8 on uint16 samples."""
import ctypes as C

import numpy as np
import pytest

ALL = 1 | 2 | 4 | 8


def p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def L(oracle):
    lib = oracle.lib()
    lib.r2o_ccso_pos.restype = C.c_int
    lib.r2o_ccso_pos_len.restype = C.c_int
    return lib


def prep(L, bo_only):
    src = np.full(16 * 16, 128, np.uint16)
    left = np.full(32, 128, np.uint16)
    top = np.full(32, 128, np.uint16)
    bottom = np.full(32, 128, np.uint16)
    dst = np.zeros(64, np.uint8)
    # ccso_prep_8bpc(dst, 8, src, 16, 0, left, top, 2, bottom, 2, max_band_log2 4, ext_filter 0,
    #                quant_step 10, edge_clf 0, bo_only, edges, 8, 8, 0, 0)
    L.r2o_ccso_prep(p(dst), 8, p(src), C.c_int64(16), C.c_int64(0), p(left), p(top), C.c_int64(2), p(bottom),
                    C.c_int64(2), 4, 0, 10, 0, int(bo_only), ALL, 8, 8, 0, 0, 8)
    return dst


def add(L, dst, idx, offset_idxs, lut, ll_mask):
    L.r2o_ccso_add(p(dst), C.c_int64(4), p(idx), 4, p(offset_idxs), p(lut), 4, 4, p(ll_mask), 8)


def test_ccso_pos_table(L):
    """ccso.rs:259-264"""
    assert (L.r2o_ccso_pos(0, 0), L.r2o_ccso_pos(0, 1)) == (-1, 0)
    assert (L.r2o_ccso_pos(6, 0), L.r2o_ccso_pos(6, 1)) == (0, 2)
    assert L.r2o_ccso_pos_len() == 7


def test_ccso_score_large_positive(L):
    """ccso.rs:266-269"""
    assert L.r2o_ccso_score(20, 10, 0) == 2


def test_ccso_score_large_positive_with_edge(L):
    """ccso.rs:271-274"""
    assert L.r2o_ccso_score(20, 10, 1) == 1


def test_ccso_score_large_negative(L):
    """ccso.rs:276-279"""
    assert L.r2o_ccso_score(-20, 10, 0) == 0


def test_ccso_score_within_range(L):
    """ccso.rs:281-285"""
    assert L.r2o_ccso_score(5, 10, 0) == 1
    assert L.r2o_ccso_score(-5, 10, 0) == 1


def test_ccso_prep_bo_only(L):
    """ccso.rs:287-320"""
    assert (prep(L, True) == 128 >> (8 - 4)).all()


def test_ccso_prep_full(L):
    """ccso.rs:322-355"""
    assert ((prep(L, False) & 0x1F) == 8).all()


def test_ccso_add_basic(L):
    """ccso.rs:357-376"""
    dst = np.full(16, 128, np.uint16)
    add(L, dst, np.zeros(16, np.uint8), np.full(8, 0x21, np.uint8),
        np.array([0, 5, -5, 10, -10, 15, -15, 20], np.int8), np.zeros(4, np.uint16))
    assert dst[0] == 133


def test_ccso_add_skip_mask(L):
    """ccso.rs:378-397"""
    dst = np.full(16, 128, np.uint16)
    add(L, dst, np.zeros(16, np.uint8), np.zeros(8, np.uint8), np.full(8, 10, np.int8),
        np.full(4, 0xFFFF, np.uint16))
    assert (dst == 128).all()


def test_ccso_score_boundary(L):
    """ccso.rs:399-405"""
    assert [L.r2o_ccso_score(d, 10, 0) for d in (10, -10, 11, -11)] == [1, 1, 2, 0]
