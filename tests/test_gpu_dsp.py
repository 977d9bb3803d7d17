"""DSP-context slot entry points (r2g_dsp_*) against the oracle.

Each slot runs one block on the GPU with the reference function's argument
meaning (neighbour rows and columns, edge flags, strides in samples); the
oracle runs the reference's restatement of the same function on the same
buffers.  Random blocks over both bit depths, every edge combination and the
strength / direction / class ranges; tolerance 0 (integer arithmetic)."""
import ctypes as C

import numpy as np
import pytest

from rav2d_b200 import synth

pytestmark = pytest.mark.gpu


def p(a):
    return C.c_void_p(a.ctypes.data)


@pytest.fixture(scope="module")
def L():
    from rav2d_b200 import gpu

    return gpu.lib()


def _st(a, bd):
    return a.astype(np.uint16 if bd > 8 else np.uint8)


@pytest.mark.parametrize("bd", [8, 10])
def test_cdef_dir(L, oracle, bd):
    rng = np.random.default_rng(bd)
    for _ in range(64):
        img = rng.integers(0, 1 << bd, (8, 12)).astype(np.uint16)
        img[:, :8] = np.clip(img[:, :8] // (1 + rng.integers(0, 8)) + rng.integers(0, 64), 0, (1 << bd) - 1)
        v0, v1 = C.c_uint32(), C.c_uint32()
        want = oracle.lib().r2o_cdef_find_dir(p(img), C.c_int64(12), C.byref(v0), bd)
        g = _st(img, bd)
        got = L.r2g_dsp_cdef_dir(p(g), 12, C.byref(v1), bd)
        assert (got, v1.value) == (want, v0.value)


@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("wh", [(8, 8), (4, 8), (4, 4)])
def test_cdef_filter(L, oracle, bd, wh):
    w, h = wh
    rng = np.random.default_rng(100 * bd + w + h)
    S = 20
    for it in range(48):
        plane = rng.integers(0, 1 << bd, (S, S)).astype(np.uint16)
        plane = np.clip(plane // 3 + (1 << (bd - 2)), 0, (1 << bd) - 1).astype(np.uint16)
        left = np.ascontiguousarray(plane[8:8 + h, 6:8])
        edges = int(it % 16)
        pri = int(rng.integers(0, 16)) << (bd - 8)
        sec = int(rng.choice([0, 1, 2, 4])) << (bd - 8)
        if pri == 0 and sec == 0:  # the reference filters only blocks with some strength
            sec = 1 << (bd - 8)
        dr, damping = int(rng.integers(0, 8)), int(rng.integers(3, 7)) + bd - 8
        ref = plane.copy().ravel()
        oracle.lib().r2o_cdef_filter_block(p(ref), C.c_int64(S), C.c_int64(8 * S + 8), p(left), p(ref),
                                           C.c_int64(6 * S + 8), p(ref), C.c_int64((8 + h) * S + 8), pri, sec, dr,
                                           damping, w, h, edges, bd)
        got = _st(plane, bd).copy()
        gl = _st(left, bd).copy()
        base = got.ctypes.data
        es = got.itemsize
        rc = L.r2g_dsp_cdef_filter(C.c_void_p(base + (8 * S + 8) * es), C.c_int64(S), p(gl),
                                   C.c_void_p(base + (6 * S + 8) * es), C.c_void_p(base + ((8 + h) * S + 8) * es),
                                   pri, sec, dr, damping, w, h, edges, bd)
        assert rc == 0
        assert np.array_equal(got.astype(np.uint16).ravel(), ref), (edges, pri, sec, dr, damping)


@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("ss", [(0, 0), (1, 1)])
def test_ccso_prep(L, oracle, bd, ss):
    rng = np.random.default_rng(7 * bd + ss[0])
    w, h = (32, 4) if ss[0] else (64, 8)
    W, H = w << ss[0], h << ss[1]
    S = W + 8
    for it in range(24):
        plane = rng.integers(0, 1 << bd, (H + 8, S)).astype(np.uint16)
        left = np.ascontiguousarray(plane[4:4 + H, 2:4])
        edges, ext = int(it % 16), int(rng.integers(0, 7))
        mbl = int(rng.integers(0, 4))
        q, clf, bo = int(rng.choice([2, 4, 8, 16])) << (bd - 8), int(rng.integers(0, 2)), int(it % 5 == 0)
        want = np.zeros(w * h, np.uint8)
        flat = plane.ravel()
        oracle.lib().r2o_ccso_prep(p(want), w, p(flat), C.c_int64(S), C.c_int64(4 * S + 4), p(left), p(flat),
                                   C.c_int64(2 * S + 4), p(flat), C.c_int64((4 + H) * S + 4), mbl, ext, q, clf, bo,
                                   edges, w, h, ss[0], ss[1], bd)
        g = _st(plane, bd)
        gl = _st(left, bd)
        es, base = g.itemsize, g.ctypes.data
        got = np.zeros(w * h, np.uint8)
        rc = L.r2g_dsp_ccso_prep(p(got), C.c_int64(w), C.c_void_p(base + (4 * S + 4) * es), C.c_int64(S), p(gl),
                                 C.c_void_p(base + (2 * S + 4) * es), C.c_void_p(base + ((4 + H) * S + 4) * es),
                                 mbl, ext, q, clf, bo, edges, w, h, ss[0], ss[1], bd)
        assert rc == 0
        assert np.array_equal(got, want), (edges, ext, mbl, q, clf, bo)


@pytest.mark.parametrize("bd", [8, 10])
def test_ccso_add_and_gdf_add(L, oracle, bd):
    rng = np.random.default_rng(11 * bd)
    w, h = 64, 16
    for _ in range(8):
        base = rng.integers(0, 1 << bd, (h, w)).astype(np.uint16)
        idx = rng.integers(0, 256, (h, w)).astype(np.uint8)
        offs = rng.integers(0, 256, 64).astype(np.uint8)
        lut = rng.integers(-15, 16, 8).astype(np.int8)
        ll = rng.integers(0, 1 << 16, (h // 4, 4)).astype(np.uint16) & rng.integers(0, 1 << 16, (h // 4, 4)).astype(
            np.uint16)
        want = base.copy()
        oracle.lib().r2o_ccso_add(p(want), C.c_int64(w), p(idx), w, p(offs), p(lut), w, h, p(ll), bd)
        got = _st(base, bd).copy()
        assert L.r2g_dsp_ccso_add(p(got), C.c_int64(w), p(idx), C.c_int64(w), p(offs), p(lut), w, h, p(ll), bd) == 0
        assert np.array_equal(got.astype(np.uint16), want)
        err = rng.integers(-128, 128, (h, w)).astype(np.int8)
        scale = int(rng.integers(1, 5))
        want = base.copy()
        oracle.lib().r2o_gdf_add(p(want), C.c_int64(w), p(err), w, w, h, scale, p(ll), bd)
        got = _st(base, bd).copy()
        assert L.r2g_dsp_gdf_add(p(got), C.c_int64(w), p(err), C.c_int64(w), w, h, scale, p(ll), bd) == 0
        assert np.array_equal(got.astype(np.uint16), want)


@pytest.mark.parametrize("bd", [8, 10])
def test_generate_grain(L, oracle, bd):
    for seed in range(3):
        sf = synth.make_frame(64, 64, bd, 0xD5A0 + seed, chain="db", grain=True)
        want = [np.zeros((73, 82), np.int16) for _ in range(3)]
        sc = [np.zeros(1 << bd, np.uint8) for _ in range(3)]
        # chroma templates whatever the scaling points: force them in the oracle call
        fgd = sf.fgd
        fgd.chroma_scaling_from_luma = 1
        oracle.lib().r2o_prep_grain(C.byref(fgd), C.c_uint32(sf.grain_seed), bd, p(want[0]), p(want[1]), p(want[2]),
                                    p(sc[0]), p(sc[1]), p(sc[2]))
        got = [np.zeros((73, 82), np.int16) for _ in range(3)]
        assert L.r2g_dsp_generate_grain(p(got[0]), p(got[1]), p(got[2]), C.byref(fgd), sf.grain_seed, bd) == 0
        for pl in range(3):
            assert np.array_equal(got[pl], want[pl]), pl
