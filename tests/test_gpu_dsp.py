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


# ---- typed loop-restoration slots (WienerFilterFn / GdfPrepFn) ----
# One plane holds the block (at row R0, column C0), its right-hand context and
# the saved rows above / below (rows R0-2, R0-1 and R0+h, R0+h+1 stand in for
# the deblocked lines); `left` is a separate [h][6] array.  The oracle runs
# the reference's function on the same buffers (in place on a copy).
R0, C0, S = 12, 16, 112


def _plane(rng, bd, rows=112, cols=S):
    yy, xx = np.mgrid[0:rows, 0:cols]
    base = ((1 << bd) // 2 + ((1 << bd) // 5) * np.sin(xx / 7.0 + yy / 11.0)).astype(np.int64)
    return np.clip(base + rng.integers(-(1 << bd) // 16, (1 << bd) // 16 + 1, (rows, cols)), 0,
                   (1 << bd) - 1).astype(np.uint16)


def _ptr(a, off):
    return C.c_void_p(a.ctypes.data + off * a.itemsize)


def _ll(rng, h, p_ll):
    return ((rng.random((h // 4 + 1, 4)) < p_ll) * rng.integers(0, 1 << 16, (h // 4 + 1, 4))).astype(np.uint16)


@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("kind", ["single", "multi", "pc"])
def test_wiener_y_slots(L, oracle, bd, kind):
    """ns_wiener_single_y / ns_wiener_multi / pc_wiener (looprestoration.rs
    :524-1143) through r2g_dsp_ns_wiener_single_y / _multi / r2g_dsp_pc_wiener."""
    from rav2d_b200 import abi

    rng = np.random.default_rng(31 * bd + len(kind))
    for it in range(40):
        w = int(rng.choice([8, 16, 32, 60, 64]))
        h = int(rng.choice([4, 8, 12, 32, 56, 64]))
        edges = it % 16
        plane = _plane(rng, bd)
        left = rng.integers(0, 1 << bd, (h, 6)).astype(np.uint16)
        ll = _ll(rng, h, 0.2)
        ref = plane.copy().ravel()
        fu = rng.integers(-8, 8, (16, 18)).astype(np.int8)
        fpt = rng.integers(-40, 40, (64, 13)).astype(np.int16)
        fpt[:, 12] += 128
        lut = rng.integers(0, 16 if kind == "multi" else 64, 256).astype(np.uint8)
        noskip = rng.integers(0, 1 << 16, h // 4 + 1).astype(np.uint16)
        base_q = int(rng.integers(4, 1200))
        single = fu[0, :16].copy()
        o = R0 * S + C0
        if kind == "single":
            oracle.lib().r2o_ns_wiener_single_y(p(ref), C.c_int64(o), C.c_int64(S), p(left), p(ref),
                                                C.c_int64(o - 2 * S), p(ref), C.c_int64(o + h * S), w, h, p(single),
                                                edges, p(ll), bd)
        else:
            oracle.lib().r2o_wiener_multi(p(ref), C.c_int64(o), C.c_int64(S), p(left), p(ref), C.c_int64(o - 2 * S),
                                          p(ref), C.c_int64(o + h * S), w, h, p(fu) if kind == "multi" else None,
                                          p(fpt) if kind == "pc" else None, p(lut), p(noskip), base_q, edges, p(ll),
                                          bd)
        got = _st(plane, bd).copy().ravel()
        gl = _st(left, bd)
        prm = abi.WienerParams()
        if kind == "single":
            prm.single.filter = single.ctypes.data
            fn = L.r2g_dsp_ns_wiener_single_y
        else:
            prm.multi.filters = (fu if kind == "multi" else fpt).ctypes.data
            prm.multi.subclass_lut = lut.ctypes.data
            prm.multi.noskip_mask = noskip.ctypes.data
            prm.multi.base_q = base_q
            fn = L.r2g_dsp_ns_wiener_multi if kind == "multi" else L.r2g_dsp_pc_wiener
        rc = fn(_ptr(got, o), S, p(gl), _ptr(got, o - 2 * S), _ptr(got, o + h * S), w, h, C.byref(prm), edges,
                p(ll), bd)
        assert rc == 0
        assert np.array_equal(got.astype(np.uint16), ref), (kind, w, h, edges)


@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("ds", [0, 1, 2])
def test_wiener_uv_slot(L, oracle, bd, ds):
    """ns_wiener_single_uv (looprestoration.rs:1145-1430) through
    r2g_dsp_ns_wiener_single_uv, 4:2:0 with each CfL downsample filter."""
    from rav2d_b200 import abi

    rng = np.random.default_rng(17 * bd + ds)
    LS = 200
    for it in range(32):
        w = int(rng.choice([8, 16, 28, 32, 64]))
        h = int(rng.choice([2, 4, 8, 16, 28, 32]))
        edges = it % 16
        plane = _plane(rng, bd)
        luma = _plane(rng, bd, rows=180, cols=LS)
        left = rng.integers(0, 1 << bd, (h, 6)).astype(np.uint16)
        ll = _ll(rng, h, 0.15)
        f = np.concatenate([rng.integers(-16, 16, 6), rng.integers(-8, 8, 12)]).astype(np.int8)
        o = R0 * S + C0
        lo, lto, lbo = 24 * LS + 16, 8 * LS + 16, (24 + 2 * h + 8) * LS + 16
        ref = plane.copy().ravel()
        lref = luma.ravel()
        oracle.lib().r2o_ns_wiener_single_uv(p(ref), C.c_int64(o), C.c_int64(S), p(left), p(ref), C.c_int64(o - 2 * S),
                                             p(ref), C.c_int64(o + h * S), w, h, p(f), p(lref), C.c_int64(lo),
                                             C.c_int64(LS), p(lref), C.c_int64(lto), p(lref), C.c_int64(lbo), 1, 1, ds,
                                             edges, p(ll), bd)
        got = _st(plane, bd).copy().ravel()
        gluma = _st(luma, bd).ravel()
        prm = abi.WienerParams()
        sp = prm.single
        sp.filter = f.ctypes.data
        sp.luma, sp.luma_top, sp.luma_bottom = (gluma.ctypes.data + k * gluma.itemsize for k in (lo, lto, lbo))
        sp.stride, sp.ss_ver, sp.ss_hor, sp.ds_flt = LS, 1, 1, ds
        gleft = _st(left, bd)  # kept alive across the call
        rc = L.r2g_dsp_ns_wiener_single_uv(_ptr(got, o), S, p(gleft), _ptr(got, o - 2 * S),
                                           _ptr(got, o + h * S), w, h, C.byref(prm), edges, p(ll), bd)
        assert rc == 0
        assert np.array_equal(got.astype(np.uint16), ref), (w, h, edges)


@pytest.mark.parametrize("bd", [8, 10])
def test_gdf_prep_slot(L, oracle, bd):
    """gdf_prep (looprestoration.rs:1432-1640) through r2g_dsp_gdf_prep, intra
    and inter tables."""
    rng = np.random.default_rng(53 * bd)
    for it in range(40):
        w = int(rng.choice([8, 16, 32, 62, 64]))
        h = int(rng.choice([6, 8, 16, 32, 56, 64]))
        edges = it % 16
        rd, qp = int(rng.integers(0, 6)), int(rng.integers(0, 6))
        plane = _plane(rng, bd)
        left = rng.integers(0, 1 << bd, (h, 6)).astype(np.uint16)
        o = R0 * S + C0
        want = np.zeros((h, w), np.int8)
        oracle.lib().r2o_gdf_prep(p(want), w, p(plane), C.c_int64(o), C.c_int64(S), p(left), p(plane),
                                  C.c_int64(o - 2 * S), p(plane), C.c_int64(o + h * S), w, h, rd, qp, edges, bd)
        got = np.full((h, w), 99, np.int8)
        g = _st(plane, bd).ravel()
        gleft = _st(left, bd)  # kept alive across the call
        rc = L.r2g_dsp_gdf_prep(p(got), w, _ptr(g, o), S, p(gleft), _ptr(g, o - 2 * S), _ptr(g, o + h * S),
                                w, h, rd, qp, edges, bd)
        assert rc == 0
        assert np.array_equal(got, want), (w, h, edges, rd, qp)


def test_lr_slots_reject_bad_arguments(L):
    from rav2d_b200 import abi

    buf = np.zeros(64 * 64, np.uint8)
    prm = abi.WienerParams()
    f = np.zeros(18, np.int8)
    prm.single.filter = f.ctypes.data
    ll = np.zeros((17, 4), np.uint16)
    for w, h, edges in ((6, 8, 0), (68, 8, 0), (8, 66, 0), (8, 8, 16), (8, 8, 32)):
        assert L.r2g_dsp_ns_wiener_single_y(p(buf), 64, None, None, None, w, h, C.byref(prm), edges, p(ll),
                                            8) == abi.R2G_E_INVALID
    assert L.r2g_dsp_ns_wiener_single_y(p(buf), 64, None, None, None, 8, 8, C.byref(prm), 1, p(ll),
                                        8) == abi.R2G_E_INVALID  # left context without `left`
    e = np.zeros(64, np.int8)
    assert L.r2g_dsp_gdf_prep(p(e), 8, p(buf), 64, None, None, None, 8, 4, 0, 0, 0, 8) == abi.R2G_E_INVALID
    assert L.r2g_dsp_gdf_prep(p(e), 8, p(buf), 64, None, None, None, 8, 8, 6, 0, 0, 8) == abi.R2G_E_INVALID


# ---- DeblockDSPContext.deblock_sb and FilmGrainDSPContext.fgy / fguv ----
@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("luma", [1, 0])
@pytest.mark.parametrize("vert", [1, 0])
def test_deblock_sb64_slot(L, oracle, bd, luma, vert):
    """deblock_{h,v}_sb64{y,uv}_bd (deblock.rs:303-548) on one 64-long edge:
    random class / lossless bits, thresholds and the `edge` clamp; a plane
    with a step across the edge so the filters engage."""
    rng = np.random.default_rng(1000 * bd + 10 * luma + vert)
    lib = oracle.lib()
    for it in range(24):
        plane = _plane(rng, bd, rows=80, cols=80)
        step = rng.integers(-(1 << bd) // 8, (1 << bd) // 8 + 1)
        if vert:
            plane[:, 40:] = np.clip(plane[:, 40:].astype(np.int64) + step, 0, (1 << bd) - 1)
        else:
            plane[40:, :] = np.clip(plane[40:, :].astype(np.int64) + step, 0, (1 << bd) - 1)
        off = (8 * 80 + 40) if vert else (40 * 80 + 8)
        vmask = (rng.integers(0, 1 << 16, 4) * (rng.random(4) < 0.6)).astype(np.uint16)
        if not luma:
            vmask[3] = 0
        ll = (rng.integers(0, 1 << 16, 2) * (rng.random(2) < 0.3)).astype(np.uint16)
        q = rng.integers(0, 1 << (bd - 2), 16).astype(np.uint16)
        sthr = rng.integers(0, 1 << bd, 16).astype(np.uint16)
        edge = int(it & 1)
        want = plane.copy()
        lib.r2o_deblock_sb64(p(want), C.c_int64(off), C.c_int64(80), p(vmask), p(ll), p(q), p(sthr), edge, luma,
                             vert, bd)
        got = _st(plane, bd)
        assert L.r2g_dsp_deblock_sb64(_ptr(got, off), 80, p(vmask), p(ll), p(q), p(sthr), edge, luma, vert, bd) == 0
        assert np.array_equal(got.astype(np.uint16), want), it


@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("chroma", [0, 1])
def test_film_grain_band_slots(L, oracle, bd, chroma):
    """fgy_32x32xn / fguv_32x32xn (filmgrain.rs:248-598) on one row band:
    band 0 and later bands (vertical overlap), with and without overlap,
    restricted range, chroma from luma or with its own multipliers."""
    lib = oracle.lib()
    lib.r2o_fgy_32x32xn.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_int, C.c_int, C.c_int]
    lib.r2o_fguv_32x32xn.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64] + [C.c_int] * 5
    rng = np.random.default_rng(77 + bd + 3 * chroma)
    for it in range(12):
        fgd, seed = synth.make_film_grain(rng)
        fgd.overlap_flag = int(it % 3 != 2)
        fgd.chroma_scaling_from_luma = int(it % 2)
        fgd.uv_mult[0], fgd.uv_mult[1] = (int(v) for v in rng.integers(-128, 128, 2))
        fgd.uv_luma_mult[0], fgd.uv_luma_mult[1] = (int(v) for v in rng.integers(-128, 128, 2))
        fgd.uv_offset[0], fgd.uv_offset[1] = (int(v) for v in rng.integers(-256, 256, 2))
        lut = rng.integers(-(128 << (bd - 8)), 128 << (bd - 8), (73, 82)).astype(np.int16)
        scaling = rng.integers(0, 256, 1 << bd).astype(np.uint8)
        row_num = int(it % 4)
        sx = sy = chroma
        pw = int(rng.integers(1, 9)) * (32 >> sx) - int(rng.integers(0, 5))
        bh = (32 >> sy) - int(rng.integers(0, 3))
        stride = pw + 7
        src = rng.integers(0, 1 << bd, (bh, stride)).astype(np.uint16)
        luma = rng.integers(0, 1 << bd, (bh << sy, (stride << sx) + 2)).astype(np.uint16)
        want = np.zeros_like(src)
        got = _st(np.zeros_like(src), bd)
        gsrc, gluma = _st(src, bd), _st(luma, bd)  # kept alive across the calls
        if chroma:
            uv, is_id = int(it & 1), int((it >> 1) & 1)
            lib.r2o_fguv_32x32xn(p(want), p(src), stride, C.byref(fgd), seed, pw, p(scaling), p(lut), bh, row_num,
                                 p(luma), luma.shape[1], uv, is_id, sx, sy, bd)
            rc = L.r2g_dsp_fguv_32x32xn(p(got), p(gsrc), stride, C.byref(fgd), seed, pw, p(scaling), p(lut),
                                        bh, row_num, p(gluma), luma.shape[1], uv, is_id, sx, sy, bd)
        else:
            lib.r2o_fgy_32x32xn(p(want), p(src), stride, C.byref(fgd), seed, pw, p(scaling), p(lut), bh, row_num, bd)
            rc = L.r2g_dsp_fgy_32x32xn(p(got), p(gsrc), stride, C.byref(fgd), seed, pw, p(scaling), p(lut),
                                       bh, row_num, bd)
        assert rc == 0
        assert np.array_equal(got[:, :pw].astype(np.uint16), want[:, :pw]), it


def test_band_slots_reject_bad_arguments(L):
    fgd, seed = synth.make_film_grain(np.random.default_rng(5))
    src = np.full((32, 64), 2000, np.uint16)
    dst = np.zeros_like(src)
    lut = np.zeros((73, 82), np.int16)
    sc = np.zeros(1024, np.uint8)
    assert L.r2g_dsp_fgy_32x32xn(p(dst), p(src), 64, C.byref(fgd), seed, 64, p(sc), p(lut), 32, 0, 10) != 0  # > 1023
    src[:] = 600
    assert L.r2g_dsp_fgy_32x32xn(p(dst), p(src), 64, C.byref(fgd), seed, 64, p(sc), p(lut), 40, 0, 10) != 0  # bh
    assert L.r2g_dsp_fgy_32x32xn(p(dst), p(src), 64, C.byref(fgd), 1 << 16, 64, p(sc), p(lut), 32, 0, 10) != 0
    vm = np.zeros(4, np.uint16)
    assert L.r2g_dsp_deblock_sb64(None, 64, p(vm), p(vm), p(vm), p(vm), 0, 1, 1, 10) != 0
