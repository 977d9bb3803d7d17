"""Byte-exact parity of the CUDA filter path against the CPU oracle.

Every test runs the same seeded synthetic frame through the oracle (the
reference's per-superblock-row sequencing) and through the C ABI of
librav2d_gpu.so, and compares every output plane sample for sample."""
import numpy as np
import pytest

from rav2d_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from rav2d_b200 import gpu

    c = gpu.Context(0)
    yield c
    c.close()


def _cmp(name, got, want, sf):
    for pl, (g, w) in enumerate(zip(got, want)):
        hh = sf.height >> (pl > 0)
        ww = sf.width >> (pl > 0)
        g, w = g[:hh, :ww], w[:hh, :ww]
        if not np.array_equal(g, w):
            ys, xs = np.nonzero(g != w)
            raise AssertionError(f"{name}: plane {pl}: {len(ys)} samples differ, first at (y={ys[0]}, x={xs[0]}) "
                                 f"gpu={g[ys[0], xs[0]]} ref={w[ys[0], xs[0]]}")


def _run(ctx, oracle, sf, inloop=None, grain=False):
    from rav2d_b200 import gpu

    if inloop is not None:
        sf.inloop = inloop
    want = oracle.filter_frame(sf)
    got = gpu.filter_frame(ctx, sf, grain=grain)
    if grain:
        got, gg = got
        _cmp("grain", gg, oracle.apply_grain(sf, want), sf)
    _cmp("filter", got, want, sf)


CASES = [
    # (w, h, bitdepth, chain, seed)
    (64, 64, 8, "db", 1),
    (352, 288, 8, "db_cdef", 0x5EED0000),  # the CPU-runnable plain-method case
    (352, 288, 10, "db_cdef", 2),
    (72, 40, 8, "full", 3),
    (128, 128, 10, "full", 4),  # height multiple of 64: two LR stripes in the last row
    (640, 360, 8, "full", 5),
    (640, 360, 10, "full", 6),
    (1280, 720, 10, "full", 7),
    (1920, 1080, 10, "full", 0x5EED0001),  # the per-frame 1080p 10-bit case
]


@pytest.mark.parametrize("w,h,bd,chain,seed", CASES)
def test_parity_frames(ctx, oracle, w, h, bd, chain, seed):
    _run(ctx, oracle, synth.make_frame(w, h, bd, seed, chain=chain, pad_fill=True))


@pytest.mark.parametrize("bit", [abi.INLOOP_DEBLOCK, abi.INLOOP_CDEF, abi.INLOOP_CCSO, abi.INLOOP_WIENER,
                                 abi.INLOOP_GDF])
@pytest.mark.parametrize("bd", [8, 10])
def test_parity_per_filter(ctx, oracle, bit, bd):
    """One filter bit at a time (the reference's per-filter sweep)."""
    sf = synth.make_frame(320, 192, bd, 100 + bit, chain="full")
    _run(ctx, oracle, sf, inloop=bit)


@pytest.mark.parametrize("ns_multi", [1, 3, 5, 7])
def test_parity_ns_multiclass(ctx, oracle, ns_multi):
    sf = synth.make_frame(256, 192, 10, 200 + ns_multi, chain="full", ns_multi=ns_multi, luma_types=(2,))
    _run(ctx, oracle, sf)


@pytest.mark.parametrize("cfl", [0, 1, 2])
def test_parity_cfl_downsample(ctx, oracle, cfl):
    sf = synth.make_frame(192, 128, 8, 300 + cfl, chain="full", cfl_ds=cfl)
    _run(ctx, oracle, sf)


@pytest.mark.parametrize("bd", [8, 10])
def test_parity_lossless(ctx, oracle, bd):
    sf = synth.make_frame(256, 128, bd, 400 + bd, chain="full", lossless=True)
    _run(ctx, oracle, sf)


@pytest.mark.parametrize("inter", [False, True])
def test_parity_gdf_ref_dst(ctx, oracle, inter):
    sf = synth.make_frame(256, 136, 10, 500 + inter, chain="full", luma_types=(3,), inter=inter)
    _run(ctx, oracle, sf)


@pytest.mark.parametrize("w,h,bd,seed", [(640, 360, 8, 11), (640, 360, 10, 12), (3840, 2160, 10, 0x5EED0002)])
def test_parity_film_grain(ctx, oracle, w, h, bd, seed):
    sf = synth.make_frame(w, h, bd, seed, chain="full", grain=True)
    _run(ctx, oracle, sf, grain=True)


def test_parity_film_grain_variants(ctx, oracle):
    """Independent chroma points, no overlap, 16x16 blocks, restricted range."""
    rng = np.random.default_rng(7)
    for k in range(4):
        sf = synth.make_frame(320, 176, 8 if k % 2 else 10, 600 + k, chain="db", grain=True)
        g = sf.fgd
        g.overlap_flag = k & 1
        g.block_size = (k >> 1) & 1
        g.clip_to_restricted_range = 1
        if k >= 2:
            g.chroma_scaling_from_luma = 0
            for pl in (1, 2):
                g.num_points[pl] = 4
                xs = np.sort(rng.choice(256, 4, replace=False))
                for i in range(4):
                    g.points[pl][i][0] = int(xs[i])
                    g.points[pl][i][1] = int(rng.integers(0, 256))
                g.uv_mult[pl - 1] = int(rng.integers(-128, 128))
                g.uv_luma_mult[pl - 1] = int(rng.integers(-128, 128))
                g.uv_offset[pl - 1] = int(rng.integers(-256, 256))
        _run(ctx, oracle, sf, grain=True)


def _tile_rows(sf, starts_sb):
    import ctypes as C

    fp = abi.FrameParams()
    C.memmove(C.byref(fp), C.byref(sf.fp), C.sizeof(fp))
    fp.tile_rows = len(starts_sb) - 1
    for i, v in enumerate(starts_sb):
        fp.tile_row_start_sb[i] = v
    sf.fp = fp
    return sf


TILE_ROW_CASES = [
    # (w, h, bitdepth, tile row starts in superblock rows, seed)
    (256, 320, 8, [0, 2, 5], 61),
    (256, 320, 10, [0, 1, 3, 5], 62),
    (640, 384, 10, [0, 3, 5, 6], 63),     # the last tile row is the last superblock row (two stripes)
    (1920, 1080, 8, [0, 5, 11, 16, 17], 64),  # a tile row of one short superblock row at the bottom
    (1920, 1080, 10, [0, 6, 12, 17], 65),
]


@pytest.mark.parametrize("w,h,bd,starts,seed", TILE_ROW_CASES)
def test_parity_tile_rows(ctx, oracle, w, h, bd, starts, seed):
    """Loop restoration over several tile rows: the split superblock row at
    each tile row's top (looprestoration.rs:2401-2548) with its integrated
    stripe edges, NS / PC / multi-class Wiener and GDF units."""
    sf = _tile_rows(synth.make_frame(w, h, bd, seed, ns_multi=3 if bd == 10 else 0), starts)
    _run(ctx, oracle, sf)
