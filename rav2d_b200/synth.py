"""Seeded synthetic reconstructed frames and filter side-info.

The reference is quoted on decoded streams; no public dataset is named, so
frames here are synthetic with the shapes and value ranges the workloads
specify, and side-info is drawn inside the reference's legal ranges:

* recon: smooth 2-D gradient + uniform noise (+-6 at 8-bit, +-24 at 10-bit),
  then each 8x8 block shifted so its mean sits on a multiple of the
  quantisation step (12 at 8-bit, 48 at 10-bit) to create block edges;
* deblock masks from a random transform quadtree (4..64 px, aligned, split
  where a block crosses the frame edge), edge class = min of the two sides'
  transform classes as `mask_outer_edge_*` writes them (lf_mask.rs:58-155),
  plus random sub-PU edge bits; per-64x64 qidx = 4 * level, level 0..63;
* CDEF: up to 8 strength presets (pri 0..15, sec code 0..3), a random preset
  per 64x64, damping 3..6, on_skiptx or random noskip masks;
* CCSO: per-plane band/edge configs with offset indices 0..4 ({0,+-1,+-3});
* LR: luma units None / NS-Wiener / PC-Wiener / GDF-only, chroma units
  None / NS-Wiener, taps uniform over NS_WIENER_COEF_RANGE_* (tables.rs:471);
* film grain: AR lag 3, 8 luma points, chroma scaling from luma, 32x32 blocks.
"""
from dataclasses import dataclass, field

import numpy as np

from . import abi

NS_RANGE_Y = [(6, -24), (6, -24), (5, -14), (5, -14), (5, -16), (5, -16)] + [(4, -8)] * 10
NS_RANGE_UV = ([(6, -24), (6, -24), (5, -14), (5, -14)] + [(5, -16)] * 6 + [(4, -8)] * 8)


def num_classes_of(idx):
    """NS-Wiener class count for num_classes_idx (obu.rs:1419-1424)."""
    return 1 + idx + max(idx - 3, 0) + 2 * max(idx - 5, 0)


@dataclass
class SynthFrame:
    fp: abi.FrameParams
    masks: np.ndarray
    lr: np.ndarray
    planes: list  # [y, u, v] 2-D arrays with the allocator geometry
    inloop: int
    fgd: object = None
    grain_seed: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def width(self):
        return self.fp.width

    @property
    def height(self):
        return self.fp.height

    @property
    def bitdepth(self):
        return self.fp.bitdepth

    def side(self):
        db = self.meta.get("db_input")
        return abi.side_info(self.masks, self.lr, db_masks=db)

    def use_db_blocks(self, blocks, hdr, garbage_rng=None):
        """Hand the deblock masks over as block records (R2gSideInfo.db_masks);
        with `garbage_rng` the given filter_y / filter_uv are overwritten with
        noise, which the device build must ignore."""
        self.meta["db_blocks"] = blocks
        self.meta["db_hdr"] = hdr
        self.meta["db_input"] = abi.db_mask_input(blocks, **hdr)
        if garbage_rng is not None:
            for k in ("filter_y", "filter_uv"):
                self.masks[k] = garbage_rng.integers(0, 1 << 16, size=self.masks[k].shape).astype(np.uint16)


def _plane(rng, w, h, rows, stride, bitdepth, pad_fill, bs=8):
    dtype = np.uint16 if bitdepth > 8 else np.uint8
    vmax = (1 << bitdepth) - 1
    k = 1 << (bitdepth - 8)
    step = 12 * k
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    a, b = rng.uniform(0.2, 0.8, 2)
    f1, f2 = rng.uniform(0.5, 3.0, 2)
    base = (0.5 + 0.35 * np.sin(f1 * np.pi * (a * xx / w + (1 - a) * yy / h))
            * np.cos(f2 * np.pi * (b * yy / h)))
    img = np.round(base * vmax).astype(np.int64)
    img += rng.integers(-6 * k, 6 * k + 1, size=img.shape)
    # block-mean quantisation (8x8 luma, the co-located 4x4 in chroma)
    blk = img.reshape(h // bs, bs, w // bs, bs)
    mean = blk.mean(axis=(1, 3), keepdims=True)
    q = np.round(mean / step) * step
    blk = blk + np.round(q - mean).astype(np.int64)
    img = np.clip(blk.reshape(h, w), 0, vmax)
    out = np.empty((rows, stride), dtype)
    if pad_fill is None:
        out[:] = 0
    else:
        out[:] = rng.integers(0, vmax + 1, size=out.shape, dtype=np.int64).astype(dtype)
    out[:h, :w] = img
    return out


def _quadtree(rng, h4p, w4p, fh4, fw4, p_split=(0.55, 0.5, 0.45, 0.4)):
    """Transform sizes in 4x4 units (16 = 64 px) over a 64-aligned grid."""
    size = np.full((h4p, w4p), 16, np.int32)
    for L, p in zip((16, 8, 4, 2), p_split):
        bh, bw = h4p // L, w4p // L
        cur = size[::L, ::L]
        ys = (np.arange(bh) * L)[:, None]
        xs = (np.arange(bw) * L)[None, :]
        cross = ((ys < fh4) & (ys + L > fh4)) | ((xs < fw4) & (xs + L > fw4))
        split = (cur == L) & ((rng.random((bh, bw)) < p) | cross)
        big = np.repeat(np.repeat(split, L, axis=0), L, axis=1)
        size = np.where(big, L // 2, size)
    return size


def _set_bits(arr, idx_tuple, bits):
    np.bitwise_or.at(arr, idx_tuple, bits.astype(arr.dtype))


def _edge_masks(rng, masks, size, fh4, fw4, sb256w, chroma, subpu_p=0.1):
    """Write vertical (dir 0) and horizontal (dir 1) edge bits for one plane
    type.  `size` is the transform size map (4x4 units of that plane)."""
    cls_cap = 2 if chroma else 3
    cls = np.minimum(np.log2(size).astype(np.int32), cls_cap)
    key = "filter_uv" if chroma else "filter_y"
    pos_mask = 31 if chroma else 63
    sb_shift = 5 if chroma else 6
    fld = masks[key]  # (n, 2, 64, 5, 4)
    H, W = fh4, fw4
    sz = size[:H, :W]
    c = cls[:H, :W]
    yy, xx = np.mgrid[0:H, 0:W]
    for d in (0, 1):
        if d == 0:
            edge = (xx >= 1) & (xx % sz == 0)
            nb = np.zeros_like(c)
            nb[:, 1:] = c[:, :-1]
        else:
            edge = (yy >= 1) & (yy % sz == 0)
            nb = np.zeros_like(c)
            nb[1:, :] = c[:-1, :]
        k = np.minimum(c, nb)
        ys, xs = np.nonzero(edge)
        ks = k[ys, xs]
        sb = (ys >> sb_shift) * sb256w + (xs >> sb_shift)
        if d == 0:
            pos = xs & pos_mask
            idx = (ys & pos_mask) >> 4
            bit = 1 << (ys & 15)
        else:
            pos = ys & pos_mask
            idx = (xs & pos_mask) >> 4
            bit = 1 << (xs & 15)
        _set_bits(fld, (sb, np.full_like(sb, d), pos, ks, idx), bit)
        sub = rng.random(len(ys)) < subpu_p
        _set_bits(fld, (sb[sub], np.full_like(sb[sub], d), pos[sub], np.full_like(sb[sub], 4),
                        idx[sub]), bit[sub])


def make_masks(rng, width, height, n_strengths, ccso_on=(1, 1, 1), gdf_p=0.5, noskip_p=0.85,
               lossless=False):
    bw4, bh4 = width // 4, height // 4
    sb256w, sb256h = (bw4 + 63) >> 6, (bh4 + 63) >> 6
    n = sb256w * sb256h
    masks = np.zeros(n, abi.AV2_FILTER_DTYPE)
    h4p, w4p = sb256h * 64, sb256w * 64
    size = _quadtree(rng, h4p, w4p, bh4, bw4)
    _edge_masks(rng, masks, size, bh4, bw4, sb256w, chroma=False)
    csize = np.maximum(size[::2, ::2] // 2, 1)
    _edge_masks(rng, masks, csize, bh4 // 2, bw4 // 2, sb256w, chroma=True)
    masks["qidx"] = 4 * rng.integers(0, 64, size=(n, 16))
    masks["gdf"] = (rng.random((n, 16)) < gdf_p).astype(np.uint8)
    cidx = rng.integers(0, n_strengths, size=(n, 16))
    cidx[rng.random((n, 16)) < 0.1] = -1
    masks["cdef_idx"] = cidx
    masks["ccso"] = np.array(ccso_on, np.uint8)[None, :]
    bits = rng.random((n, 32, 4, 8)) < noskip_p  # one decision per 8x8
    pairs = np.repeat(bits, 2, axis=3)
    masks["noskip_mask"] = (pairs * (1 << np.arange(16))).sum(axis=3).astype(np.uint16)
    masks["lr_noskip_mask"] = rng.integers(0, 1 << 16, size=(n, 64, 4)).astype(np.uint16)
    if lossless:
        masks["lossless_mask_y"] = (rng.random((n, 64, 4, 16)) < 0.05).astype(np.uint16).dot(
            (1 << np.arange(16)).astype(np.uint16)).astype(np.uint16)
        masks["lossless_mask_uv"] = (rng.random((n, 64, 4, 8)) < 0.05).astype(np.uint16).dot(
            (1 << np.arange(8)).astype(np.uint16)).astype(np.uint16)
    return masks


def _c_table(name, dtype):
    """A normative table from the generated csrc/av2_tables.h, as a flat array."""
    import os
    import re
    txt = open(os.path.join(os.path.dirname(__file__), "csrc", "av2_tables.h")).read()
    m = re.search(r"R2G_TABLE\(\w+, " + name + r"\)((?:\[\d+\])+) = \{([^}]*)\}", txt)
    dims = [int(d) for d in re.findall(r"\d+", m.group(1))]
    return np.array([int(v) for v in m.group(2).replace("\n", " ").split(",") if v.strip()], dtype).reshape(dims)


_BLOCK_TABLES = {}


def _block_tables():
    if not _BLOCK_TABLES:
        bd = _c_table("BLOCK_DIMENSIONS", np.int32)
        _BLOCK_TABLES["bs_of"] = {(int(w), int(h)): i for i, (w, h, _, _) in enumerate(bd)}
        _BLOCK_TABLES["tx_part"] = _c_table("TX_PART_TBL", np.int32)
    return _BLOCK_TABLES


def make_db_blocks(rng, width, height, *, seg_ids=1, tile_cols=(0,), tile_rows=(0,), tip_p=0.04, sub8_p=0.3,
                   intra_p=0.35, skip_p=0.4):
    """The create_db_mask calls of a random partition of the frame, in
    decode order (tiles in raster order, SB256s in raster order inside a
    tile, each partition tree depth first): a luma record per coded block and
    a chroma record per 4:2:0 chroma block (for a split 8x8, after its last
    luma block, at the 8x8's origin with BS_8X8, as decode.rs places cbx /
    cby / cbs).  Square nodes split where half of them lies outside the
    frame, as the partition syntax forces.  Returns (records, header dict
    for abi.db_mask_input)."""
    t = _block_tables()
    bs_of, txp = t["bs_of"], t["tx_part"]
    bw4, bh4 = ((width + 7) >> 3) << 1, ((height + 7) >> 3) << 1
    recs = []

    def rec(x, y, w, h, chroma, bs=None, ref0=None):
        bs = bs_of[(w, h)] if bs is None else bs
        intra = rng.random() < intra_p
        flags = (abi.DBB_CHROMA if chroma else 0) | (abi.DBB_INTRA if intra else 0)
        if not intra and rng.random() < skip_p:
            flags |= abi.DBB_SKIP_TXFM
        if rng.random() < 0.5:
            flags |= abi.DBB_TX_LL
        if rng.random() < 0.5:
            flags |= abi.DBB_REFINE_MV
        parts = np.nonzero(txp[bs] >= 0)[0]
        r0 = ref0 if ref0 is not None else (7 if rng.random() < 0.1 else int(rng.integers(0, 7)))
        r1 = -1 if rng.random() < 0.5 else int(rng.integers(0, 7))
        recs.append((x, y, bs, flags, int(rng.choice(parts)) if len(parts) else 0, int(rng.integers(0, seg_ids)),
                     int(rng.integers(0, 31)), int(rng.integers(0, 4)), r0, r1))

    def leaf(x, y, w, h):
        rec(x, y, w, h, False)
        rec(x, y, w, h, True)

    def node(x, y, w, h):
        if x >= bw4 or y >= bh4:
            return
        if w == 2 and h == 2:  # 8x8: whole, or 4x4 / 4x8 / 8x4 luma blocks sharing one chroma block
            if rng.random() < sub8_p:
                kind = int(rng.integers(0, 3))
                subs = {0: [(0, 0, 1, 1), (1, 0, 1, 1), (0, 1, 1, 1), (1, 1, 1, 1)],
                        1: [(0, 0, 1, 2), (1, 0, 1, 2)], 2: [(0, 0, 2, 1), (0, 1, 2, 1)]}[kind]
                for dx, dy, sw, sh in subs:
                    if x + dx < bw4 and y + dy < bh4:
                        rec(x + dx, y + dy, sw, sh, False)
                rec(x, y, 2, 2, True)
            else:
                leaf(x, y, 2, 2)
            return
        if w == h:
            has_rows, has_cols = y + h // 2 < bh4, x + w // 2 < bw4
            if has_rows and has_cols:
                pn = {64: 0.05, 32: 0.15, 16: 0.3, 8: 0.45, 4: 0.55}[w]
                kind = int(rng.choice(4, p=[pn, 0.6 * (1 - pn), 0.2 * (1 - pn), 0.2 * (1 - pn)]))
            elif has_cols:
                kind = 1 if rng.random() < 0.5 else 2
            elif has_rows:
                kind = 1 if rng.random() < 0.5 else 3
            else:
                kind = 1
            if kind == 0:
                leaf(x, y, w, h)
            elif kind == 1:
                for dy in (0, h // 2):
                    for dx in (0, w // 2):
                        node(x + dx, y + dy, w // 2, h // 2)
            elif kind == 2:  # horizontal halves
                for dy in (0, h // 2):
                    rect(x, y + dy, w, h // 2)
            else:
                for dx in (0, w // 2):
                    rect(x + dx, y, w // 2, h)
            return
        rect(x, y, w, h)

    def rect(x, y, w, h):
        if x >= bw4 or y >= bh4:
            return
        if min(w, h) >= 4 and rng.random() < 0.3:  # halve the long side again
            if w > h:
                for dx in (0, w // 2):
                    rect(x + dx, y, w // 2, h)
            else:
                for dy in (0, h // 2):
                    rect(x, y + dy, w, h // 2)
            return
        leaf(x, y, w, h)

    rows = list(tile_rows) + [bh4]
    cols = list(tile_cols) + [bw4]
    for tr in range(len(tile_rows)):
        for tc in range(len(tile_cols)):
            for sy in range(rows[tr], rows[tr + 1], 64):
                for sx in range(cols[tc], cols[tc + 1], 64):
                    if rng.random() < tip_p:  # a TIP superblock: one 256x256 block, chroma co-located
                        rec(sx, sy, 64, 64, False, ref0=7)
                        rec(sx, sy, 64, 64, True, ref0=7)
                    else:
                        node(sx, sy, 64, 64)
    blocks = np.array(recs, abi.DB_BLOCK_DTYPE) if recs else np.zeros(0, abi.DB_BLOCK_DTYPE)
    hdr = {"sub_pu": int(rng.random() < 0.7), "tip_frame_mode": int(rng.integers(0, 3)),
           "tip_subpel_filter": int(rng.integers(0, 4)), "tip_refine_mv": int(rng.integers(0, 2)),
           "tile_cols": tuple(tile_cols), "tile_rows": tuple(tile_rows)}
    return blocks, hdr


def _taps(rng, ranges, shape=()):
    lo = np.array([mn for nb, mn in ranges])
    hi = np.array([mn + (1 << nb) for nb, mn in ranges])
    return rng.integers(lo, hi, size=tuple(shape) + (len(ranges),)).astype(np.int8)


def make_lr(rng, n, luma_types=(0, 1, 2, 3), chroma_ns_p=0.6):
    """Per-SB256 restoration records.  Luma unit kind 0 none, 1 PC-Wiener,
    2 NS-Wiener, 3 GDF-only (type none; the gdf flag lives in the masks).
    Only class 0 of a unit's ns_filter is read for single-class NS-Wiener."""
    lr = np.zeros(n, abi.AV2_RESTORATION_DTYPE)
    kinds = rng.choice(np.array(luma_types), size=(n, 16))
    lr["lr"]["restoration_type"][:, 0, :] = np.where(kinds == 3, 0, kinds)
    lr["lr"]["ns_filter"][:, 0, :, 0, :16] = _taps(rng, NS_RANGE_Y, (n, 16))
    lr["lr"]["ns_filter"][:, 1:, :, 0, :18] = _taps(rng, NS_RANGE_UV, (n, 2, 16))
    ch = rng.random((n, 2, 16)) < chroma_ns_p
    lr["lr"]["restoration_type"][:, 1:, :] = np.where(ch, abi.RESTORE_NS_WIENER, 0)
    return lr, kinds


def make_frame_params(rng, width, height, bitdepth, *, cdef=True, ccso=True, lr=True, gdf=True,
                      ns_multi=0, cfl_ds=0, inter=None):
    fp = abi.FrameParams()
    fp.width, fp.height, fp.bitdepth, fp.layout, fp.sb128 = width, height, bitdepth, 1, 0
    fp.cfl_ds_filter_index = cfl_ds
    fp.deblock_level_y[0] = fp.deblock_level_y[1] = 1
    fp.deblock_level_u = fp.deblock_level_v = 1
    fp.deblock_delta_q_y[0], fp.deblock_delta_q_y[1] = (int(v) for v in rng.integers(-3, 4, 2))
    fp.deblock_delta_q_u, fp.deblock_delta_q_v = (int(v) for v in rng.integers(-3, 4, 2))
    fp.quant_yac = int(rng.integers(1, 256))
    fp.quant_uac_delta, fp.quant_vac_delta = (int(v) for v in rng.integers(-8, 9, 2))
    fp.seq_cdef = 1 if cdef else 0
    fp.cdef_damping = int(rng.integers(3, 7))
    fp.cdef_on_skiptx = int(rng.integers(0, 2))
    ns = int(rng.integers(1, 9))
    fp.cdef_n_strengths = ns
    for i in range(8):
        fp.cdef_y_strength[i] = int(rng.integers(0, 16)) << 2 | int(rng.integers(0, 4))
        fp.cdef_uv_strength[i] = int(rng.integers(0, 16)) << 2 | int(rng.integers(0, 4))
    for pl in range(3):
        cp = fp.ccso[pl]
        cp.enabled = 1 if ccso else 0
        cp.bo_only = int(rng.random() < 0.3)
        cp.scale_idx = 0
        cp.quant_idx = int(rng.integers(0, 3))
        cp.ext_filter_support = int(rng.integers(0, 7))
        cp.edge_clf = int(rng.integers(0, 2))
        cp.max_band_log2 = int(rng.integers(0, 8 if cp.bo_only else 4))
        offs = rng.integers(0, 5, size=128)
        for i in range(64):
            cp.filter_off[i] = int(offs[2 * i] | (offs[2 * i + 1] << 4))
    if lr:
        fp.restoration[0].restoration_type = abi.RESTORE_SWITCHABLE
        fp.restoration[1].restoration_type = abi.RESTORE_NS_WIENER
        fp.restoration[2].restoration_type = abi.RESTORE_NS_WIENER
    for pl in range(3):
        rp = fp.restoration[pl]
        rp.frame_filters_on = 0
        rp.num_classes_idx = 0
        rp.num_classes = 1
    if lr and ns_multi:
        rp = fp.restoration[0]
        rp.frame_filters_on = 1
        rp.num_classes_idx = ns_multi
        rp.num_classes = num_classes_of(ns_multi)
        for c in range(16):
            t = _taps(rng, NS_RANGE_Y)
            for i in range(16):
                rp.filter[c][i] = int(t[i])
    fp.restoration_unit_size[0] = 6
    fp.restoration_unit_size[1] = 6
    fp.gdf_enabled = 1 if gdf else 0
    fp.gdf_qp_idx = int(rng.integers(0, 6))
    fp.gdf_scale = int(rng.integers(1, 5))
    if inter is None:
        inter = bool(rng.integers(0, 2))
    fp.frame_type = 1 if inter else 0
    fp.n_ref_frames = 2 if inter else 0
    for i in range(7):
        fp.absrefdist[i] = int(rng.integers(0, 12))
    return fp


def make_film_grain(rng):
    g = abi.FilmGrainData()
    g.chroma_scaling_from_luma = 1
    g.num_points[0], g.num_points[1], g.num_points[2] = 8, 0, 0
    xs = np.sort(rng.choice(np.arange(0, 256), size=8, replace=False))
    for i in range(8):
        g.points[0][i][0] = int(xs[i])
        g.points[0][i][1] = int(rng.integers(0, 256))
    g.scaling_shift = int(rng.integers(8, 12))
    g.ar_coeff_lag = 3
    for pl in range(3):
        for i in range(28):
            g.ar_coeffs[pl][i] = int(rng.integers(-32, 32))
    g.ar_coeff_shift = int(rng.integers(6, 10))
    g.grain_scale_shift = int(rng.integers(0, 4))
    g.overlap_flag = 1
    g.clip_to_restricted_range = int(rng.integers(0, 2))
    g.mc_identity = int(rng.integers(0, 2))
    g.block_size = 1
    return g, int(rng.integers(0, 1 << 16))


def make_frame(width, height, bitdepth, seed, *, chain="full", grain=False, pad_fill=None, ns_multi=0,
               lossless=False, cfl_ds=0, luma_types=(0, 1, 2, 3), inter=None):
    """One synthetic frame.  chain: "db" (deblock), "db_cdef" (deblock+CDEF),
    "full" (deblock+CDEF+CCSO+LR+GDF)."""
    assert width % 8 == 0 and height % 8 == 0
    rng = np.random.default_rng(seed)
    ys, uvs, yrows, uvrows = abi.plane_geometry(width, height, bitdepth)
    bps = 2 if bitdepth > 8 else 1
    y = _plane(rng, width, height, yrows, ys // bps, bitdepth, pad_fill)
    u = _plane(rng, width // 2, height // 2, uvrows, uvs // bps, bitdepth, pad_fill, 4)
    v = _plane(rng, width // 2, height // 2, uvrows, uvs // bps, bitdepth, pad_fill, 4)
    full = chain == "full"
    fp = make_frame_params(rng, width, height, bitdepth, cdef=chain != "db", ccso=full, lr=full, gdf=full,
                           ns_multi=ns_multi, cfl_ds=cfl_ds, inter=inter)
    if lossless:
        fp.seg_enabled = 1
        fp.seg_lossless[1] = 1
    masks = make_masks(rng, width, height, fp.cdef_n_strengths, lossless=lossless)
    lr, kinds = make_lr(rng, masks.shape[0], luma_types=luma_types)
    # GDF-only units carry the gdf flag; others get it at random (stacked)
    masks["gdf"] = np.where(kinds == 3, 1, masks["gdf"]).astype(np.uint8)
    if chain == "db":
        inloop = abi.INLOOP_DEBLOCK
    elif chain == "db_cdef":
        inloop = abi.INLOOP_DEBLOCK | abi.INLOOP_CDEF
    else:
        inloop = abi.INLOOP_ALL
    fgd, gseed = (None, 0)
    if grain:
        fgd, gseed = make_film_grain(rng)
    return SynthFrame(fp=fp, masks=masks, lr=lr, planes=[y, u, v], inloop=inloop, fgd=fgd, grain_seed=gseed,
                      meta={"seed": seed, "chain": chain})
