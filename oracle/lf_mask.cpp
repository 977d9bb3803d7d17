/*
 * Oracle: the deblock edge-mask builders (the Av2Filter filter_y / filter_uv
 * bit planes the deblocking filter walks).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Restates crates/rav2d/src/lf_mask.rs:58-503 of the rav2d reference:
 * mask_outer_edge_l / _t, mask_inner_edges_v / _h, mask_edges_part,
 * mask_subpu_edges, subpu_flt_lvl and create_db_mask.  Masks are
 * [2][64][5][4] u16: direction (0 vertical edges, 1 horizontal), position
 * across (4x4 column or row), level 0..3 (+ 4: sub-PU), 16-bit segment of
 * the position along.
 */
#include "oracle.h"

#define R2G_TABLE(type, name) static const type name
#include "av2_tables.h"

namespace r2o {

typedef uint16_t FilterMasks[64][5][4];

enum { TXP_NONE = 0, TXP_SPLIT, TXP_H, TXP_V, TXP_H4, TXP_V4, TXP_H5, TXP_V5 };

/* TXFM_DIMENSIONS entry (tables.rs:12-21): w, h, lw, lh, min, max, sub, ctx */
struct TxfmInfo {
    int w, h, lw, lh;
};
static TxfmInfo txfm_info(int tx) {
    const uint8_t *t = TXFM_DIMENSIONS[tx];
    return {t[0], t[1], t[2], t[3]};
}

/* lf_mask.rs:58-71 */
static void mask_outer_edge_l(uint16_t (*masks)[4], int by4, int h4, int bwl4c, uint8_t *l) {
    uint64_t mask = (uint64_t)1 << by4;
    for (int y = 0; y < h4; y++) {
        int sidx = (by4 + y) >> 4;
        uint16_t smask = (uint16_t)(mask >> (sidx << 4));
        int lvl = imin(bwl4c, l[y]);
        masks[lvl][sidx] |= smask;
        mask <<= 1;
    }
    for (int y = 0; y < h4; y++) l[y] = (uint8_t)bwl4c;
}

/* lf_mask.rs:73-86 */
static void mask_outer_edge_t(uint16_t (*masks)[4], int bx4, int w4, int bhl4c, uint8_t *a) {
    uint64_t mask = (uint64_t)1 << bx4;
    for (int x = 0; x < w4; x++) {
        int sidx = (bx4 + x) >> 4;
        uint16_t smask = (uint16_t)(mask >> (sidx << 4));
        int lvl = imin(bhl4c, a[x]);
        masks[lvl][sidx] |= smask;
        mask <<= 1;
    }
    for (int x = 0; x < w4; x++) a[x] = (uint8_t)bhl4c;
}

/* lf_mask.rs:88-119 (dir 0) and :121-152 (dir 1): OR the four 16-bit parts
 * of `inner` into every hstep-th (vstep-th) position from the offset */
static void mask_inner_edges(FilterMasks masks[2], int dir, uint64_t inner, int b4, int n4, int tl4c, int off,
                             int step) {
    uint16_t parts[4] = {(uint16_t)(inner & 0xffff), (uint16_t)((inner >> 16) & 0xffff),
                         (uint16_t)((inner >> 32) & 0xffff), (uint16_t)(inner >> 48)};
    for (int i = off; i < n4; i += step) {
        int idx = b4 + i;
        for (int k = 0; k < 4; k++)
            if (parts[k]) masks[dir][idx][tl4c][k] |= parts[k];
    }
}
static void mask_inner_edges_v(FilterMasks masks[2], uint64_t inner, int bx4, int w4, int twl4c, int xoff,
                               int hstep) {
    mask_inner_edges(masks, 0, inner, bx4, w4, twl4c, xoff, hstep);
}
static void mask_inner_edges_h(FilterMasks masks[2], uint64_t inner, int by4, int h4, int thl4c, int yoff,
                               int vstep) {
    mask_inner_edges(masks, 1, inner, by4, h4, thl4c, yoff, vstep);
}

static inline uint64_t ones_shl(int n, int shift) { return (~(uint64_t)0 >> (64 - n)) << shift; }

/* lf_mask.rs:154-268 mask_edges_part */
static void mask_edges_part(FilterMasks masks[2], int by4, int bx4, int w4, int h4, int tx_part, TxfmInfo t,
                            int hlim, int vlim, uint8_t *a, uint8_t *l) {
    int tw4 = t.w, th4 = t.h;
    int twl4c = imin(hlim, t.lw), thl4c = imin(vlim, t.lh);
    if (tx_part < TXP_H5) {
        mask_outer_edge_l(masks[0][bx4], by4, h4, twl4c, l);
        mask_outer_edge_t(masks[1][by4], bx4, w4, thl4c, a);
        if (w4 > tw4) mask_inner_edges_v(masks, ones_shl(h4, by4), bx4, w4, twl4c, tw4, tw4);
        if (h4 > th4) mask_inner_edges_h(masks, ones_shl(w4, bx4), by4, h4, thl4c, th4, th4);
    } else if (tx_part == TXP_H5) {
        mask_outer_edge_t(masks[1][by4], bx4, w4, thl4c, a);
        mask_outer_edge_l(masks[0][bx4], by4, imin(th4, h4), twl4c, l);
        if (h4 > th4) {
            mask_outer_edge_l(masks[0][bx4], by4 + th4, imin(2 * th4, h4 - th4), imin(twl4c + 1, hlim), l + th4);
            if (h4 > th4 * 3)
                mask_outer_edge_l(masks[0][bx4], by4 + th4 * 3, imin(th4, h4 - 3 * th4), twl4c, l + th4 * 3);
        }
        mask_inner_edges_h(masks, ones_shl(w4, bx4), by4, h4, thl4c, th4, th4 * 2);
        uint64_t inner_a = ones_shl(h4, by4), inner_b = ones_shl(th4 * 2, by4 + th4);
        mask_inner_edges_v(masks, inner_a & ~inner_b, bx4, w4, twl4c, tw4, tw4);
    } else {
        mask_outer_edge_l(masks[0][bx4], by4, h4, twl4c, l);
        mask_outer_edge_t(masks[1][by4], bx4, imin(tw4, w4), thl4c, a);
        if (w4 > tw4) {
            mask_outer_edge_t(masks[1][by4], bx4 + tw4, imin(2 * tw4, w4 - tw4), imin(thl4c + 1, vlim), a + tw4);
            if (w4 > tw4 * 3)
                mask_outer_edge_t(masks[1][by4], bx4 + tw4 * 3, imin(tw4, w4 - 3 * tw4), thl4c, a + tw4 * 3);
        }
        mask_inner_edges_v(masks, ones_shl(h4, by4), bx4, w4, twl4c, tw4, tw4 * 2);
        uint64_t inner_a = ones_shl(w4, bx4), inner_b = ones_shl(tw4 * 2, bx4 + tw4);
        mask_inner_edges_h(masks, inner_a & ~inner_b, by4, h4, thl4c, th4, th4);
    }
}

/* lf_mask.rs:270-344 mask_subpu_edges */
static void mask_subpu_edges(FilterMasks masks[2], int by4, int bx4, int w4, int h4, int twl4c, int thl4c, int hsz,
                             int vsz, int ds_sub_pu_mask) {
    for (int dir = 0; dir < 2; dir++) {
        int sz = dir ? vsz : hsz;
        if (!sz) continue;
        uint64_t inner = dir ? ones_shl(w4, bx4) : ones_shl(h4, by4);
        uint16_t parts[4] = {(uint16_t)(inner & 0xffff), (uint16_t)((inner >> 16) & 0xffff),
                             (uint16_t)((inner >> 32) & 0xffff), (uint16_t)(inner >> 48)};
        int n4 = dir ? h4 : w4, b4 = dir ? by4 : bx4, t = dir ? thl4c : twl4c;
        for (int i = sz; i < n4; i += sz) {
            int idx = b4 + i;
            for (int e = 0; e < 4; e++)
                if (parts[e]) {
                    uint16_t m = masks[dir][idx][t][e];
                    masks[dir][idx][t][e] |= parts[e];
                    if (i & ds_sub_pu_mask) masks[dir][idx][4][e] |= (uint16_t)(parts[e] & ~m);
                }
        }
    }
}

/* The block fields create_db_mask reads (levels.rs Av2Block) and the header
 * fields subpu_flt_lvl reads. */
struct DbBlock {
    int bs, is_intra, skip_txfm, tx_part, tx_size_ll, seg_id;
    int ref0, ref1;  /* ref_pair.r; ref0 == TIP_FRAME marks a TIP block, ref1 -1 = single */
    int inter_mode, refine_mv, comp_type;
};
struct DbHeader {
    int sub_pu, tip_frame_mode, tip_subpel_filter, tip_refine_mv, lossless[8];
};
/* levels.rs:1 TIP_FRAME, :314 OpflNearMvNearMv, :326 CompInterType::Avg,
 * :246/:270 block sizes, levels.rs TxfmSize::Tx4x4; headers.rs:112-118
 * PixelLayout; lf_mask.rs:364 FILTER_8TAP_SHARP */
enum { TIP_FRAME = 7, FILTER_8TAP_SHARP = 2, OPFL_NEAR_MV_NEAR_MV = 24, COMP_AVG = 1, BS_8X8 = 24,
       BS_256X256 = 0, TX_4X4 = 0, I444 = 3, I420 = 1 };

/* lf_mask.rs:367-397 subpu_flt_lvl */
static int subpu_flt_lvl(const DbHeader &h, int bs, int bw4, int bh4, const DbBlock &b, int max_lvl) {
    const int opfl_first = OPFL_NEAR_MV_NEAR_MV;
    if (b.is_intra || !h.sub_pu) {
    } else if (b.ref0 == TIP_FRAME) {
        bool opfl = h.tip_refine_mv && (h.tip_frame_mode == 1 || h.tip_subpel_filter == FILTER_8TAP_SHARP);
        return 1 + (h.tip_frame_mode == 2 ? (int)!opfl : (int)((!opfl && imin(bw4, bh4) >= 4) || bs == BS_256X256));
    } else if (b.ref1 != -1) {
        if (b.inter_mode >= opfl_first) return 1 - (bs == BS_8X8);
        if (b.refine_mv && b.comp_type == COMP_AVG) return 2;
    }
    return max_lvl;
}

/* lf_mask.rs:399-503 create_db_mask (layout I420 = 1 .. I444 = 3 as in
 * headers.rs PixelLayout) */
static void create_db_mask(FilterMasks masks[2], const DbBlock &b, int bs, int bx, int by, int iw, int ih,
                           int layout, bool chroma, uint8_t *a, uint8_t *l, const DbHeader &h) {
    int ss_ver = chroma && layout == I420;
    int ss_hor = chroma && layout != I444;
    const uint8_t *b_dim = BLOCK_DIMENSIONS[bs];
    int bw4 = imin(iw - bx, b_dim[0]) >> ss_hor;
    int bh4 = imin(ih - by, b_dim[1]) >> ss_ver;
    int bx4 = (bx & 63) >> ss_hor;
    int by4 = (by & 63) >> ss_ver;
    int subpu_l2 = subpu_flt_lvl(h, bs, b_dim[0], b_dim[1], b, 3);
    int ds_subpu_mask = (h.tip_frame_mode != 2) * 15;
    int twl4c, thl4c;
    int chroma_i = chroma;
    int lossless = h.lossless[b.seg_id];
    if (b.is_intra || !b.skip_txfm) {
        int tx_part = chroma ? (int)TXP_NONE : b.tx_part;
        int tx;
        if (lossless)
            tx = (!chroma && b.tx_size_ll) ? (int)MAX_TXFM_SIZE_FOR_BS[bs][3] : (int)TX_4X4;
        else if (chroma)
            tx = MAX_TXFM_SIZE_FOR_BS[bs][I444 - layout];
        else
            tx = TX_PART_TBL[bs][tx_part];
        TxfmInfo t = txfm_info(tx);
        mask_edges_part(masks, by4, bx4, bw4, bh4, tx_part, t, iclip(subpu_l2 - ss_hor, 0, 3 - chroma_i),
                        iclip(subpu_l2 - ss_ver, 0, 3 - chroma_i), a, l);
        twl4c = imin(subpu_l2, t.lw);
        thl4c = imin(subpu_l2, t.lh);
    } else {
        int hlim = 0, vlim = 0;
        if (!lossless) {
            hlim = iclip(imin(subpu_l2, b_dim[2]) - ss_hor, 0, 3 - chroma_i);
            vlim = iclip(imin(subpu_l2, b_dim[3]) - ss_ver, 0, 3 - chroma_i);
        }
        mask_outer_edge_l(masks[0][bx4], by4, bh4, hlim, l);
        mask_outer_edge_t(masks[1][by4], bx4, bw4, vlim, a);
        twl4c = subpu_l2;
        thl4c = subpu_l2;
    }
    if (subpu_l2 != 3) {
        int h_subpu_l2 = twl4c - (ss_hor && twl4c);
        int v_subpu_l2 = thl4c - (ss_ver && thl4c);
        mask_subpu_edges(masks, by4, bx4, bw4, bh4, h_subpu_l2, v_subpu_l2, (1 << subpu_l2) >> ss_hor,
                         (1 << subpu_l2) >> ss_ver, ds_subpu_mask);
    }
}

/* The decoder's walk over a frame's create_db_mask calls (decode.rs:7869-
 * 7912, :12893-12928) in decode order: the left context (tx_lpf_y / _uv,
 * indexed by the 4x4 row in the SB256 row) starts at 3 / 2 (decode.rs:207
 * reset_context) for every tile column of every superblock row, the above
 * context (indexed by the 4x4 column in the SB256 column) for every tile
 * row; each call writes the masks of its SB256. */
static void build_db_masks(const R2gDbMaskInput &in, const R2gFrameParams &fp, R2gAv2Filter *masks, int n_sb256) {
    const int bw4 = ((fp.width + 7) >> 3) << 1, bh4 = ((fp.height + 7) >> 3) << 1;
    const int sb256w = (bw4 + 63) >> 6;
    for (int i = 0; i < n_sb256; i++) {
        memset(masks[i].filter_y, 0, sizeof(masks[i].filter_y));
        memset(masks[i].filter_uv, 0, sizeof(masks[i].filter_uv));
    }
    DbHeader h{in.sub_pu, in.tip_frame_mode, in.tip_subpel_filter, in.tip_refine_mv, {0}};
    for (int i = 0; i < 8; i++) h.lossless[i] = fp.seg_lossless[i];
    struct Ctx {
        uint8_t y[64], uv[64];
    };
    std::vector<std::pair<long, Ctx>> lctx, actx;  // (key, context) created on first use
    auto get = [](std::vector<std::pair<long, Ctx>> &v, long key) -> Ctx & {
        for (auto &e : v)
            if (e.first == key) return e.second;
        Ctx c;
        memset(c.y, 3, 64);
        memset(c.uv, 2, 64);
        v.push_back({key, c});
        return v.back().second;
    };
    for (int i = 0; i < in.n_blocks; i++) {
        const R2gDbBlock &r = in.blocks[i];
        int tc = 0, tr = 0;
        for (int t = 0; t < in.n_tile_cols; t++)
            if (r.bx >= in.tile_col_start4[t]) tc = t;
        for (int t = 0; t < in.n_tile_rows; t++)
            if (r.by >= in.tile_row_start4[t]) tr = t;
        Ctx &l = get(lctx, (long)tc * 4096 + (r.by >> 6));
        Ctx &a = get(actx, (long)tr * 4096 + (r.bx >> 6));
        DbBlock b{r.bs, (r.flags & R2G_DBB_INTRA) != 0, (r.flags & R2G_DBB_SKIP_TXFM) != 0, r.tx_part,
                  (r.flags & R2G_DBB_TX_LL) != 0, r.seg_id, r.ref0, r.ref1, r.inter_mode,
                  (r.flags & R2G_DBB_REFINE_MV) != 0, r.comp_type};
        R2gAv2Filter &m = masks[(r.by >> 6) * sb256w + (r.bx >> 6)];
        const bool chroma = (r.flags & R2G_DBB_CHROMA) != 0;
        const int ss = chroma ? 1 : 0;
        create_db_mask(chroma ? (FilterMasks *)m.filter_uv : (FilterMasks *)m.filter_y, b, r.bs, r.bx, r.by, bw4,
                       bh4, I420, chroma, (chroma ? a.uv : a.y) + ((r.bx & 63) >> ss),
                       (chroma ? l.uv : l.y) + ((r.by & 63) >> ss), h);
    }
}

}  // namespace r2o

/* ---- known-answer-test hooks (the reference's lf_mask.rs unit tests) ---- */
extern "C" {
/* masks_x4: [5][4] of one position */
void r2o_mask_outer_edge_l(uint16_t *masks_x4, int by4, int h4, int bwl4c, uint8_t *l) {
    r2o::mask_outer_edge_l((uint16_t(*)[4])masks_x4, by4, h4, bwl4c, l);
}
void r2o_mask_outer_edge_t(uint16_t *masks_x4, int bx4, int w4, int bhl4c, uint8_t *a) {
    r2o::mask_outer_edge_t((uint16_t(*)[4])masks_x4, bx4, w4, bhl4c, a);
}
/* masks: [2][64][5][4] */
void r2o_mask_inner_edges_v(uint16_t *masks, uint64_t inner, int bx4, int w4, int twl4c, int xoff, int hstep) {
    r2o::mask_inner_edges_v((r2o::FilterMasks *)masks, inner, bx4, w4, twl4c, xoff, hstep);
}
void r2o_mask_inner_edges_h(uint16_t *masks, uint64_t inner, int by4, int h4, int thl4c, int yoff, int vstep) {
    r2o::mask_inner_edges_h((r2o::FilterMasks *)masks, inner, by4, h4, thl4c, yoff, vstep);
}
/* t_dim: w, h, lw, lh */
void r2o_mask_edges_part(uint16_t *masks, int by4, int bx4, int w4, int h4, int tx_part, const int *t_dim, int hlim,
                         int vlim, uint8_t *a, uint8_t *l) {
    r2o::TxfmInfo t{t_dim[0], t_dim[1], t_dim[2], t_dim[3]};
    r2o::mask_edges_part((r2o::FilterMasks *)masks, by4, bx4, w4, h4, tx_part, t, hlim, vlim, a, l);
}
void r2o_mask_subpu_edges(uint16_t *masks, int by4, int bx4, int w4, int h4, int twl4c, int thl4c, int hsz, int vsz,
                          int ds_sub_pu_mask) {
    r2o::mask_subpu_edges((r2o::FilterMasks *)masks, by4, bx4, w4, h4, twl4c, thl4c, hsz, vsz, ds_sub_pu_mask);
}
/* blk: bs, is_intra, skip_txfm, tx_part, tx_size_ll, seg_id, ref0, ref1,
 * inter_mode, refine_mv, comp_type; hdr: sub_pu, tip_frame_mode,
 * tip_subpel_filter, tip_refine_mv, lossless[8] */
void r2o_create_db_mask(uint16_t *masks, const int *blk, int bs, int bx, int by, int iw, int ih, int layout,
                        int chroma, uint8_t *a, uint8_t *l, const int *hdr) {
    r2o::DbBlock b{blk[0], blk[1], blk[2], blk[3], blk[4], blk[5], blk[6], blk[7], blk[8], blk[9], blk[10]};
    r2o::DbHeader h{hdr[0], hdr[1], hdr[2], hdr[3], {0}};
    for (int i = 0; i < 8; i++) h.lossless[i] = hdr[4 + i];
    r2o::create_db_mask((r2o::FilterMasks *)masks, b, bs, bx, by, iw, ih, layout, chroma != 0, a, l, h);
}
/* the frame's edge masks from its create_db_mask calls, walked in order */
void r2o_build_db_masks(const R2gDbMaskInput *in, const R2gFrameParams *fp, R2gAv2Filter *masks, int n_sb256) {
    r2o::build_db_masks(*in, *fp, masks, n_sb256);
}
/* lf_mask.rs:21-36 Av2Filter::default (cdef_idx -1, everything else 0) and
 * :45-51 Av2Restoration::default (all zero) */
void r2o_av2_filter_default(R2gAv2Filter *f) {
    memset(f, 0, sizeof(*f));
    for (int i = 0; i < 16; i++) f->cdef_idx[i] = -1;
}
void r2o_av2_restoration_default(R2gAv2Restoration *r) { memset(r, 0, sizeof(*r)); }
/* tables.rs lookups: which 0 BLOCK_DIMENSIONS[i][k], 1 TXFM_DIMENSIONS[i][k] */
int r2o_block_table(int which, int i, int k) {
    return which == 0 ? BLOCK_DIMENSIONS[i][k] : TXFM_DIMENSIONS[i][k];
}
}
