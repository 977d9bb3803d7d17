/*
 * Oracle: per-frame driver and the exported C API of liboracle.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Restates the per-sbrow filter pass filter_sbrow (decode.rs:3718-4058) and
 * the frame-level state set-up (decode.rs:27-100, :238-330) of the rav2d
 * reference, looping filter_sbrow over every superblock row in order as the
 * Phase-B loop (decode.rs:3597-3625) does.
 */
#include "oracle.h"

namespace r2o {

/* decode.rs:27-57 init_wiener */
static void init_wiener(Frame &f) {
    const R2gFrameParams *fp = f.fp;
    f.base_q = 0;
    f.wiener_idx = 0;
    f.ns_subclass_class_idx = -1;
    int rtype = fp->restoration[0].restoration_type;
    if (rtype == R2G_RESTORE_NONE) return;
    int qidx = fp->quant_yac;
    f.base_q = dq_lookup(qidx);
    f.wiener_idx = qidx < 130 ? 0 : qidx < 190 ? 1 : qidx < 220 ? 2 : 3;
    if (rtype == R2G_RESTORE_NS_WIENER || rtype == R2G_RESTORE_SWITCHABLE) {
        int nci = fp->restoration[0].num_classes_idx;
        f.ns_subclass_class_idx = nci > 0 ? nci - 1 : -1;
    }
}

/* decode.rs:59-65 compute_restore_planes */
static int compute_restore_planes(const R2gFrameParams *fp) {
    int has_y = fp->restoration[0].restoration_type != R2G_RESTORE_NONE || fp->gdf_enabled != 0;
    int has_u = fp->restoration[1].restoration_type != R2G_RESTORE_NONE;
    int has_v = fp->restoration[2].restoration_type != R2G_RESTORE_NONE;
    return has_y | (has_u << 1) | (has_v << 2);
}

/* decode.rs:67-80 compute_gdf_ref_dst_idx */
static int compute_gdf_ref_dst_idx(const R2gFrameParams *fp) {
    if (fp->gdf_enabled == 0) return 0;
    if (!(fp->frame_type & 1)) return 0;
    int max_dist = 0;
    for (int i = 0; i < imin(fp->n_ref_frames, 2); i++) max_dist = imax(max_dist, fp->absrefdist[i]);
    static const int TBL[12] = {5, 1, 2, 3, 3, 3, 4, 4, 4, 4, 4, 5};
    return TBL[imin(max_dist, 11)];
}

/* decode.rs:3718-4058 filter_sbrow */
static void filter_sbrow(Frame &f, int sby, uint32_t inloop) {
    const R2gFrameParams *fp = f.fp;
    int sb128 = fp->sb128;
    bool deblock_on = (inloop & R2G_INLOOP_DEBLOCK) && (fp->deblock_level_y[0] != 0 || fp->deblock_level_y[1] != 0);
    size_t mask_row = (size_t)((sby >> (2 - sb128)) * f.sb256w);
    if (deblock_on) {
        deblock_crop_bottom_edge(f, mask_row, sby);
        deblock_sbrow_cols(f, mask_row, sby);
        deblock_sbrow_rows(f, mask_row, sby);
    }
    bool copy_db_on = f.restore_planes != 0 && (inloop & (R2G_INLOOP_WIENER | R2G_INLOOP_GDF));
    if (copy_db_on) {
        const size_t num_lines = 20;
        if (f.lr_db_line[0].size() != (size_t)f.stride[0] * num_lines) f.lr_db_line[0].assign(f.stride[0] * num_lines, 0);
        for (int pl = 1; pl < 3; pl++)
            if (f.lr_db_line[pl].size() != (size_t)f.stride[1] * num_lines)
                f.lr_db_line[pl].assign(f.stride[1] * num_lines, 0);
        copy_db(f, sby);
    }
    if (fp->seq_cdef && (inloop & (R2G_INLOOP_CDEF | R2G_INLOOP_CCSO))) cdef_filter_sbrow(f, mask_row, sby, inloop);
    if (f.restore_planes != 0 && (inloop & (R2G_INLOOP_WIENER | R2G_INLOOP_GDF))) lr_sbrow_apply(f, sby, inloop);
}

static bool supported(const R2gFrameParams *fp) {
    return fp && (fp->bitdepth == 8 || fp->bitdepth == 10) && fp->layout == 1 && fp->sb128 == 0 && fp->width > 0 &&
           fp->height > 0 && (fp->width & 7) == 0 && (fp->height & 7) == 0;
}

}  // namespace r2o

using namespace r2o;

extern "C" {

/* Filter one frame in place: `y/u/v` are uint16_t planes (8-bit samples
 * widened) with per-plane allocations of the reference's DefaultPicAllocator
 * geometry, strides in samples.  Returns 0, or -1 for an unsupported frame. */
int r2o_filter_frame(const R2gFrameParams *fp, const R2gSideInfo *side, uint32_t inloop, uint16_t *y, uint16_t *u,
                     uint16_t *v, int64_t y_stride, int64_t uv_stride) {
    if (!supported(fp) || !side || !side->masks || !side->lr) return -1;
    Frame f;
    f.fp = fp;
    f.bd.bitdepth = fp->bitdepth;
    f.hbd = (fp->bitdepth - 8) >> 1;
    f.bw = ((fp->width + 7) >> 3) << 1;
    f.bh = ((fp->height + 7) >> 3) << 1;
    int sb_step = 16 << fp->sb128;
    f.sbh = (f.bh + sb_step - 1) / sb_step;
    f.sb256w = (f.bw + 63) >> 6;
    f.sb256h = (f.bh + 63) >> 6;
    if (side->n_sb256 != f.sb256w * f.sb256h) return -1;
    f.p[0] = y;
    f.p[1] = u;
    f.p[2] = v;
    f.stride[0] = y_stride;
    f.stride[1] = uv_stride;
    f.mask.assign(side->masks, side->masks + side->n_sb256);
    /* edge masks handed over as the decoder's create_db_mask calls: walk
     * them as the decoder does */
    if (side->db_masks) r2o_build_db_masks(side->db_masks, fp, f.mask.data(), side->n_sb256);
    f.lr_mask = side->lr;
    f.segmap = side->segmap;
    f.b4_stride = side->segmap_stride;
    f.segmap_uv = side->segmap_uv;
    f.uv_segmap_stride = side->segmap_uv_stride;
    init_wiener(f);
    f.restore_planes = compute_restore_planes(fp);
    f.gdf_ref_dst_idx = compute_gdf_ref_dst_idx(fp);
    /* decode.rs:99-120 init_start_of_tile_row: (tile row << 1) | 1 on a
     * tile row's first superblock row, tile row << 1 on the others */
    f.start_of_tile_row.assign(f.sbh, 0);
    {
        int rows = fp->tile_rows ? fp->tile_rows : 1;
        int sby = 0;
        for (int tr = 0; tr < rows && sby < f.sbh; tr++) {
            f.start_of_tile_row[sby++] = (uint8_t)((tr << 1) | 1);
            int end = fp->tile_rows ? imin(fp->tile_row_start_sb[tr + 1], f.sbh) : f.sbh;
            while (sby < end) f.start_of_tile_row[sby++] = (uint8_t)(tr << 1);
        }
    }
    f.cdef_line_toggle = 0;
    for (int sby = 0; sby < f.sbh; sby++) filter_sbrow(f, sby, inloop);
    return 0;
}

/* ---- single-function entry points used by the known-answer tests ---- */
uint32_t r2o_deblock_quant_thr(int hbd, int qidx) { return deblock_quant_thr(hbd, qidx); }
uint32_t r2o_deblock_side_thr(int hbd, int qidx) { return deblock_side_thr(hbd, qidx); }
int r2o_dq_lookup(int qidx) { return dq_lookup(qidx); }
int r2o_filter_choice(const uint16_t *buf, int64_t s, int64_t t, int64_t stride, int mwn, int mwp, uint32_t q_thr,
                      uint32_t side_thr) {
    return filter_choice(buf, s, t, stride, mwn, mwp, q_thr, side_thr);
}
int r2o_cdef_find_dir(const uint16_t *img, int64_t stride, uint32_t *var, int bitdepth) {
    return cdef_find_dir(img, stride, var, bitdepth - 8);
}
int r2o_adjust_strength(int strength, uint32_t var) { return adjust_strength(strength, var); }
int r2o_constrain(int diff, int threshold, int shift) { return constrain(diff, threshold, shift); }
uint32_t r2o_ccso_score(int diff, int quant_step, uint32_t edge_clf) { return ccso_score(diff, quant_step, edge_clf); }
int r2o_get_qval_given_tskip(int qstep, int tskip, int i, int bitdepth_min_8) {
    return get_qval_given_tskip(qstep, tskip, i, bitdepth_min_8);
}

}  // extern "C"
