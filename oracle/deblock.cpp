/*
 * Oracle: AV2 deblocking filter and the deblocked-line backup (copy_db).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Restates crates/rav2d/src/deblock.rs, lf_mask.rs:332-364 and
 * quantizer.rs:31-50 of the rav2d reference.
 */
#include "oracle.h"

#define R2G_TABLE(type, name) static const type name
#include "av2_tables.h"

namespace r2o {

/* deblock.rs:6-11 */
static const int8_t MAX_WIDTH_Y[4] = {1, 3, 6, 8};
static const int8_t MAX_WIDTH_UV[3] = {1, 3, 4};
static const int8_t Q_FIRST[3] = {45, 40, 32};
static const int8_t Q_THRESH_MULTS[8] = {32, 25, 19, 19, 0, 18, 0, 17};
static const int8_t W_MULT[8] = {85, 51, 37, 28, 0, 20, 0, 15};

/* quantizer.rs:31-50 dq_lookup */
int dq_lookup(int qidx) {
    static const uint8_t TBL[24] = {40, 41, 43, 44, 45, 47, 48, 49, 51, 52, 54, 55,
                                    57, 59, 60, 62, 64, 66, 68, 70, 72, 74, 76, 78};
    qidx = iclip(qidx, 0, 255);
    if (qidx == 0) return 64;
    qidx -= 1;
    int shift = qidx / 24;
    return (int)TBL[qidx % 24] << shift;
}

/* lf_mask.rs:332-335 deblock_quant_thr */
uint32_t deblock_quant_thr(int hbd, int qidx) {
    int qmax = 255 + 48 * hbd;
    return (uint32_t)((dq_lookup(iclip(qidx, 0, qmax)) + 4) >> (3 + 6));
}

/* lf_mask.rs:337-342 deblock_side_thr */
uint32_t deblock_side_thr(int hbd, int qidx) {
    int bitdepth_min_8 = 2 * hbd;
    int q_ind = iclip(qidx - 24 * bitdepth_min_8, 0, 296 - 1);
    int side_thr = DEBLOCK_SIDE_THRESHOLDS[q_ind];
    return (uint32_t)imax(side_thr + ((1 << 4) >> bitdepth_min_8), 0) >> (5 - bitdepth_min_8);
}

/* deblock.rs:13-33 init_deblock_thr_lut_y */
static void init_lut_y(const Frame &f, int dir, int qidx, uint32_t lut[2][16]) {
    const R2gFrameParams *fp = f.fp;
    memset(lut, 0, sizeof(uint32_t) * 32);
    int qmax = 255 + 48 * f.hbd;
    int n = fp->seg_enabled ? 8 : 1;
    for (int i = 0; i < n; i++) {
        int yac = fp->seg_enabled ? iclip(qidx + fp->seg_delta_q[i], 0, qmax) : qidx;
        int dir_yac = yac + 8 * fp->deblock_delta_q_y[dir];
        lut[0][i] = deblock_quant_thr(f.hbd, dir_yac);
        lut[1][i] = deblock_side_thr(f.hbd, dir_yac);
    }
}

/* deblock.rs:35-57 init_deblock_thr_lut_uv */
static void init_lut_uv(const Frame &f, int qidx, uint32_t lut[2][2][16]) {
    const R2gFrameParams *fp = f.fp;
    memset(lut, 0, sizeof(uint32_t) * 64);
    int qmax = 255 + 48 * f.hbd;
    int n = fp->seg_enabled ? 8 : 1;
    for (int i = 0; i < n; i++) {
        int yac = fp->seg_enabled ? iclip(qidx + fp->seg_delta_q[i], 0, qmax) : qidx;
        int uac = yac + fp->quant_uac_delta + 8 * fp->deblock_delta_q_u;
        lut[0][0][i] = deblock_quant_thr(f.hbd, uac);
        lut[0][1][i] = deblock_side_thr(f.hbd, uac);
        int vac = yac + fp->quant_vac_delta + 8 * fp->deblock_delta_q_v;
        lut[1][0][i] = deblock_quant_thr(f.hbd, vac);
        lut[1][1][i] = deblock_side_thr(f.hbd, vac);
    }
}

/* deblock.rs:81-210 filter_choice_bd */
int filter_choice(const pixel *buf, ptrdiff_t s, ptrdiff_t t, ptrdiff_t stride, int max_width_neg,
                  int max_width_pos, uint32_t q_thr, uint32_t side_thr) {
#define AT(off) ((int)buf[(off)])
    uint32_t sd[4];
    for (int dist = -2; dist < 2; dist++) {
        ptrdiff_t d = dist;
        uint32_t ds = uabs(AT(s + (d - 1) * stride) - AT(s + d * stride) * 2 + AT(s + (d + 1) * stride));
        uint32_t dt = uabs(AT(t + (d - 1) * stride) - AT(t + d * stride) * 2 + AT(t + (d + 1) * stride));
        sd[dist + 2] = (ds + dt + 1) >> 1;
    }
    uint32_t high_deriv = sd[0] > sd[3] ? sd[0] : sd[3];
    if (high_deriv > side_thr) return 0;
    if (max_width_pos == 1) return 1;

    uint32_t side_thr2 = side_thr >> 2;
    uint32_t transition = sd[1] + sd[2];
    if (high_deriv > side_thr2) return 1;
    if (transition > q_thr * 4) return 1;

    uint32_t side_thr3 = side_thr >> 3;
    if (high_deriv > side_thr3) return 2;
    if (transition > q_thr * 3) return 2;

    uint32_t end_thr = (side_thr * 3) >> 4;
    if (max_width_neg >= 3) {
        uint32_t ds = uabs(AT(s - stride) - AT(s - 4 * stride) - 3 * (AT(s - stride) - AT(s - 2 * stride)));
        uint32_t dt = uabs(AT(t - stride) - AT(t - 4 * stride) - 3 * (AT(t - stride) - AT(t - 2 * stride)));
        if (((ds + dt + 1) >> 1) > end_thr) return 2;
    }
    {
        uint32_t ds = uabs(AT(s) - AT(s + 3 * stride) - 3 * (AT(s) - AT(s + stride)));
        uint32_t dt = uabs(AT(t) - AT(t + 3 * stride) - 3 * (AT(t) - AT(t + stride)));
        if (((ds + dt + 1) >> 1) > end_thr) return 2;
    }
    if (max_width_pos == 3) return 3;

    transition <<= 4;
    int prev_dist = 3;
    for (int dist = 4; dist <= max_width_pos; dist += 2) {
        uint32_t q_thr4 = q_thr * (uint32_t)Q_FIRST[(dist - 4) >> 1];
        uint32_t end_thr4 = (side_thr * (uint32_t)dist) >> 4;
        if (transition > q_thr4) return prev_dist;
        int dist2 = imin(7, dist);
        if (max_width_neg >= dist2) {
            uint32_t ds = uabs(AT(s - stride) - AT(s + (-(ptrdiff_t)dist2 - 1) * stride) -
                               dist2 * (AT(s - stride) - AT(s - 2 * stride)));
            uint32_t dt = uabs(AT(t - stride) - AT(t + (-(ptrdiff_t)dist2 - 1) * stride) -
                               dist2 * (AT(t - stride) - AT(t - 2 * stride)));
            if (((ds + dt + 1) >> 1) > end_thr4) return prev_dist;
        }
        uint32_t ds = uabs(AT(s) - AT(s + dist2 * stride) - dist2 * (AT(s) - AT(s + stride)));
        uint32_t dt = uabs(AT(t) - AT(t + dist2 * stride) - dist2 * (AT(t) - AT(t + stride)));
        if (((ds + dt + 1) >> 1) > end_thr4) return prev_dist;
        prev_dist = dist;
    }
    return max_width_pos;
#undef AT
}

/* deblock.rs:217-281 deblock_bd */
static void deblock_bd(const BD &bd, pixel *dst, ptrdiff_t off, uint32_t q_thr, uint32_t side_thr,
                       ptrdiff_t stridea, ptrdiff_t strideb, int max_width_pos, int max_width_neg,
                       bool pos_lossless, bool neg_lossless) {
    int bdmax = bd.bdmax();
    int width = filter_choice(dst, off, off + 3 * stridea, strideb, max_width_neg, max_width_pos,
                              q_thr, side_thr);
    int width_neg = imin(width, max_width_neg);
    int width_pos = width;
    if (width_pos < 1) return;
    int q_thr_clamp = (int)q_thr * Q_THRESH_MULTS[width - 1];
    ptrdiff_t dp = off;
    for (int l = 0; l < 4; l++) {
        int d0 = dst[dp], dm1 = dst[dp - strideb], dp1 = dst[dp + strideb],
            dm2 = dst[dp - 2 * strideb];
        int delta_m2 = iclip(4 * (3 * (d0 - dm1) - (dp1 - dm2)), -q_thr_clamp, q_thr_clamp);
        if (!neg_lossless) {
            int delta_m2_neg = delta_m2 * W_MULT[width_neg - 1];
            for (int j = 0; j < width_neg; j++) {
                ptrdiff_t idx = dp + (-(ptrdiff_t)j - 1) * strideb;
                int diff = (delta_m2_neg * (width_neg - j) + (1 << 10)) >> 11;
                dst[idx] = bd.store(iclip(dst[idx] + diff, 0, bdmax));
            }
        }
        if (!pos_lossless) {
            int delta_m2_pos = delta_m2 * W_MULT[width_pos - 1];
            for (int j = 0; j < width_pos; j++) {
                ptrdiff_t idx = dp + (ptrdiff_t)j * strideb;
                int diff = (delta_m2_pos * (width_pos - j) + (1 << 10)) >> 11;
                dst[idx] = bd.store(iclip(dst[idx] - diff, 0, bdmax));
            }
        }
        dp += stridea;
    }
}

/* deblock.rs:303-348 deblock_h_sb64y_bd (vertical edge, walks y bits);
 * :371-416 deblock_v_sb64y_bd (horizontal edge, walks x bits);
 * :439-482 / :505-548 the chroma twins.  `luma` picks the width table and
 * the edge clamp (6 for luma, 2 for chroma); `vert` the walk direction. */
static void deblock_sb64(const BD &bd, pixel *dst, ptrdiff_t dst_off, ptrdiff_t stride,
                         const uint16_t *vmask, const uint16_t *ll_mask, const uint16_t *q_thr,
                         const uint16_t *side_thr, bool edge, bool luma, bool vert) {
    uint32_t vm = (uint32_t)vmask[0] | vmask[1] | vmask[2] | (luma ? vmask[3] : 0);
    uint32_t y = 1;
    ptrdiff_t dp = dst_off;
    size_t qi = 0;
    while ((vm & ~(y - 1)) != 0) {
        if (vm & y) {
            int idx;
            if (luma) {
                idx = (vmask[3] & y) ? 3 : (vmask[2] & y) ? 2 : ((vmask[1] & y) != 0);
            } else {
                idx = (vmask[2] & y) ? 2 : ((vmask[1] & y) != 0);
            }
            int max_width_pos = luma ? MAX_WIDTH_Y[idx] : MAX_WIDTH_UV[idx];
            int max_width_neg = edge ? imin(luma ? 6 : 2, max_width_pos) : max_width_pos;
            deblock_bd(bd, dst, dp, q_thr[qi], side_thr[qi], vert ? stride : 1, vert ? 1 : stride,
                       max_width_pos, max_width_neg, (ll_mask[1] & y) != 0, (ll_mask[0] & y) != 0);
        }
        y <<= 1;
        dp += vert ? 4 * stride : 4;
        qi++;
    }
}

/* lf_mask.rs:344-358 transpose_lossless_mask */
static void transpose_lossless_mask(uint16_t dst_mask[17], const uint16_t (*src_mask)[4], int x64,
                                    int ss_hor, int ss_ver) {
    dst_mask[0] = dst_mask[16 >> ss_hor];
    for (int x = 0; x < (16 >> ss_hor); x++) {
        uint32_t col_mask = 0;
        for (int y = 0; y < (16 >> ss_ver); y++) col_mask |= (uint32_t)(1 & (src_mask[y][x64] >> x)) << y;
        dst_mask[x + 1] = (uint16_t)col_mask;
    }
}

static const uint8_t PLACEHOLDER_SEGMAP[16] = {0};

/* deblock.rs:1466-1473 edge_thr */
static inline int edge_thr(int cur, int prev) {
    return (cur != 0 && prev != 0) ? (cur + prev + 1) >> 1 : (cur | prev);
}

/* deblock.rs:1477-1515 setup_thr_cols */
static void setup_thr_cols(uint16_t q_thr_dst[256], uint16_t side_thr_dst[256], const uint8_t *segmap,
                           ptrdiff_t seg_off, ptrdiff_t seg_stride, const uint16_t (*mask)[5][4],
                           int bx4_base, const uint32_t thr_lut[2][16], uint16_t left_q_thr[16],
                           uint16_t left_side_thr[16], int y64, int ss_ver, int w4, int h4) {
    int mask_idx = y64 >> ss_ver;
    uint32_t mask_shift = (y64 & ss_ver) ? 8 : 0;
    for (int y4 = 0; y4 < h4; y4++) {
        int prev_q = left_q_thr[y4], prev_s = left_side_thr[y4];
        for (int x4 = 0; x4 < w4; x4++) {
            int seg_id = segmap[seg_off + x4 + y4 * seg_stride];
            int cur_q = (int)thr_lut[0][seg_id], cur_s = (int)thr_lut[1][seg_id];
            int subpu = 3 * ((mask[bx4_base + x4][4][mask_idx] >> (mask_shift + y4)) & 1);
            q_thr_dst[x4 * 16 + y4] = (uint16_t)(edge_thr(cur_q, prev_q) >> subpu);
            side_thr_dst[x4 * 16 + y4] = (uint16_t)(edge_thr(cur_s, prev_s) >> subpu);
            prev_q = cur_q;
            prev_s = cur_s;
        }
        left_q_thr[y4] = (uint16_t)prev_q;
        left_side_thr[y4] = (uint16_t)prev_s;
    }
}

/* deblock.rs:1519-1567 setup_thr_rows */
static void setup_thr_rows(uint16_t q_thr_dst[256], uint16_t side_thr_dst[256], const uint8_t *segmap,
                           ptrdiff_t seg_off, ptrdiff_t seg_stride, const uint16_t (*mask)[5][4],
                           int starty4, const uint32_t thr_lut[2][16], const uint32_t (*above_lut)[16],
                           const uint8_t *aseg, ptrdiff_t aoff, int sb64x, int ss_hor, int w4, int h4) {
    int mask_idx = sb64x >> ss_hor;
    uint32_t mask_shift = (sb64x & ss_hor) ? 8 : 0;
    uint16_t above_q[16] = {0}, above_s[16] = {0};
    if (above_lut && aseg) {
        for (int x4 = 0; x4 < w4; x4++) {
            int seg_id = aseg[aoff + x4];
            above_q[x4] = (uint16_t)above_lut[0][seg_id];
            above_s[x4] = (uint16_t)above_lut[1][seg_id];
        }
    }
    for (int x4 = 0; x4 < w4; x4++) {
        int prev_q = above_q[x4], prev_s = above_s[x4];
        for (int y4 = 0; y4 < h4; y4++) {
            int seg_id = segmap[seg_off + x4 + y4 * seg_stride];
            int cur_q = (int)thr_lut[0][seg_id], cur_s = (int)thr_lut[1][seg_id];
            int subpu = 3 * ((mask[starty4 + y4][4][mask_idx] >> (mask_shift + x4)) & 1);
            q_thr_dst[x4 + y4 * 16] = (uint16_t)(edge_thr(cur_q, prev_q) >> subpu);
            side_thr_dst[x4 + y4 * 16] = (uint16_t)(edge_thr(cur_s, prev_s) >> subpu);
            prev_q = cur_q;
            prev_s = cur_s;
        }
    }
}

/* deblock.rs:1572-1606 deblock_crop_bottom_edge */
void deblock_crop_bottom_edge(Frame &f, size_t mask_row, int sby) {
    int sb128 = f.fp->sb128;
    int y64_start = sby << sb128;
    int y64_end = imin((sby + 1) << sb128, (f.bh + 15) >> 4);
    for (int y64 = y64_start; y64 < y64_end; y64++) {
        if ((y64 + 1) * 16 + 4 <= f.bh) continue;
        int starty4 = (y64 * 16) & 0x30;
        int h4 = imin(f.bh - y64 * 16, 16);
        int luma_crop_y4 = starty4 + h4 - 2;
        if (luma_crop_y4 < 0) continue;
        for (int x256 = 0; x256 < f.sb256w; x256++) {
            if (mask_row + x256 >= f.mask.size()) break;
            int w = imin(64, f.bw - x256 * 64);
            uint16_t(*yv)[4] = f.mask[mask_row + x256].filter_y[1][luma_crop_y4];
            for (int i = 0; i < ((w + 15) >> 4); i++) {
                uint16_t m = yv[3][i];
                yv[3][i] = 0;
                yv[2][i] |= m;
            }
        }
    }
}

/* deblock.rs:1620-1863 deblock64_cols (single tile) */
static void deblock64_cols(Frame &f, size_t lflvl_row, ptrdiff_t y_off, ptrdiff_t uv_off, int y64) {
    const R2gFrameParams *fp = f.fp;
    int starty4 = (y64 * 16) & 0x30;
    int h4 = imin(f.bh - y64 * 16, 16);
    int uv_h4 = h4 >> SS_VER;
    int y64idx = (y64 & 3) << 2;
    ptrdiff_t seg_stride = f.segmap ? f.b4_stride : 0;
    ptrdiff_t seg_band = f.segmap ? (ptrdiff_t)y64 * 16 * seg_stride : 0;
    int n64 = (f.bw + 15) >> 4;

    if (fp->deblock_level_y[0] != 0) {
        int l_qidx = -1;
        uint32_t lut[2][16] = {{0}};
        uint16_t left_q[16] = {0}, left_s[16] = {0};
        uint16_t ll_mask[17] = {0};
        for (int x64 = 0; x64 < n64; x64++) {
            bool have_left = x64 > 0;
            size_t col = lflvl_row + (x64 >> 2);
            if (col >= f.mask.size()) break;
            const R2gAv2Filter &lf = f.mask[col];
            int cur_qidx = lf.qidx[(x64 & 3) + y64idx];
            if (cur_qidx != l_qidx) {
                init_lut_y(f, 0, cur_qidx, lut);
                l_qidx = cur_qidx;
            }
            int bx4_base = (x64 & 3) * 16;
            int w4 = imin(f.bw - x64 * 16, 16);
            uint16_t q_thr[256] = {0}, side_thr[256] = {0};
            const uint8_t *seg = f.segmap ? f.segmap : PLACEHOLDER_SEGMAP;
            ptrdiff_t seg_off = f.segmap ? seg_band + (ptrdiff_t)x64 * 16 : 0;
            setup_thr_cols(q_thr, side_thr, seg, seg_off, seg_stride, lf.filter_y[0], bx4_base, lut,
                           left_q, left_s, y64 & 3, 0, w4, h4);
            transpose_lossless_mask(ll_mask, &lf.lossless_mask_y[starty4], x64 & 3, 0, 0);
            ptrdiff_t cur_off = y_off + (ptrdiff_t)x64 * 64;
            int sb64y = y64 & 3;
            for (int x = 0; x < w4; x++) {
                if (!have_left && x == 0) continue;
                const uint16_t(*hmask)[4] = lf.filter_y[0][bx4_base + x];
                uint16_t vmask[4] = {hmask[0][sb64y], hmask[1][sb64y], hmask[2][sb64y], hmask[3][sb64y]};
                uint16_t llm[2] = {ll_mask[x], ll_mask[x + 1]};
                deblock_sb64(f.bd, f.p[0], cur_off + x * 4, f.stride[0], vmask, llm, &q_thr[x * 16],
                             &side_thr[x * 16], false, true, true);
            }
        }
    }

    if (fp->deblock_level_u == 0 && fp->deblock_level_v == 0) return;

    ptrdiff_t uv_seg_stride = f.segmap_uv ? f.uv_segmap_stride : 0;
    ptrdiff_t uv_seg_band = f.segmap_uv ? (ptrdiff_t)y64 * (16 >> SS_VER) * uv_seg_stride : 0;
    int prev_qidx = -1;
    uint32_t lut[2][2][16] = {{{0}}};
    uint16_t left_q[2][16] = {{0}}, left_s[2][16] = {{0}};
    uint16_t ll_mask[17] = {0};
    bool apply_u = fp->deblock_level_u != 0, apply_v = fp->deblock_level_v != 0;
    for (int x64 = 0; x64 < n64; x64++) {
        bool have_left = x64 > 0;
        size_t col = lflvl_row + (x64 >> 2);
        if (col >= f.mask.size()) break;
        const R2gAv2Filter &lf = f.mask[col];
        int cur_qidx = lf.qidx[(x64 & 3) + y64idx];
        if (cur_qidx != prev_qidx) {
            init_lut_uv(f, cur_qidx, lut);
            prev_qidx = cur_qidx;
        }
        int bx4_base = ((x64 & 3) * 16) >> SS_HOR;
        int uv_w4 = imin(f.bw - x64 * 16, 16) >> SS_HOR;
        const uint8_t *seg = f.segmap_uv ? f.segmap_uv : PLACEHOLDER_SEGMAP;
        ptrdiff_t seg_off = f.segmap_uv ? uv_seg_band + (ptrdiff_t)x64 * (16 >> SS_HOR) : 0;
        uint16_t q_thr[2][256] = {{0}}, side_thr[2][256] = {{0}};
        for (int pl = 0; pl < 2; pl++)
            setup_thr_cols(q_thr[pl], side_thr[pl], seg, seg_off, uv_seg_stride, lf.filter_uv[0],
                           bx4_base, lut[pl], left_q[pl], left_s[pl], y64 & 3, SS_VER, uv_w4, uv_h4);
        transpose_lossless_mask(ll_mask, &lf.lossless_mask_uv[starty4 >> SS_VER], x64 & 3, SS_HOR, SS_VER);
        ptrdiff_t cur_off = uv_off + (ptrdiff_t)x64 * (64 >> SS_HOR);
        int mask_idx = (y64 & 3) >> SS_VER;
        uint32_t mask_shift = ((y64 & 3) & SS_VER) ? 8 : 0;
        uint32_t bytes_mask = SS_VER ? 0xff : 0xffff;
        for (int x = 0; x < uv_w4; x++) {
            if (!have_left && x == 0) continue;
            const uint16_t(*hmask)[4] = lf.filter_uv[0][bx4_base + x];
            uint16_t vmask[4] = {(uint16_t)((hmask[0][mask_idx] >> mask_shift) & bytes_mask),
                                 (uint16_t)((hmask[1][mask_idx] >> mask_shift) & bytes_mask),
                                 (uint16_t)((hmask[2][mask_idx] >> mask_shift) & bytes_mask), 0};
            uint16_t llm[2] = {ll_mask[x], ll_mask[x + 1]};
            if (apply_u)
                deblock_sb64(f.bd, f.p[1], cur_off + x * 4, f.stride[1], vmask, llm, &q_thr[0][x * 16],
                             &side_thr[0][x * 16], false, false, true);
            if (apply_v)
                deblock_sb64(f.bd, f.p[2], cur_off + x * 4, f.stride[1], vmask, llm, &q_thr[1][x * 16],
                             &side_thr[1][x * 16], false, false, true);
        }
    }
}

/* deblock.rs:1866-2141 deblock64_rows (single tile) */
static void deblock64_rows(Frame &f, size_t lflvl_row, ptrdiff_t y_off, ptrdiff_t uv_off, int y64) {
    const R2gFrameParams *fp = f.fp;
    bool have_top = y64 > 0;
    int starty4 = (y64 * 16) & 0x30;
    int h4 = imin(f.bh - y64 * 16, 16);
    int uv_h4 = h4 >> SS_VER;
    int y64idx = (y64 & 3) << 2;
    int a_y64idx = ((y64 + 3) & 3) << 2;
    bool have_arow = false;
    size_t a_row = 0;
    if (have_top) {
        size_t above = starty4 == 0 ? (size_t)f.sb256w : 0;
        if (lflvl_row >= above) {
            have_arow = true;
            a_row = lflvl_row - above;
        }
    }
    ptrdiff_t seg_stride = f.segmap ? f.b4_stride : 0;
    ptrdiff_t seg_band = f.segmap ? (ptrdiff_t)y64 * 16 * seg_stride : 0;
    int n64 = (f.bw + 15) >> 4;

    if (fp->deblock_level_y[1] != 0) {
        int l_qidx = -1, al_qidx = -1;
        uint32_t lut[2][16] = {{0}}, a_lut[2][16] = {{0}};
        uint16_t ll_mask[17] = {0};
        for (int x64 = 0; x64 < n64; x64++) {
            size_t col = lflvl_row + (x64 >> 2);
            if (col >= f.mask.size()) break;
            const R2gAv2Filter &lf = f.mask[col];
            for (int y = 0; y < h4; y++) ll_mask[y + 1] = lf.lossless_mask_y[starty4 + y][x64 & 3];
            int cur_qidx = lf.qidx[(x64 & 3) + y64idx];
            if (cur_qidx != l_qidx) {
                init_lut_y(f, 1, cur_qidx, lut);
                l_qidx = cur_qidx;
            }
            const uint8_t *aseg = NULL;
            ptrdiff_t aoff = 0;
            const uint32_t(*above_lut)[16] = NULL;
            if (have_arow) {
                size_t acol = a_row + (x64 >> 2);
                if (acol < f.mask.size()) {
                    const R2gAv2Filter &al = f.mask[acol];
                    ll_mask[0] = al.lossless_mask_y[(starty4 + 63) & 63][x64 & 3];
                    int a_qidx = al.qidx[(x64 & 3) + a_y64idx];
                    if (a_qidx != al_qidx) {
                        init_lut_y(f, 1, a_qidx, a_lut);
                        al_qidx = a_qidx;
                    }
                    above_lut = a_lut;
                    if (f.segmap) {
                        aseg = f.segmap;
                        aoff = seg_band + (ptrdiff_t)x64 * 16 - seg_stride;
                    } else {
                        aseg = PLACEHOLDER_SEGMAP;
                        aoff = 0;
                    }
                }
            }
            int w4 = imin(f.bw - x64 * 16, 16);
            uint16_t q_thr[256] = {0}, side_thr[256] = {0};
            const uint8_t *seg = f.segmap ? f.segmap : PLACEHOLDER_SEGMAP;
            ptrdiff_t seg_off = f.segmap ? seg_band + (ptrdiff_t)x64 * 16 : 0;
            setup_thr_rows(q_thr, side_thr, seg, seg_off, seg_stride, lf.filter_y[1], starty4, lut,
                           above_lut, aseg, aoff, x64 & 3, 0, w4, h4);
            ptrdiff_t cur_off = y_off + (ptrdiff_t)x64 * 64;
            for (int y = 0; y < h4; y++) {
                if (!have_top && y == 0) continue;
                const uint16_t(*row)[4] = lf.filter_y[1][starty4 + y];
                uint16_t vmask[4] = {row[0][x64 & 3], row[1][x64 & 3], row[2][x64 & 3], row[3][x64 & 3]};
                uint16_t llm[2] = {ll_mask[y], ll_mask[y + 1]};
                deblock_sb64(f.bd, f.p[0], cur_off + (ptrdiff_t)y * 4 * f.stride[0], f.stride[0], vmask,
                             llm, &q_thr[y * 16], &side_thr[y * 16], y == 0, true, false);
            }
        }
    }

    if (fp->deblock_level_u == 0 && fp->deblock_level_v == 0) return;

    ptrdiff_t uv_seg_stride = f.segmap_uv ? f.uv_segmap_stride : 0;
    ptrdiff_t uv_seg_band = f.segmap_uv ? (ptrdiff_t)y64 * (16 >> SS_VER) * uv_seg_stride : 0;
    int l_qidx = -1, al_qidx = -1;
    uint32_t lut[2][2][16] = {{{0}}}, a_lut[2][2][16] = {{{0}}};
    uint16_t ll_mask[17] = {0};
    bool apply_u = fp->deblock_level_u != 0, apply_v = fp->deblock_level_v != 0;
    for (int x64 = 0; x64 < n64; x64++) {
        size_t col = lflvl_row + (x64 >> 2);
        if (col >= f.mask.size()) break;
        const R2gAv2Filter &lf = f.mask[col];
        for (int y = 0; y < uv_h4; y++) ll_mask[y + 1] = lf.lossless_mask_uv[(starty4 >> SS_VER) + y][x64 & 3];
        int cur_qidx = lf.qidx[(x64 & 3) + y64idx];
        if (cur_qidx != l_qidx) {
            init_lut_uv(f, cur_qidx, lut);
            l_qidx = cur_qidx;
        }
        const uint8_t *aseg = NULL;
        ptrdiff_t aoff = 0;
        bool above_present = false;
        if (have_arow) {
            size_t acol = a_row + (x64 >> 2);
            if (acol < f.mask.size()) {
                const R2gAv2Filter &al = f.mask[acol];
                ll_mask[0] = al.lossless_mask_uv[((starty4 + 63) & 63) >> SS_VER][x64 & 3];
                int a_qidx = al.qidx[(x64 & 3) + a_y64idx];
                if (a_qidx != al_qidx) {
                    init_lut_uv(f, a_qidx, a_lut);
                    al_qidx = a_qidx;
                }
                above_present = true;
                if (f.segmap_uv) {
                    aseg = f.segmap_uv;
                    aoff = uv_seg_band + (ptrdiff_t)x64 * (16 >> SS_HOR) - uv_seg_stride;
                } else {
                    aseg = PLACEHOLDER_SEGMAP;
                    aoff = 0;
                }
            }
        }
        int uv_w4 = imin(f.bw - x64 * 16, 16) >> SS_HOR;
        const uint8_t *seg = f.segmap_uv ? f.segmap_uv : PLACEHOLDER_SEGMAP;
        ptrdiff_t seg_off = f.segmap_uv ? uv_seg_band + (ptrdiff_t)x64 * (16 >> SS_HOR) : 0;
        uint16_t q_thr[2][256] = {{0}}, side_thr[2][256] = {{0}};
        for (int pl = 0; pl < 2; pl++)
            setup_thr_rows(q_thr[pl], side_thr[pl], seg, seg_off, uv_seg_stride, lf.filter_uv[1],
                           starty4 >> SS_VER, lut[pl], above_present ? a_lut[pl] : NULL, aseg, aoff,
                           x64 & 3, SS_HOR, uv_w4, uv_h4);
        ptrdiff_t cur_off = uv_off + (ptrdiff_t)x64 * (64 >> SS_HOR);
        int mask_idx = (x64 & 3) >> SS_HOR;
        uint32_t mask_shift = ((x64 & 3) & SS_HOR) ? 8 : 0;
        uint32_t bytes_mask = SS_HOR ? 0xff : 0xffff;
        for (int y = 0; y < uv_h4; y++) {
            if (!have_top && y == 0) continue;
            const uint16_t(*row)[4] = lf.filter_uv[1][(starty4 >> SS_VER) + y];
            uint16_t vmask[4] = {(uint16_t)((row[0][mask_idx] >> mask_shift) & bytes_mask),
                                 (uint16_t)((row[1][mask_idx] >> mask_shift) & bytes_mask),
                                 (uint16_t)((row[2][mask_idx] >> mask_shift) & bytes_mask), 0};
            uint16_t llm[2] = {ll_mask[y], ll_mask[y + 1]};
            ptrdiff_t o = cur_off + (ptrdiff_t)y * 4 * f.stride[1];
            if (apply_u)
                deblock_sb64(f.bd, f.p[1], o, f.stride[1], vmask, llm, &q_thr[0][y * 16],
                             &side_thr[0][y * 16], y == 0, false, false);
            if (apply_v)
                deblock_sb64(f.bd, f.p[2], o, f.stride[1], vmask, llm, &q_thr[1][y * 16],
                             &side_thr[1][y * 16], y == 0, false, false);
        }
    }
}

/* deblock.rs:2145-2168 deblock_sbrow_cols */
void deblock_sbrow_cols(Frame &f, size_t mask_row, int sby) {
    int sb128 = f.fp->sb128;
    int y64_start = sby << sb128;
    int y64_end = imin((sby + 1) << sb128, (f.bh + 15) >> 4);
    int sb_step = 16 << sb128;
    ptrdiff_t y_off = (ptrdiff_t)(sby * sb_step * 4) * f.stride[0];
    ptrdiff_t uv_off = ((ptrdiff_t)(sby * sb_step * 4) * f.stride[1]) >> SS_VER;
    for (int y64 = y64_start; y64 < y64_end; y64++) {
        deblock64_cols(f, mask_row, y_off, uv_off, y64);
        y_off += 64 * f.stride[0];
        uv_off += (64 * f.stride[1]) >> SS_VER;
    }
}

/* deblock.rs:2171-2190 deblock_sbrow_rows */
void deblock_sbrow_rows(Frame &f, size_t mask_row, int sby) {
    int sb128 = f.fp->sb128;
    int y64_start = sby << sb128;
    int y64_end = imin((sby + 1) << sb128, (f.bh + 15) >> 4);
    int sb_step = 16 << sb128;
    ptrdiff_t y_off = (ptrdiff_t)(sby * sb_step * 4) * f.stride[0];
    ptrdiff_t uv_off = ((ptrdiff_t)(sby * sb_step * 4) * f.stride[1]) >> SS_VER;
    for (int y64 = y64_start; y64 < y64_end; y64++) {
        deblock64_rows(f, mask_row, y_off, uv_off, y64);
        y_off += 64 * f.stride[0];
        uv_off += (64 * f.stride[1]) >> SS_VER;
    }
}

/* deblock.rs:688-729 backup_db (the filter pass runs it with n_tc = 1) */
void backup_db(pixel *dst, const pixel *src, ptrdiff_t stride, int ss_ver, bool sb128, int row,
               int row_h, int w, bool lr_backup, int n_tc) {
    int cdef_backup = !lr_backup;
    int sb128_i = sb128;
    int stripe_h = ((64 << (cdef_backup & sb128_i)) - 8 * (row == 0)) >> ss_ver;
    ptrdiff_t src_off = (ptrdiff_t)(stripe_h - 2) * stride;
    ptrdiff_t dst_off = 0;
    if (n_tc == 1) {
        if (row > 0) {
            int top = 4 << sb128_i;
            for (int i = 0; i < 4; i++)
                memmove(dst + dst_off + i * stride, dst + dst_off + (top + i) * stride, w * sizeof(pixel));
        }
        dst_off += 4 * stride;
    }
    while (row + stripe_h <= row_h) {
        for (int i = 0; i < 4; i++) {
            memcpy(dst + dst_off, src + src_off, w * sizeof(pixel));
            dst_off += stride;
            src_off += stride;
        }
        row += stripe_h;
        stripe_h = 64 >> ss_ver;
        src_off += (ptrdiff_t)(stripe_h - 4) * stride;
    }
}

/* deblock.rs:2192-2264 copy_db */
void copy_db(Frame &f, int sby) {
    bool sb128 = f.fp->sb128 != 0;
    int h = f.bh * 4;
    int w = f.bw * 4;
    int offset = 8 * (sby != 0);
    int y_stripe = (sby << (6 + sb128)) - offset;
    int row_h = imin((sby + 1) << (6 + sb128), h - 1);
    bool lr_backup = f.restore_planes != 0;
    if (y_stripe < row_h)
        backup_db(f.lr_db_line[0].data(), f.p[0] + (ptrdiff_t)y_stripe * f.stride[0], f.stride[0], 0,
                  sb128, y_stripe, row_h, w, lr_backup, 1);
    if (f.stride[1] != 0) {
        int cw = w >> SS_HOR;
        int ch = (f.bh * 4) >> SS_VER;
        int offset_uv = offset >> SS_VER;
        int cy_stripe = (sby << ((6 - SS_VER) + sb128)) - offset_uv;
        int crow_h = imin((sby + 1) << ((6 - SS_VER) + sb128), ch - 1);
        if (cy_stripe < crow_h) {
            ptrdiff_t o = (ptrdiff_t)cy_stripe * f.stride[1];
            backup_db(f.lr_db_line[1].data(), f.p[1] + o, f.stride[1], SS_VER, sb128, cy_stripe,
                      crow_h, cw, lr_backup, 1);
            backup_db(f.lr_db_line[2].data(), f.p[2] + o, f.stride[1], SS_VER, sb128, cy_stripe,
                      crow_h, cw, lr_backup, 1);
        }
    }
}

}  // namespace r2o

/* ---- known-answer-test hooks (the reference's deblock.rs unit tests) ---- */
extern "C" {
void r2o_setup_thr_cols(uint16_t *q_thr, uint16_t *side_thr, const uint8_t *segmap, int64_t seg_stride,
                        const uint16_t *mask_x4_5_4, const uint32_t *thr_lut_2x16, uint16_t *left_q,
                        uint16_t *left_side, int y64, int ss_ver, int w4, int h4) {
    r2o::setup_thr_cols(q_thr, side_thr, segmap, 0, seg_stride, (const uint16_t(*)[5][4])mask_x4_5_4, 0,
                        (const uint32_t(*)[16])thr_lut_2x16, left_q, left_side, y64, ss_ver, w4, h4);
}
void r2o_backup_db(uint16_t *dst, const uint16_t *src, int64_t stride, int ss_ver, int sb128, int row, int row_h,
                   int w, int lr_backup, int n_tc) {
    r2o::backup_db(dst, src, stride, ss_ver, sb128 != 0, row, row_h, w, lr_backup != 0, n_tc);
}
/* deblock.rs:6-11 constant tables: which 0 MAX_WIDTH_Y, 1 MAX_WIDTH_UV,
 * 2 Q_FIRST, 3 Q_THRESH_MULTS, 4 W_MULT; i = -1 gives the length */
int r2o_deblock_const(int which, int i) {
    using namespace r2o;
    switch (which) {
        case 0: return i < 0 ? 4 : MAX_WIDTH_Y[i];
        case 1: return i < 0 ? 3 : MAX_WIDTH_UV[i];
        case 2: return i < 0 ? 3 : Q_FIRST[i];
        case 3: return i < 0 ? 8 : Q_THRESH_MULTS[i];
        case 4: return i < 0 ? 8 : W_MULT[i];
    }
    return 0;
}
/* deblock.rs:13-33 / :35-57: lut [2][16] (y) or [2][2][16] (uv) */
void r2o_init_deblock_thr_lut_y(const R2gFrameParams *fp, int hbd, int dir, int qidx, uint32_t *lut) {
    r2o::Frame f;
    f.fp = fp;
    f.hbd = hbd;
    r2o::init_lut_y(f, dir, qidx, (uint32_t(*)[16])lut);
}
void r2o_init_deblock_thr_lut_uv(const R2gFrameParams *fp, int hbd, int qidx, uint32_t *lut) {
    r2o::Frame f;
    f.fp = fp;
    f.hbd = hbd;
    r2o::init_lut_uv(f, qidx, (uint32_t(*)[2][16])lut);
}
/* deblock.rs:303-548 deblock_{h,v}_sb64{y,uv}_bd: luma/chroma, vert = the
 * h (vertical edge) variants */
void r2o_deblock_sb64(uint16_t *dst, int64_t dst_off, int64_t stride, const uint16_t *vmask, const uint16_t *ll_mask,
                      const uint16_t *q_thr, const uint16_t *side_thr, int edge, int luma, int vert, int bitdepth) {
    r2o::BD bd;
    bd.bitdepth = bitdepth;
    r2o::deblock_sb64(bd, dst, dst_off, stride, vmask, ll_mask, q_thr, side_thr, edge != 0, luma != 0, vert != 0);
}
/* lf_mask.rs:344-358 transpose_lossless_mask; src is [rows][4] */
void r2o_transpose_lossless_mask(uint16_t *dst17, const uint16_t *src_x4, int x64, int ss_hor, int ss_ver) {
    r2o::transpose_lossless_mask(dst17, (const uint16_t(*)[4])src_x4, x64, ss_hor, ss_ver);
}
/* deblock.rs:1519-1567 setup_thr_rows (dst stride 16); above_lut NULL: no
 * row above; its segment ids are read at seg_off - seg_stride */
void r2o_setup_thr_rows(uint16_t *q_thr, uint16_t *side_thr, const uint8_t *segmap, int64_t seg_off,
                        int64_t seg_stride, const uint16_t *mask_x4_5_4, const uint32_t *thr_lut_2x16,
                        const uint32_t *above_lut_2x16, int sb64x, int ss_hor, int w4, int h4) {
    r2o::setup_thr_rows(q_thr, side_thr, segmap, seg_off, seg_stride, (const uint16_t(*)[5][4])mask_x4_5_4, 0,
                        (const uint32_t(*)[16])thr_lut_2x16, (const uint32_t(*)[16])above_lut_2x16,
                        above_lut_2x16 ? segmap : nullptr, seg_off - seg_stride, sb64x, ss_hor, w4, h4);
}
void r2o_deblock(uint16_t *dst, int64_t off, uint32_t q_thr, uint32_t side_thr, int64_t stridea, int64_t strideb,
                 int mwp, int mwn, int pos_ll, int neg_ll, int bitdepth) {
    r2o::BD bd;
    bd.bitdepth = bitdepth;
    r2o::deblock_bd(bd, dst, off, q_thr, side_thr, stridea, strideb, mwp, mwn, pos_ll != 0, neg_ll != 0);
}
}
