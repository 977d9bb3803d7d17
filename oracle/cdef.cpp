/*
 * Oracle: CDEF with CCSO folded in, per superblock row.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Restates crates/rav2d/src/cdef.rs:1-1182 and ccso.rs:1-254 of the rav2d
 * reference, including the toggled cdef_line banks, the 2x8 left backups and
 * the prev_flag bookkeeping of cdef_brow.
 */
#include "oracle.h"

#define R2G_TABLE(type, name) static const type name
#include "av2_tables.h"

namespace r2o {

enum { HAVE_LEFT = 1, HAVE_RIGHT = 2, HAVE_TOP = 4, HAVE_BOTTOM = 8 };
enum { BACKUP_2X8_Y = 1, BACKUP_2X8_UV = 2 };

/* ccso.rs:5-13 */
static const int8_t CCSO_POS[7][2] = {{-1, 0}, {0, -1}, {-1, -1}, {-1, 1}, {-1, -2}, {1, -2}, {0, 2}};
/* cdef.rs:605 */
static const uint8_t UV_DIRS[2][8] = {{0, 1, 2, 3, 4, 5, 6, 7}, {7, 0, 2, 4, 5, 6, 6, 6}};

typedef pixel Left2[2];

/* cdef.rs:122-128 fill: INT16_MIN over a w x h rectangle */
static void fill(int16_t *tmp, ptrdiff_t stride, int w, int h) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) tmp[y * stride + x] = INT16_MIN;
}

/* cdef.rs:218-220 cdef_pri_tap */
static int cdef_pri_tap(int pri_strength) { return 4 - (pri_strength & 1); }

/* cdef.rs:243-262 backup2lines_plane: the last 2 rows of a `height`-row
 * block (for a negative stride, the rows as the reference addresses them) */
static void backup2lines_plane(pixel *dst, ptrdiff_t dst_off, const pixel *src, ptrdiff_t src_off, ptrdiff_t stride,
                               int height) {
    ptrdiff_t abs_stride = stride < 0 ? -stride : stride, len = 2 * abs_stride;
    if (stride < 0)
        memcpy(dst + dst_off + stride, src + src_off + (height - 1) * stride, sizeof(pixel) * len);
    else
        memcpy(dst + dst_off, src + src_off + (height - 2) * abs_stride, sizeof(pixel) * len);
}

/* cdef.rs:265-280 backup2x8_plane: columns x_off-2, x_off-1 of `rows` rows */
static void backup2x8_plane(Left2 *dst, const pixel *src, ptrdiff_t src_off, ptrdiff_t stride, ptrdiff_t x_off,
                            int rows) {
    ptrdiff_t off = src_off;
    for (int y = 0; y < rows; y++) {
        ptrdiff_t s = off + x_off - 2;
        dst[y][0] = src[s];
        dst[y][1] = src[s + 1];
        off += stride;
    }
}

/* cdef.rs:37-112 cdef_padding */
static void cdef_padding(int16_t *tmp, int tmp_stride, const pixel *src, ptrdiff_t src_stride,
                         ptrdiff_t src_off, const Left2 *left, const pixel *top, ptrdiff_t top_off,
                         const pixel *bottom, ptrdiff_t bottom_off, int w, int h, int edges) {
    int o = 2 * tmp_stride + 2;
    int x_start = -2, x_end = w + 2, y_start = -2, y_end = h + 2;
    if (!(edges & HAVE_TOP)) {
        fill(tmp + o - 2 - 2 * tmp_stride, tmp_stride, w + 4, 2);
        y_start = 0;
    }
    if (!(edges & HAVE_BOTTOM)) {
        fill(tmp + o + h * tmp_stride - 2, tmp_stride, w + 4, 2);
        y_end -= 2;
    }
    if (!(edges & HAVE_LEFT)) {
        fill(tmp + o + y_start * tmp_stride - 2, tmp_stride, 2, y_end - y_start);
        x_start = 0;
    }
    if (!(edges & HAVE_RIGHT)) {
        fill(tmp + o + y_start * tmp_stride + w, tmp_stride, 2, y_end - y_start);
        x_end -= 2;
    }
    ptrdiff_t toff = top_off;
    for (int y = y_start; y < 0; y++) {
        for (int x = x_start; x < x_end; x++) tmp[o + x + y * tmp_stride] = (int16_t)top[toff + x];
        toff += src_stride;
    }
    for (int y = 0; y < h; y++)
        for (int x = x_start; x < 0; x++) tmp[o + x + y * tmp_stride] = (int16_t)left[y][2 + x];
    ptrdiff_t soff = src_off;
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < x_end; x++) tmp[o + x + y * tmp_stride] = (int16_t)src[soff + x];
        soff += src_stride;
    }
    ptrdiff_t boff = bottom_off;
    for (int y = h; y < y_end; y++) {
        for (int x = x_start; x < x_end; x++) tmp[o + x + y * tmp_stride] = (int16_t)bottom[boff + x];
        boff += src_stride;
    }
}

/* cdef.rs:114-119 constrain */
int constrain(int diff, int threshold, int shift) {
    int adiff = diff < 0 ? -diff : diff;
    return apply_sign(imin(adiff, imax(0, threshold - (adiff >> shift))), diff);
}

/* cdef.rs:134-224 cdef_find_dir_bd (wrapping u32 costs) */
int cdef_find_dir(const pixel *img, ptrdiff_t stride, uint32_t *var, int bd8) {
    int hv[2][8] = {{0}}, diag[2][15] = {{0}}, alt[4][11] = {{0}};
    for (int y = 0; y < 8; y++)
        for (int x = 0; x < 8; x++) {
            int px = ((int)img[y * stride + x] >> bd8) - 128;
            diag[0][y + x] += px;
            alt[0][y + (x >> 1)] += px;
            hv[0][y] += px;
            alt[1][3 + y - (x >> 1)] += px;
            diag[1][7 + y - x] += px;
            alt[2][3 - (y >> 1) + x] += px;
            hv[1][x] += px;
            alt[3][(y >> 1) + x] += px;
        }
    auto sq = [](int v) -> uint32_t { return (uint32_t)v * (uint32_t)v; };
    uint32_t cost[8] = {0};
    for (int n = 0; n < 8; n++) {
        cost[2] += sq(hv[0][n]);
        cost[6] += sq(hv[1][n]);
    }
    cost[2] *= 105u;
    cost[6] *= 105u;
    static const uint32_t DIV_TABLE[7] = {840, 420, 280, 210, 168, 140, 120};
    for (int n = 0; n < 7; n++) {
        uint32_t d = DIV_TABLE[n];
        cost[0] += (sq(diag[0][n]) + sq(diag[0][14 - n])) * d;
        cost[4] += (sq(diag[1][n]) + sq(diag[1][14 - n])) * d;
    }
    cost[0] += sq(diag[0][7]) * 105u;
    cost[4] += sq(diag[1][7]) * 105u;
    for (int n = 0; n < 4; n++) {
        int ci = n * 2 + 1;
        for (int m = 0; m < 5; m++) cost[ci] += sq(alt[n][3 + m]);
        cost[ci] *= 105u;
        for (int m = 0; m < 3; m++) {
            uint32_t d = DIV_TABLE[2 * m + 1];
            cost[ci] += (sq(alt[n][m]) + sq(alt[n][10 - m])) * d;
        }
    }
    int best_dir = 0;
    uint32_t best_cost = cost[0];
    for (int n = 1; n < 8; n++)
        if (cost[n] > best_cost) {
            best_cost = cost[n];
            best_dir = n;
        }
    *var = (best_cost - cost[best_dir ^ 4]) >> 10;
    return best_dir;
}

/* cdef.rs:230-241 adjust_strength */
int adjust_strength(int strength, uint32_t var) {
    if (var == 0) return 0;
    int i = (var >> 6) != 0 ? imin(ulog2(var >> 6), 12) : 0;
    return (strength * (4 + i) + 8) >> 4;
}

/* cdef.rs:320-458 cdef_filter_block */
static void cdef_filter_block(const BD &bd, pixel *dst, ptrdiff_t dst_stride, ptrdiff_t dst_off,
                              const Left2 *left, const pixel *top, ptrdiff_t top_off,
                              const pixel *bottom, ptrdiff_t bottom_off, int pri_strength,
                              int sec_strength, int dir, int damping, int w, int h, int edges) {
    const int tmp_stride = 12;
    int16_t tmp_buf[144] = {0};
    int o = 2 * tmp_stride + 2;
    cdef_padding(tmp_buf, tmp_stride, dst, dst_stride, dst_off, left, top, top_off, bottom,
                 bottom_off, w, h, edges);
    int bd8 = bd.bd8();
    ptrdiff_t dp = dst_off;
    int tp = o;
    if (pri_strength != 0) {
        int pri_tap = 4 - ((pri_strength >> bd8) & 1);
        int pri_shift = imax(0, damping - ulog2((uint32_t)pri_strength));
        if (sec_strength != 0) {
            int sec_shift = damping - ulog2((uint32_t)sec_strength);
            for (int y = 0; y < h; y++) {
                for (int x = 0; x < w; x++) {
                    int px = dst[dp + x];
                    int sum = 0, max_v = px, min_v = px, pri_tap_k = pri_tap;
                    for (int k = 0; k < 2; k++) {
                        int off1 = CDEF_DIRECTIONS[dir + 2][k];
                        int p0 = tmp_buf[tp + x + off1], p1 = tmp_buf[tp + x - off1];
                        sum += pri_tap_k * constrain(p0 - px, pri_strength, pri_shift);
                        sum += pri_tap_k * constrain(p1 - px, pri_strength, pri_shift);
                        pri_tap_k = (pri_tap_k & 3) | 2;
                        min_v = imin(p0, min_v);
                        max_v = imax(p0, max_v);
                        min_v = imin(p1, min_v);
                        max_v = imax(p1, max_v);
                        int off2 = CDEF_DIRECTIONS[dir + 4][k], off3 = CDEF_DIRECTIONS[dir][k];
                        int s0 = tmp_buf[tp + x + off2], s1 = tmp_buf[tp + x - off2];
                        int s2 = tmp_buf[tp + x + off3], s3 = tmp_buf[tp + x - off3];
                        int sec_tap = 2 - k;
                        sum += sec_tap * constrain(s0 - px, sec_strength, sec_shift);
                        sum += sec_tap * constrain(s1 - px, sec_strength, sec_shift);
                        sum += sec_tap * constrain(s2 - px, sec_strength, sec_shift);
                        sum += sec_tap * constrain(s3 - px, sec_strength, sec_shift);
                        min_v = imin(s0, min_v);
                        max_v = imax(s0, max_v);
                        min_v = imin(s1, min_v);
                        max_v = imax(s1, max_v);
                        min_v = imin(s2, min_v);
                        max_v = imax(s2, max_v);
                        min_v = imin(s3, min_v);
                        max_v = imax(s3, max_v);
                    }
                    dst[dp + x] = bd.store(iclip(px + ((sum - (sum < 0) + 8) >> 4), min_v, max_v));
                }
                dp += dst_stride;
                tp += tmp_stride;
            }
        } else {
            for (int y = 0; y < h; y++) {
                for (int x = 0; x < w; x++) {
                    int px = dst[dp + x];
                    int sum = 0, pri_tap_k = pri_tap;
                    for (int k = 0; k < 2; k++) {
                        int off = CDEF_DIRECTIONS[dir + 2][k];
                        int p0 = tmp_buf[tp + x + off], p1 = tmp_buf[tp + x - off];
                        sum += pri_tap_k * constrain(p0 - px, pri_strength, pri_shift);
                        sum += pri_tap_k * constrain(p1 - px, pri_strength, pri_shift);
                        pri_tap_k = (pri_tap_k & 3) | 2;
                    }
                    dst[dp + x] = bd.store(px + ((sum - (sum < 0) + 8) >> 4));
                }
                dp += dst_stride;
                tp += tmp_stride;
            }
        }
    } else {
        int sec_shift = damping - ulog2((uint32_t)sec_strength);
        for (int y = 0; y < h; y++) {
            for (int x = 0; x < w; x++) {
                int px = dst[dp + x];
                int sum = 0;
                for (int k = 0; k < 2; k++) {
                    int off1 = CDEF_DIRECTIONS[dir + 4][k], off2 = CDEF_DIRECTIONS[dir][k];
                    int s0 = tmp_buf[tp + x + off1], s1 = tmp_buf[tp + x - off1];
                    int s2 = tmp_buf[tp + x + off2], s3 = tmp_buf[tp + x - off2];
                    int sec_tap = 2 - k;
                    sum += sec_tap * constrain(s0 - px, sec_strength, sec_shift);
                    sum += sec_tap * constrain(s1 - px, sec_strength, sec_shift);
                    sum += sec_tap * constrain(s2 - px, sec_strength, sec_shift);
                    sum += sec_tap * constrain(s3 - px, sec_strength, sec_shift);
                }
                dst[dp + x] = bd.store(px + ((sum - (sum < 0) + 8) >> 4));
            }
            dp += dst_stride;
            tp += tmp_stride;
        }
    }
}

/* ccso.rs:16-24 ccso_score */
uint32_t ccso_score(int diff, int quant_step, uint32_t edge_classifier) {
    if (diff > quant_step && edge_classifier == 0) return 2;
    if (diff < -quant_step) return 0;
    return 1;
}

/* ccso.rs:26-61 ccso_padding */
static void ccso_padding(pixel *tmp, int tmp_stride, int o, const pixel *src, ptrdiff_t src_stride,
                         ptrdiff_t src_off, const Left2 *left, const pixel *top, ptrdiff_t top_off,
                         const pixel *bottom, ptrdiff_t bottom_off, int w, int h, int edges) {
    int x_min = (edges & HAVE_LEFT) ? -2 : 0;
    int x_max = w - 1 + ((edges & HAVE_RIGHT) ? 2 : 0);
    int y_min = (edges & HAVE_TOP) ? -2 : 0;
    int y_max = h - 1 + ((edges & HAVE_BOTTOM) ? 2 : 0);
    for (int y = -2; y < h + 2; y++) {
        int src_y = iclip(y, y_min, y_max);
        for (int x = -2; x < w + 2; x++) {
            int src_x = iclip(x, x_min, x_max);
            pixel v;
            if (src_y < 0)
                v = top[top_off + src_x + (2 + src_y) * src_stride];
            else if (src_y >= h)
                v = bottom[bottom_off + src_x + (src_y - h) * src_stride];
            else if (src_x < 0)
                v = left[src_y][2 + src_x];
            else
                v = src[src_off + src_x + src_y * src_stride];
            tmp[o + x + y * tmp_stride] = v;
        }
    }
}

/* ccso.rs:115-185 ccso_prep */
static void ccso_prep(const BD &bd, uint8_t *dst, int dst_stride, const pixel *src,
                      ptrdiff_t src_stride, ptrdiff_t src_off, const Left2 *left, const pixel *top,
                      ptrdiff_t top_off, const pixel *bottom, ptrdiff_t bottom_off,
                      uint32_t max_band_log2, int ext_filter, int quant_step, uint32_t edge_clf,
                      bool bo_only, int edges, int w, int h, int ss_hor, int ss_ver) {
    uint32_t shift = (uint32_t)bd.bitdepth - max_band_log2;
    int dy = CCSO_POS[ext_filter][0], dx = CCSO_POS[ext_filter][1];
    const int tmp_stride = 68;
    int luma_offset = dx + dy * tmp_stride;
    std::vector<pixel> tmp((size_t)tmp_stride * (imax(h, 8) * (1 << ss_ver) + 8));
    int o = 2 * tmp_stride + 2;
    ccso_padding(tmp.data(), tmp_stride, o, src, src_stride, src_off, left, top, top_off, bottom,
                 bottom_off, w << ss_hor, h << ss_ver, edges);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int ti = o + (y << ss_ver) * tmp_stride + (x << ss_hor);
            int c = tmp[ti];
            uint8_t band = (uint8_t)((uint32_t)c >> shift);
            if (bo_only) {
                dst[y * dst_stride + x] = band;
            } else {
                uint32_t cls0 = ccso_score((int)tmp[ti + luma_offset] - c, quant_step, edge_clf);
                uint32_t cls1 = ccso_score((int)tmp[ti - luma_offset] - c, quant_step, edge_clf);
                dst[y * dst_stride + x] = (uint8_t)((cls0 << 5) | (cls1 << 3)) | band;
            }
        }
}

/* ccso.rs:215-254 ccso_add */
static void ccso_add(const BD &bd, pixel *dst, ptrdiff_t dst_stride, const uint8_t *idx_buf,
                     int idx_stride, const uint8_t *offset_idxs, const int8_t *offset_lut, int w,
                     int h, const uint16_t (*ll_mask)[4]) {
    for (int yy = 0; yy < h; yy += 4) {
        int mi = yy >> 2;
        int bx = 0;
        for (int xx = 0; xx < w; xx += 4, bx++) {
            if (ll_mask[mi][0] & (1 << bx)) continue;
            for (int y = yy; y < yy + 4; y++)
                for (int x = xx; x < xx + 4; x++) {
                    uint8_t i = idx_buf[y * idx_stride + x];
                    int byte_idx = i >> 1, half_idx = i & 1;
                    uint8_t packed = byte_idx < 64 ? offset_idxs[byte_idx] : 0;
                    int offset_idx = 7 & (packed >> (4 * half_idx));
                    int cur = dst[y * dst_stride + x];
                    dst[y * dst_stride + x] = (pixel)bd.clip(cur + offset_lut[offset_idx]);
                }
        }
    }
}

/* cdef.rs:614-646 cdef_backup2lines_bank */
static void backup2lines_bank(std::vector<pixel> bank[3], Frame &f, ptrdiff_t y_off, ptrdiff_t uv_off) {
    ptrdiff_t ys = f.stride[0], uvs = f.stride[1];
    memcpy(bank[0].data(), f.p[0] + y_off + 6 * ys, sizeof(pixel) * 2 * ys);
    ptrdiff_t s = uv_off + 2 * uvs;
    memcpy(bank[1].data(), f.p[1] + s, sizeof(pixel) * 2 * uvs);
    memcpy(bank[2].data(), f.p[2] + s, sizeof(pixel) * 2 * uvs);
}

/* cdef.rs:649-663 cdef_backup2x8: backup2x8_plane with a positive stride */
static void backup2x8(Left2 *dst, const pixel *src, ptrdiff_t base, ptrdiff_t stride, int x_off, int rows) {
    backup2x8_plane(dst, src, base, stride, x_off, rows);
}

struct CcsoPlaneCfg {
    uint32_t max_band_log2;
    int ext_filter, quant_step;
    uint32_t edge_clf;
    bool bo_only;
    int scale_idx;
    const uint8_t *filter_off;
};

/* Per-brow view of one mask row (decode.rs:4061-4114 collect_*). */
struct BrowParams {
    const R2gAv2Filter *row; /* sb256w masks of the mask row */
    int n;                   /* sb256w */
    int damping;
    bool on_skip_tx, cdef_on, any_lossless, ccso_on;
    const uint8_t *y_strength, *uv_strength;
    CcsoPlaneCfg cc[3];
};

/* cdef.rs:702-1182 cdef_brow (single-thread path) */
static void cdef_brow(Frame &f, const BrowParams &p, int by_start, int by_end) {
    const BD &bd = f.bd;
    int bd8 = bd.bd8();
    int damping = p.damping + bd8;
    ptrdiff_t y_ls = f.stride[0], uv_ls = f.stride[1];
    const int ss_hor = SS_HOR, ss_ver = SS_VER;
    const uint8_t *uv_dir = UV_DIRS[0]; /* layout != I422 */
    const int sbsz = 16;
    int sb64w = (f.bw + sbsz - 1) >> 4;
    pixel *y = f.p[0], *u = f.p[1], *v = f.p[2];

    ptrdiff_t row_y = (ptrdiff_t)by_start * 4 * y_ls;
    ptrdiff_t row_uv = (ptrdiff_t)((by_start * 4) >> ss_ver) * uv_ls;
    int edge_top = by_start > 0 ? HAVE_TOP : 0;

    for (int by = by_start; by < by_end; by += 2) {
        int tf = f.cdef_line_toggle;
        int by_idx = (by & 0x3e) >> 1;
        int edges = edge_top | HAVE_BOTTOM;
        if (by + 2 >= f.bh) edges &= ~HAVE_BOTTOM;
        if (edges & HAVE_BOTTOM) backup2lines_bank(f.cdef_line[1 - tf], f, row_y, row_uv);

        Left2 lr_bak[2][3][8];
        memset(lr_bak, 0, sizeof(lr_bak));
        int bit = 0;
        edges &= ~HAVE_LEFT;
        edges |= HAVE_RIGHT;
        uint8_t prev_flag = 0;
        ptrdiff_t sb_y = row_y, sb_uv = row_uv;
        uint8_t ccso_lut_idx[3][64 * 8];
        memset(ccso_lut_idx, 0, sizeof(ccso_lut_idx));

        for (int sbx = 0; sbx < sb64w; sbx++) {
            int sb256x = sbx >> 2;
            int sb64x_idx = sbx & 3;
            int sb64_idx = ((by & 0x30) >> 2) + (sbx & 3);
            int mask_i = imin(sb256x, p.n - 1);
            int cdef_idx = sb256x < p.n ? p.row[mask_i].cdef_idx[sb64_idx] : -1;

            /* CCSO prep (cdef.rs:800-855) */
            if (p.ccso_on) {
                const uint8_t *ccm = sb256x < p.n ? p.row[sb256x].ccso : NULL;
                uint8_t c0 = ccm ? ccm[0] : 0, c1 = ccm ? ccm[1] : 0, c2 = ccm ? ccm[2] : 0;
                uint8_t ccmv[3] = {c0, c1, c2};
                uint8_t flag = c0 | c1 | c2;
                uint8_t do_left = flag & ~prev_flag;
                prev_flag |= flag;
                if (do_left && (edges & HAVE_LEFT)) {
                    if (do_left & BACKUP_2X8_Y) backup2x8(lr_bak[bit][0], y, sb_y, y_ls, 0, 8);
                    if (do_left & BACKUP_2X8_UV) {
                        backup2x8(lr_bak[bit][1], u, sb_uv, uv_ls, 0, 8 >> ss_ver);
                        backup2x8(lr_bak[bit][2], v, sb_uv, uv_ls, 0, 8 >> ss_ver);
                    }
                }
                for (int pl = 0; pl < 3; pl++) {
                    if (ccmv[pl] == 0) continue;
                    const CcsoPlaneCfg &cfg = p.cc[pl];
                    int pl_ss_hor = pl ? ss_hor : 0, pl_ss_ver = pl ? ss_ver : 0;
                    int sb_edges = edges;
                    if ((sbx + 1) * sbsz >= f.bw) sb_edges &= ~HAVE_RIGHT;
                    int w_full = imin(sbsz, f.bw - sbx * sbsz) * 4;
                    if (w_full <= 0) continue;
                    ptrdiff_t top_off = (ptrdiff_t)sbx * sbsz * 4;
                    ptrdiff_t bot_off = sb_y + 8 * y_ls;
                    ccso_prep(bd, ccso_lut_idx[pl], 64 >> pl_ss_hor, y, y_ls, sb_y, lr_bak[bit][0],
                              f.cdef_line[tf][0].data(), top_off, y, bot_off, cfg.max_band_log2,
                              cfg.ext_filter, cfg.quant_step, cfg.edge_clf, cfg.bo_only, sb_edges,
                              w_full >> pl_ss_hor, 8 >> pl_ss_ver, pl_ss_hor, pl_ss_ver);
                }
            }

            int sidx = cdef_idx < 0 ? 0 : cdef_idx;
            bool cdef_active = !(cdef_idx == -1 || !p.cdef_on ||
                                 ((sidx < 8 ? p.y_strength[sidx] : 0) == 0 &&
                                  (sidx < 8 ? p.uv_strength[sidx] : 0) == 0));
            if (cdef_active) {
                uint16_t noskip_full;
                if (p.on_skip_tx)
                    noskip_full = 0xffff;
                else if (sb256x < p.n && by_idx < 32 && sb64x_idx < 4)
                    noskip_full = p.row[mask_i].noskip_mask[by_idx][sb64x_idx];
                else
                    noskip_full = 0;
                int y_lvl = p.y_strength[cdef_idx], uv_lvl = p.uv_strength[cdef_idx];
                uint8_t flag = (uint8_t)((y_lvl != 0) + ((uv_lvl != 0) << 1));
                int y_pri_lvl = (y_lvl >> 2) << bd8;
                int y_sec_lvl = y_lvl & 3;
                y_sec_lvl += y_sec_lvl == 3;
                y_sec_lvl <<= bd8;
                int uv_pri_lvl = (uv_lvl >> 2) << bd8;
                int uv_sec_lvl = uv_lvl & 3;
                uv_sec_lvl += uv_sec_lvl == 3;
                uv_sec_lvl <<= bd8;

                uint16_t y_ll0 = 0, y_ll1 = 0, uv_ll0 = 0, uv_ll1 = 0;
                if (p.any_lossless && sb256x < p.n) {
                    const R2gAv2Filter &m = p.row[sb256x];
                    int yr = imin(2 * by_idx, 63);
                    y_ll0 = m.lossless_mask_y[yr][sb64x_idx];
                    y_ll1 = m.lossless_mask_y[imin(yr + 1, 63)][sb64x_idx];
                    int uvr = imin((2 * by_idx) >> ss_ver, 63);
                    uv_ll0 = m.lossless_mask_uv[uvr][sb64x_idx];
                    uv_ll1 = m.lossless_mask_uv[imin(uvr + (1 - ss_ver), 63)][sb64x_idx];
                }

                ptrdiff_t b_y = sb_y, b_uv = sb_uv;
                int bx = sbx * sbsz;
                int sb_bx_end = imin((sbx + 1) * sbsz, f.bw);
                for (; bx < sb_bx_end; bx += 2, b_y += 8, b_uv += 8 >> ss_hor) {
                    if (bx + 2 >= f.bw) edges &= ~HAVE_RIGHT;
                    uint16_t bx_mask = (uint16_t)(3u << (bx & 14));
                    bool y_lossless = ((y_ll0 | y_ll1) & bx_mask) != 0;
                    uint16_t uvbx_mask = (uint16_t)((3u >> ss_hor) << ((bx & 14) >> ss_hor));
                    bool uv_lossless = ((uv_ll0 | uv_ll1) & uvbx_mask) != 0;
                    if ((noskip_full & bx_mask) == 0 || (y_lossless && uv_lossless)) {
                        prev_flag = 0;
                        edges |= HAVE_LEFT;
                        continue;
                    }
                    uint8_t do_left = flag & ~prev_flag;
                    prev_flag = flag;
                    if (do_left && (edges & HAVE_LEFT)) {
                        if (do_left & BACKUP_2X8_Y) backup2x8(lr_bak[bit][0], y, b_y, y_ls, 0, 8);
                        if (do_left & BACKUP_2X8_UV) {
                            backup2x8(lr_bak[bit][1], u, b_uv, uv_ls, 0, 8 >> ss_ver);
                            backup2x8(lr_bak[bit][2], v, b_uv, uv_ls, 0, 8 >> ss_ver);
                        }
                    }
                    if (edges & HAVE_RIGHT) {
                        int other = 1 - bit;
                        if (flag & BACKUP_2X8_Y) backup2x8(lr_bak[other][0], y, b_y, y_ls, 8, 8);
                        if (flag & BACKUP_2X8_UV) {
                            backup2x8(lr_bak[other][1], u, b_uv, uv_ls, 8 >> ss_hor, 8 >> ss_ver);
                            backup2x8(lr_bak[other][2], v, b_uv, uv_ls, 8 >> ss_hor, 8 >> ss_ver);
                        }
                    }
                    uint32_t variance = 0;
                    int dir = (y_pri_lvl != 0 || uv_pri_lvl != 0) ? cdef_find_dir(y + b_y, y_ls, &variance, bd8) : 0;
                    ptrdiff_t top_col = (ptrdiff_t)bx * 4;
                    ptrdiff_t bot_y = b_y + 8 * y_ls;
                    if (y_pri_lvl != 0) {
                        int adj = adjust_strength(y_pri_lvl, variance);
                        if ((adj != 0 || y_sec_lvl != 0) && !y_lossless)
                            cdef_filter_block(bd, y, y_ls, b_y, lr_bak[bit][0], f.cdef_line[tf][0].data(),
                                              top_col, y, bot_y, adj, y_sec_lvl, dir, damping, 8, 8, edges);
                    } else if (y_sec_lvl != 0 && !y_lossless) {
                        cdef_filter_block(bd, y, y_ls, b_y, lr_bak[bit][0], f.cdef_line[tf][0].data(),
                                          top_col, y, bot_y, 0, y_sec_lvl, 0, damping, 8, 8, edges);
                    }
                    if (uv_lvl != 0 && !uv_lossless) {
                        int uvdir = uv_pri_lvl != 0 ? uv_dir[dir] : 0;
                        int cw = 8 >> ss_hor, ch = 8 >> ss_ver;
                        ptrdiff_t top_col_uv = ((ptrdiff_t)bx * 4) >> ss_hor;
                        ptrdiff_t bot_uv = b_uv + ch * uv_ls;
                        cdef_filter_block(bd, u, uv_ls, b_uv, lr_bak[bit][1], f.cdef_line[tf][1].data(),
                                          top_col_uv, u, bot_uv, uv_pri_lvl, uv_sec_lvl, uvdir,
                                          damping - 1, cw, ch, edges);
                        cdef_filter_block(bd, v, uv_ls, b_uv, lr_bak[bit][2], f.cdef_line[tf][2].data(),
                                          top_col_uv, v, bot_uv, uv_pri_lvl, uv_sec_lvl, uvdir,
                                          damping - 1, cw, ch, edges);
                    }
                    bit ^= 1;
                    edges |= HAVE_LEFT;
                }
            } else {
                prev_flag = 0;
                edges |= HAVE_LEFT;
            }

            /* CCSO add (cdef.rs:1081-1170) */
            if (p.ccso_on) {
                const uint8_t *ccm = sb256x < p.n ? p.row[sb256x].ccso : NULL;
                uint8_t c0 = ccm ? ccm[0] : 0, c1 = ccm ? ccm[1] : 0, c2 = ccm ? ccm[2] : 0;
                uint8_t ccmv[3] = {c0, c1, c2};
                uint8_t flag = (uint8_t)(c0 | ((c1 | c2) << 1));
                uint8_t do_right = flag & ~prev_flag;
                if (do_right && (sbx + 1) * sbsz < f.bw) {
                    if (do_right & BACKUP_2X8_Y) backup2x8(lr_bak[bit][0], y, sb_y, y_ls, sbsz * 4, 8);
                    if (do_right & BACKUP_2X8_UV) {
                        backup2x8(lr_bak[bit][1], u, sb_uv, uv_ls, (sbsz * 4) >> ss_hor, 8 >> ss_ver);
                        backup2x8(lr_bak[bit][2], v, sb_uv, uv_ls, (sbsz * 4) >> ss_hor, 8 >> ss_ver);
                    }
                    prev_flag |= do_right;
                }
                int by_idx_ll = 2 * by_idx;
                for (int pl = 0; pl < 3; pl++) {
                    if (ccmv[pl] == 0) continue;
                    const CcsoPlaneCfg &cfg = p.cc[pl];
                    int pl_ss_hor = pl ? ss_hor : 0, pl_ss_ver = pl ? ss_ver : 0;
                    int w_full = imin(sbsz, f.bw - sbx * sbsz) * 4;
                    pixel *dst = pl == 0 ? y : (pl == 1 ? u : v);
                    ptrdiff_t dst_off = pl == 0 ? sb_y : sb_uv;
                    ptrdiff_t dst_ls = pl == 0 ? y_ls : uv_ls;
                    uint16_t ll_buf[2][4] = {{0}};
                    if (p.any_lossless && sb256x < p.n) {
                        const R2gAv2Filter &m = p.row[sb256x];
                        const uint16_t(*src)[4] = pl == 0 ? m.lossless_mask_y : m.lossless_mask_uv;
                        int base = by_idx_ll >> pl_ss_ver;
                        for (int r = 0; r < 2; r++)
                            if (base + r < 64) ll_buf[r][0] = src[base + r][sb64x_idx];
                    }
                    ccso_add(bd, dst + dst_off, dst_ls, ccso_lut_idx[pl], 64 >> pl_ss_hor, cfg.filter_off,
                             CCSO_OFFSET[cfg.scale_idx], w_full >> pl_ss_hor, 8 >> pl_ss_ver, ll_buf);
                }
            }
            sb_y += sbsz * 4;
            sb_uv += (sbsz * 4) >> ss_hor;
        }
        row_y += 8 * y_ls;
        row_uv += (8 * uv_ls) >> ss_ver;
        f.cdef_line_toggle ^= 1;
        edge_top = HAVE_TOP;
    }
}

/* decode.rs:4117-4133 build_ccso_plane_cfg */
static CcsoPlaneCfg build_ccso_plane_cfg(const R2gFrameParams *fp, int pl) {
    const R2gCcsoPlane &cp = fp->ccso[pl];
    CcsoPlaneCfg c;
    c.max_band_log2 = cp.max_band_log2;
    c.ext_filter = cp.ext_filter_support;
    c.quant_step = CCSO_QUANT_SZ[cp.scale_idx][cp.quant_idx];
    c.edge_clf = cp.edge_clf;
    c.bo_only = cp.bo_only != 0;
    c.scale_idx = cp.scale_idx;
    c.filter_off = cp.filter_off;
    return c;
}

/* decode.rs:3855-4001: the CDEF(+CCSO) block of filter_sbrow. */
void cdef_filter_sbrow(Frame &f, size_t mask_row, int sby, uint32_t inloop) {
    const R2gFrameParams *fp = f.fp;
    int sb128 = fp->sb128;
    int sb_step = 16 << sb128;
    bool ccso_on = (inloop & R2G_INLOOP_CCSO) &&
                   (fp->ccso[0].enabled || fp->ccso[1].enabled || fp->ccso[2].enabled);
    bool any_lossless = false;
    if (fp->seg_enabled)
        for (int i = 0; i < 8; i++) any_lossless |= fp->seg_lossless[i] != 0;
    int start = sby * sb_step;

    BrowParams bp;
    bp.n = f.sb256w;
    bp.damping = fp->cdef_damping;
    bp.on_skip_tx = fp->cdef_on_skiptx != 0;
    bp.cdef_on = (inloop & R2G_INLOOP_CDEF) != 0;
    bp.any_lossless = any_lossless;
    bp.ccso_on = ccso_on;
    bp.y_strength = fp->cdef_y_strength;
    bp.uv_strength = fp->cdef_uv_strength;
    for (int pl = 0; pl < 3; pl++) bp.cc[pl] = build_ccso_plane_cfg(fp, pl);

    /* lazily sized line banks: 2 rows at the plane stride */
    for (int b = 0; b < 2; b++) {
        if (f.cdef_line[b][0].size() != (size_t)(2 * f.stride[0])) f.cdef_line[b][0].assign(2 * f.stride[0], 0);
        for (int pl = 1; pl < 3; pl++)
            if (f.cdef_line[b][pl].size() != (size_t)(2 * f.stride[1])) f.cdef_line[b][pl].assign(2 * f.stride[1], 0);
    }

    if (sby > 0) {
        size_t prev_mask_row = (size_t)(((sby - 1) >> (2 - sb128)) * f.sb256w);
        BrowParams pp = bp;
        pp.row = &f.mask[prev_mask_row];
        cdef_brow(f, pp, start - 2, start);
    }
    int n_blks = sb_step - 2 * (sby + 1 < f.sbh);
    int end = imin(start + n_blks, f.bh);
    bp.row = &f.mask[mask_row];
    cdef_brow(f, bp, start, end);
}

}  // namespace r2o

/* ---- known-answer-test hooks (the reference's ccso.rs / cdef.rs tests) ---- */
extern "C" {
void r2o_ccso_prep(uint8_t *dst, int dst_stride, const uint16_t *src, int64_t src_stride, int64_t src_off,
                   const uint16_t *left_2, const uint16_t *top, int64_t top_off, const uint16_t *bottom,
                   int64_t bottom_off, uint32_t max_band_log2, int ext_filter, int quant_step, uint32_t edge_clf,
                   int bo_only, int edges, int w, int h, int ss_hor, int ss_ver, int bitdepth) {
    r2o::BD bd;
    bd.bitdepth = bitdepth;
    r2o::ccso_prep(bd, dst, dst_stride, src, src_stride, src_off, (const r2o::Left2 *)left_2, top, top_off, bottom,
                   bottom_off, max_band_log2, ext_filter, quant_step, edge_clf, bo_only != 0, edges, w, h, ss_hor,
                   ss_ver);
}
/* ccso.rs:5-13 CCSO_POS entry [i][k] */
int r2o_ccso_pos(int i, int k) { return r2o::CCSO_POS[i][k]; }
int r2o_ccso_pos_len(void) { return (int)(sizeof(r2o::CCSO_POS) / sizeof(r2o::CCSO_POS[0])); }
/* cdef.rs:122-128, 218-224, 243-280: the helpers the reference tests */
void r2o_cdef_fill(int16_t *tmp, int64_t stride, int w, int h) { r2o::fill(tmp, stride, w, h); }
int r2o_cdef_pri_tap(int pri) { return r2o::cdef_pri_tap(pri); }
/* cdef.rs:222-224 cdef_apply_constrain */
int r2o_cdef_apply_constrain(int px, int p0, int p1, int strength, int shift, int tap) {
    return tap * r2o::constrain(p0 - px, strength, shift) + tap * r2o::constrain(p1 - px, strength, shift);
}
void r2o_backup2lines_plane(uint16_t *dst, int64_t dst_off, const uint16_t *src, int64_t src_off, int64_t stride,
                            int height) {
    r2o::backup2lines_plane(dst, dst_off, src, src_off, stride, height);
}
void r2o_backup2x8_plane(uint16_t *dst_x2, const uint16_t *src, int64_t src_off, int64_t stride, int64_t x_off,
                         int rows) {
    r2o::backup2x8_plane((r2o::Left2 *)dst_x2, src, src_off, stride, x_off, rows);
}
/* cdef.rs:37-112 cdef_padding into a tmp_stride-wide i16 buffer */
void r2o_cdef_padding(int16_t *tmp, int tmp_stride, const uint16_t *src, int64_t src_stride, int64_t src_off,
                      const uint16_t *left_2, const uint16_t *top, int64_t top_off, const uint16_t *bottom,
                      int64_t bottom_off, int w, int h, int edges) {
    r2o::cdef_padding(tmp, tmp_stride, src, src_stride, src_off, (const r2o::Left2 *)left_2, top, top_off, bottom,
                      bottom_off, w, h, edges);
}
/* cdef.rs:320-458 cdef_filter_block on a block at dst_off of a plane */
void r2o_cdef_filter_block(uint16_t *dst, int64_t dst_stride, int64_t dst_off, const uint16_t *left_2,
                           const uint16_t *top, int64_t top_off, const uint16_t *bottom, int64_t bottom_off,
                           int pri, int sec, int dir, int damping, int w, int h, int edges, int bitdepth) {
    r2o::BD bd;
    bd.bitdepth = bitdepth;
    r2o::cdef_filter_block(bd, dst, dst_stride, dst_off, (const r2o::Left2 *)left_2, top, top_off, bottom, bottom_off,
                           pri, sec, dir, damping, w, h, edges);
}
void r2o_ccso_add(uint16_t *dst, int64_t dst_stride, const uint8_t *idx_buf, int idx_stride,
                  const uint8_t *offset_idxs, const int8_t *offset_lut, int w, int h, const uint16_t *ll_mask_x4,
                  int bitdepth) {
    r2o::BD bd;
    bd.bitdepth = bitdepth;
    r2o::ccso_add(bd, dst, dst_stride, idx_buf, idx_stride, offset_idxs, offset_lut, w, h,
                  (const uint16_t(*)[4])ll_mask_x4);
}
}
