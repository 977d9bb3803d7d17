/*
 * Oracle: loop restoration (NS-Wiener single/multi, PC-Wiener, chroma
 * cross-component NS-Wiener, GDF) per superblock row.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Restates crates/rav2d/src/looprestoration.rs:1-2548 of the rav2d reference
 * (scalar arms; the 8-bit `wide` kernels in simd.rs:432-608 are tested equal
 * to these by the reference's own simd.rs tests).
 */
#include "oracle.h"

#define R2G_TABLE(type, name) static const type name
#include "av2_tables.h"

namespace r2o {

enum {
    LR_HAVE_LEFT = 1,
    LR_HAVE_RIGHT = 2,
    LR_HAVE_TOP = 4,
    LR_HAVE_BOTTOM = 8,
    LR_HAVE_TOP_INTEGRATED = 16,
    LR_HAVE_BOTTOM_INTEGRATED = 32
};
enum { FIRST_NONE = 0, FIRST_TOP = 1, FIRST_BOTTOM = 2 };

/* looprestoration.rs:13-21 */
static const uint16_t PC_WIENER_NORMALIZER[4] = {3739, 3273, 3074, 7};
static const int16_t MODE_WEIGHTS[4][3] = {{-527, 15325, 321}, {26436, -17705, 17905}, {366, -147, -194}, {202, -267, -179}};
static const int16_t MODE_OFFSETS[4] = {-547, -21565, -573, -680};
/* looprestoration.rs:334-353, :357-372, :374-387, :389-406 */
static const int8_t GDF_COORDS[18][2] = {{6, 0}, {5, 0}, {4, 0}, {3, 0}, {2, 1}, {2, 0}, {2, -1}, {1, 2}, {1, 1},
                                         {1, 0}, {1, -1}, {1, -2}, {0, 6}, {0, 5}, {0, 4}, {0, 3}, {0, 2}, {0, 1}};
static const int8_t WIENER_NS_CONFIG_UV[6][2] = {{1, 0}, {0, 1}, {1, 1}, {-1, 1}, {2, 0}, {0, 2}};
static const int8_t WIENER_NS_CONFIG_UV_FROM_Y[12][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1},
                                                        {-1, 1}, {1, -1}, {2, 0}, {-2, 0}, {0, 2}, {0, -2}};
static const int8_t PC_WIENER_CONFIG[12][2] = {{1, 0}, {0, 1}, {2, 0}, {0, 2}, {1, 1}, {-1, 1},
                                               {2, 1}, {2, -1}, {1, 2}, {1, -2}, {3, 0}, {0, 3}};
static const int8_t WIENER_NS_CONFIG_Y[16][2] = {{1, 0}, {0, 1}, {2, 0}, {0, 2}, {1, 1}, {-1, 1}, {2, 1}, {2, -1},
                                                 {1, 2}, {1, -2}, {3, 0}, {0, 3}, {4, 0}, {0, 4}, {3, 3}, {3, -3}};

enum { REST_UNIT_STRIDE = 76, ROW_ORIGIN = 6, GRADIENT_BUF_STRIDE = 33, LUMA_BUF_STRIDE = REST_UNIT_STRIDE + 64 };

typedef pixel Left6[6];
typedef pixel Row[REST_UNIT_STRIDE];
typedef pixel LRow[LUMA_BUF_STRIDE];

/* looprestoration.rs:40-50 get_qval_given_tskip */
int get_qval_given_tskip(int qstep, int tskip, int i, int bitdepth_min_8) {
    qstep = (qstep + ((1 << bitdepth_min_8) >> 1)) >> bitdepth_min_8;
    int prod = (tskip * qstep + 128) >> 8;
    int qval = MODE_WEIGHTS[i][0] * (tskip << 5) + MODE_WEIGHTS[i][1] * qstep + MODE_WEIGHTS[i][2] * prod;
    int abs_qval = qval < 0 ? -qval : qval;
    qval = apply_sign((abs_qval + (1 << 12)) >> 13, qval);
    return 255 * (MODE_OFFSETS[i] + qval);
}

/* looprestoration.rs:55-80 backup_row */
static void backup_row(pixel *dst, int o, const pixel *src, ptrdiff_t src_o, const pixel *left,
                       int left_off, int w, int edge_len, int edges) {
    if (edges & LR_HAVE_LEFT)
        for (int x = 0; x < edge_len; x++) dst[o - edge_len + x] = left[left_off - edge_len + x];
    else
        for (int x = 0; x < edge_len; x++) dst[o - edge_len + x] = src[src_o];
    memcpy(dst + o, src + src_o, sizeof(pixel) * w);
    if (edges & LR_HAVE_RIGHT)
        memcpy(dst + o + w, src + src_o + w, sizeof(pixel) * edge_len);
    else
        for (int x = 0; x < edge_len; x++) dst[o + w + x] = src[src_o + w - 1];
}

/* looprestoration.rs:85-108 backup_row_lpf */
static void backup_row_lpf(pixel *dst, int o, const pixel *src, ptrdiff_t src_o, int w, int edge_len, int edges) {
    if (edges & LR_HAVE_LEFT)
        for (int x = 0; x < edge_len; x++) dst[o - edge_len + x] = src[src_o - edge_len + x];
    else
        for (int x = 0; x < edge_len; x++) dst[o - edge_len + x] = src[src_o];
    memcpy(dst + o, src + src_o, sizeof(pixel) * w);
    if (edges & LR_HAVE_RIGHT)
        memcpy(dst + o + w, src + src_o + w, sizeof(pixel) * edge_len);
    else
        for (int x = 0; x < edge_len; x++) dst[o + w + x] = src[src_o + w - 1];
}

/* looprestoration.rs:114-193 compute_gradient_row (scalar form) */
static void compute_gradient_row(uint16_t (*dst)[4], const pixel *const *rows, int row_off, int col_off,
                                 int w, uint32_t shift) {
    static const int offs[4][2] = {{1, 0}, {0, 1}, {1, 1}, {-1, 1}};
    for (int x1 = 0; x1 < w + 2; x1 += 2)
        for (int d = 0; d < 4; d++) {
            int grad = 0;
            for (int x2 = 0; x2 < 2; x2++) {
                int x = col_off + x1 + x2;
                for (int y = 0; y < 2; y++) {
                    int dy = offs[d][0], dx = offs[d][1];
                    int ry = row_off + y;
                    int a = (int)rows[ry - 1 - dy][x - 1 - dx] >> shift;
                    int b = (int)rows[ry - 1][x - 1] >> shift;
                    int c = (int)rows[ry - 1 + dy][x - 1 + dx] >> shift;
                    int t = b * 2 - a - c;
                    grad += t < 0 ? -t : t;
                }
            }
            dst[x1 >> 1][d] = (uint16_t)grad;
        }
}

/* looprestoration.rs:195-271 get_class_lut_idx */
static int get_class_lut_idx(const pixel *const *rows, int row_center, int col_off, const uint16_t *noskip_mask,
                             int base_q, int bx, int by, int bh, int bitdepth_min_8) {
    int f[3] = {0, 0, 0};
    int s = 0;
    for (int dy = -1; dy <= 4; dy++)
        for (int dx = -1; dx <= 4; dx++) {
            int x = col_off + bx * 4 + dx;
            int y = row_center + dy;
            int m = rows[y][x];
            int vert = (int)rows[y - 1][x] - 2 * m + (int)rows[y + 1][x];
            int anti_diag = (int)rows[y - 1][x + 1] - 2 * m + (int)rows[y + 1][x - 1];
            int diag = (int)rows[y - 1][x - 1] - 2 * m + (int)rows[y + 1][x + 1];
            f[0] += vert < 0 ? -vert : vert;
            f[1] += anti_diag < 0 ? -anti_diag : anti_diag;
            f[2] += diag < 0 ? -diag : diag;
        }
    static const uint8_t num_pixels[3] = {16, 4, 1};
    for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
            int edge = (dy != 0) + (dx != 0);
            int fx = iclip((bx & 15) + dx, 0, 15);
            int fy = iclip(by + dy, 0, bh - 1);
            s += num_pixels[edge] * (((noskip_mask[fy] >> fx) & 1) == 0);
        }
    int rnd = (1 << bitdepth_min_8) >> 1;
    for (int i = 0; i < 3; i++)
        f[i] = (int)((uint32_t)f[i] * (uint32_t)PC_WIENER_NORMALIZER[i] + (uint32_t)rnd) >> bitdepth_min_8;
    s *= PC_WIENER_NORMALIZER[3];
    int qval = (imax(0, get_qval_given_tskip(base_q, s, 0, bitdepth_min_8)) + (1 << 13)) >> 14;
    qval = imin(qval, 255) >> 5;
    int lut_idx = qval << 9;
    for (int i = 0; i < 3; i++) {
        qval = (imax(0, f[i] + get_qval_given_tskip(base_q, s, i + 1, bitdepth_min_8)) + (1 << 13)) >> 14;
        qval = imin(qval, 255) >> 5;
        lut_idx |= qval << (3 * (2 - i));
    }
    return lut_idx;
}

/* looprestoration.rs:273-329 gdf_add */
static void gdf_add(pixel *p, ptrdiff_t stride, const int8_t *err, int err_stride, int w, int h, int scale,
                    const uint16_t (*ll_mask)[4], int bitdepth) {
    int shift = 12 - bitdepth;
    int rnd = (1 << shift) >> 1;
    int bdmax = (1 << bitdepth) - 1;
    int bw = w >> 2;
    for (int by = 0; by < (h >> 2); by++) {
        uint16_t skip_mask = ll_mask[by][0];
        for (int bx = 0; bx < bw; bx++) {
            if (skip_mask & (1 << bx)) continue;
            for (int y = by * 4; y < by * 4 + 4; y++)
                for (int x = bx * 4; x < bx * 4 + 4; x++) {
                    int diff = err[y * err_stride + x] * scale;
                    int ad = diff < 0 ? -diff : diff;
                    int v = (int)p[y * stride + x] + apply_sign((ad + rnd) >> shift, diff);
                    p[y * stride + x] = (pixel)iclip(v, 0, bdmax);
                }
        }
    }
}

/* looprestoration.rs:408-522 backup_row_luma (4:2:0 arm) */
static void backup_row_luma(pixel *dst, int o, const pixel *src, ptrdiff_t src_o, ptrdiff_t src_stride, int w,
                            int edges, int ss_hor, int ss_ver, int cfl_ds_flt) {
    if (ss_ver == 0) {
        backup_row_lpf(dst, o, src, src_o, w, 4, edges);
        return;
    }
    ptrdiff_t src2_o = src_o + src_stride;
    if (cfl_ds_flt == 0) {
        for (int x = 0; x < w; x += 1 + ss_hor)
            dst[o + x] = (pixel)(((int)src[src_o + x] + src[src2_o + x] + src[src_o + x + 1] + src[src2_o + x + 1]) >> 2);
    } else if (cfl_ds_flt == 1) {
        for (int x = 0; x < w; x++) dst[o + x] = (pixel)(((int)src[src_o + x] + src[src2_o + x]) >> 1);
    } else {
        memcpy(dst + o, src + src_o, sizeof(pixel) * w);
    }
    if (edges & LR_HAVE_LEFT) {
        for (int i = 0; i < 4; i++) {
            ptrdiff_t si = src_o - 4 + i, s2i = src2_o - 4 + i;
            if (cfl_ds_flt == 0)
                dst[o - 4 + i] = (pixel)(((int)src[si] + src[s2i] + src[si + 1] + src[s2i + 1]) >> 2);
            else if (cfl_ds_flt == 1)
                dst[o - 4 + i] = (pixel)(((int)src[si] + src[s2i]) >> 1);
            else
                dst[o - 4 + i] = src[si];
        }
    } else {
        pixel fill_val = dst[o];
        for (int i = 0; i < 4; i++) dst[o - 4 + i] = fill_val;
    }
    if (edges & LR_HAVE_RIGHT) {
        for (int i = 0; i < 4; i++) {
            ptrdiff_t si = src_o + w + i, s2i = src2_o + w + i;
            if (cfl_ds_flt == 0)
                dst[o + w + i] = (pixel)(((int)src[si] + src[s2i] + src[si + 1] + src[s2i + 1]) >> 2);
            else if (cfl_ds_flt == 1)
                dst[o + w + i] = (pixel)(((int)src[si] + src[s2i]) >> 1);
            else
                dst[o + w + i] = src[si];
        }
    } else {
        pixel fill_val = dst[o + w - 2];
        for (int i = 0; i < 4; i++) dst[o + w + i] = fill_val;
    }
}

/* looprestoration.rs:524-713 ns_wiener_single_y */
static void ns_wiener_single_y(pixel *p, ptrdiff_t p_off, ptrdiff_t stride, const Left6 *left, const pixel *lpf,
                               ptrdiff_t lpf_off, const pixel *lpf_bottom, ptrdiff_t lpf_bottom_off, int w, int h,
                               const int8_t filter[16], int edges, const uint16_t (*ll_mask)[4], int bitdepth) {
    Row rb[9];
    memset(rb, 0, sizeof(rb));
    int ptrs[9] = {0};
    const int o = ROW_ORIGIN;
    backup_row(rb[4], o, p, p_off, left[0], 6, w, 4, edges);
    ptrs[4] = 4;
    if (edges & LR_HAVE_TOP_INTEGRATED) {
        ptrdiff_t loff = lpf_off;
        for (int i = 0; i < 4; i++) {
            backup_row_lpf(rb[i], o, lpf, loff, w, 4, edges);
            loff += stride;
            ptrs[i] = i;
        }
    } else if (edges & LR_HAVE_TOP) {
        backup_row_lpf(rb[2], o, lpf, lpf_off, w, 4, edges);
        ptrs[2] = 2;
        backup_row_lpf(rb[3], o, lpf, lpf_off + stride, w, 4, edges);
        ptrs[3] = 3;
        ptrs[0] = 2;
        ptrs[1] = 2;
    } else {
        ptrs[0] = ptrs[1] = ptrs[2] = ptrs[3] = 4;
    }
    backup_row(rb[5], o, p, p_off + stride, left[1], 6, w, 4, edges);
    ptrs[5] = 5;
    backup_row(rb[6], o, p, p_off + 2 * stride, left[2], 6, w, 4, edges);
    ptrs[6] = 6;
    backup_row(rb[7], o, p, p_off + 3 * stride, left[3], 6, w, 4, edges);
    ptrs[7] = 7;
    int bak_idx = 8;
    int bdmax = (1 << bitdepth) - 1;
    for (int y = 0; y < h; y++) {
        if (y + 4 < h) {
            backup_row(rb[bak_idx], o, p, p_off + (y + 4) * stride, left[y + 4], 6, w, 4, edges);
            ptrs[8] = bak_idx;
        } else if (edges & LR_HAVE_BOTTOM_INTEGRATED) {
            backup_row_lpf(rb[bak_idx], o, p, p_off + (y + 4) * stride, w, 4, edges);
            ptrs[8] = bak_idx;
        } else if (y + 2 < h && (edges & LR_HAVE_BOTTOM)) {
            int offset_y = y + 4 - h;
            backup_row_lpf(rb[bak_idx], o, lpf_bottom, lpf_bottom_off + offset_y * stride, w, 4, edges);
            ptrs[8] = bak_idx;
        } else {
            ptrs[8] = ptrs[7];
        }
        if (++bak_idx == 9) bak_idx = 0;
        const pixel *refs[9];
        for (int i = 0; i < 9; i++) refs[i] = rb[ptrs[i]];
        uint16_t skip_mask = ll_mask[y >> 2][0];
        pixel *dst_row = p + p_off + y * stride;
        for (int bx = 0; bx < (w >> 2); bx++) {
            if (skip_mask & (1 << bx)) continue;
            for (int j = bx * 4; j < bx * 4 + 4; j++) {
                int c = o + j;
                int m = refs[4][c];
                int s = m << 7;
                for (int i = 0; i < 16; i++) {
                    int dy = WIENER_NS_CONFIG_Y[i][0], dx = WIENER_NS_CONFIG_Y[i][1];
                    int a = refs[4 + dy][c + dx], b = refs[4 - dy][c - dx];
                    s += (a + b - 2 * m) * filter[i];
                }
                dst_row[j] = (pixel)iclip((s + 64) >> 7, 0, bdmax);
            }
        }
        for (int r = 0; r < 8; r++) ptrs[r] = ptrs[r + 1];
    }
}

/* looprestoration.rs:715-1059 wiener_multi (NS-multi when filters_user,
 * PC-Wiener when filters_pretrained) */
static void wiener_multi(pixel *p, ptrdiff_t p_off, ptrdiff_t stride, const Left6 *left, const pixel *lpf,
                         ptrdiff_t lpf_off, const pixel *lpf_bottom, ptrdiff_t lpf_bottom_off, int w, int h,
                         const int8_t (*filters_user)[18], int filters_user_stride,
                         const int16_t (*filters_pretrained)[13], const uint8_t *subclass_lut,
                         const uint16_t *noskip_mask, int base_q, int edges, const uint16_t (*ll_mask)[4],
                         int bitdepth) {
    uint8_t classes[16] = {0};
    Row rb[10];
    memset(rb, 0, sizeof(rb));
    int ptrs[10] = {0};
    const int o = ROW_ORIGIN;
    backup_row(rb[4], o, p, p_off, left[0], 6, w, 4, edges);
    ptrs[4] = 4;
    if (edges & LR_HAVE_TOP_INTEGRATED) {
        ptrdiff_t loff = lpf_off;
        for (int i = 0; i < 4; i++) {
            backup_row_lpf(rb[i], o, lpf, loff, w, 4, edges);
            loff += stride;
            ptrs[i] = i;
        }
    } else if (edges & LR_HAVE_TOP) {
        backup_row_lpf(rb[2], o, lpf, lpf_off, w, 4, edges);
        ptrs[2] = 2;
        backup_row_lpf(rb[3], o, lpf, lpf_off + stride, w, 4, edges);
        ptrs[3] = 3;
        ptrs[0] = 2;
        ptrs[1] = 2;
    } else {
        ptrs[0] = ptrs[1] = ptrs[2] = ptrs[3] = 4;
    }
    backup_row(rb[5], o, p, p_off + stride, left[1], 6, w, 4, edges);
    ptrs[5] = 5;
    backup_row(rb[6], o, p, p_off + 2 * stride, left[2], 6, w, 4, edges);
    ptrs[6] = 6;
    backup_row(rb[7], o, p, p_off + 3 * stride, left[3], 6, w, 4, edges);
    ptrs[7] = 7;
    int bak_idx = 8;
    int bh = h >> 2, bw = w >> 2;
    int bdmax = (1 << bitdepth) - 1;
    for (int by = 0; by < bh; by++) {
        int by4 = by << 2;
        if (by + 1 < bh) {
            backup_row(rb[bak_idx], o, p, p_off + (by4 + 4) * stride, left[by4 + 4], 6, w, 4, edges);
            ptrs[8] = bak_idx;
            backup_row(rb[9], o, p, p_off + (by4 + 5) * stride, left[by4 + 5], 6, w, 4, edges);
            ptrs[9] = 9;
        } else if (edges & LR_HAVE_BOTTOM_INTEGRATED) {
            backup_row_lpf(rb[bak_idx], o, p, p_off + (by4 + 4) * stride, w, 4, edges);
            ptrs[8] = bak_idx;
            backup_row_lpf(rb[9], o, p, p_off + (by4 + 5) * stride, w, 4, edges);
            ptrs[9] = 9;
        } else if (edges & LR_HAVE_BOTTOM) {
            backup_row_lpf(rb[bak_idx], o, lpf_bottom, lpf_bottom_off, w, 4, edges);
            ptrs[8] = bak_idx;
            backup_row_lpf(rb[9], o, lpf_bottom, lpf_bottom_off + stride, w, 4, edges);
            ptrs[9] = 9;
        } else {
            ptrs[8] = ptrs[7];
            ptrs[9] = ptrs[7];
        }
        {
            const pixel *refs[10];
            for (int i = 0; i < 10; i++) refs[i] = rb[ptrs[i]];
            for (int bx = 0; bx < bw; bx++) {
                int lut_idx = get_class_lut_idx(refs, 4, o, noskip_mask, base_q, bx, by, bh, bitdepth - 8);
                int cls = PC_WIENER_LUT_TO_CLASS[lut_idx];
                classes[bx] = subclass_lut[cls];
            }
        }
        for (int y = by4; y < by4 + 4; y++) {
            if (y + 4 < h) {
                backup_row(rb[bak_idx], o, p, p_off + (y + 4) * stride, left[y + 4], 6, w, 4, edges);
                ptrs[8] = bak_idx;
            } else if (edges & LR_HAVE_BOTTOM_INTEGRATED) {
                backup_row_lpf(rb[bak_idx], o, p, p_off + (y + 4) * stride, w, 4, edges);
                ptrs[8] = bak_idx;
            } else if (y + 2 < h && (edges & LR_HAVE_BOTTOM)) {
                int offset_y = y + 4 - h;
                backup_row_lpf(rb[bak_idx], o, lpf_bottom, lpf_bottom_off + offset_y * stride, w, 4, edges);
                ptrs[8] = bak_idx;
            } else {
                ptrs[8] = ptrs[7];
            }
            if (++bak_idx == 9) bak_idx = 0;
            const pixel *refs[10];
            for (int i = 0; i < 10; i++) refs[i] = rb[ptrs[i]];
            uint16_t skip_mask = ll_mask[y >> 2][0];
            pixel *dst_row = p + p_off + y * stride;
            for (int bx = 0; bx < bw; bx++) {
                if (skip_mask & (1 << bx)) continue;
                int cls = classes[bx];
                for (int j = bx * 4; j < bx * 4 + 4; j++) {
                    int c = o + j;
                    int m = refs[4][c];
                    int s;
                    if (filters_user) {
                        const int8_t *filter = (const int8_t *)filters_user + (size_t)cls * filters_user_stride;
                        s = m << 7;
                        for (int i = 0; i < 16; i++) {
                            int dy = WIENER_NS_CONFIG_Y[i][0], dx = WIENER_NS_CONFIG_Y[i][1];
                            int a = refs[4 + dy][c + dx], b = refs[4 - dy][c - dx];
                            s += (a + b - 2 * m) * filter[i];
                        }
                    } else {
                        const int16_t *filter = filters_pretrained[cls];
                        s = m * filter[12];
                        for (int i = 0; i < 12; i++) {
                            int dy = PC_WIENER_CONFIG[i][0], dx = PC_WIENER_CONFIG[i][1];
                            int a = refs[4 + dy][c + dx], b = refs[4 - dy][c - dx];
                            s += (a + b) * filter[i];
                        }
                    }
                    dst_row[j] = (pixel)iclip((s + 64) >> 7, 0, bdmax);
                }
            }
            for (int r = 0; r < 8; r++) ptrs[r] = ptrs[r + 1];
        }
    }
}

/* looprestoration.rs:1145-1430 ns_wiener_single_uv */
static void ns_wiener_single_uv(pixel *p, ptrdiff_t p_off, ptrdiff_t stride, const Left6 *left, const pixel *lpf,
                                ptrdiff_t lpf_off, const pixel *lpf_bottom, ptrdiff_t lpf_bottom_off, int w, int h,
                                const int8_t filter[18], const pixel *luma, ptrdiff_t luma_off, ptrdiff_t lstride,
                                const pixel *luma_top, ptrdiff_t luma_top_off, const pixel *luma_bottom,
                                ptrdiff_t luma_bottom_off, int ss_hor, int ss_ver, int ds_flt, int edges,
                                const uint16_t (*ll_mask)[4], int bitdepth) {
    int bdmax = (1 << bitdepth) - 1;
    Row cb[5];
    LRow lb[5];
    memset(cb, 0, sizeof(cb));
    memset(lb, 0, sizeof(lb));
    int c_ptrs[5] = {0}, l_ptrs[5] = {0};
    const int o = ROW_ORIGIN;
    int luma_w = w << ss_hor;
    backup_row(cb[2], o, p, p_off, left[0], 6, w, 2, edges);
    c_ptrs[2] = 2;
    if (edges & (LR_HAVE_TOP_INTEGRATED | LR_HAVE_TOP)) {
        ptrdiff_t loff = lpf_off;
        for (int i = 0; i < 2; i++) {
            backup_row_lpf(cb[i], o, lpf, loff, w, 2, edges);
            c_ptrs[i] = i;
            loff += stride;
        }
    } else {
        c_ptrs[0] = 2;
        c_ptrs[1] = 2;
    }
    backup_row(cb[3], o, p, p_off + stride, left[1], 6, w, 2, edges);
    c_ptrs[3] = 3;
    int bak_idx = 4;
    backup_row_luma(lb[2], o, luma, luma_off, lstride, luma_w, edges, ss_hor, ss_ver, ds_flt);
    l_ptrs[2] = 2;
    if (edges & LR_HAVE_TOP_INTEGRATED) {
        backup_row_luma(lb[0], o, luma, luma_off - 4 * lstride, lstride, luma_w, edges, ss_hor, ss_ver, ds_flt);
        l_ptrs[0] = 0;
        backup_row_luma(lb[1], o, luma, luma_off - 2 * lstride, lstride, luma_w, edges, ss_hor, ss_ver, ds_flt);
        l_ptrs[1] = 1;
    } else if (edges & LR_HAVE_TOP) {
        backup_row_luma(lb[0], o, luma_top, luma_top_off, 0, luma_w, edges, ss_hor, ss_ver, ds_flt);
        l_ptrs[0] = 0;
        backup_row_luma(lb[1], o, luma_top, luma_top_off, lstride, luma_w, edges, ss_hor, ss_ver, ds_flt);
        l_ptrs[1] = 1;
    } else {
        l_ptrs[0] = 2;
        l_ptrs[1] = 2;
    }
    backup_row_luma(lb[3], o, luma, luma_off + (1 << ss_ver) * lstride, lstride, luma_w, edges, ss_hor, ss_ver,
                    ds_flt);
    l_ptrs[3] = 3;
    int lbak_idx = 4;
    ptrdiff_t luma_pos = luma_off;
    for (int y = 0; y < h; y++) {
        if (y + 2 < h) {
            backup_row(cb[bak_idx], o, p, p_off + (y + 2) * stride, left[y + 2], 6, w, 2, edges);
            c_ptrs[4] = bak_idx;
        } else if (edges & LR_HAVE_BOTTOM_INTEGRATED) {
            backup_row_lpf(cb[bak_idx], o, p, p_off + (y + 2) * stride, w, 2, edges);
            c_ptrs[4] = bak_idx;
        } else if (edges & LR_HAVE_BOTTOM) {
            int offset_y = y + 2 - h;
            backup_row_lpf(cb[bak_idx], o, lpf_bottom, lpf_bottom_off + offset_y * stride, w, 2, edges);
            c_ptrs[4] = bak_idx;
        } else {
            c_ptrs[4] = c_ptrs[3];
        }
        if (++bak_idx == 5) bak_idx = 0;

        if (c_ptrs[4] == c_ptrs[3]) {
            l_ptrs[4] = l_ptrs[3];
        } else if (y + 2 == h && !(edges & LR_HAVE_BOTTOM_INTEGRATED)) {
            backup_row_luma(lb[lbak_idx], o, luma_bottom, luma_bottom_off, lstride, luma_w, edges, ss_hor, ss_ver,
                            ds_flt);
            l_ptrs[4] = lbak_idx;
        } else if (y + 1 == h && !(edges & LR_HAVE_BOTTOM_INTEGRATED)) {
            backup_row_luma(lb[lbak_idx], o, luma_bottom, luma_bottom_off + lstride, 0, luma_w, edges, ss_hor,
                            ss_ver, ds_flt);
            l_ptrs[4] = lbak_idx;
        } else {
            backup_row_luma(lb[lbak_idx], o, luma, luma_pos + (2 << ss_ver) * lstride, lstride, luma_w, edges,
                            ss_hor, ss_ver, ds_flt);
            l_ptrs[4] = lbak_idx;
        }
        if (++lbak_idx == 5) lbak_idx = 0;

        for (int bx = 0; bx < (w >> 2); bx++) {
            if (ll_mask[y >> 2][0] & (1 << bx)) continue;
            for (int x = bx * 4; x < bx * 4 + 4; x++) {
                int m = cb[c_ptrs[2]][o + x];
                int s = m << 7;
                for (int i = 0; i < 6; i++) {
                    int dy = WIENER_NS_CONFIG_UV[i][0], dx = WIENER_NS_CONFIG_UV[i][1];
                    int a = cb[c_ptrs[2 + dy]][o + x + dx];
                    int b = cb[c_ptrs[2 - dy]][o + x - dx];
                    s += (a + b - 2 * m) * filter[i];
                }
                int l = lb[l_ptrs[2]][o + (x << ss_hor)];
                for (int i = 0; i < 12; i++) {
                    int dy = WIENER_NS_CONFIG_UV_FROM_Y[i][0], dx = WIENER_NS_CONFIG_UV_FROM_Y[i][1];
                    int lx = o + (x + dx) * (1 << ss_hor);
                    int lval = lb[l_ptrs[2 + dy]][lx];
                    s += (lval - l) * filter[6 + i];
                }
                p[p_off + y * stride + x] = (pixel)iclip((s + 64) >> 7, 0, bdmax);
            }
        }
        for (int r = 0; r < 4; r++) c_ptrs[r] = c_ptrs[r + 1];
        for (int r = 0; r < 4; r++) l_ptrs[r] = l_ptrs[r + 1];
        luma_pos += lstride << ss_ver;
    }
}

/* looprestoration.rs:1432-1640 gdf_prep */
static void gdf_prep(int8_t *dst, int dst_stride, const pixel *p, ptrdiff_t p_off, ptrdiff_t stride,
                     const Left6 *left, const pixel *lpf, ptrdiff_t lpf_off, const pixel *lpf_bottom,
                     ptrdiff_t lpf_bottom_off, int w, int h, int ref_dst_idx, int qp_idx, int edges, int bitdepth) {
    uint32_t down_shift = bitdepth == 12 ? 2 : 0;
    uint32_t up_shift = bitdepth == 8 ? 2 : 0;
    Row rb[13];
    memset(rb, 0, sizeof(rb));
    int ptrs[13] = {0};
    const int o = ROW_ORIGIN;
    backup_row(rb[6], o, p, p_off, left[0], 6, w, 6, edges);
    ptrs[6] = 6;
    if (edges & LR_HAVE_TOP_INTEGRATED) {
        for (int n = 0; n < 6; n++) {
            backup_row_lpf(rb[n], o, lpf, lpf_off + n * stride, w, 6, edges);
            ptrs[n] = n;
        }
    } else if (edges & LR_HAVE_TOP) {
        backup_row_lpf(rb[4], o, lpf, lpf_off, w, 6, edges);
        ptrs[4] = 4;
        backup_row_lpf(rb[5], o, lpf, lpf_off + stride, w, 6, edges);
        ptrs[5] = 5;
        ptrs[0] = ptrs[1] = ptrs[2] = ptrs[3] = 4;
    } else {
        for (int n = 0; n < 6; n++) ptrs[n] = 6;
    }
    int bak_idx = 7;
    for (int y = 1; y < 6; y++) {
        backup_row(rb[bak_idx], o, p, p_off + y * stride, left[y], 6, w, 6, edges);
        ptrs[bak_idx] = bak_idx;
        bak_idx++;
    }
    int alpha_base = ref_dst_idx * 528 + qp_idx * 88;
    int weight_base = ref_dst_idx * 1584 + qp_idx * 264;
    int bias_idx = ref_dst_idx * 6 + qp_idx;
    int error_lut_base, scale;
    if (ref_dst_idx == 0) {
        error_lut_base = qp_idx * 4096;
        scale = 8;
    } else {
        error_lut_base = (ref_dst_idx - 1) * 6000 + qp_idx * 1000;
        scale = 5;
    }
    uint16_t grad[2][GRADIENT_BUF_STRIDE][4];
    memset(grad, 0, sizeof(grad));
    {
        const pixel *refs[13];
        for (int i = 0; i < 13; i++) refs[i] = rb[ptrs[i]];
        compute_gradient_row(grad[0], refs, 6, o, w, down_shift);
    }
    int grad_bit = 1;
    for (int y = 0; y < h; y++) {
        if (y + 6 < h) {
            backup_row(rb[bak_idx], o, p, p_off + (y + 6) * stride, left[y + 6], 6, w, 6, edges);
            ptrs[12] = bak_idx;
        } else if (edges & LR_HAVE_BOTTOM_INTEGRATED) {
            backup_row_lpf(rb[bak_idx], o, p, p_off + (y + 6) * stride, w, 6, edges);
            ptrs[12] = bak_idx;
        } else if (y + 4 < h && (edges & LR_HAVE_BOTTOM)) {
            int offset_y = y + 6 - h;
            backup_row_lpf(rb[bak_idx], o, lpf_bottom, lpf_bottom_off + offset_y * stride, w, 6, edges);
            ptrs[12] = bak_idx;
        } else {
            ptrs[12] = ptrs[11];
        }
        if (++bak_idx == 13) bak_idx = 0;
        if ((y & 1) == 0) {
            const pixel *refs[13];
            for (int i = 0; i < 13; i++) refs[i] = rb[ptrs[i]];
            compute_gradient_row(grad[grad_bit], refs, 8, o, w, down_shift);
            grad_bit ^= 1;
        }
        for (int x1 = 0; x1 < w; x1 += 2) {
            int grad_sums[4];
            int hx = x1 >> 1;
            for (int d = 0; d < 4; d++)
                grad_sums[d] = grad[0][hx][d] + grad[0][hx + 1][d] + grad[1][hx][d] + grad[1][hx + 1][d];
            int cls = (grad_sums[0] <= grad_sums[1]) | ((grad_sums[2] <= grad_sums[3]) << 1);
            int shared_vals[3];
            for (int idx = 0; idx < 3; idx++) shared_vals[idx] = GDF_BIAS[bias_idx][idx];
            for (int d = 0; d < 4; d++) {
                int k = d + 18;
                int alpha = GDF_ALPHA[alpha_base + k * 4 + cls];
                int v = imin(grad_sums[d] >> (4 - up_shift), alpha);
                for (int idx = 0; idx < 3; idx++) shared_vals[idx] += v * GDF_WEIGHT[weight_base + idx * 88 + k * 4 + cls];
            }
            for (int x2 = 0; x2 < 2; x2++) {
                int x = x1 + x2;
                int idx_vals[3] = {shared_vals[0], shared_vals[1], shared_vals[2]};
                int m = (int)rb[ptrs[6]][o + x] >> down_shift;
                for (int k = 0; k < 18; k++) {
                    int alpha = GDF_ALPHA[alpha_base + k * 4 + cls];
                    int dy = GDF_COORDS[k][0], dx = GDF_COORDS[k][1];
                    int a = (int)rb[ptrs[6 - dy]][o + x - dx] >> down_shift;
                    int b = (int)rb[ptrs[6 + dy]][o + x + dx] >> down_shift;
                    int above = iclip((a - m) << up_shift, -alpha, alpha);
                    int below = iclip((b - m) << up_shift, -alpha, alpha);
                    int v = iclip(above + below, -512, 511);
                    for (int idx = 0; idx < 3; idx++) idx_vals[idx] += v * GDF_WEIGHT[weight_base + idx * 88 + k * 4 + cls];
                }
                int full_idx = 0;
                for (int idx = 0; idx < 3; idx++) {
                    int sv = idx_vals[idx] * scale;
                    int asv = sv < 0 ? -sv : sv;
                    int v = apply_sign((asv + (1 << 14)) >> 15, sv);
                    int sub_idx = iclip(v, -scale, scale - 1) + scale;
                    full_idx = full_idx * (scale * 2) + sub_idx;
                }
                dst[y * dst_stride + x] =
                    ref_dst_idx == 0 ? GDF_INTRA_ERROR[error_lut_base + full_idx] : GDF_INTER_ERROR[error_lut_base + full_idx];
            }
        }
        for (int r = 0; r < 12; r++) ptrs[r] = ptrs[r + 1];
    }
}

struct LrCtx {
    Frame *f;
    const pixel *lf_p_luma; /* luma snapshot (decode.rs:4007) */
    const uint8_t *ns_subclass_lut, *pc_subclass_lut;
    const int16_t (*pc_filters)[13];
    uint32_t inloop;
    int restore_planes;
};

/* looprestoration.rs:1847-2274 lr_stripe (single-thread: have_tt = 0) */
static void lr_stripe(const LrCtx &ctx, pixel *p, ptrdiff_t p_off, const Left6 *left, int x, int y, int plane,
                      int w, int row_h, const R2gAv2RestorationUnit *lr, int edges, int first_sby_in_tile_row) {
    Frame &f = *ctx.f;
    const R2gFrameParams *fp = f.fp;
    int chroma = plane != 0;
    int ss_ver = chroma & 1, ss_hor = chroma & 1; /* 4:2:0 */
    ptrdiff_t stride = f.stride[chroma];
    int sb128 = fp->sb128;
    int sby = (y + (y != 0 ? (8 << ss_ver) : 0)) >> (6 - ss_ver + sb128);
    int sb256x = (x << ss_hor) >> 8;
    int sb64x_idx = ((x << ss_hor) >> 6) & 3;
    int stripe_h = imin((64 - 8 * (first_sby_in_tile_row != FIRST_NONE)) >> ss_ver, row_h - y);
    int ref_dst_idx = f.gdf_ref_dst_idx, qp_idx = fp->gdf_qp_idx, gdf_scale = fp->gdf_scale;
    int wiener_type = (ctx.inloop & R2G_INLOOP_WIENER) ? lr->restoration_type : 0;
    enum { W_NONE, W_NS_SINGLE, W_NS_MULTI, W_PC } wkind;
    bool multi_wiener = false;
    uint16_t noskip_mask[66] = {0};
    const R2gRestorationPlane &pd = fp->restoration[plane];
    if (wiener_type == R2G_RESTORE_NS_WIENER) {
        if (pd.frame_filters_on) {
            if (pd.num_classes == 1)
                wkind = W_NS_SINGLE;
            else {
                multi_wiener = true;
                wkind = W_NS_MULTI;
            }
        } else
            wkind = W_NS_SINGLE;
    } else if (wiener_type == R2G_RESTORE_PC_WIENER) {
        multi_wiener = true;
        wkind = W_PC;
    } else
        wkind = W_NONE;
    size_t nmask = f.mask.size();
    if (multi_wiener) {
        int r = 0;
        for (int by = y >> 2; by < (row_h >> 2); by++, r++) {
            int by_idx = by & 63;
            size_t sb256_idx = (size_t)f.sb256w * (by >> 6) + sb256x;
            if (sb256_idx < nmask) {
                noskip_mask[r] = f.mask[sb256_idx].lr_noskip_mask[by_idx][sb64x_idx];
                if (!(edges & LR_HAVE_RIGHT) && (w & 63) != 0) {
                    int shift = ((w >> 2) & 15) - 1;
                    uint16_t edge_bit = noskip_mask[r] >> shift;
                    noskip_mask[r] |= (uint16_t)(edge_bit << (shift + 1));
                }
            }
        }
    }
    ptrdiff_t lstride = f.stride[0];
    static thread_local int8_t gdf_err[64 * 64];
    memset(gdf_err, 0, sizeof(gdf_err));
    int left_idx = 0, noskip_offset = 0;
    ptrdiff_t cur_off = p_off;
    ptrdiff_t lpf_off = x;
    ptrdiff_t llpf_off = x * 2;
    const pixel *db_line = f.lr_db_line[plane].data();
    const pixel *luma_db = f.lr_db_line[0].data();

    while (y + stripe_h <= row_h) {
        bool have_bottom = (sby + 1) != f.sbh || (y + stripe_h) != row_h;
        edges = have_bottom ? (edges | LR_HAVE_BOTTOM) : (edges & ~LR_HAVE_BOTTOM);
        int inc = ((edges & (LR_HAVE_TOP | LR_HAVE_TOP_INTEGRATED | LR_HAVE_BOTTOM_INTEGRATED)) == LR_HAVE_TOP &&
                   y + 8 < ((f.bh * 4) >> ss_ver))
                      ? 8
                      : 0;
        size_t sb256_idx = (size_t)f.sb256w * ((size_t)((y << ss_ver) + inc) >> 8) + sb256x;
        bool gdf_enabled = plane == 0 && (ctx.inloop & R2G_INLOOP_GDF) && sb256_idx < nmask &&
                           f.mask[sb256_idx].gdf[(((y + inc) >> 4) & 12) + sb64x_idx] != 0;
        /* cdef_top only applies with HAVE_TOP|HAVE_TOP_INTEGRATED, i.e. the
         * first sbrow of a second or later tile row: not reachable with one
         * tile row, which the boundary enforces. */
        if (gdf_enabled)
            gdf_prep(gdf_err, 64, p, cur_off, stride, left + left_idx, db_line, lpf_off, db_line,
                     lpf_off + 6 * stride, w, stripe_h, ref_dst_idx, qp_idx, edges, f.bd.bitdepth);

        int y4 = ((y << ss_ver) & 255) >> 2;
        int ll_rows = imax(stripe_h >> 2, 1) + 1;
        std::vector<uint16_t> llb((size_t)ll_rows * 4, 0);
        uint16_t(*ll_mask_buf)[4] = (uint16_t(*)[4])llb.data();
        if (sb256_idx < nmask) {
            const R2gAv2Filter &m = f.mask[sb256_idx];
            if (plane == 0 || ss_hor == 0) {
                const uint16_t(*src)[4] = plane == 0 ? m.lossless_mask_y : m.lossless_mask_uv;
                for (int r = 0; r < ll_rows; r++) {
                    int yy = y4 + r;
                    if (yy < 64)
                        for (int k = 0; k < 4; k++)
                            if (sb64x_idx + k < 4) ll_mask_buf[r][k] = src[yy][sb64x_idx + k];
                }
            } else {
                int init_y = y >> 2, end_y = (y + stripe_h) >> 2;
                int base = y4 >> ss_ver;
                for (int yy = init_y, r = 0; yy < end_y; yy++, r++) {
                    int src_y = base + (yy - init_y);
                    if (src_y < 64 && r < ll_rows) {
                        uint16_t lo = m.lossless_mask_uv[src_y][sb64x_idx];
                        uint16_t hi = sb64x_idx + 1 < 4 ? m.lossless_mask_uv[src_y][sb64x_idx + 1] : 0;
                        ll_mask_buf[r][0] = (uint16_t)((lo & 0xff) | ((hi & 0xff) << 8));
                    }
                }
            }
        }

        if (wkind != W_NONE) {
            ptrdiff_t bottom_off = lpf_off + 6 * stride;
            if (wkind == W_NS_SINGLE && chroma == 0) {
                int8_t filter[16];
                memcpy(filter, pd.frame_filters_on ? pd.filter[0] : lr->ns_filter[0], 16);
                ns_wiener_single_y(p, cur_off, stride, left + left_idx, db_line, lpf_off, db_line, bottom_off, w,
                                   stripe_h, filter, edges, ll_mask_buf, f.bd.bitdepth);
            } else if (wkind == W_NS_SINGLE) {
                int8_t filter[18];
                memcpy(filter, pd.frame_filters_on ? pd.filter[0] : lr->ns_filter[0], 18);
                ptrdiff_t luma_off = (ptrdiff_t)(x << ss_hor) + (ptrdiff_t)(y << ss_ver) * lstride;
                ns_wiener_single_uv(p, cur_off, stride, left + left_idx, db_line, lpf_off, db_line, bottom_off, w,
                                    stripe_h, filter, ctx.lf_p_luma, luma_off, lstride, luma_db, llpf_off, luma_db,
                                    llpf_off + 6 * lstride, ss_hor, ss_ver, fp->cfl_ds_filter_index, edges,
                                    ll_mask_buf, f.bd.bitdepth);
            } else if (wkind == W_NS_MULTI) {
                if (pd.frame_filters_on)
                    wiener_multi(p, cur_off, stride, left + left_idx, db_line, lpf_off, db_line, bottom_off, w,
                                 stripe_h, pd.filter, 18, NULL, ctx.ns_subclass_lut, noskip_mask + noskip_offset,
                                 f.base_q, edges, ll_mask_buf, f.bd.bitdepth);
                else
                    /* the reference reinterprets the [i8; 32] rows as packed
                     * [i8; 18] rows (looprestoration.rs:2148-2158): class c
                     * reads bytes c*18 .. c*18+18 of the flat array */
                    wiener_multi(p, cur_off, stride, left + left_idx, db_line, lpf_off, db_line, bottom_off, w,
                                 stripe_h, (const int8_t(*)[18])lr->ns_filter, 18, NULL, ctx.ns_subclass_lut,
                                 noskip_mask + noskip_offset, f.base_q, edges, ll_mask_buf, f.bd.bitdepth);
                noskip_offset += stripe_h >> 2;
            } else {
                wiener_multi(p, cur_off, stride, left + left_idx, db_line, lpf_off, db_line, bottom_off, w, stripe_h,
                             NULL, 0, ctx.pc_filters, ctx.pc_subclass_lut, noskip_mask + noskip_offset, f.base_q,
                             edges, ll_mask_buf, f.bd.bitdepth);
                noskip_offset += stripe_h >> 2;
            }
        }
        if (gdf_enabled)
            gdf_add(p + cur_off, stride, gdf_err, 64, w, stripe_h, gdf_scale, ll_mask_buf, f.bd.bitdepth);

        edges &= ~(LR_HAVE_BOTTOM_INTEGRATED | LR_HAVE_TOP_INTEGRATED);
        left_idx += stripe_h;
        cur_off += stripe_h * stride;
        y += stripe_h;
        edges |= LR_HAVE_TOP;
        stripe_h = imin(64 >> ss_ver, row_h - y);
        if (stripe_h == 0) break;
        lpf_off += 4 * stride;
        llpf_off += 4 * lstride;
    }
}

/* looprestoration.rs:2276-2399 lr_sbrow_plane */
static void lr_sbrow_plane(const LrCtx &ctx, pixel *p, ptrdiff_t p_off, int y, int w, int h, int row_h, int plane,
                           int first_sby_in_tile_row) {
    Frame &f = *ctx.f;
    int chroma = plane != 0;
    int ss_ver = chroma, ss_hor = chroma;
    ptrdiff_t abs_stride = f.stride[chroma];
    int unit_size_log2 = f.fp->restoration_unit_size[chroma];
    int unit_size = 1 << unit_size_log2;
    int half_unit_size = unit_size >> 1;
    int row_y = y + ((8 >> ss_ver) * (first_sby_in_tile_row != FIRST_NONE));
    int shift_hor = 8 - ss_hor;
    static thread_local Left6 pre_lr_border[2][264];
    memset(pre_lr_border, 0, sizeof(pre_lr_border));
    int aligned_unit_pos = row_y & ~(unit_size - 1);
    if (aligned_unit_pos != 0 && aligned_unit_pos + half_unit_size > h) aligned_unit_pos -= unit_size;
    aligned_unit_pos <<= ss_ver;
    int sb_idx = (aligned_unit_pos >> 8) * f.sb256w;
    int unit_idx_base = ((aligned_unit_pos >> 6) & 0x3) << 2;
    int edges = (y > 0 ? LR_HAVE_TOP : 0) | LR_HAVE_RIGHT;
    if (first_sby_in_tile_row == FIRST_TOP) edges |= LR_HAVE_BOTTOM_INTEGRATED;
    if (first_sby_in_tile_row == FIRST_BOTTOM && y > 0) edges |= LR_HAVE_TOP_INTEGRATED;
    size_t lr_idx_0 = (size_t)sb_idx;
    size_t lr_unit_0 = (size_t)unit_idx_base;
    int bit = 0, x = 0;
    ptrdiff_t cur_p_off = p_off;
    size_t n_lr = f.mask.size();
    while (x + 64 < w) {
        int next_x = x + 64;
        int next_start = next_x & ~(unit_size - 1);
        if (next_start != 0 && w - next_start < half_unit_size) next_start -= unit_size;
        int next_u_idx = unit_idx_base + ((next_start >> (shift_hor - 2)) & 3);
        int next_sb_idx = sb_idx + (next_start >> shift_hor);
        int n = plane ? 2 : 6;
        ptrdiff_t border_src_off = cur_p_off + 64;
        for (int row = 0; row < row_h - y; row++) {
            ptrdiff_t src_row = border_src_off + row * abs_stride;
            for (int i = 0; i < n; i++) pre_lr_border[bit][row][6 - n + i] = p[src_row - n + i];
        }
        if (lr_idx_0 < n_lr && lr_unit_0 < 16)
            lr_stripe(ctx, p, cur_p_off, pre_lr_border[1 - bit], x, y, plane, 64, row_h,
                      &f.lr_mask[lr_idx_0].lr[plane][lr_unit_0], edges, first_sby_in_tile_row);
        lr_idx_0 = (size_t)next_sb_idx;
        lr_unit_0 = (size_t)next_u_idx;
        x = next_x;
        cur_p_off += 64;
        edges |= LR_HAVE_LEFT;
        bit ^= 1;
    }
    edges &= ~LR_HAVE_RIGHT;
    int end_w = w - x;
    if (lr_idx_0 < n_lr && lr_unit_0 < 16)
        lr_stripe(ctx, p, cur_p_off, pre_lr_border[1 - bit], x, y, plane, end_w, row_h,
                  &f.lr_mask[lr_idx_0].lr[plane][lr_unit_0], edges, first_sby_in_tile_row);
}

/* looprestoration.rs:2401-2548 lr_sbrow_apply, with the luma snapshot and
 * table selection of decode.rs:4003-4056 */
void lr_sbrow_apply(Frame &f, int sby, uint32_t inloop) {
    const R2gFrameParams *fp = f.fp;
    std::vector<pixel> luma_snapshot(f.p[0], f.p[0] + f.stride[0] * (((f.bh * 4 + 127) & ~127)));
    LrCtx ctx;
    ctx.f = &f;
    ctx.lf_p_luma = luma_snapshot.data();
    int widx = f.wiener_idx;
    ctx.pc_subclass_lut = PC_WIENER_SUB_CLASSIFY[widx];
    ctx.pc_filters = PC_WIENER_FILTERS[widx];
    int ci = f.ns_subclass_class_idx;
    ctx.ns_subclass_lut = PC_WIENER_SUB_CLASSIFY_NS[widx][ci >= 0 ? imin(ci, 6) : 0];
    ctx.inloop = inloop;
    ctx.restore_planes = f.restore_planes;

    int restore_planes = f.restore_planes;
    int sb128 = fp->sb128;
    int not_last = sby + 1 < f.sbh;
    int start_tile_val = sby < (int)f.start_of_tile_row.size() ? f.start_of_tile_row[sby] : 0;
    int first_flag = start_tile_val & 1;

    if (restore_planes & 6) {
        int ss_ver = 1, ss_hor = 1;
        int h = (f.bh * 4) >> ss_ver;
        int w = (f.bw * 4) >> ss_hor;
        int next_row_y = (sby + 1) << ((6 - ss_ver) + sb128);
        int row_h = imin(next_row_y - (8 >> ss_ver) * not_last, h);
        int offset_uv = (8 * (sby != 0)) >> ss_ver;
        int y_stripe = (sby << ((6 - ss_ver) + sb128)) - offset_uv;
        if (sby != 0 && first_flag) {
            for (int pl = 1; pl < 3; pl++)
                if (restore_planes & (1 << pl))
                    lr_sbrow_plane(ctx, f.p[pl], (ptrdiff_t)imax(y_stripe, 0) * f.stride[1], y_stripe, w, h,
                                   y_stripe + (8 >> ss_ver), pl, FIRST_TOP);
            y_stripe += 8 >> ss_ver;
        }
        int first_bot = first_flag ? FIRST_BOTTOM : FIRST_NONE;
        for (int pl = 1; pl < 3; pl++)
            if (restore_planes & (1 << pl))
                lr_sbrow_plane(ctx, f.p[pl], (ptrdiff_t)imax(y_stripe, 0) * f.stride[1], y_stripe, w, h, row_h, pl,
                               first_bot);
    }
    if (restore_planes & 1) {
        int h = f.bh * 4, w = f.bw * 4;
        int next_row_y = (sby + 1) << (6 + sb128);
        int row_h = imin(next_row_y - 8 * not_last, h);
        int offset_y = 8 * (sby != 0);
        int y_stripe = (sby << (6 + sb128)) - offset_y;
        if (sby != 0 && first_flag) {
            lr_sbrow_plane(ctx, f.p[0], (ptrdiff_t)imax(y_stripe, 0) * f.stride[0], y_stripe, w, h, y_stripe + 8, 0,
                           FIRST_TOP);
            y_stripe += 8;
        }
        lr_sbrow_plane(ctx, f.p[0], (ptrdiff_t)imax(y_stripe, 0) * f.stride[0], y_stripe, w, h, row_h, 0,
                       first_flag ? FIRST_BOTTOM : FIRST_NONE);
    }
}

}  // namespace r2o

namespace r2o {
/* looprestoration.rs:1820-1839 backup_nxu: the n samples left of src_off on
 * each of u rows into columns 6-n .. 5 of [6]-wide rows (bounds-checked as
 * the reference does) */
static void backup_nxu(Left6 *dst, size_t dst_len, const pixel *src, size_t src_len, size_t src_off,
                       ptrdiff_t src_stride, int u, size_t n) {
    size_t abs_stride = (size_t)(src_stride < 0 ? -src_stride : src_stride);
    size_t di = 0, si = src_off;
    while (u > 0) {
        if (di < dst_len && si >= n && si + n <= src_len)
            for (size_t i = 0; i < n; i++) dst[di][6 - n + i] = src[si - n + i];
        di++;
        si += abs_stride;
        u--;
    }
}
/* looprestoration.rs:1841-1845 copy_n_lines */
static void copy_n_lines(pixel *dst, size_t dst_len, const pixel *src, size_t src_len, ptrdiff_t stride, size_t n) {
    size_t len = (size_t)(stride < 0 ? -stride : stride) * n;
    size_t copy_len = len < dst_len ? len : dst_len;
    if (src_len < copy_len) copy_len = src_len;
    memcpy(dst, src, sizeof(pixel) * copy_len);
}
}  // namespace r2o

/* ---- known-answer-test hooks (the reference's looprestoration.rs tests) ---- */
extern "C" {
/* Constant tables and flags by name: which = 0 PC_WIENER_NORMALIZER[i],
 * 1 WIENER_NS_CONFIG_Y[i][k], 2 WIENER_NS_CONFIG_UV[i][k],
 * 3 WIENER_NS_CONFIG_UV_FROM_Y[i][k], 4 PC_WIENER_CONFIG[i][k],
 * 5 GDF_COORDS[i][k], 6 LR_HAVE_* flag i (0 left .. 3 bottom), 7 MODE_OFFSETS[i];
 * i = -1 returns the table's length. */
int r2o_lr_const(int which, int i, int k) {
    using namespace r2o;
    switch (which) {
        case 0: return i < 0 ? 4 : PC_WIENER_NORMALIZER[i];
        case 1: return i < 0 ? 16 : WIENER_NS_CONFIG_Y[i][k];
        case 2: return i < 0 ? 6 : WIENER_NS_CONFIG_UV[i][k];
        case 3: return i < 0 ? 12 : WIENER_NS_CONFIG_UV_FROM_Y[i][k];
        case 4: return i < 0 ? 12 : PC_WIENER_CONFIG[i][k];
        case 5: return i < 0 ? 18 : GDF_COORDS[i][k];
        case 6: {
            static const int fl[4] = {LR_HAVE_LEFT, LR_HAVE_RIGHT, LR_HAVE_TOP, LR_HAVE_BOTTOM};
            return i < 0 ? 4 : fl[i];
        }
        case 7: return i < 0 ? 4 : MODE_OFFSETS[i];
    }
    return 0;
}
void r2o_backup_row(uint16_t *dst, int o, const uint16_t *src, int64_t src_o, const uint16_t *left, int left_off,
                    int w, int edge_len, int edges) {
    r2o::backup_row(dst, o, src, src_o, left, left_off, w, edge_len, edges);
}
void r2o_backup_row_lpf(uint16_t *dst, int o, const uint16_t *src, int64_t src_o, int w, int edge_len, int edges) {
    r2o::backup_row_lpf(dst, o, src, src_o, w, edge_len, edges);
}
/* rows: an array of row pointers, as the reference's &[&[P]] */
void r2o_compute_gradient_row(uint16_t *dst_x4, const uint16_t *const *rows, int row_off, int col_off, int w,
                              uint32_t shift) {
    r2o::compute_gradient_row((uint16_t(*)[4])dst_x4, rows, row_off, col_off, w, shift);
}
int r2o_get_class_lut_idx(const uint16_t *const *rows, int row_center, int col_off, const uint16_t *noskip_mask,
                          int base_q, int bx, int by, int bh, int bitdepth_min_8) {
    return r2o::get_class_lut_idx(rows, row_center, col_off, noskip_mask, base_q, bx, by, bh, bitdepth_min_8);
}
void r2o_ns_wiener_single_uv(uint16_t *p, int64_t p_off, int64_t stride, const uint16_t *left_6, const uint16_t *lpf,
                             int64_t lpf_off, const uint16_t *lpf_bottom, int64_t lpf_bottom_off, int w, int h,
                             const int8_t *filter18, const uint16_t *luma, int64_t luma_off, int64_t lstride,
                             const uint16_t *luma_top, int64_t luma_top_off, const uint16_t *luma_bottom,
                             int64_t luma_bottom_off, int ss_hor, int ss_ver, int ds_flt, int edges,
                             const uint16_t *ll_mask_x4, int bitdepth) {
    r2o::ns_wiener_single_uv(p, p_off, stride, (const r2o::Left6 *)left_6, lpf, lpf_off, lpf_bottom, lpf_bottom_off,
                             w, h, filter18, luma, luma_off, lstride, luma_top, luma_top_off, luma_bottom,
                             luma_bottom_off, ss_hor, ss_ver, ds_flt, edges, (const uint16_t(*)[4])ll_mask_x4,
                             bitdepth);
}
void r2o_gdf_prep(int8_t *dst, int dst_stride, const uint16_t *p, int64_t p_off, int64_t stride,
                  const uint16_t *left_6, const uint16_t *lpf, int64_t lpf_off, const uint16_t *lpf_bottom,
                  int64_t lpf_bottom_off, int w, int h, int ref_dst_idx, int qp_idx, int edges, int bitdepth) {
    r2o::gdf_prep(dst, dst_stride, p, p_off, stride, (const r2o::Left6 *)left_6, lpf, lpf_off, lpf_bottom,
                  lpf_bottom_off, w, h, ref_dst_idx, qp_idx, edges, bitdepth);
}
void r2o_backup_nxu(uint16_t *dst_x6, int64_t dst_len, const uint16_t *src, int64_t src_len, int64_t src_off,
                    int64_t src_stride, int u, int64_t n) {
    r2o::backup_nxu((r2o::Left6 *)dst_x6, dst_len, src, src_len, src_off, src_stride, u, n);
}
void r2o_copy_n_lines(uint16_t *dst, int64_t dst_len, const uint16_t *src, int64_t src_len, int64_t stride,
                      int64_t n) {
    r2o::copy_n_lines(dst, dst_len, src, src_len, stride, n);
}
/* looprestoration.rs:273-329 gdf_add */
void r2o_gdf_add(uint16_t *p, int64_t stride, const int8_t *err, int err_stride, int w, int h, int scale,
                 const uint16_t *ll_mask_x4, int bitdepth) {
    r2o::gdf_add(p, stride, err, err_stride, w, h, scale, (const uint16_t(*)[4])ll_mask_x4, bitdepth);
}
void r2o_backup_row_luma(uint16_t *dst, int o, const uint16_t *src, int64_t src_o, int64_t src_stride, int w,
                         int edges, int ss_hor, int ss_ver, int cfl_ds_flt) {
    r2o::backup_row_luma(dst, o, src, src_o, src_stride, w, edges, ss_hor, ss_ver, cfl_ds_flt);
}
void r2o_ns_wiener_single_y(uint16_t *p, int64_t p_off, int64_t stride, const uint16_t *left_6, const uint16_t *lpf,
                            int64_t lpf_off, const uint16_t *lpf_bottom, int64_t lpf_bottom_off, int w, int h,
                            const int8_t *filter16, int edges, const uint16_t *ll_mask_x4, int bitdepth) {
    r2o::ns_wiener_single_y(p, p_off, stride, (const r2o::Left6 *)left_6, lpf, lpf_off, lpf_bottom, lpf_bottom_off, w,
                            h, filter16, edges, (const uint16_t(*)[4])ll_mask_x4, bitdepth);
}
void r2o_wiener_multi(uint16_t *p, int64_t p_off, int64_t stride, const uint16_t *left_6, const uint16_t *lpf,
                      int64_t lpf_off, const uint16_t *lpf_bottom, int64_t lpf_bottom_off, int w, int h,
                      const int8_t *filters_user_x18, const int16_t *filters_pretrained_x13,
                      const uint8_t *subclass_lut, const uint16_t *noskip_mask, int base_q, int edges,
                      const uint16_t *ll_mask_x4, int bitdepth) {
    r2o::wiener_multi(p, p_off, stride, (const r2o::Left6 *)left_6, lpf, lpf_off, lpf_bottom, lpf_bottom_off, w, h,
                      (const int8_t(*)[18])filters_user_x18, 18, (const int16_t(*)[13])filters_pretrained_x13,
                      subclass_lut, noskip_mask, base_q, edges, (const uint16_t(*)[4])ll_mask_x4, bitdepth);
}
}
