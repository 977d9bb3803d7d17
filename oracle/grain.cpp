/*
 * Oracle: AV2 film-grain synthesis and apply.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Restates crates/rav2d/src/filmgrain.rs:1-941 and the picture wrapper
 * decode.rs:4641-4775 of the rav2d reference.
 */
#include "oracle.h"

#define R2G_TABLE(type, name) static const type name
#include "av2_tables.h"

namespace r2o {

enum { GRAIN_WIDTH = 82, GRAIN_HEIGHT = 73, SUB_GRAIN_WIDTH = 44, SUB_GRAIN_HEIGHT = 38 };
typedef int16_t GrainLut[GRAIN_HEIGHT][GRAIN_WIDTH];

/* filmgrain.rs:11-16 get_random_number */
uint32_t get_random_number(uint32_t bits, uint32_t *state) {
    uint32_t r = *state;
    uint32_t bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1;
    *state = (r >> 1) | (bit << 15);
    return (*state >> (16 - bits)) & ((1u << bits) - 1);
}

/* filmgrain.rs:18-20 round2 */
int round2(int x, uint32_t shift) { return (x + ((1 << shift) >> 1)) >> shift; }

/* filmgrain.rs:22-57 generate_scaling_8bpc and :59-113 generate_scaling_hbd */
void generate_scaling(int bitdepth, const uint8_t (*points)[2], int num, uint8_t *scaling) {
    int shift_x = bitdepth - 8;
    int scaling_size = 1 << bitdepth;
    if (num == 0) {
        memset(scaling, 0, scaling_size);
        return;
    }
    memset(scaling, points[0][1], (size_t)points[0][0] << shift_x);
    for (int i = 0; i < num - 1; i++) {
        int bx = points[i][0], by = points[i][1], ex = points[i + 1][0], ey = points[i + 1][1];
        int dx = ex - bx, dy = ey - by;
        if (dx <= 0) continue;
        int delta = dy * ((0x10000 + (dx >> 1)) / dx);
        int d = 0x8000;
        for (int x = 0; x < dx; x++) {
            scaling[(bx + x) << shift_x] = (uint8_t)(by + (d >> 16));
            d += delta;
        }
    }
    int n = points[num - 1][0] << shift_x;
    memset(scaling + n, points[num - 1][1], scaling_size - n);
    if (bitdepth == 8) return;
    int pad = 1 << shift_x, rnd = pad >> 1;
    for (int i = 0; i < num - 1; i++) {
        int bx = points[i][0] << shift_x, ex = points[i + 1][0] << shift_x;
        int dx = ex - bx;
        for (int x = 0; x < dx; x += pad) {
            int base = scaling[bx + x];
            int range = scaling[bx + x + pad] - base;
            int r = rnd;
            for (int n2 = 1; n2 < pad; n2++) {
                r += range;
                scaling[bx + x + n2] = (uint8_t)(base + (r >> shift_x));
            }
        }
    }
}

/* filmgrain.rs:115-158 generate_grain_y */
static void generate_grain_y(GrainLut buf, const R2gFilmGrainData &data, uint32_t seed, int bitdepth) {
    int bitdepth_min_8 = bitdepth - 8;
    int shift = 4 - bitdepth_min_8 + data.grain_scale_shift;
    int grain_ctr = 128 << bitdepth_min_8;
    int grain_min = -grain_ctr, grain_max = grain_ctr - 1;
    for (int y = 0; y < GRAIN_HEIGHT; y++)
        for (int x = 0; x < GRAIN_WIDTH; x++) {
            uint32_t value = get_random_number(11, &seed);
            buf[y][x] = (int16_t)round2(GAUSSIAN_SEQUENCE[value], shift);
        }
    const int ar_pad = 3;
    int ar_lag = data.ar_coeff_lag;
    for (int y = ar_pad; y < GRAIN_HEIGHT; y++)
        for (int x = ar_pad; x < GRAIN_WIDTH - ar_pad; x++) {
            const int8_t *coeff = data.ar_coeffs[0];
            int sum = 0, ci = 0;
            for (int dy = y - ar_lag; dy <= y; dy++) {
                int dx_end = dy == y ? x : x + ar_lag + 1;
                for (int dx = x - ar_lag; dx < dx_end; dx++) {
                    if (dy == y && dx == x) break;
                    sum += coeff[ci] * buf[dy][dx];
                    ci++;
                }
            }
            int grain = buf[y][x] + round2(sum, data.ar_coeff_shift);
            buf[y][x] = (int16_t)iclip(grain, grain_min, grain_max);
        }
}

/* filmgrain.rs:160-229 generate_grain_uv */
static void generate_grain_uv(GrainLut buf, const GrainLut buf_y, const R2gFilmGrainData &data, uint32_t seed,
                              int uv, bool subx, bool suby, int bitdepth) {
    seed ^= uv ? 0x49d8 : 0xb524;
    int bitdepth_min_8 = bitdepth - 8;
    int shift = 4 - bitdepth_min_8 + data.grain_scale_shift;
    int grain_ctr = 128 << bitdepth_min_8;
    int grain_min = -grain_ctr, grain_max = grain_ctr - 1;
    int chroma_w = subx ? SUB_GRAIN_WIDTH : GRAIN_WIDTH;
    int chroma_h = suby ? SUB_GRAIN_HEIGHT : GRAIN_HEIGHT;
    for (int y = 0; y < chroma_h; y++)
        for (int x = 0; x < chroma_w; x++) {
            uint32_t value = get_random_number(11, &seed);
            buf[y][x] = (int16_t)round2(GAUSSIAN_SEQUENCE[value], shift);
        }
    const int ar_pad = 3;
    int ar_lag = data.ar_coeff_lag;
    int subx_i = subx, suby_i = suby;
    for (int y = ar_pad; y < chroma_h; y++)
        for (int x = ar_pad; x < chroma_w - ar_pad; x++) {
            const int8_t *coeff = data.ar_coeffs[1 + uv];
            int sum = 0, ci = 0;
            bool done = false;
            for (int dy = y - ar_lag; dy <= y && !done; dy++) {
                int dx_end = dy == y ? x + 1 : x + ar_lag + 1;
                for (int dx = x - ar_lag; dx < dx_end; dx++) {
                    if (dy == y && dx == x) {
                        if (data.num_points[0] > 0) {
                            int luma_x = ((x - ar_pad) << subx_i) + ar_pad;
                            int luma_y = ((y - ar_pad) << suby_i) + ar_pad;
                            int luma = 0;
                            for (int i = 0; i <= suby_i; i++)
                                for (int j = 0; j <= subx_i; j++) luma += buf_y[luma_y + i][luma_x + j];
                            luma = round2(luma, subx_i + suby_i);
                            sum += luma * coeff[ci];
                        }
                        done = true;
                        break;
                    }
                    sum += coeff[ci] * buf[dy][dx];
                    ci++;
                }
            }
            int grain = buf[y][x] + round2(sum, data.ar_coeff_shift);
            buf[y][x] = (int16_t)iclip(grain, grain_min, grain_max);
        }
}

/* filmgrain.rs:231-246 sample_lut */
static inline int sample_lut(const GrainLut lut, int bs, const int offsets[2][2][2], int subx, int suby, int bx,
                             int by, int x, int y) {
    const int *off = offsets[bx][by];
    int offx = 3 + (2 >> subx) * (3 + off[1]);
    int offy = 3 + (2 >> suby) * (3 + off[0]);
    return lut[offy + y + (bs >> suby) * by][offx + x + (bs >> subx) * bx];
}

/* The per-block offset draws shared by fgy_32x32xn (:248-407) and
 * fguv_32x32xn (:409-598). */
static void init_seeds(uint32_t seed[2], int rows, uint32_t in_seed, int row_num) {
    for (int i = 0; i < rows; i++) {
        seed[i] = in_seed;
        seed[i] ^= (uint32_t)((((row_num - i) * 37 + 178) & 0xFF)) << 8;
        seed[i] ^= (uint32_t)(((row_num - i) * 173 + 105) & 0xFF);
    }
}
static void draw_offsets(int offsets[2][2][2], uint32_t seed[2], int rows, const R2gFilmGrainData &data, int bx) {
    if (data.overlap_flag && bx > 0)
        for (int i = 0; i < rows; i++)
            for (int n = 0; n < 2; n++) offsets[1][i][n] = offsets[0][i][n];
    for (int i = 0; i < rows; i++)
        for (int n = 0; n < 2; n++) {
            offsets[0][i][n] = (int)(((uint32_t)(3 - data.block_size) * get_random_number(9, &seed[i])) >> 6);
            for (int k = 0; k < 3; k++) get_random_number(16, &seed[i]);
        }
}

/* filmgrain.rs:248-407 fgy_32x32xn */
static void fgy_32x32xn(pixel *dst, const pixel *src, ptrdiff_t stride, const R2gFilmGrainData &data,
                        uint32_t in_seed, int pw, const uint8_t *scaling, const GrainLut lut, int bh, int row_num,
                        int bitdepth) {
    int rows = 1 + (data.overlap_flag && row_num > 0);
    int bitdepth_min_8 = bitdepth - 8;
    int grain_ctr = 128 << bitdepth_min_8;
    int grain_min = -grain_ctr, grain_max = grain_ctr - 1;
    int bs = 16 << data.block_size;
    int min_value, max_value;
    if (data.clip_to_restricted_range) {
        min_value = 16 << bitdepth_min_8;
        max_value = 235 << bitdepth_min_8;
    } else {
        min_value = 0;
        max_value = (1 << bitdepth) - 1;
    }
    uint32_t seed[2] = {0, 0};
    init_seeds(seed, rows, in_seed, row_num);
    int offsets[2][2][2] = {{{0}}};
    static const int w[2][2] = {{27, 17}, {17, 27}};
    for (int bx = 0; bx < pw; bx += bs) {
        int bw = imin(bs, pw - bx);
        draw_offsets(offsets, seed, rows, data, bx);
        int ystart = (data.overlap_flag && row_num > 0) ? imin(2, bh) : 0;
        int xstart = (data.overlap_flag && bx > 0) ? imin(2, bw) : 0;
        auto add = [&](int x, int y, int grain) {
            ptrdiff_t si = y * stride + x + bx;
            int sv = src[si];
            int noise = round2(scaling[sv] * grain, data.scaling_shift);
            dst[si] = (pixel)iclip(sv + noise, min_value, max_value);
        };
        for (int y = ystart; y < bh; y++) {
            for (int x = xstart; x < bw; x++) add(x, y, sample_lut(lut, bs, offsets, 0, 0, 0, 0, x, y));
            for (int x = 0; x < xstart; x++) {
                int grain = sample_lut(lut, bs, offsets, 0, 0, 0, 0, x, y);
                int old = sample_lut(lut, bs, offsets, 0, 0, 1, 0, x, y);
                grain = iclip(round2(old * w[x][0] + grain * w[x][1], 5), grain_min, grain_max);
                add(x, y, grain);
            }
        }
        for (int y = 0; y < ystart; y++) {
            for (int x = xstart; x < bw; x++) {
                int grain = sample_lut(lut, bs, offsets, 0, 0, 0, 0, x, y);
                int old = sample_lut(lut, bs, offsets, 0, 0, 0, 1, x, y);
                grain = iclip(round2(old * w[y][0] + grain * w[y][1], 5), grain_min, grain_max);
                add(x, y, grain);
            }
            for (int x = 0; x < xstart; x++) {
                int top = sample_lut(lut, bs, offsets, 0, 0, 0, 1, x, y);
                int old = sample_lut(lut, bs, offsets, 0, 0, 1, 1, x, y);
                top = iclip(round2(old * w[x][0] + top * w[x][1], 5), grain_min, grain_max);
                int grain = sample_lut(lut, bs, offsets, 0, 0, 0, 0, x, y);
                int old2 = sample_lut(lut, bs, offsets, 0, 0, 1, 0, x, y);
                grain = iclip(round2(old2 * w[x][0] + grain * w[x][1], 5), grain_min, grain_max);
                grain = iclip(round2(top * w[y][0] + grain * w[y][1], 5), grain_min, grain_max);
                add(x, y, grain);
            }
        }
    }
}

/* filmgrain.rs:409-598 fguv_32x32xn */
static void fguv_32x32xn(pixel *dst, const pixel *src, ptrdiff_t stride, const R2gFilmGrainData &data,
                         uint32_t in_seed, int pw, const uint8_t *scaling, const GrainLut lut, int bh, int row_num,
                         const pixel *luma_row, ptrdiff_t luma_stride, int uv, bool is_id, int sx, int sy,
                         int bitdepth) {
    int rows = 1 + (data.overlap_flag && row_num > 0);
    int bitdepth_min_8 = bitdepth - 8;
    int grain_ctr = 128 << bitdepth_min_8;
    int grain_min = -grain_ctr, grain_max = grain_ctr - 1;
    int bs = 16 << data.block_size;
    int min_value, max_value;
    if (data.clip_to_restricted_range) {
        min_value = 16 << bitdepth_min_8;
        max_value = (is_id ? 235 : 240) << bitdepth_min_8;
    } else {
        min_value = 0;
        max_value = (1 << bitdepth) - 1;
    }
    uint32_t seed[2] = {0, 0};
    init_seeds(seed, rows, in_seed, row_num);
    int offsets[2][2][2] = {{{0}}};
    static const int w[2][2][2] = {{{27, 17}, {17, 27}}, {{23, 22}, {0, 0}}};
    for (int bx = 0; bx < pw; bx += bs >> sx) {
        int bw = imin(bs >> sx, pw - bx);
        draw_offsets(offsets, seed, rows, data, bx);
        int ystart = (data.overlap_flag && row_num > 0) ? imin(2 >> sy, bh) : 0;
        int xstart = (data.overlap_flag && bx > 0) ? imin(2 >> sx, bw) : 0;
        auto add = [&](int x, int y, int grain) {
            ptrdiff_t lx = (ptrdiff_t)(bx + x) << sx;
            ptrdiff_t ly = (ptrdiff_t)y << sy;
            int luma = luma_row[ly * luma_stride + lx];
            int avg = sx ? (luma + luma_row[ly * luma_stride + lx + 1] + 1) >> 1 : luma;
            ptrdiff_t si = y * stride + bx + x;
            int sv = src[si];
            int val;
            if (!data.chroma_scaling_from_luma) {
                int combined = avg * data.uv_luma_mult[uv] + sv * data.uv_mult[uv];
                val = iclip((combined >> 6) + data.uv_offset[uv] * (1 << bitdepth_min_8), 0, (1 << bitdepth) - 1);
            } else {
                val = avg;
            }
            int noise = round2(scaling[val] * grain, data.scaling_shift);
            dst[si] = (pixel)iclip(sv + noise, min_value, max_value);
        };
        for (int y = ystart; y < bh; y++) {
            for (int x = xstart; x < bw; x++) add(x, y, sample_lut(lut, bs, offsets, sx, sy, 0, 0, x, y));
            for (int x = 0; x < xstart; x++) {
                int grain = sample_lut(lut, bs, offsets, sx, sy, 0, 0, x, y);
                int old = sample_lut(lut, bs, offsets, sx, sy, 1, 0, x, y);
                grain = iclip(round2(old * w[sx][x][0] + grain * w[sx][x][1], 5), grain_min, grain_max);
                add(x, y, grain);
            }
        }
        for (int y = 0; y < ystart; y++) {
            for (int x = xstart; x < bw; x++) {
                int grain = sample_lut(lut, bs, offsets, sx, sy, 0, 0, x, y);
                int old = sample_lut(lut, bs, offsets, sx, sy, 0, 1, x, y);
                grain = iclip(round2(old * w[sy][y][0] + grain * w[sy][y][1], 5), grain_min, grain_max);
                add(x, y, grain);
            }
            for (int x = 0; x < xstart; x++) {
                int top = sample_lut(lut, bs, offsets, sx, sy, 0, 1, x, y);
                int old = sample_lut(lut, bs, offsets, sx, sy, 1, 1, x, y);
                top = iclip(round2(old * w[sx][x][0] + top * w[sx][x][1], 5), grain_min, grain_max);
                int grain = sample_lut(lut, bs, offsets, sx, sy, 0, 0, x, y);
                int old2 = sample_lut(lut, bs, offsets, sx, sy, 1, 0, x, y);
                grain = iclip(round2(old2 * w[sx][x][0] + grain * w[sx][x][1], 5), grain_min, grain_max);
                grain = iclip(round2(top * w[sy][y][0] + grain * w[sy][y][1], 5), grain_min, grain_max);
                add(x, y, grain);
            }
        }
    }
}

}  // namespace r2o

using namespace r2o;

extern "C" {

/* filmgrain.rs:617-686 prep_grain: the three grain templates (82x73 luma,
 * 44x38 4:2:0 chroma in the top-left of 82x73 arrays) and scaling LUTs. */
int r2o_prep_grain(const R2gFilmGrainData *fgd, uint32_t seed, int bitdepth, int16_t *lut_y, int16_t *lut_u,
                   int16_t *lut_v, uint8_t *scaling_y, uint8_t *scaling_u, uint8_t *scaling_v) {
    GrainLut *ly = (GrainLut *)lut_y, *lu = (GrainLut *)lut_u, *lv = (GrainLut *)lut_v;
    memset(*ly, 0, sizeof(GrainLut));
    memset(*lu, 0, sizeof(GrainLut));
    memset(*lv, 0, sizeof(GrainLut));
    generate_grain_y(*ly, *fgd, seed, bitdepth);
    if (fgd->num_points[1] > 0 || fgd->chroma_scaling_from_luma)
        generate_grain_uv(*lu, *ly, *fgd, seed, 0, true, true, bitdepth);
    if (fgd->num_points[2] > 0 || fgd->chroma_scaling_from_luma)
        generate_grain_uv(*lv, *ly, *fgd, seed, 1, true, true, bitdepth);
    int sz = 1 << bitdepth;
    memset(scaling_y, 0, sz);
    memset(scaling_u, 0, sz);
    memset(scaling_v, 0, sz);
    if (fgd->num_points[0] > 0) generate_scaling(bitdepth, fgd->points[0], fgd->num_points[0], scaling_y);
    if (!fgd->chroma_scaling_from_luma)
        for (int uv = 0; uv < 2; uv++)
            if (fgd->num_points[uv + 1] > 0)
                generate_scaling(bitdepth, fgd->points[uv + 1], fgd->num_points[uv + 1], uv ? scaling_v : scaling_u);
    return 0;
}

/* decode.rs:4672-4775 apply_grain_to_picture_mt with filmgrain.rs:847-941
 * apply_grain_mt (n_threads = 1): dst starts as a copy of src, then each
 * grained plane is overwritten band by band (filmgrain.rs:688-822). */
int r2o_apply_grain(const R2gFilmGrainData *fgd, uint32_t seed, int w, int h, int bitdepth, const uint16_t *src_y,
                    const uint16_t *src_u, const uint16_t *src_v, uint16_t *dst_y, uint16_t *dst_u,
                    uint16_t *dst_v, int64_t y_stride, int64_t uv_stride) {
    const R2gFilmGrainData &d = *fgd;
    int aligned_h = (h + 127) & ~127;
    memcpy(dst_y, src_y, sizeof(uint16_t) * y_stride * aligned_h);
    memcpy(dst_u, src_u, sizeof(uint16_t) * uv_stride * (aligned_h >> 1));
    memcpy(dst_v, src_v, sizeof(uint16_t) * uv_stride * (aligned_h >> 1));
    bool has = d.num_points[0] || d.num_points[1] || d.num_points[2] ||
               (d.clip_to_restricted_range && d.chroma_scaling_from_luma);
    if (!has) return 0;
    static thread_local GrainLut lut[3];
    static thread_local uint8_t scaling[3][4096];
    r2o_prep_grain(fgd, seed, bitdepth, &lut[0][0][0], &lut[1][0][0], &lut[2][0][0], scaling[0], scaling[1],
                   scaling[2]);
    int bs = 16 << d.block_size;
    int rows = (h + bs - 1) / bs;
    const int ss_x = 1, ss_y = 1;
    for (int row = 0; row < rows; row++) {
        int row_start = row * bs;
        if (d.num_points[0] > 0) {
            int bh = imin(h - row_start, bs);
            ptrdiff_t off = (ptrdiff_t)row_start * y_stride;
            fgy_32x32xn(dst_y + off, src_y + off, y_stride, d, seed, w, scaling[0], lut[0], bh, row, bitdepth);
        }
        int ch = (imin(h - row_start, bs) + ss_y) >> ss_y;
        int cw = (w + ss_x) >> ss_x;
        ptrdiff_t uv_off = (ptrdiff_t)(row_start >> ss_y) * uv_stride;
        ptrdiff_t luma_off = (ptrdiff_t)row_start * y_stride;
        for (int uv = 0; uv < 2; uv++) {
            if (!(d.num_points[uv + 1] > 0 || d.chroma_scaling_from_luma)) continue;
            /* scaling_for_uv (filmgrain.rs:824-830) hands chroma the luma LUT
             * under chroma_scaling_from_luma; an ungenerated LUT is empty and
             * has_uv() then skips the plane */
            if (d.chroma_scaling_from_luma && d.num_points[0] == 0) continue;
            const uint8_t *sc = d.chroma_scaling_from_luma ? scaling[0] : scaling[uv + 1];
            const uint16_t *s = uv ? src_v : src_u;
            uint16_t *dd = uv ? dst_v : dst_u;
            fguv_32x32xn(dd + uv_off, s + uv_off, uv_stride, d, seed, cw, sc, lut[1 + uv], ch, row,
                         src_y + luma_off, y_stride, uv, d.mc_identity != 0, ss_x, ss_y, bitdepth);
        }
    }
    return 0;
}

/* Single-function hooks for the reference's filmgrain.rs unit tests
 * (:943-1342).  Templates are 73 x 82 int16 arrays (GrainLut). */
void r2o_generate_grain_y(int16_t *buf, const R2gFilmGrainData *fgd, uint32_t seed, int bitdepth) {
    generate_grain_y(*(GrainLut *)buf, *fgd, seed, bitdepth);
}
void r2o_generate_grain_uv(int16_t *buf, const int16_t *buf_y, const R2gFilmGrainData *fgd, uint32_t seed, int uv,
                           int subx, int suby, int bitdepth) {
    generate_grain_uv(*(GrainLut *)buf, *(const GrainLut *)buf_y, *fgd, seed, uv, subx != 0, suby != 0, bitdepth);
}
/* offsets: [bx][by][n] as 8 ints */
int r2o_sample_lut(const int16_t *lut, int bs, const int *offsets, int subx, int suby, int bx, int by, int x, int y) {
    return sample_lut(*(const GrainLut *)lut, bs, (const int(*)[2][2])offsets, subx, suby, bx, by, x, y);
}
void r2o_fgy_32x32xn(uint16_t *dst, const uint16_t *src, int64_t stride, const R2gFilmGrainData *fgd, uint32_t seed,
                     int pw, const uint8_t *scaling, const int16_t *lut, int bh, int row_num, int bitdepth) {
    fgy_32x32xn(dst, src, stride, *fgd, seed, pw, scaling, *(const GrainLut *)lut, bh, row_num, bitdepth);
}
void r2o_fguv_32x32xn(uint16_t *dst, const uint16_t *src, int64_t stride, const R2gFilmGrainData *fgd, uint32_t seed,
                      int pw, const uint8_t *scaling, const int16_t *lut, int bh, int row_num, const uint16_t *luma,
                      int64_t luma_stride, int uv, int is_id, int sx, int sy, int bitdepth) {
    fguv_32x32xn(dst, src, stride, *fgd, seed, pw, scaling, *(const GrainLut *)lut, bh, row_num, luma, luma_stride, uv,
                 is_id != 0, sx, sy, bitdepth);
}

uint32_t r2o_get_random_number(uint32_t bits, uint32_t *state) { return get_random_number(bits, state); }
int r2o_round2(int x, uint32_t shift) { return round2(x, shift); }
int r2o_generate_scaling(int bitdepth, const uint8_t *points, int num, uint8_t *scaling) {
    generate_scaling(bitdepth, (const uint8_t(*)[2])points, num, scaling);
    return 0;
}

}  // extern "C"
