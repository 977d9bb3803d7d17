// AV2 deblocking on the GPU: one launch for all vertical edges of a frame
// (luma + both chroma planes), then one for all horizontal edges.
//
// Reference: crates/rav2d/src/deblock.rs (deblock_bd :217, filter_choice_bd
// :81, deblock64_cols :1623, deblock64_rows :1866, setup_thr_* :1477/:1520)
// and lf_mask.rs:332-358.  The reference walks the frame per 64-row band,
// edge by edge; here every 4-line edge segment is one thread.  Transform
// sizes bound each edge's filter length (MAX_WIDTH_* by edge class), so the
// pixels one edge reads never overlap the pixels another edge of the same
// direction writes, and the segments can run in any order in place.
//
// Each thread keeps a 4 x 16 window of the edge neighbourhood in registers:
// line l (0..3) along the edge, position j (0..15) across it, j = 8 is the
// first sample on the positive side.  Vertical edges load each line as four
// 4-sample vectors; horizontal edges load each position row as one 4-sample
// vector covering all four lines.
#include "r2g_common.cuh"

namespace {

__constant__ uint8_t c_dq_tbl[24] = {40, 41, 43, 44, 45, 47, 48, 49, 51, 52, 54, 55,
                                     57, 59, 60, 62, 64, 66, 68, 70, 72, 74, 76, 78};
__constant__ int8_t c_max_width_y[4] = {1, 3, 6, 8};
__constant__ int8_t c_max_width_uv[3] = {1, 3, 4};
__constant__ int8_t c_q_first[3] = {45, 40, 32};
__constant__ int8_t c_q_thresh_mults[8] = {32, 25, 19, 19, 0, 18, 0, 17};
__constant__ int8_t c_w_mult[8] = {85, 51, 37, 28, 0, 20, 0, 15};

// quantizer.rs:31-50
R2G_D int dq_lookup(int qidx) {
    qidx = iclip_(qidx, 0, 255);
    if (qidx == 0) return 64;
    qidx -= 1;
    return (int)c_dq_tbl[qidx % 24] << (qidx / 24);
}

// lf_mask.rs:332-342 (quant) and :337-342 (side)
R2G_D uint32_t quant_thr(int hbd, int qidx) {
    int qmax = 255 + 48 * hbd;
    return (uint32_t)((dq_lookup(iclip_(qidx, 0, qmax)) + 4) >> 9);
}
R2G_D uint32_t side_thr(const int16_t *tab, int hbd, int qidx) {
    int b8 = 2 * hbd;
    int q_ind = iclip_(qidx - 24 * b8, 0, 295);
    return (uint32_t)imax_(__ldg(tab + q_ind) + ((1 << 4) >> b8), 0) >> (5 - b8);
}

// init_deblock_thr_lut_{y,uv} (deblock.rs:13-57) evaluated for one 4x4:
// kind 0/1 = luma dir 0/1, 2 = U, 3 = V.  Segments beyond the LUT's filled
// range read 0, as the reference's zero-initialised LUT does.
R2G_D void thr_of(const DevFrame &f, int kind, int qidx, int seg, int &q, int &s) {
    const R2gFrameParams &fp = f.fp;
    int n = fp.seg_enabled ? 8 : 1;
    if (seg >= n) {
        q = s = 0;
        return;
    }
    int qmax = 255 + 48 * f.hbd;
    int yac = fp.seg_enabled ? iclip_(qidx + fp.seg_delta_q[seg], 0, qmax) : qidx;
    int v;
    if (kind < 2)
        v = yac + 8 * fp.deblock_delta_q_y[kind];
    else if (kind == 2)
        v = yac + fp.quant_uac_delta + 8 * fp.deblock_delta_q_u;
    else
        v = yac + fp.quant_vac_delta + 8 * fp.deblock_delta_q_v;
    q = (int)quant_thr(f.hbd, v);
    s = (int)side_thr(f.tab.DEBLOCK_SIDE_THRESHOLDS, f.hbd, v);
}

// deblock.rs:1466 edge_thr
R2G_D int edge_thr(int cur, int prev) { return (cur != 0 && prev != 0) ? (cur + prev + 1) >> 1 : (cur | prev); }

R2G_D uint32_t uabs_(int v) { return (uint32_t)(v < 0 ? -v : v); }

// filter_choice_bd (deblock.rs:81-210) on window lines ls and lt; position
// p(k) = win[line][8 + k].
R2G_D int filter_choice(const int (*win)[16], int ls, int lt, int mwn, int mwp, uint32_t q_thr, uint32_t side_thr) {
#define S(k) win[ls][8 + (k)]
#define T(k) win[lt][8 + (k)]
    uint32_t sd[4];
#pragma unroll
    for (int d = -2; d < 2; d++) {
        uint32_t ds = uabs_(S(d - 1) - S(d) * 2 + S(d + 1));
        uint32_t dt = uabs_(T(d - 1) - T(d) * 2 + T(d + 1));
        sd[d + 2] = (ds + dt + 1) >> 1;
    }
    uint32_t high = sd[0] > sd[3] ? sd[0] : sd[3];
    if (high > side_thr) return 0;
    if (mwp == 1) return 1;
    uint32_t transition = sd[1] + sd[2];
    if (high > (side_thr >> 2)) return 1;
    if (transition > q_thr * 4) return 1;
    if (high > (side_thr >> 3)) return 2;
    if (transition > q_thr * 3) return 2;
    uint32_t end_thr = (side_thr * 3) >> 4;
    if (mwn >= 3) {
        uint32_t ds = uabs_(S(-1) - S(-4) - 3 * (S(-1) - S(-2)));
        uint32_t dt = uabs_(T(-1) - T(-4) - 3 * (T(-1) - T(-2)));
        if (((ds + dt + 1) >> 1) > end_thr) return 2;
    }
    {
        uint32_t ds = uabs_(S(0) - S(3) - 3 * (S(0) - S(1)));
        uint32_t dt = uabs_(T(0) - T(3) - 3 * (T(0) - T(1)));
        if (((ds + dt + 1) >> 1) > end_thr) return 2;
    }
    if (mwp == 3) return 3;
    transition <<= 4;
    int prev = 3;
    for (int dist = 4; dist <= mwp; dist += 2) {
        uint32_t q4 = q_thr * (uint32_t)c_q_first[(dist - 4) >> 1];
        uint32_t e4 = (side_thr * (uint32_t)dist) >> 4;
        if (transition > q4) return prev;
        int d2 = imin_(7, dist);
        if (mwn >= d2) {
            uint32_t ds = uabs_(S(-1) - S(-d2 - 1) - d2 * (S(-1) - S(-2)));
            uint32_t dt = uabs_(T(-1) - T(-d2 - 1) - d2 * (T(-1) - T(-2)));
            if (((ds + dt + 1) >> 1) > e4) return prev;
        }
        uint32_t ds = uabs_(S(0) - S(d2) - d2 * (S(0) - S(1)));
        uint32_t dt = uabs_(T(0) - T(d2) - d2 * (T(0) - T(1)));
        if (((ds + dt + 1) >> 1) > e4) return prev;
        prev = dist;
    }
    return mwp;
#undef S
#undef T
}

// deblock_bd (deblock.rs:217-281) on the register window.  Returns the
// number of modified samples on each side through wn / wp.
R2G_D void deblock_window(int (*win)[16], uint32_t q_thr, uint32_t side_thr, int mwp, int mwn, bool pos_ll,
                          bool neg_ll, int bdmax, int &wn_out, int &wp_out) {
    wn_out = wp_out = 0;
    int width = filter_choice(win, 0, 3, mwn, mwp, q_thr, side_thr);
    if (width < 1) return;
    int wn = imin_(width, mwn), wp = width;
    int clampv = (int)q_thr * c_q_thresh_mults[width - 1];
    int mneg = c_w_mult[wn - 1], mpos = c_w_mult[wp - 1];
#pragma unroll
    for (int l = 0; l < 4; l++) {
        int *L = win[l];
        int delta = iclip_(4 * (3 * (L[8] - L[7]) - (L[9] - L[6])), -clampv, clampv);
        if (!neg_ll) {
            int dn = delta * mneg;
            for (int j = 0; j < wn; j++) {
                int diff = (dn * (wn - j) + (1 << 10)) >> 11;
                L[7 - j] = iclip_(L[7 - j] + diff, 0, bdmax);
            }
        }
        if (!pos_ll) {
            int dp = delta * mpos;
            for (int j = 0; j < wp; j++) {
                int diff = (dp * (wp - j) + (1 << 10)) >> 11;
                L[8 + j] = iclip_(L[8 + j] - diff, 0, bdmax);
            }
        }
    }
    wn_out = neg_ll ? 0 : wn;
    wp_out = pos_ll ? 0 : wp;
}

template <typename P>
struct Vec4;
template <>
struct Vec4<uint8_t> {
    typedef uint32_t T;
    R2G_D static void unpack(T v, int *o) {
        o[0] = v & 0xff;
        o[1] = (v >> 8) & 0xff;
        o[2] = (v >> 16) & 0xff;
        o[3] = v >> 24;
    }
    R2G_D static T pack(const int *i) {
        return (uint32_t)i[0] | ((uint32_t)i[1] << 8) | ((uint32_t)i[2] << 16) | ((uint32_t)i[3] << 24);
    }
};
template <>
struct Vec4<uint16_t> {
    typedef uint2 T;
    R2G_D static void unpack(T v, int *o) {
        o[0] = v.x & 0xffff;
        o[1] = v.x >> 16;
        o[2] = v.y & 0xffff;
        o[3] = v.y >> 16;
    }
    R2G_D static T pack(const int *i) {
        return make_uint2((uint32_t)i[0] | ((uint32_t)i[1] << 16), (uint32_t)i[2] | ((uint32_t)i[3] << 16));
    }
};

R2G_D bool ll_y(const R2gAv2Filter &m, int x4, int y4) {
    return (m.lossless_mask_y[y4 & 63][(x4 >> 4) & 3] >> (x4 & 15)) & 1;
}
R2G_D bool ll_uv(const R2gAv2Filter &m, int cx4, int cy4) {
    return (m.lossless_mask_uv[cy4 & 31][(cx4 >> 3) & 3] >> (cx4 & 7)) & 1;
}

R2G_D int seg_y(const DevFrame &f, int x4, int y4) {
    return f.segmap ? f.segmap[(int64_t)y4 * f.segmap_stride + x4] : 0;
}
R2G_D int seg_uv(const DevFrame &f, int cx4, int cy4) {
    return f.segmap_uv ? f.segmap_uv[(int64_t)cy4 * f.segmap_uv_stride + cx4] : 0;
}

// Edge-threshold pair for a luma 4x4 and its neighbour (setup_thr_* :1477).
R2G_D void luma_thr(const DevFrame &f, int dir, int x4, int y4, int nx4, int ny4, bool subpu, uint32_t &q,
                    uint32_t &s) {
    const R2gAv2Filter &mc = f.masks[(y4 >> 6) * f.sb256w + (x4 >> 6)];
    const R2gAv2Filter &mn = f.masks[(ny4 >> 6) * f.sb256w + (nx4 >> 6)];
    int cq, cs, pq, ps;
    thr_of(f, dir, mc.qidx[((x4 >> 4) & 3) + (((y4 >> 4) & 3) << 2)], seg_y(f, x4, y4), cq, cs);
    thr_of(f, dir, mn.qidx[((nx4 >> 4) & 3) + (((ny4 >> 4) & 3) << 2)], seg_y(f, nx4, ny4), pq, ps);
    int sh = subpu ? 3 : 0;
    q = (uint32_t)(uint16_t)(edge_thr(cq, pq) >> sh);
    s = (uint32_t)(uint16_t)(edge_thr(cs, ps) >> sh);
}
R2G_D void chroma_thr(const DevFrame &f, int pl, int cx4, int cy4, int nx4, int ny4, bool subpu, uint32_t &q,
                      uint32_t &s) {
    const R2gAv2Filter &mc = f.masks[(cy4 >> 5) * f.sb256w + (cx4 >> 5)];
    const R2gAv2Filter &mn = f.masks[(ny4 >> 5) * f.sb256w + (nx4 >> 5)];
    int cq, cs, pq, ps;
    thr_of(f, 2 + pl, mc.qidx[((cx4 >> 3) & 3) + (((cy4 >> 3) & 3) << 2)], seg_uv(f, cx4, cy4), cq, cs);
    thr_of(f, 2 + pl, mn.qidx[((nx4 >> 3) & 3) + (((ny4 >> 3) & 3) << 2)], seg_uv(f, nx4, ny4), pq, ps);
    int sh = subpu ? 3 : 0;
    q = (uint32_t)(uint16_t)(edge_thr(cq, pq) >> sh);
    s = (uint32_t)(uint16_t)(edge_thr(cs, ps) >> sh);
}

// Vertical edge at sample column x (x % 4 == 0), rows y..y+3.
// Window samples outside the plane (pw x ph) read as 0; the edge classes of
// a valid stream never let the filter use them.
template <typename P>
R2G_D void vert_edge(P *plane, int64_t stride, int pw, int x, int y, uint32_t q, uint32_t s, int mwp, int mwn,
                     bool pos_ll, bool neg_ll, int bdmax) {
    typedef Vec4<P> V;
    int win[4][16];
#pragma unroll
    for (int l = 0; l < 4; l++) {
        const P *row = plane + (int64_t)(y + l) * stride;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            int x0 = x - 8 + 4 * c;
            if (x0 >= 0 && x0 + 3 < pw)
                V::unpack(*reinterpret_cast<const typename V::T *>(row + x0), &win[l][4 * c]);
            else
                win[l][4 * c] = win[l][4 * c + 1] = win[l][4 * c + 2] = win[l][4 * c + 3] = 0;
        }
    }
    int wn, wp;
    deblock_window(win, q, s, mwp, mwn, pos_ll, neg_ll, bdmax, wn, wp);
    if (wn == 0 && wp == 0) return;
#pragma unroll
    for (int l = 0; l < 4; l++) {
        P *row = plane + (int64_t)(y + l) * stride;
        for (int j = 8 - wn; j < 8 + wp; j++) row[x - 8 + j] = (P)win[l][j];
    }
}

// Horizontal edge at sample row y (y % 4 == 0), columns x..x+3.
template <typename P>
R2G_D void horz_edge(P *plane, int64_t stride, int ph, int x, int y, uint32_t q, uint32_t s, int mwp, int mwn,
                     bool pos_ll, bool neg_ll, int bdmax) {
    typedef Vec4<P> V;
    int win[4][16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        int yy = y - 8 + j;
        int v[4] = {0, 0, 0, 0};
        if (yy >= 0 && yy < ph) V::unpack(*reinterpret_cast<const typename V::T *>(plane + (int64_t)yy * stride + x), v);
#pragma unroll
        for (int l = 0; l < 4; l++) win[l][j] = v[l];
    }
    int wn, wp;
    deblock_window(win, q, s, mwp, mwn, pos_ll, neg_ll, bdmax, wn, wp);
    for (int j = 8 - wn; j < 8 + wp; j++) {
        int v[4] = {win[0][j], win[1][j], win[2][j], win[3][j]};
        *reinterpret_cast<typename V::T *>(plane + (int64_t)(y - 8 + j) * stride + x) = V::pack(v);
    }
}

// One launch per direction; items [0, nl) are luma 4x4s, [nl, nl + nc)
// chroma 4x4s (U and V share mask decode and run in the same thread).
template <typename P, int DIR>
__global__ void __launch_bounds__(256) deblock_kernel(const DevFrame f) {
    const int nl = f.bw4 * f.bh4;
    const int cbw4 = f.bw4 >> 1, cbh4 = f.bh4 >> 1;
    const int nc = cbw4 * cbh4;
    const R2gFrameParams &fp = f.fp;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < nl + nc; it += gridDim.x * blockDim.x) {
        if (it < nl) {
            if (!fp.deblock_level_y[DIR]) continue;
            int x4 = it % f.bw4, y4 = it / f.bw4;
            if ((DIR == 0 ? x4 : y4) == 0) continue;
            const R2gAv2Filter &m = f.masks[(y4 >> 6) * f.sb256w + (x4 >> 6)];
            int pos = DIR == 0 ? (x4 & 63) : (y4 & 63);
            int idx = DIR == 0 ? ((y4 >> 4) & 3) : ((x4 >> 4) & 3);
            int bit = DIR == 0 ? (y4 & 15) : (x4 & 15);
            const uint16_t(*km)[4] = m.filter_y[DIR][pos];
            int k3 = (km[3][idx] >> bit) & 1, k2 = (km[2][idx] >> bit) & 1, k1 = (km[1][idx] >> bit) & 1,
                k0 = (km[0][idx] >> bit) & 1;
            if (!(k0 | k1 | k2 | k3)) continue;
            int cls = k3 ? 3 : k2 ? 2 : k1;
            int mwp = c_max_width_y[cls];
            int mwn = (DIR == 1 && (y4 & 15) == 0) ? imin_(6, mwp) : mwp;
            bool subpu = (km[4][idx] >> bit) & 1;
            int nx4 = DIR == 0 ? x4 - 1 : x4, ny4 = DIR == 0 ? y4 : y4 - 1;
            uint32_t q, s;
            luma_thr(f, DIR, x4, y4, nx4, ny4, subpu, q, s);
            const R2gAv2Filter &mn = f.masks[(ny4 >> 6) * f.sb256w + (nx4 >> 6)];
            bool pos_ll = ll_y(m, x4, y4), neg_ll = ll_y(mn, nx4, ny4);
            P *pl = plane_ptr<P>(f.R[0]);
            if (DIR == 0)
                vert_edge<P>(pl, f.stride[0], f.w, x4 * 4, y4 * 4, q, s, mwp, mwn, pos_ll, neg_ll, f.bdmax);
            else
                horz_edge<P>(pl, f.stride[0], f.h, x4 * 4, y4 * 4, q, s, mwp, mwn, pos_ll, neg_ll, f.bdmax);
        } else {
            if (!fp.deblock_level_u && !fp.deblock_level_v) continue;
            int c = it - nl;
            int cx4 = c % cbw4, cy4 = c / cbw4;
            if ((DIR == 0 ? cx4 : cy4) == 0) continue;
            const R2gAv2Filter &m = f.masks[(cy4 >> 5) * f.sb256w + (cx4 >> 5)];
            int pos = DIR == 0 ? (cx4 & 31) : (cy4 & 31);
            int idx = DIR == 0 ? ((cy4 & 31) >> 4) : ((cx4 & 31) >> 4);
            int bit = DIR == 0 ? (cy4 & 15) : (cx4 & 15);
            const uint16_t(*km)[4] = m.filter_uv[DIR][pos];
            int k2 = (km[2][idx] >> bit) & 1, k1 = (km[1][idx] >> bit) & 1, k0 = (km[0][idx] >> bit) & 1;
            if (!(k0 | k1 | k2)) continue;
            int cls = k2 ? 2 : k1;
            int mwp = c_max_width_uv[cls];
            int mwn = (DIR == 1 && (cy4 & 7) == 0) ? imin_(2, mwp) : mwp;
            bool subpu = (km[4][idx] >> bit) & 1;
            int nx4 = DIR == 0 ? cx4 - 1 : cx4, ny4 = DIR == 0 ? cy4 : cy4 - 1;
            const R2gAv2Filter &mn = f.masks[(ny4 >> 5) * f.sb256w + (nx4 >> 5)];
            bool pos_ll = ll_uv(m, cx4, cy4), neg_ll = ll_uv(mn, nx4, ny4);
            for (int pl = 0; pl < 2; pl++) {
                if (!(pl ? fp.deblock_level_v : fp.deblock_level_u)) continue;
                uint32_t q, s;
                chroma_thr(f, pl, cx4, cy4, nx4, ny4, subpu, q, s);
                P *plane = plane_ptr<P>(f.R[1 + pl]);
                if (DIR == 0)
                    vert_edge<P>(plane, f.stride[1], f.cw, cx4 * 4, cy4 * 4, q, s, mwp, mwn, pos_ll, neg_ll, f.bdmax);
                else
                    horz_edge<P>(plane, f.stride[1], f.ch, cx4 * 4, cy4 * 4, q, s, mwp, mwn, pos_ll, neg_ll, f.bdmax);
            }
        }
    }
}

}  // namespace

int r2g_launch_deblock_dir(const DevFrame &f, int dir, cudaStream_t s) {
    if (!f.deblock_on) return 0;
    int items = f.bw4 * f.bh4 + (f.bw4 >> 1) * (f.bh4 >> 1);
    int blocks = (items + 255) / 256;
    if (f.bitdepth > 8) {
        if (dir == 0)
            deblock_kernel<uint16_t, 0><<<blocks, 256, 0, s>>>(f);
        else
            deblock_kernel<uint16_t, 1><<<blocks, 256, 0, s>>>(f);
    } else {
        if (dir == 0)
            deblock_kernel<uint8_t, 0><<<blocks, 256, 0, s>>>(f);
        else
            deblock_kernel<uint8_t, 1><<<blocks, 256, 0, s>>>(f);
    }
    return 1;
}
