// AV2 deblocking on the GPU, fused and out of place: recon R -> deblocked D.
//
// Reference: crates/rav2d/src/deblock.rs (deblock_bd :217, filter_choice_bd
// :81, deblock64_cols :1623, deblock64_rows :1866, setup_thr_* :1477/:1520)
// and lf_mask.rs:332-358.  The reference walks the frame per 64-row band,
// all vertical edges of a band, then its horizontal edges.  Transform sizes
// bound each edge's filter length (MAX_WIDTH_* by edge class), so the samples
// one edge reads never overlap the samples another edge of the same direction
// writes: the edges of one direction can run in any order, and the result is
// "all vertical edges of the frame, then all horizontal edges".
//
// One CTA produces one 64x64 luma tile and its 32x32 chroma tiles.  A luma
// edge moves samples at most 8 away and reads at most 8 away, so the tile
// stages R over [-12, 76) in both directions (chroma: width <= 4, reads <= 5,
// staged over [-8, 40)), applies every vertical edge whose effect can reach a
// sample the horizontal pass reads, synchronises, applies every horizontal
// edge that can reach the tile, and writes the tile.  Each edge segment (4
// lines) is one thread working on a 4 x 16 register window read from shared
// memory: line l along the edge, position j across it, j = 8 the first sample
// on the positive side.
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

// filter_choice_bd (deblock.rs:81-210) on window lines 0 and 3; position
// p(k) = win[line][8 + k].  Every index is a compile-time constant.
R2G_D int filter_choice(const int *ws, const int *wt, int mwn, int mwp, uint32_t q_thr, uint32_t side_thr) {
#define S(k) ws[8 + (k)]
#define T(k) wt[8 + (k)]
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
#pragma unroll
    for (int di = 0; di < 3; di++) {
        const int dist = 4 + 2 * di;
        if (dist > mwp) break;
        const int d2 = dist < 7 ? dist : 7;
        uint32_t q4 = q_thr * (uint32_t)c_q_first[di];
        uint32_t e4 = (side_thr * (uint32_t)dist) >> 4;
        if (transition > q4) return prev;
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

// deblock_bd (deblock.rs:217-281) on a shared-memory edge: `e` points at the
// first positive-side sample of line 0; `along` steps between the 4 lines,
// `across` steps across the edge.
R2G_D void filter_edge(int16_t *e, int along, int across, uint32_t q_thr, uint32_t side_thr, int mwp, int mwn,
                       bool pos_ll, bool neg_ll, int bdmax) {
    int width;
    {
        int w0[16], w3[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            w0[j] = e[(j - 8) * across];
            w3[j] = e[3 * along + (j - 8) * across];
        }
        width = filter_choice(w0, w3, mwn, mwp, q_thr, side_thr);
    }
    if (width < 1) return;
    int wn = imin_(width, mwn), wp = width;
    int clampv = (int)q_thr * c_q_thresh_mults[width - 1];
    int mneg = c_w_mult[wn - 1], mpos = c_w_mult[wp - 1];
    // lines are independent once the width is chosen: two at a time, both
    // loaded before either is written
#pragma unroll 1
    for (int l = 0; l < 4; l += 2) {
        int16_t *ln0 = e + l * along, *ln1 = ln0 + along;
        int L0[16], L1[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            L0[j] = ln0[(j - 8) * across];
            L1[j] = ln1[(j - 8) * across];
        }
        const int delta0 = iclip_(4 * (3 * (L0[8] - L0[7]) - (L0[9] - L0[6])), -clampv, clampv);
        const int delta1 = iclip_(4 * (3 * (L1[8] - L1[7]) - (L1[9] - L1[6])), -clampv, clampv);
        const int dn0 = delta0 * mneg, dp0 = delta0 * mpos, dn1 = delta1 * mneg, dp1 = delta1 * mpos;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (!neg_ll && j < wn) {
                ln0[(-j - 1) * across] = (int16_t)clip_px_(L0[7 - j] + ((dn0 * (wn - j) + (1 << 10)) >> 11), bdmax);
                ln1[(-j - 1) * across] = (int16_t)clip_px_(L1[7 - j] + ((dn1 * (wn - j) + (1 << 10)) >> 11), bdmax);
            }
            if (!pos_ll && j < wp) {
                ln0[j * across] = (int16_t)clip_px_(L0[8 + j] - ((dp0 * (wp - j) + (1 << 10)) >> 11), bdmax);
                ln1[j * across] = (int16_t)clip_px_(L1[8 + j] - ((dp1 * (wp - j) + (1 << 10)) >> 11), bdmax);
            }
        }
    }
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

// Shared-memory tile geometry.
constexpr int DB_NT = 256;  // threads per tile CTA
constexpr int LT = 88;   // luma staged span: tile origin - 12 .. + 76
constexpr int LO = 12;   // luma halo
constexpr int LP = 90;   // luma row pitch (int16)
constexpr int CT = 48;   // chroma staged span: origin - 8 .. + 40
constexpr int CO = 8;    // chroma halo
constexpr int CP = 50;   // chroma row pitch

// One resolved edge segment: thresholds and geometry in the staged span.
//   qs  = q_thr | side_thr << 16
//   geo = x | y << 8 | mwp << 16 | mwn << 20 | pos_ll << 24 | neg_ll << 25
struct EdgeDesc {
    uint32_t qs, geo;
};

// Per-tile edge lists (upper bounds: every segment position of the span).
constexpr int NVL = 19 * 22, NVC = 2 * 9 * 12, NHL = 19 * 16, NHC = 2 * 9 * 8;

// The side-info one tile's edges read, staged once per tile with independent
// loads (so resolving an edge touches shared memory only).  Coordinates in
// 4x4 units; tile origin (X0, Y0) luma, (CX0, CY0) chroma.
//   vy[j][s][k]: vertical luma edge masks of column X0-1+j, 16-row segment
//                s of rows Y0-3 .., level k (4 = sub-PU)
//   hy[i][k]:    horizontal luma edge masks of row Y0-1+i (columns X0..X0+15)
//   vc, hc:      the chroma twins (columns CX0+j, rows CY0-2.. / CY0+i)
//   lly[r][g]:   luma lossless bits of row Y0-4+r, 16-column group X0/16-1+g
//   llc[r][g]:   chroma lossless bits of row CY0-3+r, 8-column group tx-1+g
//   thr[kind][b][seg]: q_thr | side_thr << 16 of 64x64 block b (3x3 around
//                the tile), kind 0/1 luma dir 0/1, 2 U, 3 V
//   segy / segc: segment ids (when the frame has a segment map)
struct DbSide {
    uint16_t vy[19][3][5], hy[19][5], vc[9][2][5], hc[9][5];
    uint16_t lly[23][3], llc[13][3];
    uint32_t thr[4][9][8];
    uint8_t segy[23][20], segc[13][10];
};

struct DeblockSmem {
    int16_t y[LT * LP];
    int16_t uv[2][CT * CP];
    EdgeDesc vl[NVL], vc[NVC], hl[NHL], hc[NHC];  // vertical / horizontal, luma / chroma
    int n[4];  // list lengths: vl, vc, hl, hc
    DbSide side;
};

// Appends to a list with one shared atomic per group of converged lanes
// pushing to the same list (the lists' order does not matter: the edges of
// one direction are independent).
R2G_D void push_edge(DeblockSmem &sm, int list, EdgeDesc d) {
    EdgeDesc *dst = list == 0 ? sm.vl : list == 1 ? sm.vc : list == 2 ? sm.hl : sm.hc;
    const unsigned peers = __match_any_sync(__activemask(), list);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&sm.n[list], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    dst[base + __popc(peers & ((1u << lane) - 1))] = d;
}

R2G_D uint32_t pack_geo(int x, int y, int mwp, int mwn, bool pos_ll, bool neg_ll) {
    return (uint32_t)x | ((uint32_t)y << 8) | ((uint32_t)mwp << 16) | ((uint32_t)mwn << 20) |
           ((uint32_t)pos_ll << 24) | ((uint32_t)neg_ll << 25);
}

// Stages the tile's side-info (all loads independent, spread over the CTA).
R2G_D void stage_side(const DevFrame &f, DbSide &sd, int tx, int ty, int tid, int nt) {
    const int X0 = tx * 16, Y0 = ty * 16, CX0 = tx * 8, CY0 = ty * 8;
    const int bw4 = f.bw4, bh4 = f.bh4, cbw4 = bw4 >> 1, cbh4 = bh4 >> 1;
    const int nsb = f.sb256w * f.sb256h;
    auto mask_at = [&](int sbrow, int sbcol) -> const R2gAv2Filter * {
        const int i = sbrow * f.sb256w + sbcol;
        return (sbrow >= 0 && sbcol >= 0 && sbcol < f.sb256w && i < nsb) ? &f.masks[i] : nullptr;
    };
    const int gy0 = (Y0 - 3) >> 4, gc0 = (CY0 - 2) >> 4;
    constexpr int NV = 19 * 3 * 5, NH = 19 * 5, NVCW = 9 * 2 * 5, NHCW = 9 * 5, NLY = 23 * 3, NLC = 13 * 3;
    constexpr int NQ = 9, NSY = 23 * 20, NSC = 13 * 10;
    const bool segs = f.segmap != nullptr, segsc = f.segmap_uv != nullptr;
    const int total = NV + NH + NVCW + NHCW + NLY + NLC + NQ + (segs ? NSY : 0) + (segsc ? NSC : 0);
    __shared__ uint16_t q64[9];
    for (int i = tid; i < total; i += nt) {
        int j = i;
        if (j < NV) {
            const int c = j / 15, s = (j / 5) % 3, k = j % 5;
            const int x4 = X0 - 1 + c, g = gy0 + s;
            const R2gAv2Filter *m = (x4 >= 0 && x4 < bw4 && g >= 0 && 16 * g < bh4) ? mask_at(g >> 2, x4 >> 6) : nullptr;
            sd.vy[c][s][k] = m ? m->filter_y[0][x4 & 63][k][g & 3] : 0;
            continue;
        }
        j -= NV;
        if (j < NH) {
            const int r = j / 5, k = j % 5;
            const int y4 = Y0 - 1 + r;
            const R2gAv2Filter *m = (y4 >= 0 && y4 < bh4 && X0 < bw4) ? mask_at(y4 >> 6, X0 >> 6) : nullptr;
            sd.hy[r][k] = m ? m->filter_y[1][y4 & 63][k][(X0 >> 4) & 3] : 0;
            continue;
        }
        j -= NH;
        if (j < NVCW) {
            const int c = j / 10, s = (j / 5) % 2, k = j % 5;
            const int cx4 = CX0 + c, g = gc0 + s;
            const R2gAv2Filter *m =
                (cx4 < cbw4 && g >= 0 && 16 * g < cbh4) ? mask_at(g >> 1, cx4 >> 5) : nullptr;
            sd.vc[c][s][k] = m ? m->filter_uv[0][cx4 & 31][k][g & 1] : 0;
            continue;
        }
        j -= NVCW;
        if (j < NHCW) {
            const int r = j / 5, k = j % 5;
            const int cy4 = CY0 + r;
            const R2gAv2Filter *m = (cy4 < cbh4 && CX0 < cbw4) ? mask_at(cy4 >> 5, CX0 >> 5) : nullptr;
            sd.hc[r][k] = m ? m->filter_uv[1][cy4 & 31][k][(CX0 & 31) >> 4] : 0;
            continue;
        }
        j -= NHCW;
        if (j < NLY) {
            const int r = j / 3, g = X0 / 16 - 1 + j % 3, y4 = Y0 - 4 + r;
            const R2gAv2Filter *m = (y4 >= 0 && y4 < bh4 && g >= 0 && 16 * g < bw4) ? mask_at(y4 >> 6, g >> 2) : nullptr;
            sd.lly[r][j % 3] = m ? m->lossless_mask_y[y4 & 63][g & 3] : 0;
            continue;
        }
        j -= NLY;
        if (j < NLC) {
            const int r = j / 3, g = tx - 1 + j % 3, cy4 = CY0 - 3 + r;
            const R2gAv2Filter *m =
                (cy4 >= 0 && cy4 < cbh4 && g >= 0 && 8 * g < cbw4) ? mask_at(cy4 >> 5, g >> 2) : nullptr;
            sd.llc[r][j % 3] = m ? m->lossless_mask_uv[cy4 & 31][g & 3] : 0;
            continue;
        }
        j -= NLC;
        if (j < NQ) {
            const int bx = tx - 1 + j % 3, by = ty - 1 + j / 3;
            const R2gAv2Filter *m = (bx >= 0 && by >= 0 && 16 * bx < bw4 && 16 * by < bh4) ? mask_at(by >> 2, bx >> 2)
                                                                                          : nullptr;
            q64[j] = m ? m->qidx[(bx & 3) + ((by & 3) << 2)] : 0;
            continue;
        }
        j -= NQ;
        if (segs && j < NSY) {
            const int r = j / 20, c = j % 20, y4 = Y0 - 4 + r, x4 = X0 - 2 + c;
            sd.segy[r][c] =
                (x4 >= 0 && y4 >= 0 && x4 < bw4 && y4 < bh4) ? f.segmap[(int64_t)y4 * f.segmap_stride + x4] : 0;
            continue;
        }
        if (segs) j -= NSY;
        const int r = j / 10, c = j % 10, cy4 = CY0 - 3 + r, cx4 = CX0 - 1 + c;
        sd.segc[r][c] = (cx4 >= 0 && cy4 >= 0 && cx4 < cbw4 && cy4 < cbh4)
                            ? f.segmap_uv[(int64_t)cy4 * f.segmap_uv_stride + cx4]
                            : 0;
    }
    __syncthreads();
    // thresholds of every (kind, block, segment id < 8) the tile can use
    // (thr_of gives 0 for ids the frame's segmentation does not define)
    for (int i = tid; i < 4 * 9 * 8; i += nt) {
        const int kind = i / 72, b = (i / 8) % 9, seg = i % 8;
        int q, s;
        thr_of(f, kind, q64[b], seg, q, s);
        sd.thr[kind][b][seg] = (uint32_t)q | ((uint32_t)s << 16);
    }
    __syncthreads();
}

// Threshold pair (setup_thr_*, deblock.rs:1477-1567) of a 4x4 and its
// neighbour (left for vertical edges, above for horizontal ones), from the
// staged table: block index relative to the 3x3 around the tile.
R2G_D uint32_t edge_q_s(const DbSide &sd, int kind, int bc, int sc, int bn, int sn, bool subpu) {
    const uint32_t c = sc < 8 ? sd.thr[kind][bc][sc] : 0, n = sn < 8 ? sd.thr[kind][bn][sn] : 0;
    const int sh = subpu ? 3 : 0;
    const uint32_t q = (uint32_t)(uint16_t)(edge_thr((int)(c & 0xffff), (int)(n & 0xffff)) >> sh);
    const uint32_t s = (uint32_t)(uint16_t)(edge_thr((int)(c >> 16), (int)(n >> 16)) >> sh);
    return q | (s << 16);
}

// Resolve one luma edge segment (masks, class, widths, thresholds, lossless
// sides) into the tile's list.  dir 0: vertical edge at column x, rows
// y..y+3; dir 1: horizontal edge at row y, columns x..x+3.  (x, y) are frame
// coordinates; `sx`/`sy` the origin of the staged span.
R2G_D void luma_edge(const DevFrame &f, DeblockSmem &sm, int dir, int x, int y, int sx, int sy, int tx, int ty) {
    const DbSide &sd = sm.side;
    const int x4 = x >> 2, y4 = y >> 2;
    if (x4 >= f.bw4 || y4 >= f.bh4 || x < 0 || y < 0) return;
    if ((dir == 0 ? x4 : y4) == 0) return;
    const int X0 = tx * 16, Y0 = ty * 16;
    const uint16_t *km = dir == 0 ? sd.vy[x4 - X0 + 1][(y4 >> 4) - ((Y0 - 3) >> 4)] : sd.hy[y4 - Y0 + 1];
    const int bit = dir == 0 ? (y4 & 15) : (x4 & 15);
    int k3 = (km[3] >> bit) & 1, k2 = (km[2] >> bit) & 1, k1 = (km[1] >> bit) & 1, k0 = (km[0] >> bit) & 1;
    if (dir == 1) {
        // deblock_crop_bottom_edge (deblock.rs:1572-1606), applied as the
        // masks are read: in a 64-row band that overhangs the frame bottom
        // (by more than the last 4 rows of 4x4s), the horizontal edges of the
        // band's second-to-last 4x4 row lose class 3 (32-long) to class 2
        const int y64 = y4 >> 4;
        if ((y64 + 1) * 16 + 4 > f.bh4 && (y4 & 15) == imin_(f.bh4 - y64 * 16, 16) - 2) {
            k2 |= k3;
            k3 = 0;
        }
    }
    if (!(k0 | k1 | k2 | k3)) return;
    const int cls = k3 ? 3 : k2 ? 2 : k1;
    const int mwp = c_max_width_y[cls];
    const int mwn = (dir == 1 && (y4 & 15) == 0) ? imin_(6, mwp) : mwp;
    const bool subpu = (km[4] >> bit) & 1;
    const int nx4 = dir == 0 ? x4 - 1 : x4, ny4 = dir == 0 ? y4 : y4 - 1;
    auto blk = [&](int a4, int b4) { return ((b4 >> 4) - ty + 1) * 3 + ((a4 >> 4) - tx + 1); };
    auto seg = [&](int a4, int b4) { return f.segmap ? (int)sd.segy[b4 - Y0 + 4][a4 - X0 + 2] : 0; };
    auto ll = [&](int a4, int b4) { return (sd.lly[b4 - Y0 + 4][(a4 >> 4) - tx + 1] >> (a4 & 15)) & 1; };
    const uint32_t qs = edge_q_s(sd, dir, blk(x4, y4), seg(x4, y4), blk(nx4, ny4), seg(nx4, ny4), subpu);
    push_edge(sm, dir == 0 ? 0 : 2,
              EdgeDesc{qs, pack_geo(x - sx, y - sy, mwp, mwn, ll(x4, y4) != 0, ll(nx4, ny4) != 0)});
}

// One chroma edge segment position: a descriptor per enabled plane (U and V
// share masks and widths; thresholds differ); plane 1 (V) is flagged by
// bit 26 of the geometry word.
R2G_D void chroma_edge(const DevFrame &f, DeblockSmem &sm, int dir, int cx, int cy, int sx, int sy, int tx, int ty) {
    const DbSide &sd = sm.side;
    const R2gFrameParams &fp = f.fp;
    const int cx4 = cx >> 2, cy4 = cy >> 2;
    const int cbw4 = f.bw4 >> 1, cbh4 = f.bh4 >> 1;
    if (cx4 >= cbw4 || cy4 >= cbh4 || cx < 0 || cy < 0) return;
    if ((dir == 0 ? cx4 : cy4) == 0) return;
    const int CX0 = tx * 8, CY0 = ty * 8;
    const uint16_t *km = dir == 0 ? sd.vc[cx4 - CX0][(cy4 >> 4) - ((CY0 - 2) >> 4)] : sd.hc[cy4 - CY0];
    const int bit = dir == 0 ? (cy4 & 15) : (cx4 & 15);
    const int k2 = (km[2] >> bit) & 1, k1 = (km[1] >> bit) & 1, k0 = (km[0] >> bit) & 1;
    if (!(k0 | k1 | k2)) return;
    const int cls = k2 ? 2 : k1;
    const int mwp = c_max_width_uv[cls];
    const int mwn = (dir == 1 && (cy4 & 7) == 0) ? imin_(2, mwp) : mwp;
    const bool subpu = (km[4] >> bit) & 1;
    const int nx4 = dir == 0 ? cx4 - 1 : cx4, ny4 = dir == 0 ? cy4 : cy4 - 1;
    auto blk = [&](int a4, int b4) { return ((b4 >> 3) - ty + 1) * 3 + ((a4 >> 3) - tx + 1); };
    auto seg = [&](int a4, int b4) { return f.segmap_uv ? (int)sd.segc[b4 - CY0 + 3][a4 - CX0 + 1] : 0; };
    auto ll = [&](int a4, int b4) { return (sd.llc[b4 - CY0 + 3][(a4 >> 3) - tx + 1] >> (a4 & 7)) & 1; };
    const bool pos_ll = ll(cx4, cy4), neg_ll = ll(nx4, ny4);
    for (int pl = 0; pl < 2; pl++) {
        if (!(pl ? fp.deblock_level_v : fp.deblock_level_u)) continue;
        const uint32_t qs = edge_q_s(sd, 2 + pl, blk(cx4, cy4), seg(cx4, cy4), blk(nx4, ny4), seg(nx4, ny4), subpu);
        push_edge(sm, dir == 0 ? 1 : 3,
                  EdgeDesc{qs, pack_geo(cx - sx, cy - sy, mwp, mwn, pos_ll, neg_ll) | ((uint32_t)pl << 26)});
    }
}

// Filter the listed luma edges, then the chroma edges, of one direction.
template <int DIR>
R2G_D void run_edges(DeblockSmem &sm, const EdgeDesc *lum, int nl, const EdgeDesc *chr, int nc, int bdmax) {
    for (int i = threadIdx.x; i < nl + nc; i += blockDim.x) {
        const bool luma = i < nl;
        const EdgeDesc d = luma ? lum[i] : chr[i - nl];
        const int x = d.geo & 0xff, y = (d.geo >> 8) & 0xff, mwp = (d.geo >> 16) & 15, mwn = (d.geo >> 20) & 15;
        const bool pos_ll = (d.geo >> 24) & 1, neg_ll = (d.geo >> 25) & 1;
        const uint32_t q = d.qs & 0xffff, s = d.qs >> 16;
        if (luma) {
            int16_t *e = &sm.y[y * LP + x];
            filter_edge(e, DIR == 0 ? LP : 1, DIR == 0 ? 1 : LP, q, s, mwp, mwn, pos_ll, neg_ll, bdmax);
        } else {
            int16_t *e = &sm.uv[(d.geo >> 26) & 1][y * CP + x];
            filter_edge(e, DIR == 0 ? CP : 1, DIR == 0 ? 1 : CP, q, s, mwp, mwn, pos_ll, neg_ll, bdmax);
        }
    }
}

// The deblock work of one tile (tx, ty); callable from the per-frame kernel
// and from the batched persistent kernel.
template <typename P>
R2G_D void deblock_tile(const DevFrame &f, DeblockSmem &sm, int tx, int ty) {
    const R2gFrameParams &fp = f.fp;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int x0 = tx * 64, y0 = ty * 64, cx0 = x0 >> 1, cy0 = y0 >> 1;
    const int lsx = x0 - LO, lsy = y0 - LO, csx = cx0 - CO, csy = cy0 - CO;
    const P *Ry = plane_ptr<const P>(f.R[0]);
    const int64_t ys = f.stride[0], uvs = f.stride[1];
    if (tid < 4) sm.n[tid] = 0;
    __syncthreads();  // list counters reset before any thread appends
    // ---- stage R (samples outside the frame read 0; no valid edge uses them)
    for (int i = tid; i < LT * (LT / 4); i += nt) {
        int r = i / (LT / 4), c4 = (i % (LT / 4)) * 4;
        int gy = lsy + r, gx = lsx + c4;
        int v[4] = {0, 0, 0, 0};
        if (gy >= 0 && gy < f.h) {
            if (gx >= 0 && gx + 3 < f.w)
                Vec4<P>::unpack(*reinterpret_cast<const typename Vec4<P>::T *>(Ry + gy * ys + gx), v);
            else
                for (int k = 0; k < 4; k++)
                    if (gx + k >= 0 && gx + k < f.w) v[k] = Ry[gy * ys + gx + k];
        }
        for (int k = 0; k < 4; k++) sm.y[r * LP + c4 + k] = (int16_t)v[k];
    }
    for (int i = tid; i < 2 * CT * (CT / 4); i += nt) {
        int pl = i / (CT * (CT / 4)), j = i % (CT * (CT / 4));
        int r = j / (CT / 4), c4 = (j % (CT / 4)) * 4;
        int gy = csy + r, gx = csx + c4;
        const P *Rc = plane_ptr<const P>(f.R[1 + pl]);
        int v[4] = {0, 0, 0, 0};
        if (gy >= 0 && gy < f.ch) {
            if (gx >= 0 && gx + 3 < f.cw)
                Vec4<P>::unpack(*reinterpret_cast<const typename Vec4<P>::T *>(Rc + gy * uvs + gx), v);
            else
                for (int k = 0; k < 4; k++)
                    if (gx + k >= 0 && gx + k < f.cw) v[k] = Rc[gy * uvs + gx + k];
        }
        for (int k = 0; k < 4; k++) sm.uv[pl][r * CP + c4 + k] = (int16_t)v[k];
    }
    // the tile's side-info (its loads are in flight together with the
    // sample loads above); stage_side ends with a barrier
    stage_side(f, sm.side, tx, ty, tid, nt);
    const bool do_y_v = fp.deblock_level_y[0] != 0, do_y_h = fp.deblock_level_y[1] != 0;
    const bool do_uv = fp.deblock_level_u || fp.deblock_level_v;
    // ---- resolve every edge segment that can matter into the tile's lists:
    // vertical luma columns x0-4 .. x0+68 on rows y0-12 .. y0+75, chroma
    // columns cx0 .. cx0+32 on rows cy0-8 .. cy0+39; horizontal luma rows
    // y0-4 .. y0+68 on columns x0 .. x0+63, chroma rows cy0 .. cy0+32 on
    // columns cx0 .. cx0+31
    {
        const int nlv = do_y_v ? NVL : 0, ncv = do_uv ? NVC / 2 : 0;
        const int nlh = do_y_h ? NHL : 0, nch = do_uv ? NHC / 2 : 0;
        for (int i = tid; i < nlv + ncv + nlh + nch; i += nt) {
            int j = i;
            if (j < nlv) {
                luma_edge(f, sm, 0, x0 - 4 + 4 * (j % 19), lsy + 4 * (j / 19), lsx, lsy, tx, ty);
                continue;
            }
            j -= nlv;
            if (j < ncv) {
                chroma_edge(f, sm, 0, cx0 + 4 * (j % 9), csy + 4 * (j / 9), csx, csy, tx, ty);
                continue;
            }
            j -= ncv;
            if (j < nlh) {
                luma_edge(f, sm, 1, x0 + 4 * (j % 16), y0 - 4 + 4 * (j / 16), lsx, lsy, tx, ty);
                continue;
            }
            j -= nlh;
            chroma_edge(f, sm, 1, cx0 + 4 * (j % 8), cy0 + 4 * (j / 8), csx, csy, tx, ty);
        }
    }
    __syncthreads();
    run_edges<0>(sm, sm.vl, sm.n[0], sm.vc, sm.n[1], f.bdmax);
    __syncthreads();
    run_edges<1>(sm, sm.hl, sm.n[2], sm.hc, sm.n[3], f.bdmax);
    __syncthreads();
    // ---- write the tile (the previous kernel on the stream may still read
    // this frame's deblocked planes: wait for it first)
    pdl_wait();
    P *Dy = plane_ptr<P>(f.D[0]);
    for (int i = tid; i < 64 * 16; i += nt) {
        int r = i >> 4, c4 = (i & 15) * 4;
        int gy = y0 + r, gx = x0 + c4;
        if (gy >= f.h || gx >= f.w) continue;
        const int16_t *src = &sm.y[(r + LO) * LP + c4 + LO];
        int v[4] = {src[0], src[1], src[2], src[3]};
        *reinterpret_cast<typename Vec4<P>::T *>(Dy + gy * ys + gx) = Vec4<P>::pack(v);
    }
    for (int i = tid; i < 2 * 32 * 8; i += nt) {
        int pl = i >> 8, j = i & 255;
        int r = j >> 3, c4 = (j & 7) * 4;
        int gy = cy0 + r, gx = cx0 + c4;
        if (gy >= f.ch || gx >= f.cw) continue;
        P *Dc = plane_ptr<P>(f.D[1 + pl]);
        const int16_t *src = &sm.uv[pl][(r + CO) * CP + c4 + CO];
        int v[4] = {src[0], src[1], src[2], src[3]};
        *reinterpret_cast<typename Vec4<P>::T *>(Dc + gy * uvs + gx) = Vec4<P>::pack(v);
    }
}

template <typename P>
__global__ void __launch_bounds__(DB_NT, 4) deblock_tile_kernel(const DevFrame f) {
    pdl_trigger();
    __shared__ DeblockSmem sm;
    deblock_tile<P>(f, sm, blockIdx.x, blockIdx.y);
}

// Persistent kernel over a cross-frame work list: item = frame << 22 | ty *
// tiles_w + tx.
__global__ void __launch_bounds__(DB_NT, 4) deblock_batch_kernel(BatchArgs a) {
    pdl_trigger();
    __shared__ DeblockSmem sm;
    const int n = a.count[0];
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const uint32_t it = a.work[0][w];
        const DevFrame &f = a.frames[it >> 22];
        const int b = it & 0x3fffff, tw = (f.w + 63) >> 6;
        if (f.bitdepth > 8)
            deblock_tile<uint16_t>(f, sm, b % tw, b / tw);
        else
            deblock_tile<uint8_t>(f, sm, b % tw, b / tw);
        __syncthreads();
    }
}

}  // namespace

void r2g_batch_launch_deblock(const BatchArgs &a, int grid, cudaStream_t s) {
    r2g_launch_pdl(deblock_batch_kernel, dim3(grid), dim3(DB_NT), s, a);
}
int r2g_batch_occupancy_deblock() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, deblock_batch_kernel, DB_NT, 0);
    return nb;
}
int r2g_deblock_items(const DevFrame &f) { return f.deblock_on ? ((f.w + 63) >> 6) * ((f.h + 63) >> 6) : 0; }

int r2g_launch_deblock(const DevFrame &f, cudaStream_t s) {
    if (!f.deblock_on) return 0;
    dim3 grid((f.w + 63) / 64, (f.h + 63) / 64);
    if (f.bitdepth > 8)
        r2g_launch_pdl(deblock_tile_kernel<uint16_t>, grid, dim3(DB_NT), s, f);
    else
        r2g_launch_pdl(deblock_tile_kernel<uint8_t>, grid, dim3(DB_NT), s, f);
    return 1;
}

// ---------------------------------------------------------------- DSP slot
// DeblockDSPContext.deblock_sb[dir][plane] (dsp.rs:86-89): one call of
// deblock_{h,v}_sb64{y,uv}_bd (deblock.rs:303-548) on a staged strip: `strip`
// holds the 16 samples across the edge (-8 .. 7) for every line along it
// (line-major: strip[line * 16 + 8 + j]), one thread per 4-line segment
// whose bit is set in the class masks.
namespace {
__global__ void dsp_deblock_sb64_kernel(int16_t *strip, uint32_t vm0, uint32_t vm1, uint32_t vm2, uint32_t vm3,
                                        uint32_t ll_pos, uint32_t ll_neg, const uint16_t *thr, int edge, int luma,
                                        int bdmax) {
    const int seg = threadIdx.x;
    const uint32_t y = 1u << seg;
    const uint32_t vm = vm0 | vm1 | vm2 | (luma ? vm3 : 0);
    if (seg >= 16 || !(vm & y)) return;
    const int idx = luma ? ((vm3 & y) ? 3 : (vm2 & y) ? 2 : ((vm1 & y) != 0)) : ((vm2 & y) ? 2 : ((vm1 & y) != 0));
    const int mwp = luma ? c_max_width_y[idx] : c_max_width_uv[idx];
    const int mwn = edge ? imin_(luma ? 6 : 2, mwp) : mwp;
    filter_edge(strip + seg * 4 * 16 + 8, 16, 1, thr[seg], thr[16 + seg], mwp, mwn, (ll_pos & y) != 0,
                (ll_neg & y) != 0, bdmax);
}
}  // namespace

void r2g_dsp_launch_deblock_sb64(int16_t *strip, const uint16_t vmask[4], const uint16_t ll_mask[2],
                                 const uint16_t *thr, int edge, int luma, int bitdepth, cudaStream_t s) {
    dsp_deblock_sb64_kernel<<<1, 16, 0, s>>>(strip, vmask[0], vmask[1], vmask[2], vmask[3], ll_mask[1], ll_mask[0],
                                             thr, edge, luma, (1 << bitdepth) - 1);
}
