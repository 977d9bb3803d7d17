// CDEF with CCSO folded in, out of place: deblocked frame D -> C.
//
// Reference: crates/rav2d/src/cdef.rs (cdef_brow :702, cdef_find_dir_bd
// :134, adjust_strength :226, cdef_filter_block :320, cdef_padding :37) and
// ccso.rs (ccso_prep :115, ccso_padding :26, ccso_add :215).  The reference
// filters in place per 8-row band and keeps pre-CDEF copies of every sample
// a later block reads (toggled top-line banks, 2x8 left backups, the 8-row
// seam pass), so every tap it takes is a deblocked, pre-CDEF sample.  Here
// that is expressed directly: the kernel reads D and writes C.
//
// One CTA covers a 64x32 luma region of a 64-wide superblock column (32
// 8x8 blocks) plus the co-located 32x16 chroma region.  The region and its
// halo are staged in shared memory in aligned 8-sample chunks (one 8- or
// 16-byte load each; columns -8 .. 71 luma, -8 .. 39 chroma, rows -2 .. +1
// beyond the region): coordinates clamped to the frame, which is CCSO's
// padding, and a copy with INT16_MIN for taps outside the frame, CDEF's
// padding; plus a block-major copy of the region's luma for the direction
// search.
//   phase 1: warp 0 decodes each block's strengths and skip / lossless state
//            (lane = block);
//   phase 2: warp d computes direction d's cost for every block (lane =
//            block): partial sums in registers, no atomics;
//   phase 3: warp 0 picks each block's direction (first maximum wins, as in
//            the reference), its variance and adjusted strengths;
//   phase 4: warp w filters blocks w, w+8, w+16, w+24: each lane two luma
//            samples of one row and one chroma sample, plus the CCSO offset.
#include "r2g_common.cuh"

namespace {

constexpr int RH = 32;   // luma rows per CTA region
constexpr int NB = 32;   // 8x8 blocks per region (8 wide, 4 high)
constexpr int XO = 8;    // tile column of the region's first sample
// Tile pitches: TW / 2 = 4 (mod 8) words puts the 8 rows a warp reads in the
// filter phase (4 lanes per row, 4 consecutive words) on 32 distinct banks;
// CW = 56 does the same for the 2 planes x 4 rows of the chroma lanes.
constexpr int TW = 88;   // luma tile pitch (columns -8 .. 71 used)
constexpr int TH = RH + 4;   // luma tile height (-2 .. RH+1)
constexpr int TCH = 10;  // 8-sample chunks per luma tile row
constexpr int CW = 56;   // chroma tile pitch (columns -8 .. 39 used)
constexpr int CH = RH / 2 + 4;  // chroma tile height
constexpr int CCH = 6;   // 8-sample chunks per chroma tile row
constexpr int BKP = 66;  // block-major pitch (int16): conflict-free per-lane reads
constexpr int NCHUNK = TH * TCH + 2 * CH * CCH;

__constant__ int8_t c_ccso_pos[7][2] = {{-1, 0}, {0, -1}, {-1, -1}, {-1, 1}, {-1, -2}, {1, -2}, {0, 2}};
__constant__ uint8_t c_uv_dirs[8] = {0, 1, 2, 3, 4, 5, 6, 7};
__constant__ uint32_t c_div_table[7] = {840, 420, 280, 210, 168, 140, 120};

struct BlockParams {
    int active;   // any CDEF filtering of this 8x8 (luma or chroma)
    int need_dir;
    int y_pri, y_sec, y_dir, y_on;
    int uv_pri, uv_sec, uv_dir, uv_on;
    int y_ll;     // luma lossless rows mask bits for CCSO: bit r>>2 of the block
};

// constrain (cdef.rs:117-120): min(|d|, max(0, t - (|d| >> s))) equals
// max(0, min(|d|, t - (|d| >> s))) since |d| >= 0 - one fused min/relu.
R2G_D int constrain(int diff, int threshold, int shift) {
    int adiff = diff < 0 ? -diff : diff;
    return apply_sign_(__vimin_s32_relu(adiff, threshold - (adiff >> shift)), diff);
}

// CDEF_DIRECTIONS entries are offsets in a 12-wide padded block; decode to
// (dy, dx) with dx in [-2, 2].
R2G_D void dir_off(int off, int &dy, int &dx) {
    dy = (off + 26) / 12 - 2;  // off in [-26, 26]
    dx = off - 12 * dy;
    if (dx > 2) {
        dy += 1;
        dx -= 12;
    } else if (dx < -2) {
        dy -= 1;
        dx += 12;
    }
}

// cdef_filter_block (cdef.rs:320-458) for one sample.  `t` points at the
// sample in a padded tile (INT16_MIN outside the frame, as cdef_padding
// writes); off[0..1] are the primary taps (dir + 2, k = 0, 1), off[2..3] the
// secondary taps of dir + 4 and off[4..5] those of dir, as linear offsets.
R2G_D int cdef_px(const int16_t *t, int pri, int sec, const int *off, int damping, int bd8) {
    const int px = t[0];
    if (pri != 0) {
        int pri_tap = 4 - ((pri >> bd8) & 1);
        int pri_shift = imax_(0, damping - ulog2_((uint32_t)pri));
        int sum = 0, mx = px, mn = px, tk = pri_tap;
        if (sec != 0) {
            int sec_shift = damping - ulog2_((uint32_t)sec);
#pragma unroll
            for (int k = 0; k < 2; k++) {
                int p0 = t[off[k]], p1 = t[-off[k]];
                sum += tk * constrain(p0 - px, pri, pri_shift);
                sum += tk * constrain(p1 - px, pri, pri_shift);
                tk = (tk & 3) | 2;
                int s0 = t[off[2 + k]], s1 = t[-off[2 + k]], s2 = t[off[4 + k]], s3 = t[-off[4 + k]];
                int st = 2 - k;
                sum += st * (constrain(s0 - px, sec, sec_shift) + constrain(s1 - px, sec, sec_shift) +
                             constrain(s2 - px, sec, sec_shift) + constrain(s3 - px, sec, sec_shift));
                // the six taps of this k and the running bounds, 3-input min / max
                mn = __vimin3_s32(__vimin3_s32(p0, p1, s0), __vimin3_s32(s1, s2, s3), mn);
                mx = __vimax3_s32(__vimax3_s32(p0, p1, s0), __vimax3_s32(s1, s2, s3), mx);
            }
            return iclip_(px + ((sum - (sum < 0) + 8) >> 4), mn, mx);
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            int p0 = t[off[k]], p1 = t[-off[k]];
            sum += tk * constrain(p0 - px, pri, pri_shift);
            sum += tk * constrain(p1 - px, pri, pri_shift);
            tk = (tk & 3) | 2;
        }
        return px + ((sum - (sum < 0) + 8) >> 4);
    }
    int sec_shift = damping - ulog2_((uint32_t)sec);
    int sum = 0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        int s0 = t[off[2 + k]], s1 = t[-off[2 + k]], s2 = t[off[4 + k]], s3 = t[-off[4 + k]];
        int st = 2 - k;
        sum += st * (constrain(s0 - px, sec, sec_shift) + constrain(s1 - px, sec, sec_shift) +
                     constrain(s2 - px, sec, sec_shift) + constrain(s3 - px, sec, sec_shift));
    }
    return px + ((sum - (sum < 0) + 8) >> 4);
}

// ccso_score (ccso.rs:16-24)
R2G_D uint32_t ccso_score(int diff, int q, uint32_t clf) {
    if (diff > q && clf == 0) return 2;
    if (diff < -q) return 0;
    return 1;
}

// Cost of direction D for one 8x8 block (cdef_find_dir_bd, cdef.rs:134-224):
// `b` holds the block's 64 values (px >> bd8) - 128 in raster order.  The
// per-direction lines are summed in registers (every index is a constant
// after unrolling); squares and sums wrap in 32 bits as in the reference.
template <int D>
R2G_D uint32_t dir_cost(const int16_t *b) {
    constexpr int NBIN = (D == 2 || D == 6) ? 8 : ((D == 0 || D == 4) ? 15 : 11);
    int bin[NBIN];
#pragma unroll
    for (int n = 0; n < NBIN; n++) bin[n] = 0;
#pragma unroll
    for (int y = 0; y < 8; y++)
#pragma unroll
        for (int x = 0; x < 8; x++) {
            const int v = b[y * 8 + x];
            int k;
            if (D == 0) k = y + x;
            else if (D == 1) k = y + (x >> 1);
            else if (D == 2) k = y;
            else if (D == 3) k = 3 + y - (x >> 1);
            else if (D == 4) k = 7 + y - x;
            else if (D == 5) k = 3 - (y >> 1) + x;
            else if (D == 6) k = x;
            else k = (y >> 1) + x;
            bin[k] += v;
        }
    auto sq = [](int v) -> uint32_t { return (uint32_t)v * (uint32_t)v; };
    uint32_t cost = 0;
    if (D == 2 || D == 6) {
#pragma unroll
        for (int n = 0; n < 8; n++) cost += sq(bin[n]);
        cost *= 105u;
    } else if (D == 0 || D == 4) {
#pragma unroll
        for (int n = 0; n < 7; n++) cost += (sq(bin[n]) + sq(bin[14 - n])) * c_div_table[n];
        cost += sq(bin[7]) * 105u;
    } else {
#pragma unroll
        for (int m = 0; m < 5; m++) cost += sq(bin[3 + m]);
        cost *= 105u;
#pragma unroll
        for (int m = 0; m < 3; m++) cost += (sq(bin[m]) + sq(bin[10 - m])) * c_div_table[2 * m + 1];
    }
    return cost;
}

struct CdefSmem {
    alignas(16) int16_t ty[TH][TW];  // clamped to the frame (CCSO padding)
    alignas(16) int16_t tc[2][CH][CW];
    alignas(16) int16_t pty[TH][TW];  // INT16_MIN outside the frame (CDEF padding)
    alignas(16) int16_t ptc[2][CH][CW];
    int16_t blk[NB][BKP]; // per block: (px >> bd8) - 128, raster order
    uint32_t cost[8][NB];
    BlockParams bp[NB];
    int toff_y[8][6], toff_c[8][6];  // tap offsets per direction (tile pitches)
    int s_ccso[3];
    // per plane, the CCSO offset of every class index (ccso_add's lookup
    // of the plane's packed filter_off nibble in CCSO_OFFSET), so the
    // per-pixel lookup is one shared-memory byte instead of a
    // lane-dependent read of the kernel parameters
    int8_t ccso_off[3][256];
    // chroma CCSO parameters per plane (U, V): band shift, band-only flag,
    // quantiser step, tap offset in the luma tile, edge classifier
    int ccso_c[2][5];
};

// Eight consecutive samples x0 .. x0+7 of one row as four int16 pairs (low
// half = even sample), clamped to [0, w).  A chunk inside the row is one
// 8-byte (8-bit) or 16-byte (16-bit) load: plane rows start 64-byte aligned
// and x0 is a multiple of 8.  Chunks crossing a frame edge clamp per sample.
template <typename P>
R2G_D void load_chunk(const P *row, int x0, int w, uint32_t (&v)[4]) {
    if (x0 >= 0 && x0 + 8 <= w) {
        if (sizeof(P) == 1) {
            const uint2 q = __ldg(reinterpret_cast<const uint2 *>(row + x0));
            v[0] = __byte_perm(q.x, 0, 0x4140);
            v[1] = __byte_perm(q.x, 0, 0x4342);
            v[2] = __byte_perm(q.y, 0, 0x4140);
            v[3] = __byte_perm(q.y, 0, 0x4342);
        } else {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(row + x0));
            v[0] = q.x;
            v[1] = q.y;
            v[2] = q.z;
            v[3] = q.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++)
            v[k] = (uint32_t)__ldg(row + iclip_(x0 + 2 * k, 0, w - 1)) |
                   ((uint32_t)__ldg(row + iclip_(x0 + 2 * k + 1, 0, w - 1)) << 16);
    }
}

// The same chunk with CDEF's padding (cdef_padding, cdef.rs:37): INT16_MIN
// for samples outside the frame.
R2G_D void pad_chunk(const uint32_t (&v)[4], bool row_out, int x0, int w, uint32_t (&pv)[4]) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const bool lo = !row_out && x0 + 2 * k >= 0 && x0 + 2 * k < w;
        const bool hi = !row_out && x0 + 2 * k + 1 >= 0 && x0 + 2 * k + 1 < w;
        pv[k] = (lo ? (v[k] & 0xffffu) : 0x8000u) | (hi ? (v[k] & 0xffff0000u) : 0x80000000u);
    }
}

// One 64x32 region (superblock column sbx, region row rr) of the frame; the
// work of one CTA, shared by the per-frame and the batched kernels.  LB:
// staging chunks whose loads a thread issues before their stores (more
// loads in flight, more registers).
template <typename P, int LB>
R2G_D void cdef_region(const DevFrame &f, CdefSmem &sm, int sbx, int rr) {
    const int gx0 = sbx * 64, gy0 = rr * RH;
    const int cx0 = gx0 >> 1, cy0 = gy0 >> 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int bd8 = f.bitdepth - 8;
    const P *Dy = plane_ptr<const P>(f.D[0]);
    const P *Du = plane_ptr<const P>(f.D[1]);
    const P *Dv = plane_ptr<const P>(f.D[2]);
    const int64_t ys = f.stride[0], uvs = f.stride[1];

    // ---- tap offsets of every direction in both tile pitches ----
    if (tid < 96) {
        const int chroma = tid >= 48, e = tid % 48, dir = e / 6, w = (e % 6) >> 1, k = e & 1;
        const int which = w == 0 ? dir + 2 : (w == 1 ? dir + 4 : dir);
        int dy, dx;
        dir_off(f.tab.CDEF_DIRECTIONS[which * 2 + k], dy, dx);
        if (chroma)
            sm.toff_c[dir][w * 2 + k] = dy * CW + dx;
        else
            sm.toff_y[dir][w * 2 + k] = dy * TW + dx;
    }
    // ---- phase 1: superblock and per-block parameters (cdef.rs:787-907) ----
    const int sb256x = sbx >> 2, sb64x_idx = sbx & 3;
    const int by0 = gy0 >> 2;  // 4x4 row of the region's top
    const R2gAv2Filter &m = f.masks[(by0 >> 6) * f.sb256w + sb256x];
    const R2gFrameParams &fp = f.fp;
    if (tid < 3) sm.s_ccso[tid] = f.ccso_on ? m.ccso[tid] : 0;
    if (f.ccso_on)
        for (int i = tid; i < 3 * 256; i += blockDim.x) {
            const int pl = i >> 8, idx = i & 255, bi = idx >> 1;
            const R2gCcsoPlane &c = fp.ccso[pl];
            const int packed = bi < 64 ? c.filter_off[bi] : 0;
            sm.ccso_off[pl][idx] = f.tab.CCSO_OFFSET[c.scale_idx * 8 + (7 & (packed >> (4 * (idx & 1))))];
        }
    if (tid < 2) {
        const R2gCcsoPlane &c = fp.ccso[1 + tid];
        sm.ccso_c[tid][0] = f.bitdepth - c.max_band_log2;
        sm.ccso_c[tid][1] = c.bo_only;
        sm.ccso_c[tid][2] = f.tab.CCSO_QUANT_SZ[c.scale_idx * 4 + c.quant_idx];
        sm.ccso_c[tid][3] = c_ccso_pos[c.ext_filter_support][0] * TW + c_ccso_pos[c.ext_filter_support][1];
        sm.ccso_c[tid][4] = c.edge_clf;
    }
    const int cdef_idx = m.cdef_idx[((by0 & 0x30) >> 2) + (sbx & 3)];
    const int sidx = cdef_idx < 0 ? 0 : cdef_idx;
    const bool cdef_active = !(cdef_idx == -1 || !f.cdef_on ||
                               ((sidx < 8 ? fp.cdef_y_strength[sidx] : 0) == 0 &&
                                (sidx < 8 ? fp.cdef_uv_strength[sidx] : 0) == 0));
    const int damping = fp.cdef_damping + bd8;
    if (warp == 0) {
        const int b = lane, br = b >> 3, bc = b & 7;
        const int bx = sbx * 16 + bc * 2;  // 4x4 column of this 8x8
        const int by = by0 + br * 2;       // 4x4 row
        const int by_idx = (by & 0x3e) >> 1;
        BlockParams p = {};
        const bool in_frame = bx < f.bw4 && gy0 + br * 8 < f.h;
        if (f.any_lossless && in_frame) {
            const int yr = imin_(2 * by_idx, 63);
            const uint16_t l0 = m.lossless_mask_y[yr][sb64x_idx], l1 = m.lossless_mask_y[imin_(yr + 1, 63)][sb64x_idx];
            // CCSO's luma lossless test is per 4x4: bits (row in block >> 2) * 2
            // + (column in block >> 2)
            p.y_ll = ((l0 >> (bc * 2)) & 3) | (((l1 >> (bc * 2)) & 3) << 2);
        }
        if (cdef_active && in_frame) {
            const uint16_t noskip = fp.cdef_on_skiptx ? 0xffff : m.noskip_mask[by_idx][sb64x_idx];
            uint16_t y_ll0 = 0, y_ll1 = 0, uv_ll = 0;
            if (f.any_lossless) {
                const int yr = imin_(2 * by_idx, 63);
                y_ll0 = m.lossless_mask_y[yr][sb64x_idx];
                y_ll1 = m.lossless_mask_y[imin_(yr + 1, 63)][sb64x_idx];
                uv_ll = m.lossless_mask_uv[imin_(by_idx, 63)][sb64x_idx];
            }
            const uint16_t bx_mask = (uint16_t)(3u << (bx & 14));
            const bool y_lossless = ((y_ll0 | y_ll1) & bx_mask) != 0;
            const bool uv_lossless = (uv_ll & (uint16_t)(1u << ((bx & 14) >> 1))) != 0;
            if ((noskip & bx_mask) != 0 && !(y_lossless && uv_lossless)) {
                const int y_lvl = fp.cdef_y_strength[cdef_idx], uv_lvl = fp.cdef_uv_strength[cdef_idx];
                int y_sec = y_lvl & 3, uv_sec = uv_lvl & 3;
                y_sec += y_sec == 3;
                uv_sec += uv_sec == 3;
                p.active = 1;
                p.y_pri = (y_lvl >> 2) << bd8;
                p.y_sec = y_sec << bd8;
                p.uv_pri = (uv_lvl >> 2) << bd8;
                p.uv_sec = uv_sec << bd8;
                p.y_on = !y_lossless;
                p.uv_on = uv_lvl != 0 && !uv_lossless;
                p.need_dir = p.y_pri != 0 || p.uv_pri != 0;
            }
        }
        sm.bp[b] = p;
    }
    // the deblocked planes come from the previous kernel on the stream:
    // wait for it before staging (everything above reads side-info only)
    pdl_wait();
    // ---- stage the region and its halo, one 8-sample chunk per thread and
    // step; every step's loads are issued before any of its stores ----
    for (int base = tid; base < NCHUNK; base += LB * 256) {
    uint32_t v[LB][4];
#pragma unroll
    for (int k = 0; k < LB; k++) {
        const int i = base + 256 * k;
        if (i >= NCHUNK) break;
        if (i < TH * TCH) {
            const int r = i / TCH, kk = i - r * TCH;
            load_chunk(Dy + iclip_(gy0 - 2 + r, 0, f.h - 1) * ys, gx0 - XO + 8 * kk, f.w, v[k]);
        } else {
            const int j = i - TH * TCH, pl = j / (CH * CCH), j2 = j - pl * (CH * CCH);
            const int r = j2 / CCH, kk = j2 - r * CCH;
            load_chunk((pl ? Dv : Du) + iclip_(cy0 - 2 + r, 0, f.ch - 1) * uvs, cx0 - XO + 8 * kk, f.cw, v[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < LB; k++) {
        const int i = base + 256 * k;
        if (i >= NCHUNK) break;
        uint32_t pv[4];
        uint32_t *dt, *dp;
        int yy = -1, bc = 0;
        if (i < TH * TCH) {
            const int r = i / TCH, kk = i - r * TCH;
            const int ry = gy0 - 2 + r;
            pad_chunk(v[k], ry < 0 || ry >= f.h, gx0 - XO + 8 * kk, f.w, pv);
            dt = reinterpret_cast<uint32_t *>(&sm.ty[r][8 * kk]);
            dp = reinterpret_cast<uint32_t *>(&sm.pty[r][8 * kk]);
            if (r >= 2 && r < RH + 2 && kk >= 1 && kk <= 8) {
                yy = r - 2;
                bc = kk - 1;
            }
        } else {
            const int j = i - TH * TCH, pl = j / (CH * CCH), j2 = j - pl * (CH * CCH);
            const int r = j2 / CCH, kk = j2 - r * CCH;
            const int ry = cy0 - 2 + r;
            pad_chunk(v[k], ry < 0 || ry >= f.ch, cx0 - XO + 8 * kk, f.cw, pv);
            dt = reinterpret_cast<uint32_t *>(&sm.tc[pl][r][8 * kk]);
            dp = reinterpret_cast<uint32_t *>(&sm.ptc[pl][r][8 * kk]);
        }
        *reinterpret_cast<uint4 *>(dt) = make_uint4(v[k][0], v[k][1], v[k][2], v[k][3]);
        *reinterpret_cast<uint4 *>(dp) = make_uint4(pv[0], pv[1], pv[2], pv[3]);
        if (yy >= 0) {
            uint32_t *d = reinterpret_cast<uint32_t *>(&sm.blk[(yy >> 3) * 8 + bc][(yy & 7) * 8]);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int lo = (int)((v[k][q] & 0xffffu) >> bd8) - 128, hi = (int)((v[k][q] >> 16) >> bd8) - 128;
                d[q] = ((uint32_t)lo & 0xffffu) | ((uint32_t)hi << 16);
            }
        }
    }
    }

    __syncthreads();

    // ---- phase 2: direction costs, warp = direction, lane = block ----
    {
        const int b = lane;
        if (sm.bp[b].need_dir) {
            const int16_t *bk = sm.blk[b];
            uint32_t c;
            switch (warp) {
                case 0: c = dir_cost<0>(bk); break;
                case 1: c = dir_cost<1>(bk); break;
                case 2: c = dir_cost<2>(bk); break;
                case 3: c = dir_cost<3>(bk); break;
                case 4: c = dir_cost<4>(bk); break;
                case 5: c = dir_cost<5>(bk); break;
                case 6: c = dir_cost<6>(bk); break;
                default: c = dir_cost<7>(bk); break;
            }
            sm.cost[warp][b] = c;
        }
    }
    __syncthreads();

    // ---- phase 3: direction, variance, strength adjust (cdef.rs:969-1012) ----
    if (warp == 0) {
        BlockParams &p = sm.bp[lane];
        int dir = 0;
        uint32_t var = 0;
        if (p.need_dir) {
            uint32_t best = sm.cost[0][lane];
#pragma unroll
            for (int d = 1; d < 8; d++) {
                const uint32_t c = sm.cost[d][lane];
                if (c > best) {
                    best = c;
                    dir = d;
                }
            }
            var = (best - sm.cost[dir ^ 4][lane]) >> 10;
        }
        p.y_dir = dir;
        if (p.active) {
            int yp = 0, yd = 0;
            bool yon = false;
            if (p.y_pri != 0) {
                int adj = 0;
                if (var != 0) {
                    const int i = (var >> 6) != 0 ? imin_(31 - __clz((int)(var >> 6)), 12) : 0;
                    adj = (p.y_pri * (4 + i) + 8) >> 4;
                }
                yon = (adj != 0 || p.y_sec != 0) && p.y_on;
                yp = adj;
                yd = dir;
            } else if (p.y_sec != 0 && p.y_on) {
                yon = true;
            }
            p.y_on = yon;
            p.y_pri = yp;
            p.y_dir = yd;
            p.uv_dir = p.uv_pri != 0 ? c_uv_dirs[dir] : 0;
        }
    }
    __syncthreads();

    // ---- phase 4: filter + CCSO; warp w produces blocks w, w+8, w+16, w+24
    // (uniform parameters per warp), lane -> 2 luma samples, 1 chroma sample
    const int bitdepth = f.bitdepth, bdmax = f.bdmax;
    P *Cy = plane_ptr<P>(f.C[0]);
    const R2gCcsoPlane &cp = fp.ccso[0];
    const int cq = f.tab.CCSO_QUANT_SZ[cp.scale_idx * 4 + cp.quant_idx];
    const int coff = c_ccso_pos[cp.ext_filter_support][0] * TW + c_ccso_pos[cp.ext_filter_support][1];
#pragma unroll 1
    for (int b = warp; b < NB; b += 8) {
        const int br = b >> 3, bc = b & 7;
        if (gx0 + bc * 8 >= f.w || gy0 + br * 8 >= f.h) continue;
        const BlockParams &p = sm.bp[b];
        int yoff[6], uvoff[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            yoff[k] = sm.toff_y[p.y_dir][k];
            uvoff[k] = sm.toff_c[p.uv_dir][k];
        }
        // luma
        const int r = br * 8 + (lane >> 2), c0 = bc * 8 + (lane & 3) * 2;
        const int gy = gy0 + r;
        int out[2];
        const bool lossy_row = !(f.any_lossless && ((p.y_ll >> (((lane >> 2) >> 2) * 2 + ((lane & 3) >> 1))) & 1));
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int c = c0 + k;
            const int16_t *t = &sm.ty[2 + r][XO + c];
            const int px = t[0];
            int v = px;
            if (p.active && p.y_on) {
                v = cdef_px(&sm.pty[2 + r][XO + c], p.y_pri, p.y_sec, yoff, damping, bd8);
                v = bitdepth == 8 ? (v & 0xff) : (v & 0xffff);
            }
            if (sm.s_ccso[0] && lossy_row) {
                // ccso_prep (ccso.rs:115-185): the clamped tile is the padding
                const int band_ = (int)((uint32_t)px >> (bitdepth - cp.max_band_log2));
                int idx;
                if (cp.bo_only)
                    idx = band_ & 0xff;
                else
                    idx = ((int)((ccso_score(t[coff] - px, cq, cp.edge_clf) << 5) |
                                 (ccso_score(t[-coff] - px, cq, cp.edge_clf) << 3)) |
                           band_) & 0xff;
                v = clip_px_(v + sm.ccso_off[0][idx], bdmax);
            }
            out[k] = v;
        }
        // the pair is 2-sample aligned (c0 even, 64-aligned region): one store
        if (sizeof(P) == 1)
            *reinterpret_cast<uint16_t *>(Cy + gy * ys + gx0 + c0) = (uint16_t)(out[0] | (out[1] << 8));
        else
            *reinterpret_cast<uint32_t *>(Cy + gy * ys + gx0 + c0) = (uint32_t)out[0] | ((uint32_t)out[1] << 16);
        // chroma: lane -> plane lane/16, row (lane%16)/4, column lane%4
        const int pl = lane >> 4, cr = br * 4 + ((lane & 15) >> 2), cc = bc * 4 + (lane & 3);
        const int cgy = cy0 + cr, cgx = cx0 + cc;
        P *Cp = plane_ptr<P>(f.C[1 + pl]);
        const int px = sm.tc[pl][2 + cr][XO + cc];
        int v = px;
        if (p.active && p.uv_on) {
            v = cdef_px(&sm.ptc[pl][2 + cr][XO + cc], p.uv_pri, p.uv_sec, uvoff, damping - 1, bd8);
            v = bitdepth == 8 ? (v & 0xff) : (v & 0xffff);
        }
        if (sm.s_ccso[1 + pl]) {
            const int *cpc = sm.ccso_c[pl];
            const int by_idx = ((by0 + br * 2) & 0x3e) >> 1;
            const bool ll = f.any_lossless && ((m.lossless_mask_uv[by_idx][sb64x_idx] >> (cc >> 2)) & 1);
            if (!ll) {
                // co-located luma of the chroma sample (ccso_prep, 4:2:0)
                const int16_t *t = &sm.ty[2 + 2 * cr][XO + 2 * cc];
                const int cl = t[0];
                const int band_ = (int)((uint32_t)cl >> cpc[0]);
                int idx;
                if (cpc[1]) {
                    idx = band_ & 0xff;
                } else {
                    const int q = cpc[2], o = cpc[3];
                    idx = ((int)((ccso_score(t[o] - cl, q, cpc[4]) << 5) | (ccso_score(t[-o] - cl, q, cpc[4]) << 3)) |
                           band_) & 0xff;
                }
                v = clip_px_(v + sm.ccso_off[1 + pl][idx], bdmax);
            }
        }
        Cp[cgy * uvs + cgx] = (P)v;
    }
}

template <typename P>
__global__ void __launch_bounds__(256, 7) cdef_ccso_kernel(const DevFrame f) {
    pdl_trigger();
    __shared__ CdefSmem sm;
    cdef_region<P, 1>(f, sm, blockIdx.x, blockIdx.y);
}

// Persistent kernel over a cross-frame work list: item = frame << 22 |
// region row * sb64w + sbx.
__global__ void __launch_bounds__(256, 6) cdef_batch_kernel(BatchArgs a) {
    pdl_trigger();
    __shared__ CdefSmem sm;
    const int n = a.count[1];
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const uint32_t it = a.work[1][w];
        const DevFrame &f = a.frames[it >> 22];
        const int b = it & 0x3fffff, sb64w = (f.w + 63) >> 6;
        if (f.bitdepth > 8)
            cdef_region<uint16_t, 1>(f, sm, b % sb64w, b / sb64w);
        else
            cdef_region<uint8_t, 1>(f, sm, b % sb64w, b / sb64w);
        __syncthreads();
    }
}


// ---- DSP-context slot kernels (r2g_dsp_*): one block per call ----
// `tile` holds the block and a 2-sample ring around it, (h + 4) x (w + 4),
// as the caller's buffers provide it; positions whose edge flag is absent
// are not read.

// cdef_filter_block (cdef.rs:320-458) with cdef_padding (:37-114): absent
// edges become INT16_MIN.
__global__ void dsp_cdef_filter_kernel(const uint16_t *tile, int w, int h, int edges, int pri, int sec, int dir,
                                       int damping, int bitdepth, const DevTables tab, uint16_t *out) {
    __shared__ int16_t t[12 * 12];
    __shared__ int off[6];
    const int tid = threadIdx.x;
    for (int i = tid; i < 144; i += blockDim.x) {
        const int y = i / 12 - 2, x = i % 12 - 2;
        int16_t v = (int16_t)INT16_MIN;
        if (y < h + 2 && x < w + 2) {
            const bool absent = (y < 0 && !(edges & 4)) || (y >= h && !(edges & 8)) || (x < 0 && !(edges & 1)) ||
                                (x >= w && !(edges & 2));
            if (!absent) v = (int16_t)tile[(y + 2) * (w + 4) + x + 2];
        }
        t[i] = v;
    }
    if (tid < 6) {
        const int wh = tid >> 1, k = tid & 1;
        const int which = wh == 0 ? dir + 2 : (wh == 1 ? dir + 4 : dir);
        int dy, dx;
        dir_off(tab.CDEF_DIRECTIONS[which * 2 + k], dy, dx);
        off[tid] = dy * 12 + dx;
    }
    __syncthreads();
    if (tid < w * h) {
        const int y = tid / w, x = tid % w;
        int o[6];
#pragma unroll
        for (int k = 0; k < 6; k++) o[k] = off[k];
        const int v = cdef_px(&t[(y + 2) * 12 + x + 2], pri, sec, o, damping, bitdepth - 8);
        out[tid] = (uint16_t)(bitdepth == 8 ? (v & 0xff) : (v & 0xffff));
    }
}

// cdef_find_dir_bd (cdef.rs:134-224) on one 8x8 block; out = {dir, var}.
__global__ void dsp_cdef_dir_kernel(const uint16_t *blk, int bitdepth, uint32_t *out) {
    __shared__ int16_t b[64];
    __shared__ uint32_t cost[8];
    const int tid = threadIdx.x;
    if (tid < 64) b[tid] = (int16_t)(((int)blk[tid] >> (bitdepth - 8)) - 128);
    __syncthreads();
    switch (tid) {
        case 0: cost[0] = dir_cost<0>(b); break;
        case 1: cost[1] = dir_cost<1>(b); break;
        case 2: cost[2] = dir_cost<2>(b); break;
        case 3: cost[3] = dir_cost<3>(b); break;
        case 4: cost[4] = dir_cost<4>(b); break;
        case 5: cost[5] = dir_cost<5>(b); break;
        case 6: cost[6] = dir_cost<6>(b); break;
        case 7: cost[7] = dir_cost<7>(b); break;
        default: break;
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t best = cost[0];
        int dir = 0;
        for (int d = 1; d < 8; d++)
            if (cost[d] > best) {
                best = cost[d];
                dir = d;
            }
        out[0] = (uint32_t)dir;
        out[1] = (best - cost[dir ^ 4]) >> 10;
    }
}

// ccso_prep (ccso.rs:115-187) with ccso_padding (:26-65): coordinates clamp
// to the available area.  The tile covers the luma region W x H = w << ss_hor
// by h << ss_ver.
__global__ void dsp_ccso_prep_kernel(const uint16_t *tile, int w, int h, int ss_hor, int ss_ver, int edges,
                                     int max_band_log2, int ext, int quant_step, int edge_clf, int bo_only,
                                     int bitdepth, uint8_t *out) {
    const int W = w << ss_hor, H = h << ss_ver, tw = W + 4;
    const int x_min = (edges & 1) ? -2 : 0, x_max = W - 1 + ((edges & 2) ? 2 : 0);
    const int y_min = (edges & 4) ? -2 : 0, y_max = H - 1 + ((edges & 8) ? 2 : 0);
    auto px = [&](int yy, int xx) -> int {
        yy = iclip_(yy, y_min, y_max);
        xx = iclip_(xx, x_min, x_max);
        return tile[(yy + 2) * tw + xx + 2];
    };
    const int dy = c_ccso_pos[ext][0], dx = c_ccso_pos[ext][1];
    for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
        const int y = i / w, x = i % w, yl = y << ss_ver, xl = x << ss_hor;
        const int c = px(yl, xl);
        const uint8_t band = (uint8_t)((uint32_t)c >> (bitdepth - max_band_log2));
        if (bo_only) {
            out[i] = band;
        } else {
            const uint32_t c0 = ccso_score(px(yl + dy, xl + dx) - c, quant_step, (uint32_t)edge_clf);
            const uint32_t c1 = ccso_score(px(yl - dy, xl - dx) - c, quant_step, (uint32_t)edge_clf);
            out[i] = (uint8_t)((c0 << 5) | (c1 << 3)) | band;
        }
    }
}

// ccso_add (ccso.rs:215-254) on a w x h block.
__global__ void dsp_ccso_add_kernel(uint16_t *dst, const uint8_t *idx, const uint8_t *offs, const int8_t *lut, int w,
                                    int h, const uint16_t *llm, int bdmax) {
    for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
        const int y = i / w, x = i % w;
        if ((llm[(y >> 2) * 4] >> (x >> 2)) & 1) continue;
        const int k = idx[i];
        const int packed = (k >> 1) < 64 ? offs[k >> 1] : 0;
        dst[i] = (uint16_t)iclip_((int)dst[i] + lut[7 & (packed >> (4 * (k & 1)))], 0, bdmax);
    }
}

}  // namespace

void r2g_batch_launch_cdef(const BatchArgs &a, int grid, cudaStream_t s) {
    r2g_launch_pdl(cdef_batch_kernel, dim3(grid), dim3(256), s, a);
}
int r2g_batch_occupancy_cdef() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, cdef_batch_kernel, 256, 0);
    return nb;
}
int r2g_cdef_items(const DevFrame &f) { return f.cdef_stage_on ? ((f.w + 63) >> 6) * ((f.h + RH - 1) / RH) : 0; }

int r2g_launch_cdef(const DevFrame &f, cudaStream_t s) {
    if (!f.cdef_stage_on) return 0;
    dim3 grid((f.w + 63) / 64, (f.h + RH - 1) / RH);
    if (f.bitdepth > 8)
        r2g_launch_pdl(cdef_ccso_kernel<uint16_t>, grid, dim3(256), s, f);
    else
        r2g_launch_pdl(cdef_ccso_kernel<uint8_t>, grid, dim3(256), s, f);
    return 1;
}

void r2g_dsp_launch_cdef_filter(const uint16_t *tile, int w, int h, int edges, int pri, int sec, int dir, int damping,
                                int bitdepth, const DevTables &tab, uint16_t *out, cudaStream_t s) {
    dsp_cdef_filter_kernel<<<1, 64, 0, s>>>(tile, w, h, edges, pri, sec, dir, damping, bitdepth, tab, out);
}
void r2g_dsp_launch_cdef_dir(const uint16_t *blk, int bitdepth, uint32_t *out, cudaStream_t s) {
    dsp_cdef_dir_kernel<<<1, 64, 0, s>>>(blk, bitdepth, out);
}
void r2g_dsp_launch_ccso_prep(const uint16_t *tile, int w, int h, int ss_hor, int ss_ver, int edges, int max_band_log2,
                              int ext, int quant_step, int edge_clf, int bo_only, int bitdepth, uint8_t *out,
                              cudaStream_t s) {
    dsp_ccso_prep_kernel<<<1, 256, 0, s>>>(tile, w, h, ss_hor, ss_ver, edges, max_band_log2, ext, quant_step, edge_clf,
                                     bo_only, bitdepth, out);
}
void r2g_dsp_launch_ccso_add(uint16_t *dst, const uint8_t *idx, const uint8_t *offs, const int8_t *lut, int w, int h,
                             const uint16_t *llm, int bdmax, cudaStream_t s) {
    dsp_ccso_add_kernel<<<1, 256, 0, s>>>(dst, idx, offs, lut, w, h, llm, bdmax);
}
