// Deblock edge masks built on the device from the decoder's create_db_mask
// calls (one R2gDbBlock record per call).
//
// Reference: crates/rav2d/src/lf_mask.rs:58-503 (mask_outer_edge_l / _t,
// mask_inner_edges_v / _h, mask_edges_part, mask_subpu_edges,
// subpu_flt_lvl, create_db_mask) and the calls in decode.rs:7869-7912 and
// :12893-12928, whose above / left edge-level contexts (tx_lpf_y /
// tx_lpf_uv) decode.rs:207 resets to 3 (luma) / 2 (chroma) at every tile row
// (above) and at every tile column of every superblock row (left).
//
// The reference walks the blocks in decode order and threads the contexts
// through the walk: an outer edge's level is min(this block's level, the
// level the previous block on that row / column left in the context), and
// the block then leaves its own level there.  In a partition tree every
// block that covers a row left of a block B is decoded before B, left to
// right, so the value B reads is the one its left neighbour on that row
// left; likewise above.  The device form is two passes over the records:
//   pass 1 (one warp per record): write the level the block leaves in the
//          left context for each of its rows at its right-most 4x4 column,
//          and the level it leaves in the above context for each column at
//          its bottom 4x4 row, into frame-sized u16 maps;
//   pass 2 (one warp per record): resolve the outer edges against the
//          neighbour's cell in those maps (or the reset value at a tile
//          start) and OR every edge bit into the SB256's masks with 32-bit
//          atomics.  Inner and sub-PU edges need no context.  mask_subpu_
//          edges reads the mask before OR-ing; only this block sets bits on
//          its own rows at its interior positions, so the old value that
//          atomicOr returns gives the same new bits as the sequential walk.
// A 1:2:1 transform split (H5 / V5) whose parts do not reach the block's
// far side (a lossless 4x4 transform in a taller block) leaves some rows /
// columns of the context untouched: their cells hold 0x8000 | the block's
// first column / row, and a reader steps over such blocks to the value
// further left / up, as the walk carries it through.
// Records that the reference could not have produced (out-of-range fields,
// a block crossing its SB256, a transform size the tables do not give) are
// skipped and counted in the context's bad-record word.
#include "r2g_common.cuh"

namespace {

enum { TXP_NONE = 0, TXP_H5 = 6, TXP_V5 = 7 };
// levels.rs: TIP_FRAME, CompInterPredMode::OpflNearMvNearMv,
// CompInterType::Avg, BlockSize::Bs8x8 / Bs256x256, TxfmSize::Tx4x4;
// lf_mask.rs:364 FILTER_8TAP_SHARP
enum { TIP_FRAME = 7, OPFL_NEAR_MV_NEAR_MV = 24, COMP_AVG = 1, BS_8X8 = 24, BS_256X256 = 0, TX_4X4 = 0,
       FILTER_8TAP_SHARP = 2 };

struct MaskArgs {
    const R2gDbBlock *blk;
    int n;
    R2gAv2Filter *masks;  // the frame's SB256 records (filter_y / filter_uv zeroed)
    int sb256w;
    int bw4, bh4;         // luma 4x4 units (the reference's fi.bw / fi.bh)
    uint16_t *lv[4];      // left / above maps: luma (bh4 x bw4), chroma (bh4/2 x bw4/2)
    int sub_pu, tip_frame_mode, tip_subpel_filter, tip_refine_mv;
    uint8_t lossless[8];
    uint32_t col_start[64], row_start[64];  // tile starts, bit per luma 4x4 column / row
    DevTables tab;
    unsigned *bad;
};

// Everything create_db_mask derives from one record before touching masks.
struct Geo {
    bool ok, chroma;
    int ssh, ssv;
    int w4, h4;        // bw4 / bh4 of create_db_mask (clipped to the frame)
    int bx4, by4;      // position in the SB256 (plane 4x4 units)
    int X, Y;          // position in the frame (plane 4x4 units)
    int sb;            // SB256 index
    int subpu_l2;
    bool txb;          // is_intra || !skip_txfm: the transform-partition branch
    int tx_part, tw4, th4, twl4c, thl4c;  // transform branch
    int hlim, vlim;    // the limits mask_edges_part gets (transform branch)
    int lvl_l, lvl_t;  // skip branch: the outer edge levels
    int sub_twl, sub_thl;  // twl4c / thl4c create_db_mask hands to the sub-PU step
};

// lf_mask.rs:367-397 subpu_flt_lvl (bw4 / bh4 are the block's full size)
R2G_D int subpu_flt_lvl(const MaskArgs &a, const R2gDbBlock &b, int bs, int bw4, int bh4) {
    if ((b.flags & R2G_DBB_INTRA) || !a.sub_pu) {
    } else if (b.ref0 == TIP_FRAME) {
        const bool opfl = a.tip_refine_mv && (a.tip_frame_mode == 1 || a.tip_subpel_filter == FILTER_8TAP_SHARP);
        return 1 + (a.tip_frame_mode == 2 ? (int)!opfl : (int)((!opfl && imin_(bw4, bh4) >= 4) || bs == BS_256X256));
    } else if (b.ref1 != -1) {
        if (b.inter_mode >= OPFL_NEAR_MV_NEAR_MV) return 1 - (bs == BS_8X8);
        if ((b.flags & R2G_DBB_REFINE_MV) && b.comp_type == COMP_AVG) return 2;
    }
    return 3;
}

// create_db_mask (lf_mask.rs:399-503) up to the first mask write, for the
// 4:2:0 layout.
R2G_D Geo geometry(const MaskArgs &a, const R2gDbBlock &b) {
    Geo g;
    g.ok = false;
    const int bs = b.bs;
    if (bs >= 31 || b.tx_part >= 8 || b.seg_id >= 8 || b.bx >= a.bw4 || b.by >= a.bh4) return g;
    const uint8_t *bd = a.tab.BLOCK_DIMENSIONS + bs * 4;
    if ((b.bx & 63) + bd[0] > 64 || (b.by & 63) + bd[1] > 64) return g;
    g.chroma = (b.flags & R2G_DBB_CHROMA) != 0;
    g.ssh = g.ssv = g.chroma;
    g.w4 = imin_(a.bw4 - b.bx, bd[0]) >> g.ssh;
    g.h4 = imin_(a.bh4 - b.by, bd[1]) >> g.ssv;
    if (g.w4 <= 0 || g.h4 <= 0) return g;
    g.bx4 = (b.bx & 63) >> g.ssh;
    g.by4 = (b.by & 63) >> g.ssv;
    g.X = b.bx >> g.ssh;
    g.Y = b.by >> g.ssv;
    g.sb = (b.by >> 6) * a.sb256w + (b.bx >> 6);
    g.subpu_l2 = subpu_flt_lvl(a, b, bs, bd[0], bd[1]);
    const int ci = g.chroma;
    const bool lossless = a.lossless[b.seg_id] != 0;
    g.txb = (b.flags & R2G_DBB_INTRA) || !(b.flags & R2G_DBB_SKIP_TXFM);
    if (g.txb) {
        g.tx_part = g.chroma ? TXP_NONE : b.tx_part;
        int tx;
        if (lossless)
            tx = (!g.chroma && (b.flags & R2G_DBB_TX_LL)) ? a.tab.MAX_TXFM_SIZE_FOR_BS[bs * 4 + 3] : TX_4X4;
        else if (g.chroma)
            tx = a.tab.MAX_TXFM_SIZE_FOR_BS[bs * 4 + 2];  // I444 - I420
        else
            tx = a.tab.TX_PART_TBL[bs * 8 + g.tx_part];
        if (tx < 0 || tx >= 25) return g;
        const uint8_t *t = a.tab.TXFM_DIMENSIONS + tx * 8;
        g.tw4 = t[0];
        g.th4 = t[1];
        g.hlim = iclip_(g.subpu_l2 - g.ssh, 0, 3 - ci);
        g.vlim = iclip_(g.subpu_l2 - g.ssv, 0, 3 - ci);
        g.twl4c = imin_(g.hlim, t[2]);
        g.thl4c = imin_(g.vlim, t[3]);
        g.sub_twl = imin_(g.subpu_l2, t[2]);
        g.sub_thl = imin_(g.subpu_l2, t[3]);
    } else {
        g.lvl_l = g.lvl_t = 0;
        if (!lossless) {
            g.lvl_l = iclip_(imin_(g.subpu_l2, bd[2]) - g.ssh, 0, 3 - ci);
            g.lvl_t = iclip_(imin_(g.subpu_l2, bd[3]) - g.ssv, 0, 3 - ci);
        }
        g.sub_twl = g.sub_thl = g.subpu_l2;
    }
    g.ok = true;
    return g;
}

constexpr int UNTOUCHED = -1;

// The level this block's call(s) of mask_outer_edge_l write for row y (and
// leave in the left context), or UNTOUCHED; mask_edges_part,
// lf_mask.rs:154-268.
R2G_D int level_l(const Geo &g, int y) {
    if (!g.txb) return g.lvl_l;
    if (g.tx_part == TXP_H5) {
        if (y >= g.th4 && y < 3 * g.th4) return imin_(g.twl4c + 1, g.hlim);
        if (y >= 4 * g.th4) return UNTOUCHED;
    }
    return g.twl4c;
}
// The same for column x and mask_outer_edge_t.
R2G_D int level_t(const Geo &g, int x) {
    if (!g.txb) return g.lvl_t;
    if (g.tx_part == TXP_V5) {
        if (x >= g.tw4 && x < 3 * g.tw4) return imin_(g.thl4c + 1, g.vlim);
        if (x >= 4 * g.tw4) return UNTOUCHED;
    }
    return g.thl4c;
}

// The context value a block starting at `pos` (column for the left context,
// row for the above one) reads: the neighbour's cell at pos - 1 along
// `step`, stepping over blocks that left it untouched, or the reset value
// at a tile start.  `starts` is the tile-start bitmap along that axis (in
// luma 4x4 units, `sh` the plane's subsampling).
R2G_D int context_at(const uint16_t *map, size_t cell, int step, int pos, const uint32_t *starts, int sh, int reset) {
    for (int guard = 0; guard < 4096; guard++) {
        const int lp = pos << sh;
        if ((starts[lp >> 5] >> (lp & 31)) & 1) return reset;
        const uint16_t v = map[cell - step];
        if (!(v & 0x8000)) return v;
        const int start = v & 0x7fff;  // the untouched block's first column / row
        if (start >= pos) return reset;   // only a stale cell (an incomplete record set) gets here
        cell -= (size_t)(pos - start) * step;
        pos = start;
    }
    return reset;
}

R2G_D uint64_t ones_shl(int n, int shift) { return (~0ull >> (64 - n)) << shift; }

// OR `bits` (64 positions along) into masks[dir][pos][lvl][0..3]; returns
// the old 64 bits of the positions this call touched (the parts it ORs).
R2G_D uint64_t or_along(uint16_t (*m)[5][4], int pos, int lvl, uint64_t bits) {
    uint64_t old = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t part = (uint32_t)(bits >> (16 * k)) & 0xffffu;
        if (!part) continue;
        uint16_t *p = &m[pos][lvl][k];
        uint32_t *w = reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(p) & ~(uintptr_t)3);
        const int sh = (reinterpret_cast<uintptr_t>(p) & 2) ? 16 : 0;
        const uint32_t o = atomicOr(w, part << sh);
        old |= (uint64_t)((o >> sh) & 0xffffu) << (16 * k);
    }
    return old;
}

// One warp per record in both passes: its lanes take the block's rows,
// columns or edge positions, so large blocks cost no more than small ones.
__global__ void __launch_bounds__(128) db_levels_kernel(const __grid_constant__ MaskArgs a) {
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= a.n) return;
    const R2gDbBlock b = a.blk[i];
    const Geo g = geometry(a, b);
    if (!g.ok) return;
    const int pw = a.bw4 >> g.ssh;  // map pitch
    uint16_t *L = a.lv[g.chroma ? 2 : 0], *T = a.lv[g.chroma ? 3 : 1];
    for (int y = lane; y < g.h4; y += 32) {
        const int l = level_l(g, y);
        L[(size_t)(g.Y + y) * pw + g.X + g.w4 - 1] = (uint16_t)(l == UNTOUCHED ? 0x8000 | g.X : l);
    }
    for (int x = lane; x < g.w4; x += 32) {
        const int l = level_t(g, x);
        T[(size_t)(g.Y + g.h4 - 1) * pw + g.X + x] = (uint16_t)(l == UNTOUCHED ? 0x8000 | g.Y : l);
    }
}

// The four per-level bit sets of one outer edge, gathered by ballots (lane =
// row or column of the block), then ORed in by lanes 0..3.
R2G_D void outer_edge(uint16_t (*m)[5][4], int pos, int start, int n, int lane, bool left, const Geo &g,
                      const MaskArgs &a, const uint16_t *map, int pw, int reset) {
    uint64_t bits[4] = {0, 0, 0, 0};
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        int lvl = -1;
        if (j < n) {
            const int own = left ? level_l(g, j) : level_t(g, j);
            if (own != UNTOUCHED) {
                const int nb = left ? context_at(map, (size_t)(g.Y + j) * pw + g.X, 1, g.X, a.col_start, g.ssh, reset)
                                    : context_at(map, (size_t)g.Y * pw + g.X + j, pw, g.Y, a.row_start, g.ssv, reset);
                lvl = imin_(own, nb) & 3;
            }
        }
#pragma unroll
        for (int l = 0; l < 4; l++) bits[l] |= (uint64_t)__ballot_sync(0xffffffffu, lvl == l) << (start + j0);
    }
    const uint64_t mine = lane == 0 ? bits[0] : lane == 1 ? bits[1] : lane == 2 ? bits[2] : bits[3];
    if (lane < 4 && mine) or_along(m, pos, lane, mine);
}

__global__ void __launch_bounds__(128) db_masks_kernel(const __grid_constant__ MaskArgs a) {
    pdl_wait();
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= a.n) return;
    const R2gDbBlock b = a.blk[i];
    const Geo g = geometry(a, b);
    if (!g.ok) {
        if (lane == 0) atomicAdd(a.bad, 1u);
        return;
    }
    R2gAv2Filter &f = a.masks[g.sb];
    uint16_t(*m)[64][5][4] = g.chroma ? f.filter_uv : f.filter_y;
    const int pw = a.bw4 >> g.ssh, ci = g.chroma;
    const int reset = 3 - ci;

    // ---- outer edges against the neighbours' context levels (tile starts
    // are superblock-aligned, so chroma column X starts a tile when luma
    // column 2X does; levels read from the maps are 0..3) ----
    outer_edge(m[0], g.bx4, g.by4, g.h4, lane, true, g, a, a.lv[ci ? 2 : 0], pw, reset);
    outer_edge(m[1], g.by4, g.bx4, g.w4, lane, false, g, a, a.lv[ci ? 3 : 1], pw, reset);

    // ---- inner transform edges (mask_edges_part): a lane per position ----
    if (g.txb) {
        const uint64_t rows = ones_shl(g.h4, g.by4), cols = ones_shl(g.w4, g.bx4);
        const int tw = g.tw4, th = g.th4;
        if (g.tx_part < TXP_H5) {
            for (int x = tw * (1 + lane); x < g.w4; x += 32 * tw) or_along(m[0], g.bx4 + x, g.twl4c, rows);
            for (int y = th * (1 + lane); y < g.h4; y += 32 * th) or_along(m[1], g.by4 + y, g.thl4c, cols);
        } else if (g.tx_part == TXP_H5) {
            for (int y = th + 2 * th * lane; y < g.h4; y += 64 * th) or_along(m[1], g.by4 + y, g.thl4c, cols);
            const uint64_t v = rows & ~ones_shl(2 * th, g.by4 + th);
            if (v)
                for (int x = tw * (1 + lane); x < g.w4; x += 32 * tw) or_along(m[0], g.bx4 + x, g.twl4c, v);
        } else {
            for (int x = tw + 2 * tw * lane; x < g.w4; x += 64 * tw) or_along(m[0], g.bx4 + x, g.twl4c, rows);
            const uint64_t h = cols & ~ones_shl(2 * tw, g.bx4 + tw);
            if (h)
                for (int y = th * (1 + lane); y < g.h4; y += 32 * th) or_along(m[1], g.by4 + y, g.thl4c, h);
        }
    }
    // the sub-PU step reads what the inner edges wrote (other lanes' atomics)
    __syncwarp();

    // ---- sub-PU edges (create_db_mask's tail, mask_subpu_edges): a lane
    // per position ----
    if (g.subpu_l2 != 3) {
        const int ds = (a.tip_frame_mode != 2) * 15;
        const int hl = g.sub_twl - (g.ssh && g.sub_twl), vl = g.sub_thl - (g.ssv && g.sub_thl);
        const int hsz = (1 << g.subpu_l2) >> g.ssh, vsz = (1 << g.subpu_l2) >> g.ssv;
        if (hsz) {
            const uint64_t parts = ones_shl(g.h4, g.by4);
            for (int x = hsz * (1 + lane); x < g.w4; x += 32 * hsz) {
                const uint64_t old = or_along(m[0], g.bx4 + x, hl, parts);
                if (x & ds) {
                    const uint64_t nb = parts & ~old;
                    if (nb) or_along(m[0], g.bx4 + x, 4, nb);
                }
            }
        }
        if (vsz) {
            const uint64_t parts = ones_shl(g.w4, g.bx4);
            for (int y = vsz * (1 + lane); y < g.h4; y += 32 * vsz) {
                const uint64_t old = or_along(m[1], g.by4 + y, vl, parts);
                if (y & ds) {
                    const uint64_t nb = parts & ~old;
                    if (nb) or_along(m[1], g.by4 + y, 4, nb);
                }
            }
        }
    }
}

}  // namespace

// Zero the frame's filter_y / filter_uv, then the two passes; returns the
// number of kernels launched.
int r2g_launch_db_masks(const R2gDbMaskInput &in, const R2gDbBlock *dev_blocks, R2gAv2Filter *dev_masks,
                        int n_sb256, int sb256w, int bw4, int bh4, void *dev_levels, const uint8_t lossless[8],
                        const DevTables &tab, unsigned *bad, cudaStream_t s) {
    cudaMemset2DAsync(dev_masks, sizeof(R2gAv2Filter), 0, sizeof(dev_masks->filter_y) + sizeof(dev_masks->filter_uv),
                      n_sb256, s);
    if (in.n_blocks <= 0) return 0;
    MaskArgs a;
    memset(&a, 0, sizeof(a));
    a.blk = dev_blocks;
    a.n = in.n_blocks;
    a.masks = dev_masks;
    a.sb256w = sb256w;
    a.bw4 = bw4;
    a.bh4 = bh4;
    const size_t ly = (size_t)bw4 * bh4, lc = ly / 4;
    uint16_t *lv = static_cast<uint16_t *>(dev_levels);
    a.lv[0] = lv;
    a.lv[1] = lv + ly;
    a.lv[2] = lv + 2 * ly;
    a.lv[3] = lv + 2 * ly + lc;
    a.sub_pu = in.sub_pu;
    a.tip_frame_mode = in.tip_frame_mode;
    a.tip_subpel_filter = in.tip_subpel_filter;
    a.tip_refine_mv = in.tip_refine_mv;
    memcpy(a.lossless, lossless, 8);
    for (int t = 0; t < in.n_tile_cols && t < 64; t++)
        if (in.tile_col_start4[t] < 2048) a.col_start[in.tile_col_start4[t] >> 5] |= 1u << (in.tile_col_start4[t] & 31);
    for (int t = 0; t < in.n_tile_rows && t < 64; t++)
        if (in.tile_row_start4[t] < 2048) a.row_start[in.tile_row_start4[t] >> 5] |= 1u << (in.tile_row_start4[t] & 31);
    a.col_start[0] |= 1u;  // the frame's first column and row start a tile
    a.row_start[0] |= 1u;
    a.tab = tab;
    a.bad = bad;
    const int grid = (in.n_blocks + 3) / 4;  // four warps (records) per CTA
    db_levels_kernel<<<grid, 128, 0, s>>>(a);
    r2g_launch_pdl(db_masks_kernel, dim3(grid), dim3(128), s, a);
    return 2;
}

// Bytes of the level maps r2g_launch_db_masks needs for a frame.
size_t r2g_db_levels_bytes(int bw4, int bh4) { return (size_t)bw4 * bh4 * 5; }
