// Loop restoration (NS-Wiener single/multi, PC-Wiener, chroma NS-Wiener with
// cross-component luma taps, GDF) out of place: C (CDEF+CCSO output) and D
// (deblocked frame) -> L.
//
// Reference: crates/rav2d/src/looprestoration.rs (lr_sbrow_apply :2401,
// lr_sbrow_plane :2276, lr_stripe :1847, ns_wiener_single_y :524,
// wiener_multi :715, get_class_lut_idx :195, ns_wiener_single_uv :1145,
// backup_row_luma :408, gdf_prep :1432, compute_gradient_row :114, gdf_add
// :273) and decode.rs:4003-4056.  The reference filters in place, stripe by
// stripe, through rings of row buffers; the rows a stripe sees are:
//   rows inside the stripe: pre-LR samples (C), left context from the saved
//     pre-LR border of the unit to the left, right context in place (C);
//   the 2 rows above / below a stripe boundary: deblocked rows saved by
//     copy_db (D); rows further out repeat the outermost saved row;
//   at the frame top / bottom: the stripe's first / last row repeated;
//   at the frame left / right: the row's first / last sample repeated.
//
// Work items are (plane, stripe, 64-wide unit, row part): luma parts of
// f.lr_rows (32 or 16) rows, chroma parts of 16 rows.  The kernel is
// persistent and warp-specialised:
//   * one producer warp takes items (blockIdx.x first, then a shared atomic
//     counter), decodes their geometry, unit kind, lossless and no-skip rows
//     from the side-info, and stages every source row of the item's window
//     (C or D by the rule above; the unit's width plus a 16-byte margin on
//     each side) into one of two shared-memory slots, one bulk copy
//     (cp.async.bulk) per row completing on the slot's "full" mbarrier;
//   * eight consumer warps take the slots in turn: they turn the raw rows
//     into the filter window (edge replication at the frame's left / right
//     border; each position holds its sample and the right neighbour as a
//     16x2 pair), release the slot through its "empty" mbarrier, and filter
//     (GDF gradient cells and PC classes, then per pixel pair: GDF error,
//     FIR, GDF add, one 2-sample store).
// So the producer loads items k+1 and k+2 while the consumers filter item
// k, and a frame's GDF / PC-Wiener tables are staged once per CTA.
#include <atomic>
#include <type_traits>

#include "r2g_common.cuh"

namespace {

enum { LR_HAVE_LEFT = 1, LR_HAVE_RIGHT = 2, LR_HAVE_TOP = 4, LR_HAVE_BOTTOM = 8, LR_HAVE_TOP_INTEGRATED = 16,
       LR_HAVE_BOTTOM_INTEGRATED = 32 };
enum { W_NONE = 0, W_NS_SINGLE = 1, W_NS_MULTI = 2, W_PC = 3 };

constexpr int NCW = 8;           // consumer warps
constexpr int NCT = NCW * 32;    // consumer threads
constexpr int LR_NT = NCT + 32;  // plus the producer warp
constexpr int CROWS = 16;        // chroma rows per work item
constexpr int LW = 76, LH = 44;  // luma window: columns -6 .. 69, rows -6 .. nr + 5 (nr <= 32)
constexpr int CW2 = 68, CH2 = 20;  // chroma windows: columns -2 .. 65, rows -2 .. 17
constexpr int RAW_BYTES = 14720;   // one staging slot (largest item: 10-bit chroma with its CfL luma)

// Raw staging rows start 16 bytes left of the unit origin (every copy is
// 16-byte aligned) and hold the unit's 64 samples plus 16 bytes on each
// side; the CfL luma rows of a chroma item hold 128 luma samples plus the
// same margins.
template <typename P>
struct RawGeom {
    static constexpr int XO = 16 / (int)sizeof(P);                // margin in samples
    static constexpr int RB = (64 + 2 * XO) * (int)sizeof(P);    // bytes per raw row
    static constexpr int LRB = (128 + 2 * XO) * (int)sizeof(P);  // bytes per raw CfL luma row
    static constexpr int LOFF = CH2 * RB;                         // offset of the CfL luma rows
};
static_assert(LH * RawGeom<uint16_t>::RB <= RAW_BYTES, "luma window slot");
static_assert(RawGeom<uint16_t>::LOFF + 2 * CH2 * RawGeom<uint16_t>::LRB <= RAW_BYTES, "chroma slot");
static_assert(RawGeom<uint8_t>::LOFF + 2 * CH2 * RawGeom<uint8_t>::LRB <= RAW_BYTES, "chroma slot");

__constant__ uint16_t c_pcw_norm[4] = {3739, 3273, 3074, 7};
__constant__ int16_t c_mode_weights[4][3] = {{-527, 15325, 321}, {26436, -17705, 17905}, {366, -147, -194}, {202, -267, -179}};
__constant__ int16_t c_mode_offsets[4] = {-547, -21565, -573, -680};

struct UnitGeom {
    int plane, x0, uw, y0, sh, edges, valid;
    int l45;  // top-integrated luma stripe: the deblocked row behind saved rows 4 and 5
    int sb256x, sb64x_idx;
    const LrUnitPacked *unit;
};

// looprestoration.rs:40-50
R2G_D int get_qval(int qstep, int tskip, int i, int b8) {
    qstep = (qstep + ((1 << b8) >> 1)) >> b8;
    int prod = (tskip * qstep + 128) >> 8;
    int qval = c_mode_weights[i][0] * (tskip << 5) + c_mode_weights[i][1] * qstep + c_mode_weights[i][2] * prod;
    int aq = qval < 0 ? -qval : qval;
    qval = apply_sign_((aq + (1 << 12)) >> 13, qval);
    return 255 * (c_mode_offsets[i] + qval);
}

R2G_D bool tile_row_first(const DevFrame &f, int sby) {
    return sby > 0 && sby < 128 && ((f.tr_first[sby >> 5] >> (sby & 31)) & 1);
}

// Stripe geometry and unit selection, following lr_sbrow_apply /
// lr_sbrow_plane / lr_stripe (sb128 = 0).  A superblock row's LR call
// covers [y_call, row_h); its first stripe is 56 (luma) rows high on the
// first superblock row of a tile row and 64 otherwise, so a call holds one
// stripe, or two when the frame height is a multiple of 64 and this is the
// last superblock row (mode 1 is that second stripe).  On the first
// superblock row of a later tile row the call is split
// (looprestoration.rs:2424-2548): mode 2 is the 8-row stripe above the tile
// row's top edge, which reads the rows below it in place
// (LR_HAVE_BOTTOM_INTEGRATED), and the call's first stripe starts at the
// edge and reads four saved deblocked rows above it (LR_HAVE_TOP_INTEGRATED).
R2G_D void unit_geom(const DevFrame &f, int plane, int sby, int mode, int ux, UnitGeom &g) {
    const int chroma = plane != 0;
    const int ss = chroma;  // 4:2:0: ss_hor = ss_ver = 1 for chroma
    const int W = chroma ? f.cw : f.w, H = chroma ? f.ch : f.h;
    const int not_last = sby + 1 < f.sbh;
    const int next_row_y = (sby + 1) << (6 - ss);
    const int trf = tile_row_first(f, sby);
    const int first = sby == 0 || trf;  // FirstSbInTileRow other than None
    int row_h = imin_(next_row_y - (8 >> ss) * not_last, H);
    const int y_call = (sby << (6 - ss)) - (first ? 0 : (8 >> ss));
    int y0, sh, edges;
    if (mode == 2) {
        // the 8 rows above the tile row's top edge (FirstSbInTileRow::Top)
        y0 = y_call - (8 >> ss);
        row_h = y_call;
        sh = row_h - y0;
        edges = LR_HAVE_TOP | LR_HAVE_BOTTOM_INTEGRATED;
    } else {
        const int sh0 = imin_((first ? 56 : 64) >> ss, row_h - y_call);
        y0 = y_call;
        sh = sh0;
        edges = y0 > 0 ? LR_HAVE_TOP : 0;
        if (trf && mode == 0) edges |= LR_HAVE_TOP_INTEGRATED;
        if (mode == 1) {
            y0 = y_call + sh0;
            sh = imin_(64 >> ss, row_h - y0);
            edges = LR_HAVE_TOP;
        }
    }
    g.plane = plane;
    g.y0 = y0;
    g.sh = sh;
    g.x0 = ux * 64;
    g.uw = imin_(64, W - g.x0);
    g.edges = edges | (ux > 0 ? LR_HAVE_LEFT : 0) | (g.x0 + 64 < W ? LR_HAVE_RIGHT : 0) |
              ((not_last || y0 + sh != row_h) ? LR_HAVE_BOTTOM : 0);
    // saved deblocked rows 4 and 5 of a top-integrated luma stripe: the
    // superblock row's own backup (copy_db / backup_db, deblock.rs:2192-2264)
    // when it saved a stripe boundary, else the previous one left in place
    g.l45 = (y0 + 56 <= f.h - 1) ? y0 + 54 : y0 - 10;
    g.sb256x = (g.x0 << ss) >> 8;
    g.sb64x_idx = ((g.x0 << ss) >> 6) & 3;
    // unit selection (looprestoration.rs:2295-2331) from the call's first
    // row, 8 (luma) rows lower on a tile row's first superblock row
    const int unit_size = 1 << f.fp.restoration_unit_size[chroma];
    const int half = unit_size >> 1;
    const int row_y = (mode == 2 ? y0 : y_call) + ((8 >> ss) * (first || mode == 2));
    int aligned = row_y & ~(unit_size - 1);
    if (aligned != 0 && aligned + half > H) aligned -= unit_size;
    aligned <<= ss;
    const int sb_idx = (aligned >> 8) * f.sb256w;
    const int unit_idx_base = ((aligned >> 6) & 3) << 2;
    int lr_sb = sb_idx, lr_u = unit_idx_base;
    if (g.x0 > 0) {
        int start = g.x0 & ~(unit_size - 1);
        if (start != 0 && W - start < half) start -= unit_size;
        const int shift_hor = 8 - ss;
        lr_u = unit_idx_base + ((start >> (shift_hor - 2)) & 3);
        lr_sb = sb_idx + (start >> shift_hor);
    }
    g.valid = sh > 0 && lr_sb < f.sb256w * f.sb256h && lr_u < 16;
    g.unit = g.valid ? &f.lr[lr_sb].lr[plane][lr_u] : nullptr;
}

// Source row of window row r (stripe-relative) and whether it is deblocked.
R2G_D void row_src(const UnitGeom &g, int r, int &row, bool &from_d) {
    if (r >= 0 && r < g.sh) {
        row = g.y0 + r;
        from_d = false;
    } else if (r < 0 && (g.edges & LR_HAVE_TOP_INTEGRATED)) {
        // the saved deblocked rows 0.. of the line store (the previous stripe
        // boundary's four rows, then the superblock row's own): luma window
        // rows -6 .. -1 hold saved rows 0 .. 5 as gdf_prep reads them (the
        // Wiener filters read rows 0 .. 3 as -4 .. -1, see filter_luma);
        // chroma rows -2, -1 hold saved rows 0, 1
        from_d = true;
        if (g.plane) {
            row = g.y0 - 6 + (r + 2);
        } else {
            const int k = r + 6;
            row = k < 4 ? g.y0 - 10 + k : g.l45 + (k - 4);
        }
    } else if (r >= g.sh && (g.edges & LR_HAVE_BOTTOM_INTEGRATED)) {
        // the rows below, read in place: not yet restored
        row = g.y0 + r;
        from_d = false;
    } else if (r < 0) {
        if (g.edges & LR_HAVE_TOP) {
            row = g.y0 + (r < -2 ? -2 : r);
            from_d = true;
        } else {
            row = g.y0;
            from_d = false;
        }
    } else {
        if (g.edges & LR_HAVE_BOTTOM) {
            row = g.y0 + g.sh + (r - g.sh > 1 ? 1 : r - g.sh);
            from_d = true;
        } else {
            row = g.y0 + g.sh - 1;
            from_d = false;
        }
    }
}

// Window column x (unit-relative) -> the column whose sample it holds.
R2G_D int col_clamp(int x, int uw, int edges) {
    if (x < 0 && !(edges & LR_HAVE_LEFT)) return 0;
    if (x >= uw && !(edges & LR_HAVE_RIGHT)) return uw - 1;
    return x;
}

// Compile-time tap tables (the reference's WIENER_NS_CONFIG_Y :389,
// PC_WIENER_CONFIG :374, GDF_COORDS :334, WIENER_NS_CONFIG_UV[_FROM_Y]
// :357/:359): with the loops unrolled every window offset is an immediate.
namespace TapsY {
__device__ constexpr int8_t ns[16][2] = {{1, 0}, {0, 1}, {2, 0}, {0, 2}, {1, 1}, {-1, 1}, {2, 1}, {2, -1},
                                         {1, 2}, {1, -2}, {3, 0}, {0, 3}, {4, 0}, {0, 4}, {3, 3}, {3, -3}};
__device__ constexpr int8_t pc[12][2] = {{1, 0}, {0, 1}, {2, 0}, {0, 2}, {1, 1}, {-1, 1},
                                         {2, 1}, {2, -1}, {1, 2}, {1, -2}, {3, 0}, {0, 3}};
__device__ constexpr int8_t gdf[18][2] = {{6, 0}, {5, 0}, {4, 0}, {3, 0}, {2, 1}, {2, 0}, {2, -1}, {1, 2}, {1, 1},
                                          {1, 0}, {1, -1}, {1, -2}, {0, 6}, {0, 5}, {0, 4}, {0, 3}, {0, 2}, {0, 1}};
__device__ constexpr int8_t uv[6][2] = {{1, 0}, {0, 1}, {1, 1}, {-1, 1}, {2, 0}, {0, 2}};
__device__ constexpr int8_t uvy[12][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1},
                                          {-1, 1}, {1, -1}, {2, 0}, {-2, 0}, {0, 2}, {0, -2}};
}  // namespace TapsY

// One work item as the producer publishes it to the consumers.
struct LrDesc {
    int b;   // per-frame item index; -1: no more items
    int fi;  // frame of the batch (0 in a per-frame launch)
    int plane, x0, y0, sh, ro, nr, uw, edges, kind, gdf, copy;
    int c0, c1;           // single-class FIR constants (sums of the taps)
    int8_t f[20];         // single-class NS-Wiener taps (the unit's or the frame's)
    uint16_t llm[18];     // lossless 4x4 bits per 4 rows of the stripe
    uint16_t noskip[18];  // no-skip 4x4 bits per 4 rows of the stripe (multi-class)
};

struct LrSmem {
    uint64_t full[2], empty[2];
    LrDesc desc[2];
    alignas(16) unsigned char raw[2][RAW_BYTES];
    union {
        // luma: every window position holds its sample and the right
        // neighbour as a 16x2 pair (low half = the sample), so a pixel pair
        // (x, x + 1) reads one tap of both pixels with one 32-bit load
        uint32_t wp[LH * LW];
        struct {
            uint32_t win[CH2 * CW2];   // chroma window, same pairing
            uint32_t lwin[CH2 * CW2];  // downsampled luma window, same pairing
        } ch;
    } u;
    // a top-integrated luma item's rows -4 .. 8 as the Wiener filters and the
    // classification read them (saved rows 0 .. 3 above the stripe; the
    // window holds gdf_prep's saved rows 0 .. 5 there), same layout as wp
    // (rows -6, -5 unused)
    uint32_t wtop[15 * LW];
    alignas(8) uint16_t gcell[17 * 33 * 4];  // GDF 2x2 gradient cells, 4 directions
    uint8_t classes[8][16];
    // consumer-side copies of the item's row data (the slot is released
    // before filtering)
    int8_t f[20];
    uint16_t llm[18];
    uint16_t noskip[18];
    // frame tables and the parameters they were staged for (-1: none)
    int gdf_key, pc_key, nsm_key;
    int bias[3];
    uint2 s_aa[4][18];       // per class and tap: (alpha, alpha), (-alpha, -alpha) as s16x2
    int4 s_w[4][22];         // per class and tap / feature: weights 0..2, alpha
    int16_t s_pcf[64 * 13];  // PC-Wiener filters of the frame's wiener_idx
    int8_t s_nsm[16][16];    // multi-class NS-Wiener filters of the frame
    int s_nsm_c0[16];
    int8_t s_err[4096];
};

// Sign-extended low / high halves of a 16x2 pair; unsigned halves.
R2G_D int lo16(uint32_t v) { return (int)(int16_t)(v & 0xffff); }
R2G_D int hi16(uint32_t v) { return (int)v >> 16; }
R2G_D int ulo(uint32_t v) { return (int)(v & 0xffff); }
R2G_D int uhi(uint32_t v) { return (int)(v >> 16); }

// Per-frame item index b -> geometry (luma items first: stripe slot, row
// part, unit; then U, then V: stripe slot, row part, unit).  Slots
// 0 .. sbh-1 are the superblock rows' first stripes; slot sbh is the second
// stripe only the last superblock row can have; slots sbh+1 .. sbh+n_tr are
// the 8-row stripes above the tile rows after the first.  False: an empty
// item.
R2G_D bool item_geom(const DevFrame &f, int b, UnitGeom &g, int &ro, int &nr) {
    const int nux_l = (f.w + 63) >> 6, nux_c = (f.cw + 63) >> 6;
    const int nparts = 64 / f.lr_rows;
    const int nslots = f.sbh + 1 + f.n_tr;
    const int n_luma = nslots * nparts * nux_l;
    int plane, ux, part, slot;
    if (b < n_luma) {
        plane = 0;
        ux = b % nux_l;
        b /= nux_l;
        part = b % nparts;
        slot = b / nparts;
    } else {
        b -= n_luma;
        const int per = nslots * 2 * nux_c;
        plane = 1 + b / per;
        b %= per;
        ux = b % nux_c;
        b /= nux_c;
        part = b & 1;
        slot = b >> 1;
    }
    if (slot > f.sbh)
        unit_geom(f, plane, f.tr_sby[slot - f.sbh - 1], 2, ux, g);
    else if (slot == f.sbh)
        unit_geom(f, plane, f.sbh - 1, 1, ux, g);
    else
        unit_geom(f, plane, slot, 0, ux, g);
    const int rows = plane ? CROWS : f.lr_rows;
    ro = part * rows;
    nr = imin_(rows, g.sh - ro);
    return g.sh > 0 && nr > 0;
}

// ---------------------------------------------------------------- producer
// Issues (issue = true) or only sizes the bulk copies of one item's raw
// rows, spread over the warp's lanes; returns this lane's bytes.
template <typename P>
R2G_D uint32_t item_copies(const DevFrame &f, const UnitGeom &g, int plane, int ro, int nr, int kind, bool copy,
                           unsigned char *raw, uint64_t *bar, int lane, bool issue) {
    typedef RawGeom<P> RG;
    constexpr int bps = (int)sizeof(P);
    const int64_t stride = f.stride[plane != 0];
    const char *Cp = (const char *)f.C[plane];
    const char *Dp = (const char *)f.D[plane];
    uint32_t total = 0;
    if (copy) {
        // unfiltered unit: its output rows only, from the unit origin
        const uint32_t bytes = (uint32_t)((g.uw * bps + 15) & ~15);
        if (!issue) return lane == 0 ? (uint32_t)nr * bytes : 0u;
        for (int r = lane; r < nr; r += 32) {
            if (issue)
                bulk_g2s(raw + r * RG::RB, Cp + ((int64_t)(g.y0 + ro + r) * stride + g.x0) * bps, bytes, bar);
            total += bytes;
        }
        return total;
    }
    // window columns [x0 - XO, x0 + 64 + XO), clipped to the plane row
    int cs = g.x0 - RG::XO, doff = 0;
    if (cs < 0) {
        doff = -cs * bps;
        cs = 0;
    }
    const int ce = imin_(g.x0 + 64 + RG::XO, (int)stride);
    const uint32_t bytes = (uint32_t)((ce - cs) * bps);
    const int halo = plane ? 2 : 6;
    const int wrows = nr + 2 * halo;
    if (!issue) {
        // every row copy of the item has the same length: the byte count
        // the slot's barrier expects, without walking the rows
        uint32_t t = (uint32_t)wrows * bytes;
        if (plane && kind == W_NS_SINGLE) {
            int lcs = 2 * g.x0 - RG::XO;
            if (lcs < 0) lcs = 0;
            const int lce = imin_(2 * g.x0 + 128 + RG::XO, (int)f.stride[0]);
            t += (uint32_t)(2 * wrows) * (uint32_t)((lce - lcs) * bps);
        }
        return lane == 0 ? t : 0u;
    }
    for (int r = lane; r < wrows; r += 32) {
        int row;
        bool from_d;
        row_src(g, ro + r - halo, row, from_d);
        if (issue) bulk_g2s(raw + r * RG::RB + doff, (from_d ? Dp : Cp) + ((int64_t)row * stride + cs) * bps, bytes, bar);
        total += bytes;
    }
    if (plane && kind == W_NS_SINGLE) {
        // CfL luma rows (backup_row_luma with ns_wiener_single_uv's row
        // selection, looprestoration.rs:1207-1350): two luma rows per window
        // row, C inside the stripe, D at the stripe boundaries
        const int64_t ls = f.stride[0];
        const char *Cy = (const char *)f.C[0];
        const char *Dy = (const char *)f.D[0];
        int lcs = 2 * g.x0 - RG::XO, ldoff = 0;
        if (lcs < 0) {
            ldoff = -lcs * bps;
            lcs = 0;
        }
        const int lce = imin_(2 * g.x0 + 128 + RG::XO, (int)ls);
        const uint32_t lbytes = (uint32_t)((lce - lcs) * bps);
        const bool topi = g.edges & LR_HAVE_TOP_INTEGRATED, boti = g.edges & LR_HAVE_BOTTOM_INTEGRATED;
        for (int q = lane; q < 2 * wrows; q += 32) {
            int rr = ro + (q >> 1) - 2;
            if (!(g.edges & LR_HAVE_TOP) && rr < 0) rr = 0;
            if (!(g.edges & LR_HAVE_BOTTOM) && !boti && rr >= g.sh) rr = g.sh - 1;
            const char *src;
            int ra, rb;
            if ((rr < 0 && topi) || (rr >= g.sh && boti)) {
                // integrated edges read the luma rows in place (pre-LR)
                src = Cy;
                ra = 2 * (g.y0 + rr);
                rb = ra + 1;
            } else if (rr == -2) {
                src = Dy;
                ra = rb = 2 * g.y0 - 2;
            } else if (rr == -1) {
                src = Dy;
                ra = 2 * g.y0 - 2;
                rb = 2 * g.y0 - 1;
            } else if (rr == g.sh) {
                src = Dy;
                ra = 2 * (g.y0 + g.sh);
                rb = ra + 1;
            } else if (rr == g.sh + 1) {
                src = Dy;
                ra = rb = 2 * (g.y0 + g.sh) + 1;
            } else {
                src = Cy;
                ra = 2 * (g.y0 + rr);
                rb = ra + 1;
            }
            const int lrow = (q & 1) ? rb : ra;
            if (issue)
                bulk_g2s(raw + RG::LOFF + q * RG::LRB + ldoff, src + ((int64_t)lrow * ls + lcs) * bps, lbytes, bar);
            total += lbytes;
        }
    }
    return total;
}

// Produces one work item into slot k & 1, after waiting for the slot's
// release when it was used before.  Returns 0 for an empty item (nothing
// published), 1 when published, -1 when a wait ran out.
template <typename P>
R2G_D int produce_item(const DevFrame &f, int fi, int b, LrSmem &sm, int k, int lane, bool &waited) {
    UnitGeom g;
    int ro, nr;
    if (!item_geom(f, b, g, ro, nr)) return 0;
    const int plane = g.plane, chroma = plane != 0;
    const R2gFrameParams &fp = f.fp;
    // ---- kernel selection (looprestoration.rs:1880-1920) ----
    int wkind = W_NONE;
    const bool plane_on = (f.restore_planes >> plane) & 1;
    if (plane_on && g.valid) {
        const int wt = (f.inloop & R2G_INLOOP_WIENER) ? g.unit->type : 0;
        const R2gRestorationPlane &pd = fp.restoration[plane];
        if (wt == R2G_RESTORE_NS_WIENER)
            wkind = (pd.frame_filters_on && pd.num_classes != 1) ? W_NS_MULTI : W_NS_SINGLE;
        else if (wt == R2G_RESTORE_PC_WIENER)
            wkind = W_PC;
    }
    const int inc = ((g.edges & (LR_HAVE_TOP | LR_HAVE_TOP_INTEGRATED | LR_HAVE_BOTTOM_INTEGRATED)) == LR_HAVE_TOP &&
                     g.y0 + 8 < ((f.bh4 * 4) >> chroma))
                        ? 8
                        : 0;
    const int sb256_idx = f.sb256w * (((g.y0 << chroma) + inc) >> 8) + g.sb256x;
    const int nsb = f.sb256w * f.sb256h;
    const bool gdf_on = plane_on && g.valid && plane == 0 && (f.inloop & R2G_INLOOP_GDF) && sb256_idx < nsb &&
                        f.masks[sb256_idx].gdf[(((g.y0 + inc) >> 4) & 12) + g.sb64x_idx] != 0;
    const bool copy = wkind == W_NONE && !gdf_on;
    // ---- per-lane side-info: lossless rows (looprestoration.rs:2037-2075),
    // multi-class no-skip rows (:1922-1944), single-class taps ----
    uint16_t llm = 0, nsk = 0;
    int tap = 0;
    if (!copy) {
        if (lane < 17) {
            const int ll_rows = imax_(g.sh >> 2, 1) + 1;
            if (lane < ll_rows && sb256_idx < nsb) {
                const R2gAv2Filter &m = f.masks[sb256_idx];
                const int y4 = ((g.y0 << chroma) & 255) >> 2;
                if (plane == 0) {
                    const int yy = y4 + lane;
                    if (yy < 64) llm = m.lossless_mask_y[yy][g.sb64x_idx];
                } else {
                    const int init_y = g.y0 >> 2, end_y = (g.y0 + g.sh) >> 2;
                    const int sy = (y4 >> 1) + lane;
                    if (init_y + lane < end_y && sy < 64) {
                        const uint16_t lo = m.lossless_mask_uv[sy][g.sb64x_idx];
                        const uint16_t hi = g.sb64x_idx + 1 < 4 ? m.lossless_mask_uv[sy][g.sb64x_idx + 1] : 0;
                        llm = (uint16_t)((lo & 0xff) | ((hi & 0xff) << 8));
                    }
                }
            }
        }
        if ((wkind == W_NS_MULTI || wkind == W_PC) && lane < 18) {
            const int by = (g.y0 >> 2) + lane;
            if (by < ((g.y0 + g.sh) >> 2)) {
                const int sidx = f.sb256w * (by >> 6) + g.sb256x;
                if (sidx < nsb) {
                    uint16_t v = f.masks[sidx].lr_noskip_mask[by & 63][g.sb64x_idx];
                    if (!(g.edges & LR_HAVE_RIGHT) && (g.uw & 63) != 0) {
                        const int s = ((g.uw >> 2) & 15) - 1;
                        const uint16_t eb = (uint16_t)(v >> s);
                        v = (uint16_t)(v | (uint16_t)(eb << (s + 1)));
                    }
                    nsk = v;
                }
            }
        }
        if (wkind == W_NS_SINGLE && lane < 18) {
            const R2gRestorationPlane &pd = fp.restoration[plane];
            tap = pd.frame_filters_on ? pd.filter[0][lane] : g.unit->f[lane];
        }
    }
    // single-class FIR constants: s = m * c0 + sum (a + b) f [- l * c1 + sum l' f]
    // equals the reference's (m << 7) + sum (a + b - 2m) f [+ sum (l' - l) f]
    const int nsym = chroma ? 6 : 16;
    const int fsym = __reduce_add_sync(0xffffffffu, lane < nsym ? tap : 0);
    const int fcc = __reduce_add_sync(0xffffffffu, (chroma && lane >= 6 && lane < 18) ? tap : 0);

    // C and D (and L, which the consumers write) belong to the previous
    // kernels on the stream: wait for them before the first copy
    if (!waited) {
        pdl_wait();
        waited = true;
    }
    const int s = k & 1;
    if (k >= 2 && !mbar_wait(&sm.empty[s], ((k >> 1) - 1) & 1)) return -1;
    LrDesc &d = sm.desc[s];
    if (lane == 0) {
        d.b = b;
        d.fi = fi;
        d.plane = plane;
        d.x0 = g.x0;
        d.y0 = g.y0;
        d.sh = g.sh;
        d.ro = ro;
        d.nr = nr;
        d.uw = g.uw;
        d.edges = g.edges;
        d.kind = wkind;
        d.gdf = gdf_on;
        d.copy = copy;
        d.c0 = 128 - 2 * fsym;
        d.c1 = fcc;
    }
    if (lane < 18) {
        d.llm[lane] = llm;
        d.noskip[lane] = nsk;
        d.f[lane] = (int8_t)tap;
    }
    const uint32_t total =
        __reduce_add_sync(0xffffffffu, item_copies<P>(f, g, plane, ro, nr, wkind, copy, sm.raw[s], &sm.full[s], lane,
                                                      false));
    // the consumers' reads of this slot (ordered before by the empty
    // barrier) precede the copies' writes
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(&sm.full[s], total);
    __syncwarp();
    item_copies<P>(f, g, plane, ro, nr, wkind, copy, sm.raw[s], &sm.full[s], lane, true);
    return 1;
}

template <int HB>
R2G_D bool is_hbd(const DevFrame &f) {
    return HB == 1 || (HB == 2 && f.bitdepth > 8);
}

// The producer warp: work-list positions blockIdx.x, then
// gridDim.x + atomicAdd(next), until the list is exhausted.
template <int HB, typename Src>
R2G_D void lr_producer(const Src &src, LrSmem &sm, int lane) {
    const int n = src.count();
    StageSched *sched = src.sched();
    int k = 0;  // items published
    int w = blockIdx.x;
    bool waited = false, ok = true;
    while (w < n) {
        int fi, b;
        src.item(w, fi, b);
        const DevFrame &f = src.frame(fi);
        const int rc = is_hbd<HB>(f) ? produce_item<uint16_t>(f, fi, b, sm, k, lane, waited)
                                     : produce_item<uint8_t>(f, fi, b, sm, k, lane, waited);
        if (rc < 0) {
            ok = false;
            break;
        }
        k += rc;
        if (!waited) {
            pdl_wait();
            waited = true;
        }
        // near the end of the list (fewer than two items per CTA left) take
        // the next item only once the consumers are on the last one
        // published (one item queued rather than two), so the CTAs run out
        // of work closer together; from three items per CTA on it made the
        // kernel shorter alone but the frame's pipelined step longer
        if (k >= 1) {
            unsigned taken = 0;
            if (lane == 0) taken = *reinterpret_cast<volatile unsigned *>(&sched->next);
            taken = __shfl_sync(0xffffffffu, taken, 0);
            if ((int)(2 * gridDim.x + taken) >= n && !mbar_wait(&sm.empty[(k - 1) & 1], ((k - 1) >> 1) & 1)) {
                ok = false;
                break;
            }
        }
        int nx = 0;
        if (lane == 0) nx = (int)(gridDim.x + atomicAdd(&sched->next, 1u));
        w = __shfl_sync(0xffffffffu, nx, 0);
    }
    if (!waited) pdl_wait();
    if (ok) {
        // no more items: publish the stop marker
        const int s = k & 1;
        if (k >= 2 && !mbar_wait(&sm.empty[s], ((k >> 1) - 1) & 1)) {
            ok = false;
        } else {
            if (lane == 0) {
                sm.desc[s].b = -1;
                mbar_arrive_expect_tx(&sm.full[s], 0);
            }
            __syncwarp();
        }
    }
    if (!ok && lane == 0) {
        // a wait ran out: record it, and let this CTA's copies in flight land
        // before the CTA (and its shared memory) goes away
        atomicAdd(src.fault(), 1u);
        for (int s = 0; s < 2; s++) {
            const int uses = (k + 1 - s) / 2;
            if (uses > 0) mbar_wait(&sm.full[s], (uses - 1) & 1);
        }
    }
    __syncwarp();
    if (lane == 0) sched_retire(sched);
}

// ---------------------------------------------------------------- consumers
// Stages the frame tables an item needs (GDF alpha / weights / bias / error
// LUT of the frame's ref_dst_idx and qp_idx; PC-Wiener filters of its
// wiener_idx; multi-class NS-Wiener filters).  Uniform over the consumers.
// Returns what it staged; after a consumer barrier, commit_tables records it
// (the keys are read by every consumer before any of them may change them).
R2G_D int stage_tables(const DevFrame &f, int fi, LrSmem &sm, bool gdf, bool pc, bool nsm, int tid) {
    const R2gFrameParams &fp = f.fp;
    const int ref_dst_idx = f.gdf_ref_dst_idx, qp_idx = fp.gdf_qp_idx;
    const int gkey = ref_dst_idx * 8 + qp_idx;
    const bool do_gdf = gdf && sm.gdf_key != gkey;
    const bool do_pc = pc && sm.pc_key != f.wiener_idx;
    const bool do_nsm = nsm && sm.nsm_key != fi;
    if (do_gdf) {
        const int alpha_base = ref_dst_idx * 528 + qp_idx * 88;
        const int weight_base = ref_dst_idx * 1584 + qp_idx * 264;
        const int8_t *errtab = ref_dst_idx == 0 ? f.tab.GDF_INTRA_ERROR + qp_idx * 4096
                                                : f.tab.GDF_INTER_ERROR + (ref_dst_idx - 1) * 6000 + qp_idx * 1000;
        const int nerr = ref_dst_idx == 0 ? 4096 : 1000;
        for (int i = tid; i < 88; i += NCT) {
            const int k = i >> 2, c = i & 3;
            const int a = f.tab.GDF_ALPHA[alpha_base + i];
            sm.s_w[c][k] = make_int4(f.tab.GDF_WEIGHT[weight_base + 0 * 88 + i],
                                     f.tab.GDF_WEIGHT[weight_base + 1 * 88 + i],
                                     f.tab.GDF_WEIGHT[weight_base + 2 * 88 + i], a);
            if (k < 18) {
                const uint32_t pa = (uint32_t)a & 0xffff, na = (uint32_t)(-a) & 0xffff;
                sm.s_aa[c][k] = make_uint2(pa | (pa << 16), na | (na << 16));
            }
        }
        if (tid < 3) sm.bias[tid] = f.tab.GDF_BIAS[(ref_dst_idx * 6 + qp_idx) * 3 + tid];
#pragma unroll 4
        for (int i = tid; i < nerr; i += NCT) sm.s_err[i] = __ldg(errtab + i);
    }
    if (do_pc)
        for (int i = tid; i < 64 * 13; i += NCT) sm.s_pcf[i] = __ldg(f.tab.PC_WIENER_FILTERS + f.wiener_idx * 64 * 13 + i);
    if (do_nsm) {
        sm.s_nsm[tid >> 4][tid & 15] = fp.restoration[0].filter[tid >> 4][tid & 15];
        if (tid < 16) {
            int s = 0;
            for (int k = 0; k < 16; k++) s += fp.restoration[0].filter[tid][k];
            sm.s_nsm_c0[tid] = 128 - 2 * s;
        }
    }
    return (do_gdf ? 1 : 0) | (do_pc ? 2 : 0) | (do_nsm ? 4 : 0);
}
R2G_D void commit_tables(const DevFrame &f, int fi, LrSmem &sm, int staged) {
    if (staged & 1) sm.gdf_key = f.gdf_ref_dst_idx * 8 + f.fp.gdf_qp_idx;
    if (staged & 2) sm.pc_key = f.wiener_idx;
    if (staged & 4) sm.nsm_key = fi;
}

template <typename P>
R2G_D int raw_at(const unsigned char *row, int x) {
    return (int)reinterpret_cast<const P *>(row)[x];
}

// Raw rows -> luma pair window (window column c holds source column c - 6),
// replicating the frame's left / right edge samples.
template <typename P>
R2G_D void build_luma_window(LrSmem &sm, const unsigned char *raw, int nr, int uw, int edges, int tid) {
    typedef RawGeom<P> RG;
    const int wh = nr + 12;
    if ((edges & LR_HAVE_LEFT) && (edges & LR_HAVE_RIGHT)) {
        // interior unit (uw == 64): four window columns 4q .. 4q + 3 per
        // step, from raw samples 4q + 2 .. 4q + 6 (u16) / 4q + 10 .. 4q + 14 (u8)
        for (int i = tid; i < wh * 19; i += NCT) {
            const int r = i / 19, q = i - r * 19;
            const unsigned char *row = raw + r * RG::RB;
            uint4 o;
            if (sizeof(P) == 2) {
                const uint32_t w0 = *reinterpret_cast<const uint32_t *>(row + 8 * q + 4);
                const uint32_t w1 = *reinterpret_cast<const uint32_t *>(row + 8 * q + 8);
                const uint32_t s4 = *reinterpret_cast<const uint16_t *>(row + 8 * q + 12);
                o = make_uint4(w0, __byte_perm(w0, w1, 0x5432), w1, __byte_perm(w1, s4, 0x5432));
            } else {
                const uint32_t w0 = *reinterpret_cast<const uint32_t *>(row + 4 * q + 8);
                const uint32_t w1 = *reinterpret_cast<const uint32_t *>(row + 4 * q + 12);
                const uint32_t e0 = __byte_perm(w0, 0, 0x4342), e1 = __byte_perm(w1, 0, 0x4140),
                               e2 = __byte_perm(w1, 0, 0x4442);
                o = make_uint4(e0, __byte_perm(e0, e1, 0x5432), e1, __byte_perm(e1, e2, 0x5432));
            }
            *reinterpret_cast<uint4 *>(&sm.u.wp[r * LW + 4 * q]) = o;
        }
    } else {
        const int ww = uw + 12;
        for (int i = tid; i < wh * ww; i += NCT) {
            const int r = i / ww, c = i - r * ww;
            const unsigned char *row = raw + r * RG::RB;
            const int a = raw_at<P>(row, col_clamp(c - 6, uw, edges) + RG::XO);
            const int b = raw_at<P>(row, col_clamp(c - 5, uw, edges) + RG::XO);
            sm.u.wp[r * LW + c] = (uint32_t)a | ((uint32_t)b << 16);
        }
    }
}

// Raw rows -> chroma pair window and (CfL) downsampled luma pair window
// (window column j holds chroma column j - 2).
template <typename P>
R2G_D void build_chroma_windows(LrSmem &sm, const unsigned char *raw, int nr, int uw, int edges, bool cfl, int ds,
                                int tid) {
    typedef RawGeom<P> RG;
    const int wh = nr + 4, ww = uw + 4;
    for (int i = tid; i < wh * ww; i += NCT) {
        const int r = i / ww, j = i - r * ww;
        const unsigned char *row = raw + r * RG::RB;
        const int a = raw_at<P>(row, col_clamp(j - 2, uw, edges) + RG::XO);
        const int b = raw_at<P>(row, col_clamp(j - 1, uw, edges) + RG::XO);
        sm.u.ch.win[r * CW2 + j] = (uint32_t)a | ((uint32_t)b << 16);
    }
    if (!cfl) return;
    const int lw = uw << 1;
    for (int i = tid; i < wh * ww; i += NCT) {
        const int r = i / ww, j = i - r * ww;
        const unsigned char *ra = raw + RG::LOFF + (2 * r) * RG::LRB;
        const unsigned char *rb = ra + RG::LRB;
        int l[2];
#pragma unroll
        for (int t = 0; t < 2; t++) {
            int pos = 2 * (j + t - 2);
            if (pos < 0 && !(edges & LR_HAVE_LEFT)) pos = 0;
            if (pos >= lw && !(edges & LR_HAVE_RIGHT)) pos = lw - 2;
            pos += RG::XO;
            if (ds == 0)
                l[t] = (raw_at<P>(ra, pos) + raw_at<P>(rb, pos) + raw_at<P>(ra, pos + 1) + raw_at<P>(rb, pos + 1)) >> 2;
            else if (ds == 1)
                l[t] = (raw_at<P>(ra, pos) + raw_at<P>(rb, pos)) >> 1;
            else
                l[t] = raw_at<P>(ra, pos);
        }
        sm.u.ch.lwin[r * CW2 + j] = (uint32_t)l[0] | ((uint32_t)l[1] << 16);
    }
}

// An unfiltered unit: staged rows -> L, 16 bytes per store.
template <typename P>
R2G_D void copy_unit(const DevFrame &f, const unsigned char *raw, int plane, int x0, int y, int nr, int uw, int tid) {
    typedef RawGeom<P> RG;
    const int bytes = uw * (int)sizeof(P);
    const int nch = (bytes + 15) >> 4;
    const int64_t stride = f.stride[plane != 0] * (int64_t)sizeof(P);
    char *L = (char *)f.L[plane] + (int64_t)y * stride + (int64_t)x0 * sizeof(P);
    for (int i = tid; i < nr * nch; i += NCT) {
        const int r = i / nch, q = i - r * nch;
        const unsigned char *src = raw + r * RG::RB + 16 * q;
        char *dst = L + r * stride + 16 * q;
        const int left = bytes - 16 * q;
        if (left >= 16) {
            *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(src);
        } else if (left >= 8) {
            *reinterpret_cast<uint2 *>(dst) = *reinterpret_cast<const uint2 *>(src);
            if (left >= 12) *reinterpret_cast<uint32_t *>(dst + 8) = *reinterpret_cast<const uint32_t *>(src + 8);
        } else {
            *reinterpret_cast<uint32_t *>(dst) = *reinterpret_cast<const uint32_t *>(src);
        }
    }
}

// GDF error of a luma pixel pair (x1, x1 + 1), x1 even, window row y
// (gdf_prep, looprestoration.rs:1540-1640): both pixels share the 2x2
// gradient cell and so the class; their 18 clipped symmetric differences run
// as 16x2 pairs.
template <typename P>
R2G_D void gdf_pair(const DevFrame &f, const LrSmem &sm, const uint32_t *wc, int y, int x1, int uw, int &e0, int &e1) {
    constexpr int up = sizeof(P) == 1 ? 2 : 0;  // the 10-bit internal domain
    const int ci = (uw >> 1) + 1;
    const int j = y >> 1, c = x1 >> 1;
    // the four cells' 16-bit direction sums add as 16x2 pairs without a
    // carry between the halves: a cell holds at most 4 x 2046 per direction
    const uint2 *gc = reinterpret_cast<const uint2 *>(sm.gcell);
    const uint2 ca = gc[j * ci + c], cb = gc[j * ci + c + 1], cc = gc[(j + 1) * ci + c], cd = gc[(j + 1) * ci + c + 1];
    const uint32_t s01 = ca.x + cb.x + cc.x + cd.x, s23 = ca.y + cb.y + cc.y + cd.y;
    const int gsum[4] = {(int)(s01 & 0xffff), (int)(s01 >> 16), (int)(s23 & 0xffff), (int)(s23 >> 16)};
    const int cls = (gsum[0] <= gsum[1]) | ((gsum[2] <= gsum[3]) << 1);
    const int4 *wt = sm.s_w[cls];
    const uint2 *aa = sm.s_aa[cls];
    int sh0 = sm.bias[0], sh1 = sm.bias[1], sh2 = sm.bias[2];
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const int4 p = wt[18 + d];
        const int v = imin_(gsum[d] >> (4 - up), p.w);
        sh0 += v * p.x;
        sh1 += v * p.y;
        sh2 += v * p.z;
    }
    const uint32_t mm = wc[0] << up;  // samples < 2^10: no carry between the halves
    const uint32_t nm = __vneg2(mm);
    int i0 = sh0, i1 = sh1, i2 = sh2, j0 = sh0, j1 = sh1, j2 = sh2;
#pragma unroll
    for (int k = 0; k < 18; k++) {
        const int o = TapsY::gdf[k][0] * LW + TapsY::gdf[k][1];
        const uint2 al = aa[k];
        const int4 p = wt[k];
        // clip(a - m, -alpha, alpha) as the fused add-max / add-min
        const uint32_t above = __viaddmin_s16x2(__viaddmax_s16x2(wc[-o] << up, nm, al.y), 0u, al.x);
        const uint32_t below = __viaddmin_s16x2(__viaddmax_s16x2(wc[o] << up, nm, al.y), 0u, al.x);
        const uint32_t v = __viaddmin_s16x2(__viaddmax_s16x2(above, below, 0xfe00fe00u), 0u, 0x01ff01ffu);
        const int v0 = lo16(v), v1 = hi16(v);
        i0 += v0 * p.x;
        i1 += v0 * p.y;
        i2 += v0 * p.z;
        j0 += v1 * p.x;
        j1 += v1 * p.y;
        j2 += v1 * p.z;
    }
    const int scale = f.gdf_ref_dst_idx == 0 ? 8 : 5;
    int full0 = 0, full1 = 0;
    const int iv0[3] = {i0, i1, i2}, iv1[3] = {j0, j1, j2};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        int sv = iv0[q] * scale;
        int v = apply_sign_(((sv < 0 ? -sv : sv) + (1 << 14)) >> 15, sv);
        full0 = full0 * (scale * 2) + iclip_(v, -scale, scale - 1) + scale;
        sv = iv1[q] * scale;
        v = apply_sign_(((sv < 0 ? -sv : sv) + (1 << 14)) >> 15, sv);
        full1 = full1 * (scale * 2) + iclip_(v, -scale, scale - 1) + scale;
    }
    e0 = sm.s_err[full0];
    e1 = sm.s_err[full1];
}

// Filters one staged luma item (everything after the window is built).
template <typename P>
R2G_D void filter_luma(const DevFrame &f, LrSmem &sm, int x0, int y0, int sh, int ro, int nr, int uw, int kind,
                       bool gdf, int c0, bool topi, int tid) {
    const int warp = tid >> 5, lane = tid & 31;
    const R2gFrameParams &fp = f.fp;
    const int16_t *W16 = reinterpret_cast<const int16_t *>(sm.u.wp);  // scalar sample i at W16[2 * i]
    const int16_t *WT16 = reinterpret_cast<const int16_t *>(sm.wtop);
    const int bh4 = nr >> 2, bw4 = uw >> 2, sbh4 = sh >> 2;
    const int b8 = f.bitdepth - 8;
    // ---- phase 1: GDF gradient cells (compute_gradient_row :114-193) and
    // multi-class 4x4 classes (get_class_lut_idx :195-271, :870-896) ----
    if (gdf) {
        // cell (j, i): window rows 2j-1, 2j; columns 2i-1, 2i; pair (y, x1)
        // sums cells (y/2 .. y/2+1, x1/2 .. x1/2+1)
        constexpr int down = 0;
        const int cj = (nr >> 1) + 1, ci = (uw >> 1) + 1;
        for (int i = tid; i < cj * ci; i += NCT) {
            const int j = i / ci, c = i - j * ci;
            int gs[4] = {0, 0, 0, 0};
#pragma unroll
            for (int yy = 0; yy < 2; yy++)
#pragma unroll
                for (int xx = 0; xx < 2; xx++) {
                    const int16_t *w = &W16[2 * ((2 * j - 1 + yy + 6) * LW + 2 * c - 1 + xx + 6)];
                    constexpr int R = 2 * LW, C1 = 2;
                    const int bv = w[0] >> down;
                    int t;
                    t = 2 * bv - (w[-R] >> down) - (w[R] >> down);
                    gs[0] += t < 0 ? -t : t;
                    t = 2 * bv - (w[-C1] >> down) - (w[C1] >> down);
                    gs[1] += t < 0 ? -t : t;
                    t = 2 * bv - (w[-R - C1] >> down) - (w[R + C1] >> down);
                    gs[2] += t < 0 ? -t : t;
                    t = 2 * bv - (w[R - C1] >> down) - (w[-R + C1] >> down);
                    gs[3] += t < 0 ? -t : t;
                }
            *reinterpret_cast<uint2 *>(&sm.gcell[i * 4]) =
                make_uint2((uint32_t)gs[0] | ((uint32_t)gs[1] << 16), (uint32_t)gs[2] | ((uint32_t)gs[3] << 16));
        }
    }
    if (kind == W_NS_MULTI || kind == W_PC) {
        const uint8_t *sub_lut = kind == W_PC
                                     ? f.tab.PC_WIENER_SUB_CLASSIFY + f.wiener_idx * 256
                                     : f.tab.PC_WIENER_SUB_CLASSIFY_NS +
                                           (f.wiener_idx * 7 + (f.ns_ci >= 0 ? imin_(f.ns_ci, 6) : 0)) * 256;
        // two adjacent lanes per 4x4 block, each summing three of the six
        // feature rows; the trip count is uniform over the consumers so
        // the pair's partial sums combine with one shuffle
        const int nblk = bh4 * bw4;
        for (int base = 0; base < 2 * nblk; base += NCT) {
            const int i = base + tid;
            const bool act = i < 2 * nblk;
            const int blk = act ? (i >> 1) : 0, half = i & 1;
            const int by = blk / bw4, bx = blk - by * bw4;
            int fs0 = 0, fs1 = 0, fs2 = 0;
            if (act) {
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    const int dy = 3 * half - 1 + t;
#pragma unroll
                    for (int dx = -1; dx <= 4; dx++) {
                        const int16_t *w =
                            &(topi && by == 0 ? WT16 : W16)[2 * ((by * 4 + dy + 6) * LW + bx * 4 + dx + 6)];
                        constexpr int R = 2 * LW, C1 = 2;
                        const int m2 = 2 * w[0];
                        const int vert = w[-R] - m2 + w[R];
                        const int anti = w[-R + C1] - m2 + w[R - C1];
                        const int diag = w[-R - C1] - m2 + w[R + C1];
                        fs0 += vert < 0 ? -vert : vert;
                        fs1 += anti < 0 ? -anti : anti;
                        fs2 += diag < 0 ? -diag : diag;
                    }
                }
            }
            fs0 += __shfl_xor_sync(0xffffffffu, fs0, 1);
            fs1 += __shfl_xor_sync(0xffffffffu, fs1, 1);
            fs2 += __shfl_xor_sync(0xffffffffu, fs2, 1);
            if (!act || half) continue;
            int s = 0;
            const int np[3] = {16, 4, 1};
#pragma unroll
            for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    const int e = (dy != 0) + (dx != 0);
                    const int fx = iclip_((bx & 15) + dx, 0, 15);
                    const int fy = iclip_((ro >> 2) + by + dy, 0, sbh4 - 1);
                    s += np[e] * (((sm.noskip[fy] >> fx) & 1) == 0);
                }
            const int rnd = (1 << b8) >> 1;
            int fs[3] = {fs0, fs1, fs2};
#pragma unroll
            for (int k = 0; k < 3; k++) fs[k] = (int)((uint32_t)fs[k] * (uint32_t)c_pcw_norm[k] + (uint32_t)rnd) >> b8;
            s *= c_pcw_norm[3];
            int qv = (imax_(0, get_qval(f.base_q, s, 0, b8)) + (1 << 13)) >> 14;
            qv = imin_(qv, 255) >> 5;
            int lut_idx = qv << 9;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                qv = (imax_(0, fs[k] + get_qval(f.base_q, s, k + 1, b8)) + (1 << 13)) >> 14;
                qv = imin_(qv, 255) >> 5;
                lut_idx |= qv << (3 * (2 - k));
            }
            sm.classes[by][bx] = __ldg(sub_lut + __ldg(f.tab.PC_WIENER_LUT_TO_CLASS + lut_idx));
        }
    }
    if (gdf || kind == W_NS_MULTI || kind == W_PC) bar_sync_n(NCT);
    // ---- phase 2: per pixel pair: GDF error, FIR, GDF add, store ----
    const int bdmax = f.bdmax;
    const int gshift = 12 - f.bitdepth, grnd = (1 << gshift) >> 1, gscale = fp.gdf_scale;
    const int64_t stride = f.stride[0];
    P *Lp = plane_ptr<P>(f.L[0]) + (int64_t)(y0 + ro) * stride + x0;
    const int x1 = 2 * lane;
    if (x1 >= uw) return;
    for (int y = warp; y < nr; y += NCW) {
        const uint32_t *wc = &sm.u.wp[(y + 6) * LW + x1 + 6];
        const uint32_t *wf = topi && y < 4 ? &sm.wtop[(y + 6) * LW + x1 + 6] : wc;  // the Wiener taps' rows
        const uint32_t mm = wc[0];
        int v0 = ulo(mm), v1 = uhi(mm);
        const bool ll = (sm.llm[(ro + y) >> 2] >> (x1 >> 2)) & 1;
        if (!ll) {
            int e0 = 0, e1 = 0;
            if (gdf) gdf_pair<P>(f, sm, wc, y, x1, uw, e0, e1);
            if (kind != W_NONE) {
                int s0, s1;
                if (kind == W_PC) {
                    const int16_t *flt = sm.s_pcf + sm.classes[y >> 2][x1 >> 2] * 13;
                    s0 = v0 * flt[12];
                    s1 = v1 * flt[12];
#pragma unroll
                    for (int k = 0; k < 12; k++) {
                        const int o = TapsY::pc[k][0] * LW + TapsY::pc[k][1];
                        const uint32_t t = wf[o] + wf[-o];  // both halves < 2^11: no carry
                        const int fk = flt[k];
                        s0 += ulo(t) * fk;
                        s1 += uhi(t) * fk;
                    }
                } else {
                    const int8_t *flt;
                    int cc;
                    if (kind == W_NS_SINGLE) {
                        flt = sm.f;
                        cc = c0;
                    } else {
                        const int cls = sm.classes[y >> 2][x1 >> 2];
                        flt = sm.s_nsm[cls];
                        cc = sm.s_nsm_c0[cls];
                    }
                    s0 = v0 * cc;
                    s1 = v1 * cc;
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const int o = TapsY::ns[k][0] * LW + TapsY::ns[k][1];
                        const uint32_t t = wf[o] + wf[-o];
                        const int fk = flt[k];
                        s0 += ulo(t) * fk;
                        s1 += uhi(t) * fk;
                    }
                }
                v0 = clip_px_((s0 + 64) >> 7, bdmax);
                v1 = clip_px_((s1 + 64) >> 7, bdmax);
            }
            if (gdf) {
                int diff = e0 * gscale;
                v0 = clip_px_(v0 + apply_sign_(((diff < 0 ? -diff : diff) + grnd) >> gshift, diff), bdmax);
                diff = e1 * gscale;
                v1 = clip_px_(v1 + apply_sign_(((diff < 0 ? -diff : diff) + grnd) >> gshift, diff), bdmax);
            }
        }
        if (sizeof(P) == 2)
            *reinterpret_cast<uint32_t *>(Lp + (int64_t)y * stride + x1) = (uint32_t)v0 | ((uint32_t)v1 << 16);
        else
            *reinterpret_cast<uint16_t *>(Lp + (int64_t)y * stride + x1) = (uint16_t)(v0 | (v1 << 8));
    }
}

// Filters one staged chroma item: NS-Wiener with 6 chroma taps and 12
// cross-component taps on the downsampled luma (ns_wiener_single_uv
// :1145-1430).
template <typename P>
R2G_D void filter_chroma(const DevFrame &f, LrSmem &sm, int plane, int x0, int y0, int ro, int nr, int uw, int c0,
                         int c1, int tid) {
    const int warp = tid >> 5, lane = tid & 31;
    const int bdmax = f.bdmax;
    const int64_t stride = f.stride[1];
    P *Lp = plane_ptr<P>(f.L[plane]) + (int64_t)(y0 + ro) * stride + x0;
    const int x = 2 * lane;
    if (x >= uw) return;
    for (int y = warp; y < nr; y += NCW) {
        const uint32_t *w = &sm.u.ch.win[(y + 2) * CW2 + x + 2];
        const uint32_t *l = &sm.u.ch.lwin[(y + 2) * CW2 + x + 2];
        const uint32_t mm = w[0];
        int v0 = ulo(mm), v1 = uhi(mm);
        const bool ll = (sm.llm[(ro + y) >> 2] >> (x >> 2)) & 1;
        if (!ll) {
            const uint32_t lm = l[0];
            int s0 = v0 * c0 - ulo(lm) * c1, s1 = v1 * c0 - uhi(lm) * c1;
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const int o = TapsY::uv[k][0] * CW2 + TapsY::uv[k][1];
                const uint32_t t = w[o] + w[-o];
                const int fk = sm.f[k];
                s0 += ulo(t) * fk;
                s1 += uhi(t) * fk;
            }
#pragma unroll
            for (int k = 0; k < 12; k++) {
                const int o = TapsY::uvy[k][0] * CW2 + TapsY::uvy[k][1];
                const uint32_t t = l[o];
                const int fk = sm.f[6 + k];
                s0 += ulo(t) * fk;
                s1 += uhi(t) * fk;
            }
            v0 = clip_px_((s0 + 64) >> 7, bdmax);
            v1 = clip_px_((s1 + 64) >> 7, bdmax);
        }
        if (sizeof(P) == 2)
            *reinterpret_cast<uint32_t *>(Lp + (int64_t)y * stride + x) = (uint32_t)v0 | ((uint32_t)v1 << 16);
        else
            *reinterpret_cast<uint16_t *>(Lp + (int64_t)y * stride + x) = (uint16_t)(v0 | (v1 << 8));
    }
}

// One consumed item: tables, window, slot release, filtering.
template <typename P>
R2G_D void consume_item(const DevFrame &f, LrSmem &sm, int s, int tid) {
    const LrDesc &d = sm.desc[s];
    const int fi = d.fi, plane = d.plane, x0 = d.x0, y0 = d.y0, sh = d.sh, ro = d.ro, nr = d.nr, uw = d.uw;
    const int edges = d.edges, kind = d.kind, c0 = d.c0, c1 = d.c1;
    const bool gdf = d.gdf, copy = d.copy;
    const unsigned char *raw = sm.raw[s];
    if (copy) {
        copy_unit<P>(f, raw, plane, x0, y0 + ro, nr, uw, tid);
        __syncwarp();
        if ((tid & 31) == 0) mbar_arrive(&sm.empty[s]);
        return;
    }
    const int staged = stage_tables(f, fi, sm, gdf, kind == W_PC, kind == W_NS_MULTI, tid);
    if (tid < 18) {
        sm.llm[tid] = d.llm[tid];
        sm.noskip[tid] = d.noskip[tid];
        sm.f[tid] = d.f[tid];
    }
    if (plane == 0)
        build_luma_window<P>(sm, raw, nr, uw, edges, tid);
    else
        build_chroma_windows<P>(sm, raw, nr, uw, edges, kind == W_NS_SINGLE, f.fp.cfl_ds_filter_index, tid);
    __syncwarp();
    if ((tid & 31) == 0) mbar_arrive(&sm.empty[s]);
    bar_sync_n(NCT);
    if (tid == 0 && staged) commit_tables(f, fi, sm, staged);
    // a top-integrated luma item: the Wiener filters' rows -4 .. -1 are the
    // saved rows 0 .. 3, which the window holds as rows -6 .. -3
    const bool topi = plane == 0 && ro == 0 && (edges & LR_HAVE_TOP_INTEGRATED) && kind != W_NONE;
    if (topi) {
        for (int i = 2 * LW + tid; i < 15 * LW; i += NCT) {
            const int r = i / LW - 6;
            sm.wtop[i] = sm.u.wp[i + (r < 0 ? -2 * LW : 0)];
        }
        bar_sync_n(NCT);
    }
    if (plane == 0)
        filter_luma<P>(f, sm, x0, y0, sh, ro, nr, uw, kind, gdf, c0, topi, tid);
    else
        filter_chroma<P>(f, sm, plane, x0, y0, ro, nr, uw, c0, c1, tid);
}

// The consumer warps: slots in publication order until the stop marker.
template <int HB, typename Src>
R2G_D void lr_consumers(const Src &src, LrSmem &sm, int tid) {
    for (int k = 0;; k++) {
        const int s = k & 1;
        const bool got = mbar_wait(&sm.full[s], (k >> 1) & 1);
        // one vote per item: the previous item is finished by every consumer
        // and all of them saw the slot (or all stop)
        if (bar_or(!got, NCT)) {
            if (tid == 0) atomicAdd(src.fault(), 1u);
            return;
        }
        if (sm.desc[s].b < 0) return;
        const DevFrame &f = src.frame(sm.desc[s].fi);
        if (is_hbd<HB>(f))
            consume_item<uint16_t>(f, sm, s, tid);
        else
            consume_item<uint8_t>(f, sm, s, tid);
    }
}

template <int HB, typename Src>
R2G_D void lr_run(const Src &src, LrSmem &sm) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&sm.full[0], 1);
        mbar_init(&sm.full[1], 1);
        mbar_init(&sm.empty[0], NCW);
        mbar_init(&sm.empty[1], NCW);
        sm.gdf_key = sm.pc_key = sm.nsm_key = -1;
        mbar_init_fence();
    }
    __syncthreads();
    if (tid >= NCT) {
        lr_producer<HB>(src, sm, tid & 31);
    } else {
        src.prologue(sm, tid);
        pdl_wait();
        lr_consumers<HB>(src, sm, tid);
    }
}

// Work sources: one frame (kernel parameter) or a batch's LR work list.
struct FrameSrc {
    const DevFrame *f;
    int n;
    R2G_D int count() const { return n; }
    R2G_D const DevFrame &frame(int) const { return *f; }
    R2G_D void item(int w, int &fi, int &b) const {
        fi = 0;
        b = w;
    }
    R2G_D StageSched *sched() const { return f->sched + 2; }
    R2G_D unsigned *fault() const { return f->fault; }
    // the frame's tables, staged before the dependency wait
    R2G_D void prologue(LrSmem &sm, int tid) const {
        const bool gdf = (f->inloop & R2G_INLOOP_GDF) && f->fp.gdf_enabled;
        const int rt = f->fp.restoration[0].restoration_type;
        const bool pc = (f->inloop & R2G_INLOOP_WIENER) && (rt == R2G_RESTORE_PC_WIENER || rt == R2G_RESTORE_SWITCHABLE);
        const bool nsm = (f->inloop & R2G_INLOOP_WIENER) && f->fp.restoration[0].frame_filters_on &&
                         f->fp.restoration[0].num_classes != 1;
        const int staged = stage_tables(*f, 0, sm, gdf, pc, nsm, tid);
        bar_sync_n(NCT);
        if (tid == 0 && staged) commit_tables(*f, 0, sm, staged);
    }
};
struct BatchSrc {
    const BatchArgs *a;
    R2G_D int count() const { return a->count[2]; }
    R2G_D const DevFrame &frame(int fi) const { return a->frames[fi]; }
    R2G_D void item(int w, int &fi, int &b) const {
        const uint32_t it = a->work[2][w];
        fi = (int)(it >> 22);
        b = (int)(it & 0x3fffff);
    }
    R2G_D StageSched *sched() const { return a->sched + 2; }
    R2G_D unsigned *fault() const { return a->fault; }
    R2G_D void prologue(LrSmem &, int) const {}
};

template <typename P>
__global__ void __launch_bounds__(LR_NT, 3) lr_kernel(const __grid_constant__ DevFrame f, int n) {
    pdl_trigger();
    extern __shared__ __align__(128) unsigned char lr_smem[];
    LrSmem &sm = *reinterpret_cast<LrSmem *>(lr_smem);
    FrameSrc src{&f, n};
    lr_run<sizeof(P) == 2 ? 1 : 0>(src, sm);
}

__global__ void __launch_bounds__(LR_NT, 3) lr_batch_kernel(const __grid_constant__ BatchArgs a) {
    pdl_trigger();
    extern __shared__ __align__(128) unsigned char lr_smem[];
    LrSmem &sm = *reinterpret_cast<LrSmem *>(lr_smem);
    BatchSrc src{&a};
    lr_run<2>(src, sm);
}

// ---- DSP-context slot kernel (r2g_dsp_gdf_add): gdf_add
// (looprestoration.rs:273-329) on a w x h block ----
__global__ void dsp_gdf_add_kernel(uint16_t *p, const int8_t *err, int w, int h, int scale, const uint16_t *llm,
                                   int bitdepth) {
    const int shift = 12 - bitdepth, rnd = (1 << shift) >> 1, bdmax = (1 << bitdepth) - 1;
    for (int i = threadIdx.x; i < (w & ~3) * (h & ~3); i += blockDim.x) {
        const int ww = w & ~3, y = i / ww, x = i % ww;
        if ((llm[(y >> 2) * 4] >> (x >> 2)) & 1) continue;
        const int diff = err[y * w + x] * scale;
        const int ad = diff < 0 ? -diff : diff;
        p[y * w + x] = (uint16_t)clip_px_((int)p[y * w + x] + apply_sign_((ad + rnd) >> shift, diff), bdmax);
    }
}

// ---- DSP-context slot kernels for the typed LR slots (WienerFilterFn,
// GdfPrepFn).  The host (dsp.cu) stages the block's rows as the reference's
// row rings hold them: `rows` is a table of staged rows of `rs` samples
// (column 0 of the block at index e), and per output row (and per
// classification row / gradient event) the row ids each ring slot points at.
// One CTA computes the block; results go to `out` ([h][w]).

R2G_D int trow(const uint16_t *rows, int rs, int e, int id, int x) { return (int)rows[(size_t)id * rs + e + x]; }

// ns_wiener_single_y / ns_wiener_multi / pc_wiener (looprestoration.rs
// :524-1143): ref [h][9] FIR rows (ring slot 4 = the output row), cref
// [h/4][10] classification rows.  kind: 1 single, 2 NS multi, 3 PC.
__global__ void dsp_wiener_y_kernel(const uint16_t *rows, int rs, int e, const int *ref, const int *cref, int w, int h,
                                    int kind, const int8_t *taps, int taps_stride, const int16_t *pcf,
                                    const uint8_t *sub_lut, const uint16_t *noskip, int base_q, const uint16_t *llm,
                                    int bitdepth, const DevTables tab, uint16_t *out) {
    __shared__ uint8_t classes[16][16];
    const int tid = threadIdx.x, bh = h >> 2, bw = w >> 2, b8 = bitdepth - 8, bdmax = (1 << bitdepth) - 1;
    if (kind != W_NS_SINGLE) {
        // get_class_lut_idx (:195-271) with the ring rows of block row by
        for (int i = tid; i < bh * bw; i += blockDim.x) {
            const int by = i / bw, bx = i % bw;
            const int *r = cref + by * 10;
            int f0 = 0, f1 = 0, f2 = 0;
            for (int dy = -1; dy <= 4; dy++)
                for (int dx = -1; dx <= 4; dx++) {
                    const int x = bx * 4 + dx, y = 4 + dy;
                    const int m2 = 2 * trow(rows, rs, e, r[y], x);
                    int t = trow(rows, rs, e, r[y - 1], x) - m2 + trow(rows, rs, e, r[y + 1], x);
                    f0 += t < 0 ? -t : t;
                    t = trow(rows, rs, e, r[y - 1], x + 1) - m2 + trow(rows, rs, e, r[y + 1], x - 1);
                    f1 += t < 0 ? -t : t;
                    t = trow(rows, rs, e, r[y - 1], x - 1) - m2 + trow(rows, rs, e, r[y + 1], x + 1);
                    f2 += t < 0 ? -t : t;
                }
            const int np[3] = {16, 4, 1};
            int s = 0;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const int fx = iclip_((bx & 15) + dx, 0, 15), fy = iclip_(by + dy, 0, bh - 1);
                    s += np[(dy != 0) + (dx != 0)] * (((noskip[fy] >> fx) & 1) == 0);
                }
            const int rnd = (1 << b8) >> 1;
            int fs[3] = {f0, f1, f2};
            for (int k = 0; k < 3; k++) fs[k] = (int)((uint32_t)fs[k] * (uint32_t)c_pcw_norm[k] + (uint32_t)rnd) >> b8;
            s *= c_pcw_norm[3];
            int qv = (imax_(0, get_qval(base_q, s, 0, b8)) + (1 << 13)) >> 14;
            int lut_idx = (imin_(qv, 255) >> 5) << 9;
            for (int k = 0; k < 3; k++) {
                qv = (imax_(0, fs[k] + get_qval(base_q, s, k + 1, b8)) + (1 << 13)) >> 14;
                lut_idx |= (imin_(qv, 255) >> 5) << (3 * (2 - k));
            }
            classes[by][bx] = sub_lut[tab.PC_WIENER_LUT_TO_CLASS[lut_idx]];
        }
        __syncthreads();
    }
    for (int i = tid; i < w * h; i += blockDim.x) {
        const int y = i / w, x = i % w;
        const int *r = ref + y * 9;
        const int m = trow(rows, rs, e, r[4], x);
        int v = m;
        if (!((llm[(y >> 2) * 4] >> (x >> 2)) & 1)) {
            int s;
            if (kind == W_PC) {
                const int16_t *flt = pcf + classes[y >> 2][x >> 2] * 13;
                s = m * flt[12];
                for (int k = 0; k < 12; k++) {
                    const int dy = TapsY::pc[k][0], dx = TapsY::pc[k][1];
                    s += (trow(rows, rs, e, r[4 + dy], x + dx) + trow(rows, rs, e, r[4 - dy], x - dx)) * flt[k];
                }
            } else {
                const int8_t *flt = kind == W_NS_SINGLE ? taps : taps + classes[y >> 2][x >> 2] * taps_stride;
                s = m << 7;
                for (int k = 0; k < 16; k++) {
                    const int dy = TapsY::ns[k][0], dx = TapsY::ns[k][1];
                    s += (trow(rows, rs, e, r[4 + dy], x + dx) + trow(rows, rs, e, r[4 - dy], x - dx) - 2 * m) * flt[k];
                }
            }
            v = iclip_((s + 64) >> 7, 0, bdmax);
        }
        out[i] = (uint16_t)v;
    }
}

// ns_wiener_single_uv (:1145-1430): chroma rows (margin 2) and downsampled
// luma rows (margin 4, luma columns); cref / lref [h][5], slot 2 = the
// output row.
__global__ void dsp_wiener_uv_kernel(const uint16_t *crows, int crs, const uint16_t *lrows, int lrs, const int *cref,
                                     const int *lref, int w, int h, int ss_hor, const int8_t *f, const uint16_t *llm,
                                     int bitdepth, uint16_t *out) {
    const int bdmax = (1 << bitdepth) - 1;
    for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
        const int y = i / w, x = i % w;
        const int *cr = cref + y * 5, *lr = lref + y * 5;
        const int m = trow(crows, crs, 2, cr[2], x);
        int v = m;
        if (!((llm[(y >> 2) * 4] >> (x >> 2)) & 1)) {
            int s = m << 7;
            for (int k = 0; k < 6; k++) {
                const int dy = TapsY::uv[k][0], dx = TapsY::uv[k][1];
                s += (trow(crows, crs, 2, cr[2 + dy], x + dx) + trow(crows, crs, 2, cr[2 - dy], x - dx) - 2 * m) * f[k];
            }
            const int l = trow(lrows, lrs, 4, lr[2], x << ss_hor);
            for (int k = 0; k < 12; k++) {
                const int dy = TapsY::uvy[k][0], dx = TapsY::uvy[k][1];
                s += (trow(lrows, lrs, 4, lr[2 + dy], (x + dx) * (1 << ss_hor)) - l) * f[6 + k];
            }
            v = iclip_((s + 64) >> 7, 0, bdmax);
        }
        out[i] = (uint16_t)v;
    }
}

// gdf_prep (:1432-1640): gradient events gref [ng][13] (event 0 with row
// offset 6, the others with 8), per output row pref [h][13] (slot 6 = the
// output row).
__global__ void dsp_gdf_prep_kernel(const uint16_t *rows, int rs, int e, const int *gref, int ng, const int *pref, int w,
                                    int h, int ref_dst_idx, int qp_idx, int bitdepth, const DevTables tab,
                                    int8_t *out) {
    __shared__ uint16_t cells[33][34][4];
    const int up = bitdepth == 8 ? 2 : 0;
    const int nc = (w + 2 + 1) >> 1;
    // compute_gradient_row (:114-193) per event and cell
    for (int i = threadIdx.x; i < ng * nc; i += blockDim.x) {
        const int g = i / nc, c = i % nc, x1 = 2 * c;
        const int *r = gref + g * 13;
        const int row_off = g == 0 ? 6 : 8;
        const int offs[4][2] = {{1, 0}, {0, 1}, {1, 1}, {-1, 1}};
        for (int d = 0; d < 4; d++) {
            int grad = 0;
            for (int x2 = 0; x2 < 2; x2++)
                for (int yy = 0; yy < 2; yy++) {
                    const int dy = offs[d][0], dx = offs[d][1], ry = row_off + yy, x = x1 + x2;
                    const int a = trow(rows, rs, e, r[ry - 1 - dy], x - 1 - dx);
                    const int b = trow(rows, rs, e, r[ry - 1], x - 1);
                    const int cc = trow(rows, rs, e, r[ry - 1 + dy], x - 1 + dx);
                    const int t = b * 2 - a - cc;
                    grad += t < 0 ? -t : t;
                }
            cells[g][c][d] = (uint16_t)grad;
        }
    }
    __syncthreads();
    const int alpha_base = ref_dst_idx * 528 + qp_idx * 88, weight_base = ref_dst_idx * 1584 + qp_idx * 264;
    const int bias_idx = ref_dst_idx * 6 + qp_idx;
    const int scale = ref_dst_idx == 0 ? 8 : 5;
    const int8_t *errtab = ref_dst_idx == 0 ? tab.GDF_INTRA_ERROR + qp_idx * 4096
                                            : tab.GDF_INTER_ERROR + (ref_dst_idx - 1) * 6000 + qp_idx * 1000;
    for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
        const int y = i / w, x = i % w, x1 = x & ~1, hx = x1 >> 1;
        const int k1 = (y >> 1) + 1, k0 = k1 - 1;  // the two gradient rows in use at row y
        int gs[4];
        for (int d = 0; d < 4; d++)
            gs[d] = cells[k0][hx][d] + cells[k0][hx + 1][d] + cells[k1][hx][d] + cells[k1][hx + 1][d];
        const int cls = (gs[0] <= gs[1]) | ((gs[2] <= gs[3]) << 1);
        int iv[3];
        for (int q = 0; q < 3; q++) iv[q] = tab.GDF_BIAS[bias_idx * 3 + q];
        for (int d = 0; d < 4; d++) {
            const int k = d + 18;
            const int v = imin_(gs[d] >> (4 - up), tab.GDF_ALPHA[alpha_base + k * 4 + cls]);
            for (int q = 0; q < 3; q++) iv[q] += v * tab.GDF_WEIGHT[weight_base + q * 88 + k * 4 + cls];
        }
        const int *r = pref + y * 13;
        const int m = trow(rows, rs, e, r[6], x);
        for (int k = 0; k < 18; k++) {
            const int alpha = tab.GDF_ALPHA[alpha_base + k * 4 + cls];
            const int dy = TapsY::gdf[k][0], dx = TapsY::gdf[k][1];
            const int a = trow(rows, rs, e, r[6 - dy], x - dx), b = trow(rows, rs, e, r[6 + dy], x + dx);
            const int above = iclip_((a - m) << up, -alpha, alpha), below = iclip_((b - m) << up, -alpha, alpha);
            const int v = iclip_(above + below, -512, 511);
            for (int q = 0; q < 3; q++) iv[q] += v * tab.GDF_WEIGHT[weight_base + q * 88 + k * 4 + cls];
        }
        int full = 0;
        for (int q = 0; q < 3; q++) {
            const int sv = iv[q] * scale;
            const int v = apply_sign_(((sv < 0 ? -sv : sv) + (1 << 14)) >> 15, sv);
            full = full * (scale * 2) + iclip_(v, -scale, scale - 1) + scale;
        }
        out[i] = errtab[full];
    }
}

// Per device: dynamic shared memory opted in, SM count and CTAs per SM.
struct LrLaunchInfo {
    std::atomic<int> ready{0};
    int sms = 0, occ[3] = {0, 0, 0};
};
LrLaunchInfo g_lr_info[64];

const LrLaunchInfo &lr_info() {
    int dev = 0;
    cudaGetDevice(&dev);
    LrLaunchInfo &li = g_lr_info[dev & 63];
    if (!li.ready.load(std::memory_order_acquire)) {
        const int bytes = (int)sizeof(LrSmem);
        cudaFuncSetAttribute(lr_kernel<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaFuncSetAttribute(lr_kernel<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaFuncSetAttribute(lr_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaDeviceGetAttribute(&li.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&li.occ[0], lr_kernel<uint8_t>, LR_NT, bytes);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&li.occ[1], lr_kernel<uint16_t>, LR_NT, bytes);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&li.occ[2], lr_batch_kernel, LR_NT, bytes);
        for (int &o : li.occ)
            if (o < 1) o = 1;
        li.ready.store(1, std::memory_order_release);
    }
    return li;
}

}  // namespace

void r2g_batch_launch_lr(const BatchArgs &a, int grid, cudaStream_t s) {
    lr_info();
    r2g_launch_pdl_smem(lr_batch_kernel, dim3(grid), dim3(LR_NT), sizeof(LrSmem), s, a);
}
int r2g_batch_occupancy_lr() { return lr_info().occ[2]; }
int r2g_lr_items(const DevFrame &f) {
    const int nslots = f.sbh + 1 + f.n_tr;
    if (!f.lr_on) return 0;
    return nslots * (64 / f.lr_rows) * ((f.w + 63) >> 6) + 2 * nslots * 2 * ((f.cw + 63) >> 6);
}

int r2g_launch_lr(const DevFrame &f, cudaStream_t s) {
    if (!f.lr_on) return 0;
    const LrLaunchInfo &li = lr_info();
    const int n = r2g_lr_items(f);
    const int hbd = f.bitdepth > 8;
    int grid = li.sms * li.occ[hbd];
    if (grid > n) grid = n;
    if (hbd)
        r2g_launch_pdl_smem(lr_kernel<uint16_t>, dim3(grid), dim3(LR_NT), sizeof(LrSmem), s, f, n);
    else
        r2g_launch_pdl_smem(lr_kernel<uint8_t>, dim3(grid), dim3(LR_NT), sizeof(LrSmem), s, f, n);
    return 1;
}

void r2g_dsp_launch_gdf_add(uint16_t *p, const int8_t *err, int w, int h, int scale, const uint16_t *llm, int bitdepth,
                            cudaStream_t s) {
    dsp_gdf_add_kernel<<<1, 256, 0, s>>>(p, err, w, h, scale, llm, bitdepth);
}

void r2g_dsp_launch_wiener_y(const uint16_t *rows, int rs, int e, const int *ref, const int *cref, int w, int h,
                             int kind, const int8_t *taps, int taps_stride, const int16_t *pcf, const uint8_t *sub_lut,
                             const uint16_t *noskip, int base_q, const uint16_t *llm, int bitdepth,
                             const DevTables &tab, uint16_t *out, cudaStream_t s) {
    dsp_wiener_y_kernel<<<1, 256, 0, s>>>(rows, rs, e, ref, cref, w, h, kind, taps, taps_stride, pcf, sub_lut, noskip,
                                          base_q, llm, bitdepth, tab, out);
}
void r2g_dsp_launch_wiener_uv(const uint16_t *crows, int crs, const uint16_t *lrows, int lrs, const int *cref,
                              const int *lref, int w, int h, int ss_hor, const int8_t *f, const uint16_t *llm,
                              int bitdepth, uint16_t *out, cudaStream_t s) {
    dsp_wiener_uv_kernel<<<1, 256, 0, s>>>(crows, crs, lrows, lrs, cref, lref, w, h, ss_hor, f, llm, bitdepth, out);
}
void r2g_dsp_launch_gdf_prep(const uint16_t *rows, int rs, int e, const int *gref, int ng, const int *pref, int w,
                             int h, int ref_dst_idx, int qp_idx, int bitdepth, const DevTables &tab, int8_t *out,
                             cudaStream_t s) {
    dsp_gdf_prep_kernel<<<1, 256, 0, s>>>(rows, rs, e, gref, ng, pref, w, h, ref_dst_idx, qp_idx, bitdepth, tab, out);
}
