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
// Each CTA materialises exactly that window for one (plane, stripe, 64-wide
// unit) in shared memory and evaluates every restoration tap from it.
#include <type_traits>

#include "r2g_common.cuh"

namespace {

enum { LR_HAVE_LEFT = 1, LR_HAVE_RIGHT = 2, LR_HAVE_TOP = 4, LR_HAVE_BOTTOM = 8 };

constexpr int LW = 76;   // luma window width: -6 .. 69
constexpr int LH = 44;   // luma window height: -6 .. 37 (a work item has <= 32 rows)
constexpr int CWW = 68;  // chroma window width: -2 .. 65
constexpr int CWH = 36;  // chroma window height: -2 .. 33 (stripe <= 32 rows)

__constant__ uint16_t c_pcw_norm[4] = {3739, 3273, 3074, 7};
__constant__ int16_t c_mode_weights[4][3] = {{-527, 15325, 321}, {26436, -17705, 17905}, {366, -147, -194}, {202, -267, -179}};
__constant__ int16_t c_mode_offsets[4] = {-547, -21565, -573, -680};

enum { W_NONE = 0, W_NS_SINGLE = 1, W_NS_MULTI = 2, W_PC = 3 };

struct UnitGeom {
    int plane, x0, uw, y0, sh, edges, valid;
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

// Work item -> geometry, following lr_sbrow_apply / lr_sbrow_plane /
// lr_stripe for one tile row (sb128 = 0).  A superblock row's LR call covers
// [y_call, row_h); its first stripe is 56 (luma) rows high on superblock row
// 0 and 64 otherwise, so a call holds one stripe, or two when the frame
// height is a multiple of 64 and this is the last superblock row.
R2G_D void unit_geom(const DevFrame &f, int plane, int sby, int sub, int ux, UnitGeom &g) {
    const int chroma = plane != 0;
    const int ss = chroma;  // 4:2:0: ss_hor = ss_ver = 1 for chroma
    const int W = chroma ? f.cw : f.w, H = chroma ? f.ch : f.h;
    const int not_last = sby + 1 < f.sbh;
    const int next_row_y = (sby + 1) << (6 - ss);
    const int row_h = imin_(next_row_y - (8 >> ss) * not_last, H);
    const int y_call = (sby << (6 - ss)) - ((8 * (sby != 0)) >> ss);
    const int sh0 = imin_((sby == 0 ? 56 : 64) >> ss, row_h - y_call);
    int y0 = y_call, sh = sh0;
    if (sub) {
        y0 = y_call + sh0;
        sh = imin_(64 >> ss, row_h - y0);
    }
    g.plane = plane;
    g.y0 = y0;
    g.sh = sh;
    g.x0 = ux * 64;
    g.uw = imin_(64, W - g.x0);
    g.edges = (y0 > 0 ? LR_HAVE_TOP : 0) | (ux > 0 ? LR_HAVE_LEFT : 0) | (g.x0 + 64 < W ? LR_HAVE_RIGHT : 0) |
              ((not_last || y0 + sh != row_h) ? LR_HAVE_BOTTOM : 0);
    g.sb256x = (g.x0 << ss) >> 8;
    g.sb64x_idx = ((g.x0 << ss) >> 6) & 3;
    // unit selection (looprestoration.rs:2295-2331) from the call's first
    // row; only sby 0 is the first superblock row of the (single) tile row
    const int unit_size = 1 << f.fp.restoration_unit_size[chroma];
    const int half = unit_size >> 1;
    int row_y = y_call + ((8 >> ss) * (sby == 0));
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

R2G_D int col_src(const UnitGeom &g, int c) {
    if (c < 0 && !(g.edges & LR_HAVE_LEFT)) return g.x0;
    if (c >= g.uw && !(g.edges & LR_HAVE_RIGHT)) return g.x0 + g.uw - 1;
    return g.x0 + c;
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

struct LrSmem {
    union {
        // luma: every window position holds the sample and its right
        // neighbour as a signed 16x2 pair, so GDF can work on two adjacent
        // pixels (which share a GDF class) with one 32-bit load per tap;
        // a scalar sample is the low half (16-bit loads at a 4-byte stride)
        uint32_t wp[LH * LW];
        struct {
            int16_t win[CWH * CWW];   // chroma window
            int16_t lwin[CWH * CWW];  // downsampled luma window
        } ch;
    } u;
    uint16_t gcell[17 * 33 * 4];  // GDF 2x2 gradient cells, 4 directions
    int8_t gerr[32 * 64];
    int8_t s_err[4096];
    uint2 s_aa[4][18];   // per class and tap: (alpha, alpha), (-alpha, -alpha) as s16x2
    int4 s_w[4][22];     // per class and tap / feature: weights 0..2, alpha
    int16_t s_pcf[64 * 13];  // PC-Wiener filters of this frame's wiener_idx
    uint8_t classes[8][16];
    uint16_t noskip[18];
    uint16_t llm[17];
};

// Sign-extended low / high halves of a 16x2 pair.
R2G_D int lo16(uint32_t v) { return (int)(int16_t)(v & 0xffff); }
R2G_D int hi16(uint32_t v) { return (int)v >> 16; }

// One (plane, stripe, 64-wide unit) work item; b is the per-frame item index:
// luma items first (stripe slot, row part, unit), then U, then V (stripe
// slot, unit).  Slots 0 .. sbh-1 are the superblock rows' first stripes;
// slot sbh is the second stripe that only the last superblock row can have.
// A luma stripe is split into parts of f.lr_rows rows (32: two halves, or
// 16: four quarters; separate CTAs) so that a frame gives more, lighter work
// items.
template <typename P, int NT>
R2G_D void lr_unit(const DevFrame &f, LrSmem &sm, int b) {
    constexpr int NW = NT / 32;  // warps of the CTA
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nux_l = (f.w + 63) >> 6, nux_c = (f.cw + 63) >> 6;
    const int nparts = 64 / f.lr_rows;
    const int n_luma_units = (f.sbh + 1) * nparts * nux_l;
    int plane, sby, sub, ux, part = 0;
    if (b < n_luma_units) {
        plane = 0;
        ux = b % nux_l;
        b /= nux_l;
        part = b % nparts;
        b /= nparts;
    } else {
        b -= n_luma_units;
        const int per = (f.sbh + 1) * nux_c;
        plane = 1 + b / per;
        b %= per;
        ux = b % nux_c;
        b /= nux_c;
    }
    sub = b >= f.sbh;
    sby = sub ? f.sbh - 1 : b;
    UnitGeom g;
    unit_geom(f, plane, sby, sub, ux, g);
    if (g.sh <= 0) return;
    const int chroma = plane != 0;
    // rows [ro, ro + nr) of the stripe are this item's output rows (luma: one
    // part of f.lr_rows rows; chroma: the whole stripe)
    const int ro = part * f.lr_rows, nr = chroma ? g.sh : imin_(f.lr_rows, g.sh - ro);
    if (nr <= 0) return;
    const int64_t stride = f.stride[chroma];
    const P *Cp = plane_ptr<const P>(f.C[plane]);
    const P *Dp = plane_ptr<const P>(f.D[plane]);
    P *Lp = plane_ptr<P>(f.L[plane]);
    const R2gFrameParams &fp = f.fp;
    const int bitdepth = f.bitdepth, bdmax = f.bdmax;

    // ---- kernel selection (looprestoration.rs:1880-1920) ----
    int wkind = W_NONE;
    bool plane_on = (f.restore_planes >> plane) & 1;
    if (plane_on && g.valid) {
        int wt = (f.inloop & R2G_INLOOP_WIENER) ? g.unit->type : 0;
        const R2gRestorationPlane &pd = fp.restoration[plane];
        if (wt == R2G_RESTORE_NS_WIENER)
            wkind = (pd.frame_filters_on && pd.num_classes != 1) ? W_NS_MULTI : W_NS_SINGLE;
        else if (wt == R2G_RESTORE_PC_WIENER)
            wkind = W_PC;
    }
    const int inc = ((g.edges & LR_HAVE_TOP) && g.y0 + 8 < ((f.bh4 * 4) >> chroma)) ? 8 : 0;
    const int sb256_idx = f.sb256w * (((g.y0 << chroma) + inc) >> 8) + g.sb256x;
    const int nsb = f.sb256w * f.sb256h;
    const bool gdf_on = plane_on && g.valid && plane == 0 && (f.inloop & R2G_INLOOP_GDF) && sb256_idx < nsb &&
                        f.masks[sb256_idx].gdf[(((g.y0 + inc) >> 4) & 12) + g.sb64x_idx] != 0;

    // ---- lossless rows of the stripe (looprestoration.rs:2037-2075) ----
    const int ll_rows = imax_(g.sh >> 2, 1) + 1;
    if (tid < 17) {
        uint16_t v = 0;
        if (tid < ll_rows && sb256_idx < nsb) {
            const R2gAv2Filter &m = f.masks[sb256_idx];
            int y4 = ((g.y0 << chroma) & 255) >> 2;
            if (plane == 0) {
                int yy = y4 + tid;
                if (yy < 64) v = m.lossless_mask_y[yy][g.sb64x_idx];
            } else {
                int init_y = g.y0 >> 2, end_y = (g.y0 + g.sh) >> 2;
                int base = y4 >> 1;
                if (init_y + tid < end_y) {
                    int sy = base + tid;
                    if (sy < 64) {
                        uint16_t lo = m.lossless_mask_uv[sy][g.sb64x_idx];
                        uint16_t hi = g.sb64x_idx + 1 < 4 ? m.lossless_mask_uv[sy][g.sb64x_idx + 1] : 0;
                        v = (uint16_t)((lo & 0xff) | ((hi & 0xff) << 8));
                    }
                }
            }
        }
        sm.llm[tid] = v;
    }
    // ---- multi-class noskip rows (looprestoration.rs:1922-1944) ----
    if ((wkind == W_NS_MULTI || wkind == W_PC) && tid < 18) {
        uint16_t v = 0;
        int by = (g.y0 >> 2) + tid;
        if (by < ((g.y0 + g.sh) >> 2)) {
            int sidx = f.sb256w * (by >> 6) + g.sb256x;
            if (sidx < nsb) {
                v = f.masks[sidx].lr_noskip_mask[by & 63][g.sb64x_idx];
                if (!(g.edges & LR_HAVE_RIGHT) && (g.uw & 63) != 0) {
                    int sh = ((g.uw >> 2) & 15) - 1;
                    uint16_t eb = (uint16_t)(v >> sh);
                    v = (uint16_t)(v | (uint16_t)(eb << (sh + 1)));
                }
            }
        }
        sm.noskip[tid] = v;
    }
    // GDF and PC-Wiener parameters of the frame (tables only)
    if (gdf_on && !chroma) {
        const int ref_dst_idx = f.gdf_ref_dst_idx, qp_idx = fp.gdf_qp_idx;
        const int alpha_base = ref_dst_idx * 528 + qp_idx * 88;
        const int weight_base = ref_dst_idx * 1584 + qp_idx * 264;
        const int8_t *errtab = ref_dst_idx == 0 ? f.tab.GDF_INTRA_ERROR + qp_idx * 4096
                                                : f.tab.GDF_INTER_ERROR + (ref_dst_idx - 1) * 6000 + qp_idx * 1000;
        const int nerr = ref_dst_idx == 0 ? 4096 : 1000;
        for (int i = tid; i < 88; i += NT) {
            int k = i >> 2, c = i & 3;
            const int a = f.tab.GDF_ALPHA[alpha_base + i];
            sm.s_w[c][k] = make_int4(f.tab.GDF_WEIGHT[weight_base + 0 * 88 + i],
                                     f.tab.GDF_WEIGHT[weight_base + 1 * 88 + i],
                                     f.tab.GDF_WEIGHT[weight_base + 2 * 88 + i], a);
            if (k < 18) {
                const uint32_t pa = (uint32_t)a & 0xffff, na = (uint32_t)(-a) & 0xffff;
                sm.s_aa[c][k] = make_uint2(pa | (pa << 16), na | (na << 16));
            }
        }
        for (int i = tid; i < nerr; i += NT) sm.s_err[i] = errtab[i];
    }
    if (wkind == W_PC)
        for (int i = tid; i < 64 * 13; i += NT) sm.s_pcf[i] = f.tab.PC_WIENER_FILTERS[f.wiener_idx * 64 * 13 + i];
    // C and D come from the previous kernels on the stream: wait for them
    // (everything above reads side-info and tables only; a CTA that only
    // copies has staged a few unused rows and parameters)
    pdl_wait();
    if (wkind == W_NONE && !gdf_on) {
        // unfiltered unit: copy C -> L in 4-byte words (unit widths are
        // multiples of 4 samples; rows and unit origins are 64-byte aligned)
        const int wpr = g.uw * (int)sizeof(P) / 4;
        for (int i = tid; i < nr * wpr; i += NT) {
            const int r = ro + i / wpr, q = i % wpr;
            const int64_t o = (int64_t)(g.y0 + r) * stride + g.x0;
            reinterpret_cast<uint32_t *>(Lp + o)[q] = __ldg(reinterpret_cast<const uint32_t *>(Cp + o) + q);
        }
        return;
    }


    if (chroma) {
        // ---- chroma window: rows -2 .. sh+1, columns -2 .. uw+1 ----
        const int wh = g.sh + 4, ww = g.uw + 4;
        for (int r = warp; r < wh; r += NW) {
            int row;
            bool from_d;
            row_src(g, r - 2, row, from_d);
            const P *src = (from_d ? Dp : Cp) + (int64_t)row * stride;
            for (int c = lane; c < ww; c += 32) sm.u.ch.win[r * CWW + c] = (int16_t)src[col_src(g, c - 2)];
        }
        if (wkind == W_NS_SINGLE) {
            // downsampled luma for chroma rows -2 .. sh+1 at chroma columns
            // -2 .. uw+1 (backup_row_luma with the ns_wiener_single_uv row
            // selection, looprestoration.rs:1207-1350)
            const P *Cy = plane_ptr<const P>(f.C[0]);
            const P *Dy = plane_ptr<const P>(f.D[0]);
            const int64_t ls = f.stride[0];
            const int ds = fp.cfl_ds_filter_index;
            const int lw = g.uw << 1, lx0 = g.x0 << 1;
            for (int r = warp; r < wh; r += NW) {
                int rr = r - 2;
                if (!(g.edges & LR_HAVE_TOP) && rr < 0) rr = 0;
                if (!(g.edges & LR_HAVE_BOTTOM) && rr >= g.sh) rr = g.sh - 1;
                const P *src;
                int ra, rb;
                if (rr == -2) {
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
                const P *rowa = src + (int64_t)ra * ls + lx0;
                const P *rowb = src + (int64_t)rb * ls + lx0;
                for (int j = lane; j < ww; j += 32) {
                    int pos = 2 * (j - 2);
                    if (pos < 0 && !(g.edges & LR_HAVE_LEFT)) pos = 0;
                    if (pos >= lw && !(g.edges & LR_HAVE_RIGHT)) pos = lw - 2;
                    int v;
                    if (ds == 0)
                        v = ((int)rowa[pos] + rowb[pos] + rowa[pos + 1] + rowb[pos + 1]) >> 2;
                    else if (ds == 1)
                        v = ((int)rowa[pos] + rowb[pos]) >> 1;
                    else
                        v = rowa[pos];
                    sm.u.ch.lwin[r * CWW + j] = (int16_t)v;
                }
            }
        }
        __syncthreads();
        // ---- chroma NS-Wiener with cross-component luma taps (:1145-1430) ----
        int8_t flt[18];
        if (wkind == W_NS_SINGLE) {
            const int8_t *src = fp.restoration[plane].frame_filters_on ? fp.restoration[plane].filter[0]
                                                                       : g.unit->f;
#pragma unroll
            for (int k = 0; k < 18; k++) flt[k] = src[k];
        }
        for (int y = warp; y < g.sh; y += NW)
            for (int x = lane; x < g.uw; x += 32) {
                const int16_t *w = &sm.u.ch.win[(y + 2) * CWW + x + 2];
                const int16_t *lw_ = &sm.u.ch.lwin[(y + 2) * CWW + x + 2];
                int m = w[0];
                int v = m;
                bool ll = (sm.llm[y >> 2] >> (x >> 2)) & 1;
                if (!ll && wkind == W_NS_SINGLE) {
                    int s = m << 7;
#pragma unroll
                    for (int k = 0; k < 6; k++) {
                        const int o = TapsY::uv[k][0] * CWW + TapsY::uv[k][1];
                        s += (w[o] + w[-o] - 2 * m) * flt[k];
                    }
                    int l = lw_[0];
#pragma unroll
                    for (int k = 0; k < 12; k++) {
                        const int o = TapsY::uvy[k][0] * CWW + TapsY::uvy[k][1];
                        s += (lw_[o] - l) * flt[6 + k];
                    }
                    v = clip_px_((s + 64) >> 7, bdmax);
                }
                Lp[(int64_t)(g.y0 + y) * stride + g.x0 + x] = (P)v;
            }
        return;
    }

    // ---- luma window: rows ro-6 .. ro+nr+5 of the stripe, columns -6 .. uw+5 ----
    const int wh = nr + 12, ww = g.uw + 12;
    if ((g.edges & LR_HAVE_LEFT) && (g.edges & LR_HAVE_RIGHT) && g.uw == 64) {
        // interior unit: window columns are source columns x0-6 .. x0+69, all
        // inside the frame.  Read them as 2-sample words U_j (samples
        // x0-6+2j, x0-5+2j): pair 2j is U_j, pair 2j+1 joins U_j's second
        // sample with U_{j+1}'s first.  Each thread issues four words' loads
        // before storing any pair.
        typedef typename std::conditional<sizeof(P) == 2, uint32_t, uint16_t>::type U;
        constexpr int NJ = 38, SH = 8 * (int)sizeof(P);
        constexpr uint32_t MK = (1u << SH) - 1;
        const int total = wh * NJ;
        for (int base = 0; base < total; base += 4 * NT) {
            uint32_t a[4], nb[4];
            int dst[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = base + q * NT + tid;
                dst[q] = -1;
                a[q] = nb[q] = 0;
                if (i < total) {
                    const int r = i / NJ, j = i - r * NJ;
                    int row;
                    bool from_d;
                    row_src(g, ro + r - 6, row, from_d);
                    const U *src = reinterpret_cast<const U *>((from_d ? Dp : Cp) + (int64_t)row * stride + g.x0 - 6);
                    a[q] = __ldg(src + j);
                    nb[q] = __ldg(src + j + 1);
                    dst[q] = r * LW + 2 * j;
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (dst[q] >= 0) {
                    const uint32_t s0 = a[q] & MK, s1 = a[q] >> SH, t0 = nb[q] & MK;
                    sm.u.wp[dst[q]] = s0 | (s1 << 16);
                    sm.u.wp[dst[q] + 1] = s1 | (t0 << 16);
                }
        }
    } else {
        // source columns of this lane's window columns (the same on every row)
        int cs0[3], cs1[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int c = lane + 32 * j;
            cs0[j] = col_src(g, c - 6);
            cs1[j] = c + 1 < ww ? col_src(g, c - 5) : cs0[j];
        }
        for (int r = warp; r < wh; r += NW) {
            int row;
            bool from_d;
            row_src(g, ro + r - 6, row, from_d);
            const P *src = (from_d ? Dp : Cp) + (int64_t)row * stride;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int c = lane + 32 * j;
                if (c < ww) sm.u.wp[r * LW + c] = (uint32_t)src[cs0[j]] | ((uint32_t)src[cs1[j]] << 16);
            }
        }
    }
    const int16_t *W16 = reinterpret_cast<const int16_t *>(sm.u.wp);  // scalar sample i at W16[2 * i]
    __syncthreads();

    const int b8 = bitdepth - 8;
    const int bh4 = nr >> 2, bw4 = g.uw >> 2, sbh4 = g.sh >> 2;
    // ---- GDF prep (looprestoration.rs:1432-1640) ----
    if (gdf_on) {
        // GDF works in a 10-bit domain (looprestoration.rs:1450-1453): 8-bit
        // samples shift up by 2; 12-bit (not accepted at the boundary) would
        // shift down by 2.
        constexpr int down = 0, up = sizeof(P) == 1 ? 2 : 0;
        // gradient cell (j, i): rows 2j-1, 2j; columns 2i-1, 2i
        // (compute_gradient_row :114-193); pair (y1, x1) sums cells
        // (y1/2 .. y1/2+1, x1/2 .. x1/2+1)
        const int cj = (nr >> 1) + 1, ci = (g.uw >> 1) + 1;
        for (int i = tid; i < cj * ci; i += NT) {
            int j = i / ci, c = i % ci;
            int gs[4] = {0, 0, 0, 0};
#pragma unroll
            for (int yy = 0; yy < 2; yy++)
#pragma unroll
                for (int xx = 0; xx < 2; xx++) {
                    const int16_t *w = &W16[2 * ((2 * j - 1 + yy + 6) * LW + 2 * c - 1 + xx + 6)];
                    constexpr int R = 2 * LW, C1 = 2;
                    int bv = w[0] >> down;
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
#pragma unroll
            for (int d = 0; d < 4; d++) sm.gcell[i * 4 + d] = (uint16_t)gs[d];
        }
        __syncthreads();
        const int ref_dst_idx = f.gdf_ref_dst_idx;
        const int bias_idx = ref_dst_idx * 6 + fp.gdf_qp_idx;
        const int scale = ref_dst_idx == 0 ? 8 : 5;
        const int b0 = f.tab.GDF_BIAS[bias_idx * 3], b1 = f.tab.GDF_BIAS[bias_idx * 3 + 1],
                  b2 = f.tab.GDF_BIAS[bias_idx * 3 + 2];
        const int npairs = nr * (g.uw >> 1);
        for (int i = tid; i < npairs; i += NT) {
            int y = i / (g.uw >> 1), x1 = (i % (g.uw >> 1)) * 2;
            int j = y >> 1, c = x1 >> 1;
            int gsum[4];
#pragma unroll
            for (int d = 0; d < 4; d++)
                gsum[d] = sm.gcell[(j * ci + c) * 4 + d] + sm.gcell[(j * ci + c + 1) * 4 + d] +
                          sm.gcell[((j + 1) * ci + c) * 4 + d] + sm.gcell[((j + 1) * ci + c + 1) * 4 + d];
            int cls = (gsum[0] <= gsum[1]) | ((gsum[2] <= gsum[3]) << 1);
            const int4 *wt = sm.s_w[cls];
            const uint2 *aa = sm.s_aa[cls];
            int sh0 = b0, sh1 = b1, sh2 = b2;
#pragma unroll
            for (int d = 0; d < 4; d++) {
                int4 p = wt[18 + d];
                int v = imin_(gsum[d] >> (4 - up), p.w);
                sh0 += v * p.x;
                sh1 += v * p.y;
                sh2 += v * p.z;
            }
            // the 18 clipped symmetric differences of both pixels at once,
            // as signed 16x2 pairs: (pixel x, pixel x + 1)
            const uint32_t *wc = &sm.u.wp[(y + 6) * LW + x1 + 6];
            const uint32_t mm = wc[0] << up;  // samples < 2^10: no carry between halves
            const uint32_t nm = __vneg2(mm);
            int i0 = sh0, i1 = sh1, i2 = sh2, j0 = sh0, j1 = sh1, j2 = sh2;
#pragma unroll
            for (int k = 0; k < 18; k++) {
                const int o = TapsY::gdf[k][0] * LW + TapsY::gdf[k][1];
                const uint2 al = aa[k];
                const int4 p = wt[k];
                // (min as the fused add-min with 0: one instruction, where a
                // plain packed min is slower on this part)
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
#pragma unroll
            for (int x2 = 0; x2 < 2; x2++) {
                const int iv[3] = {x2 ? j0 : i0, x2 ? j1 : i1, x2 ? j2 : i2};
                int full = 0;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    int sv = iv[q] * scale;
                    int asv = sv < 0 ? -sv : sv;
                    int v = apply_sign_((asv + (1 << 14)) >> 15, sv);
                    int subi = iclip_(v, -scale, scale - 1) + scale;
                    full = full * (scale * 2) + subi;
                }
                sm.gerr[y * 64 + x1 + x2] = sm.s_err[full];
            }
        }
    }
    // ---- classification for PC-Wiener / NS-multi (:195-271, :870-896) ----
    if (wkind == W_NS_MULTI || wkind == W_PC) {
        const uint8_t *sub_lut = wkind == W_PC
                                     ? f.tab.PC_WIENER_SUB_CLASSIFY + f.wiener_idx * 256
                                     : f.tab.PC_WIENER_SUB_CLASSIFY_NS +
                                           (f.wiener_idx * 7 + (f.ns_ci >= 0 ? imin_(f.ns_ci, 6) : 0)) * 256;
        for (int i = tid; i < bh4 * bw4; i += NT) {
            int by = i / bw4, bx = i % bw4;
            int fs0 = 0, fs1 = 0, fs2 = 0;
#pragma unroll
            for (int dy = -1; dy <= 4; dy++)
#pragma unroll
                for (int dx = -1; dx <= 4; dx++) {
                    const int16_t *w = &W16[2 * ((by * 4 + dy + 6) * LW + bx * 4 + dx + 6)];
                    constexpr int R = 2 * LW, C1 = 2;
                    int m2 = 2 * w[0];
                    int vert = w[-R] - m2 + w[R];
                    int anti = w[-R + C1] - m2 + w[R - C1];
                    int diag = w[-R - C1] - m2 + w[R + C1];
                    fs0 += vert < 0 ? -vert : vert;
                    fs1 += anti < 0 ? -anti : anti;
                    fs2 += diag < 0 ? -diag : diag;
                }
            int s = 0;
            const int np[3] = {16, 4, 1};
#pragma unroll
            for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    int e = (dy != 0) + (dx != 0);
                    int fx = iclip_((bx & 15) + dx, 0, 15);
                    int fy = iclip_((ro >> 2) + by + dy, 0, sbh4 - 1);
                    s += np[e] * (((sm.noskip[fy] >> fx) & 1) == 0);
                }
            int rnd = (1 << b8) >> 1;
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
            sm.classes[by][bx] = sub_lut[f.tab.PC_WIENER_LUT_TO_CLASS[lut_idx]];
        }
    }
    __syncthreads();
    // ---- Wiener FIR + GDF add, one output sample per iteration ----
    int8_t single[16];
    if (wkind == W_NS_SINGLE) {
        const int8_t *src = fp.restoration[0].frame_filters_on ? fp.restoration[0].filter[0] : g.unit->f;
#pragma unroll
        for (int k = 0; k < 16; k++) single[k] = src[k];
    }
    const int gshift = 12 - bitdepth, grnd = (1 << gshift) >> 1, gscale = fp.gdf_scale;
    for (int y = warp; y < nr; y += NW)
        for (int x = lane; x < g.uw; x += 32) {
            const int16_t *w = &W16[2 * ((y + 6) * LW + x + 6)];
            int m = w[0];
            int v = m;
            bool ll = (sm.llm[(ro + y) >> 2] >> (x >> 2)) & 1;
            if (!ll && wkind != W_NONE) {
                int s;
                if (wkind == W_PC) {
                    const int16_t *flt = sm.s_pcf + sm.classes[y >> 2][x >> 2] * 13;
                    s = m * flt[12];
#pragma unroll
                    for (int k = 0; k < 12; k++) {
                        const int o = 2 * (TapsY::pc[k][0] * LW + TapsY::pc[k][1]);
                        s += (w[o] + w[-o]) * flt[k];
                    }
                } else {
                    const int8_t *flt =
                        wkind == W_NS_SINGLE ? single : fp.restoration[0].filter[sm.classes[y >> 2][x >> 2]];
                    s = m << 7;
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const int o = 2 * (TapsY::ns[k][0] * LW + TapsY::ns[k][1]);
                        s += (w[o] + w[-o] - 2 * m) * flt[k];
                    }
                }
                v = clip_px_((s + 64) >> 7, bdmax);
            }
            if (gdf_on && !ll) {
                int diff = sm.gerr[y * 64 + x] * gscale;
                int ad = diff < 0 ? -diff : diff;
                v = clip_px_(v + apply_sign_((ad + grnd) >> gshift, diff), bdmax);
            }
            Lp[(int64_t)(g.y0 + ro + y) * stride + g.x0 + x] = (P)v;
        }
}

// Per-frame kernel: one CTA per work item (the hardware hands items to SMs
// as CTAs finish, which balances light and heavy items).
constexpr int LR_FRAME_NT = 256;
template <typename P>
__global__ void __launch_bounds__(LR_FRAME_NT, 4) lr_kernel(const DevFrame f) {
    pdl_trigger();
    __shared__ LrSmem sm;
    lr_unit<P, LR_FRAME_NT>(f, sm, blockIdx.x);
}

// Persistent kernel over a cross-frame work list: item = frame << 22 |
// per-frame item index.
// (one call per sample type, kept out of line so the two instantiations do
// not share one register allocation)
__device__ __noinline__ void lr_unit_hbd(const DevFrame &f, LrSmem &sm, int b) { lr_unit<uint16_t, 256>(f, sm, b); }
__device__ __noinline__ void lr_unit_8(const DevFrame &f, LrSmem &sm, int b) { lr_unit<uint8_t, 256>(f, sm, b); }

__global__ void __launch_bounds__(256, 4) lr_batch_kernel(BatchArgs a) {
    pdl_trigger();
    __shared__ LrSmem sm;
    const int n = a.count[2];
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const uint32_t it = a.work[2][w];
        const DevFrame &f = a.frames[it >> 22];
        if (f.bitdepth > 8)
            lr_unit_hbd(f, sm, it & 0x3fffff);
        else
            lr_unit_8(f, sm, it & 0x3fffff);
        __syncthreads();
    }
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

}  // namespace

void r2g_batch_launch_lr(const BatchArgs &a, int grid, cudaStream_t s) {
    r2g_launch_pdl(lr_batch_kernel, dim3(grid), dim3(256), s, a);
}
int r2g_batch_occupancy_lr() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, lr_batch_kernel, 256, 0);
    return nb;
}
int r2g_lr_items(const DevFrame &f) {
    if (!f.lr_on) return 0;
    return (f.sbh + 1) * (64 / f.lr_rows) * ((f.w + 63) >> 6) + 2 * (f.sbh + 1) * ((f.cw + 63) >> 6);
}

int r2g_launch_lr(const DevFrame &f, cudaStream_t s) {
    if (!f.lr_on) return 0;
    int n = r2g_lr_items(f);
    if (f.bitdepth > 8)
        r2g_launch_pdl(lr_kernel<uint16_t>, dim3(n), dim3(LR_FRAME_NT), s, f);
    else
        r2g_launch_pdl(lr_kernel<uint8_t>, dim3(n), dim3(LR_FRAME_NT), s, f);
    return 1;
}

void r2g_dsp_launch_gdf_add(uint16_t *p, const int8_t *err, int w, int h, int scale, const uint16_t *llm, int bitdepth,
                            cudaStream_t s) {
    dsp_gdf_add_kernel<<<1, 256, 0, s>>>(p, err, w, h, scale, llm, bitdepth);
}
