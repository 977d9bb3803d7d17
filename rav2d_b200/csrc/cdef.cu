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
// One CTA covers one 64x8 luma band of a 64-wide superblock column plus the
// co-located 32x4 chroma bands.  The band and a 2-sample halo are staged in
// shared memory (coordinates clamped to the frame, which is CCSO's padding;
// CDEF substitutes INT16_MIN for taps outside the frame, its padding).
//   phase 1: warp w runs the direction search of 8x8 block w: per-direction
//            partial sums in shared memory, the 8 costs on lanes 0..7 and a
//            shuffle argmax (first maximum wins, as in the reference);
//   phase 2: every thread filters two luma samples of one row and one chroma
//            sample, adds the CCSO offset and stores row-contiguous.
#include "r2g_common.cuh"

namespace {

constexpr int TW = 68;  // luma tile width  (-2 .. 65)
constexpr int TH = 12;  // luma tile height (-2 .. 9)
constexpr int CW = 36;  // chroma tile width (-2 .. 33)
constexpr int CH = 8;   // chroma tile height (-2 .. 5)

__constant__ int8_t c_ccso_pos[7][2] = {{-1, 0}, {0, -1}, {-1, -1}, {-1, 1}, {-1, -2}, {1, -2}, {0, 2}};
__constant__ uint8_t c_uv_dirs[8] = {0, 1, 2, 3, 4, 5, 6, 7};
__constant__ uint32_t c_div_table[7] = {840, 420, 280, 210, 168, 140, 120};

struct BlockParams {
    int active;   // any CDEF filtering of this 8x8 (luma or chroma)
    int y_pri, y_sec, y_dir, y_on;
    int uv_pri, uv_sec, uv_dir, uv_on;
    int yoff[6], uvoff[6];  // tap offsets in the luma / chroma padded tiles
};

R2G_D int constrain(int diff, int threshold, int shift) {
    int adiff = diff < 0 ? -diff : diff;
    return apply_sign_(imin_(adiff, imax_(0, threshold - (adiff >> shift))), diff);
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

template <typename P>
R2G_D int load_px(const P *p) {
    return (int)*p;
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
                mn = imin_(imin_(p0, p1), mn);
                mx = imax_(imax_(p0, p1), mx);
                int s0 = t[off[2 + k]], s1 = t[-off[2 + k]], s2 = t[off[4 + k]], s3 = t[-off[4 + k]];
                int st = 2 - k;
                sum += st * (constrain(s0 - px, sec, sec_shift) + constrain(s1 - px, sec, sec_shift) +
                             constrain(s2 - px, sec, sec_shift) + constrain(s3 - px, sec, sec_shift));
                mn = imin_(imin_(imin_(s0, s1), imin_(s2, s3)), mn);
                mx = imax_(imax_(imax_(s0, s1), imax_(s2, s3)), mx);
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

// Linear tap offsets of direction `dir` in a tile of row pitch `pitch`.
R2G_D void tap_offsets(const int8_t *dirs, int dir, int pitch, int *off) {
    const int which[3] = {dir + 2, dir + 4, dir};
#pragma unroll
    for (int w = 0; w < 3; w++)
#pragma unroll
        for (int k = 0; k < 2; k++) {
            int dy, dx;
            dir_off(dirs[which[w] * 2 + k], dy, dx);
            off[w * 2 + k] = dy * pitch + dx;
        }
}

// ccso_score (ccso.rs:16-24)
R2G_D uint32_t ccso_score(int diff, int q, uint32_t clf) {
    if (diff > q && clf == 0) return 2;
    if (diff < -q) return 0;
    return 1;
}

struct CdefSmem {
    int16_t ty[TH][TW];   // clamped to the frame (CCSO padding)
    int16_t tc[2][CH][CW];
    int16_t pty[TH][TW];  // INT16_MIN outside the frame (CDEF padding)
    int16_t ptc[2][CH][CW];
    int bins[8][96];
    BlockParams bp[8];
    int s_ccso[3];
};

// One 64x8 band of superblock column sbx (the work of one CTA); shared by
// the per-frame kernel and the batched persistent kernel.
template <typename P>
R2G_D void cdef_band(const DevFrame &f, CdefSmem &sm, int sbx, int band) {
    auto &ty = sm.ty;
    auto &tc = sm.tc;
    auto &pty = sm.pty;
    auto &ptc = sm.ptc;
    auto &bins = sm.bins;
    auto &bp = sm.bp;
    auto &s_ccso = sm.s_ccso;
    const int gx0 = sbx * 64, gy0 = band * 8;
    const int cx0 = gx0 >> 1, cy0 = gy0 >> 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int bd8 = f.bitdepth - 8;
    const P *Dy = plane_ptr<const P>(f.D[0]);
    const P *Du = plane_ptr<const P>(f.D[1]);
    const P *Dv = plane_ptr<const P>(f.D[2]);
    const int64_t ys = f.stride[0], uvs = f.stride[1];

    // ---- stage the band (clamped coordinates) ----
    for (int r = warp; r < TH; r += 8) {
        const int ry = gy0 - 2 + r, gy = iclip_(ry, 0, f.h - 1);
        const P *row = Dy + gy * ys;
        for (int c = lane; c < TW; c += 32) {
            int rx = gx0 - 2 + c;
            int16_t v = (int16_t)row[iclip_(rx, 0, f.w - 1)];
            ty[r][c] = v;
            pty[r][c] = (ry < 0 || ry >= f.h || rx < 0 || rx >= f.w) ? (int16_t)INT16_MIN : v;
        }
    }
    for (int rr = warp; rr < 2 * CH; rr += 8) {
        const int pl = rr / CH, r = rr % CH;
        const int ry = cy0 - 2 + r, gy = iclip_(ry, 0, f.ch - 1);
        const P *row = (pl ? Dv : Du) + gy * uvs;
        for (int c = lane; c < CW; c += 32) {
            int rx = cx0 - 2 + c;
            int16_t v = (int16_t)row[iclip_(rx, 0, f.cw - 1)];
            tc[pl][r][c] = v;
            ptc[pl][r][c] = (ry < 0 || ry >= f.ch || rx < 0 || rx >= f.cw) ? (int16_t)INT16_MIN : v;
        }
    }
    for (int i = tid; i < 8 * 96; i += 256) (&bins[0][0])[i] = 0;

    // ---- superblock parameters (cdef.rs:787-907) ----
    const int sb256x = sbx >> 2, sb64x_idx = sbx & 3;
    const int by = band * 2;  // 4x4 row of the band
    const int by_idx = (by & 0x3e) >> 1;
    const R2gAv2Filter &m = f.masks[(by >> 6) * f.sb256w + sb256x];
    const R2gFrameParams &fp = f.fp;
    if (tid < 3) s_ccso[tid] = f.ccso_on ? m.ccso[tid] : 0;
    const int cdef_idx = m.cdef_idx[((by & 0x30) >> 2) + (sbx & 3)];
    const int sidx = cdef_idx < 0 ? 0 : cdef_idx;
    const bool cdef_active = !(cdef_idx == -1 || !f.cdef_on ||
                               ((sidx < 8 ? fp.cdef_y_strength[sidx] : 0) == 0 &&
                                (sidx < 8 ? fp.cdef_uv_strength[sidx] : 0) == 0));
    const int damping = fp.cdef_damping + bd8;
    __syncthreads();

    // ---- phase 1: per-8x8 decisions and direction search (warp = block) ----
    {
        const int bx = sbx * 16 + warp * 2;  // 4x4 column of this 8x8
        BlockParams p = {};
        bool in_frame = bx < f.bw4;
        bool need_dir = false;
        if (cdef_active && in_frame) {
            uint16_t noskip = fp.cdef_on_skiptx ? 0xffff : m.noskip_mask[by_idx][sb64x_idx];
            uint16_t y_ll0 = 0, y_ll1 = 0, uv_ll = 0;
            if (f.any_lossless) {
                int yr = imin_(2 * by_idx, 63);
                y_ll0 = m.lossless_mask_y[yr][sb64x_idx];
                y_ll1 = m.lossless_mask_y[imin_(yr + 1, 63)][sb64x_idx];
                uv_ll = m.lossless_mask_uv[imin_(by_idx, 63)][sb64x_idx];
            }
            uint16_t bx_mask = (uint16_t)(3u << (bx & 14));
            bool y_lossless = ((y_ll0 | y_ll1) & bx_mask) != 0;
            bool uv_lossless = (uv_ll & (uint16_t)(1u << ((bx & 14) >> 1))) != 0;
            if ((noskip & bx_mask) != 0 && !(y_lossless && uv_lossless)) {
                int y_lvl = fp.cdef_y_strength[cdef_idx], uv_lvl = fp.cdef_uv_strength[cdef_idx];
                int y_pri = (y_lvl >> 2) << bd8;
                int y_sec = y_lvl & 3;
                y_sec += y_sec == 3;
                y_sec <<= bd8;
                int uv_pri = (uv_lvl >> 2) << bd8;
                int uv_sec = uv_lvl & 3;
                uv_sec += uv_sec == 3;
                uv_sec <<= bd8;
                p.active = 1;
                p.y_pri = y_pri;
                p.y_sec = y_sec;
                p.uv_pri = uv_pri;
                p.uv_sec = uv_sec;
                p.y_on = !y_lossless;
                p.uv_on = uv_lvl != 0 && !uv_lossless;
                need_dir = y_pri != 0 || uv_pri != 0;
            }
        }
        int dir = 0;
        uint32_t var = 0;
        if (need_dir) {
            // cdef_find_dir_bd (cdef.rs:134-224): lane handles 2 samples
            int *b = bins[warp];
            int ly = lane >> 2, lx0 = (lane & 3) * 2;
#pragma unroll
            for (int k = 0; k < 2; k++) {
                int x = lx0 + k, y = ly;
                int px = ((int)ty[2 + y][2 + warp * 8 + x] >> bd8) - 128;
                atomicAdd(&b[0 + (y + x)], px);            // diag0[15]
                atomicAdd(&b[15 + (y + (x >> 1))], px);    // alt0[11]
                atomicAdd(&b[26 + y], px);                 // hv0[8]
                atomicAdd(&b[34 + (3 + y - (x >> 1))], px);  // alt1[11]
                atomicAdd(&b[45 + (7 + y - x)], px);       // diag1[15]
                atomicAdd(&b[60 + (3 - (y >> 1) + x)], px);  // alt2[11]
                atomicAdd(&b[71 + x], px);                 // hv1[8]
                atomicAdd(&b[79 + ((y >> 1) + x)], px);    // alt3[11]
            }
            __syncwarp();
            uint32_t cost = 0;
            if (lane < 8) {
                auto sq = [](int v) -> uint32_t { return (uint32_t)v * (uint32_t)v; };
                if (lane == 2 || lane == 6) {
                    const int *hv = b + (lane == 2 ? 26 : 71);
                    for (int n = 0; n < 8; n++) cost += sq(hv[n]);
                    cost *= 105u;
                } else if (lane == 0 || lane == 4) {
                    const int *dg = b + (lane == 0 ? 0 : 45);
                    for (int n = 0; n < 7; n++) cost += (sq(dg[n]) + sq(dg[14 - n])) * c_div_table[n];
                    cost += sq(dg[7]) * 105u;
                } else {
                    const int alt_base[4] = {15, 34, 60, 79};
                    const int *al = b + alt_base[lane >> 1];
                    for (int mm = 0; mm < 5; mm++) cost += sq(al[3 + mm]);
                    cost *= 105u;
                    for (int mm = 0; mm < 3; mm++) cost += (sq(al[mm]) + sq(al[10 - mm])) * c_div_table[2 * mm + 1];
                }
            }
            // argmax over lanes 0..7, first maximum wins
            uint32_t best = cost;
            int bdir = lane;
#pragma unroll
            for (int st = 1; st < 8; st <<= 1) {
                uint32_t oc = __shfl_xor_sync(0xffffffff, best, st);
                int od = __shfl_xor_sync(0xffffffff, bdir, st);
                if (oc > best || (oc == best && od < bdir)) {
                    best = oc;
                    bdir = od;
                }
            }
            uint32_t opp = __shfl_sync(0xffffffff, cost, bdir ^ 4);
            dir = bdir;
            var = (best - opp) >> 10;
        }
        if (lane == 0) {
            // luma strength adjust / path selection (cdef.rs:969-1012)
            p.y_dir = dir;
            if (p.active) {
                int yp = 0, yd = 0;
                bool yon = false;
                if (p.y_pri != 0) {
                    int adj = 0;
                    if (var != 0) {
                        int i = (var >> 6) != 0 ? imin_(31 - __clz((int)(var >> 6)), 12) : 0;
                        adj = (p.y_pri * (4 + i) + 8) >> 4;
                    }
                    yon = (adj != 0 || p.y_sec != 0) && p.y_on;
                    yp = adj;
                    yd = dir;
                } else if (p.y_sec != 0 && p.y_on) {
                    yon = true;
                    yp = 0;
                    yd = 0;
                }
                p.y_on = yon;
                p.y_pri = yp;
                p.y_dir = yd;
                p.uv_dir = p.uv_pri != 0 ? c_uv_dirs[dir] : 0;
                tap_offsets(f.tab.CDEF_DIRECTIONS, p.y_dir, TW, p.yoff);
                tap_offsets(f.tab.CDEF_DIRECTIONS, p.uv_dir, CW, p.uvoff);
            }
            bp[warp] = p;
        }
    }
    __syncthreads();

    // ---- phase 2: filter + CCSO; warp w produces 8x8 block w (uniform
    // parameters per warp), lane -> 2 luma samples and 1 chroma sample ----
    const int bitdepth = f.bitdepth, bdmax = f.bdmax;
    const BlockParams &p = bp[warp];
    const int bx0 = warp * 8;
    if (gx0 + bx0 < f.w) {
        // luma
        const int r = lane >> 2, c0 = bx0 + (lane & 3) * 2;
        P *Cy = plane_ptr<P>(f.C[0]);
        const int gy = gy0 + r;
        int out[2];
        const R2gCcsoPlane &cp = fp.ccso[0];
        const int cq = f.tab.CCSO_QUANT_SZ[cp.scale_idx * 4 + cp.quant_idx];
        const int coff = c_ccso_pos[cp.ext_filter_support][0] * TW + c_ccso_pos[cp.ext_filter_support][1];
        const bool lossy_row = !(f.any_lossless &&
                                 ((m.lossless_mask_y[2 * by_idx + (r >> 2)][sb64x_idx] >> (c0 >> 2)) & 1));
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int c = c0 + k;
            const int16_t *t = &ty[2 + r][2 + c];
            const int px = t[0];
            int v = px;
            if (p.active && p.y_on) {
                v = cdef_px(&pty[2 + r][2 + c], p.y_pri, p.y_sec, p.yoff, damping, bd8);
                v = bitdepth == 8 ? (v & 0xff) : (v & 0xffff);
            }
            if (s_ccso[0] && lossy_row) {
                // ccso_prep (ccso.rs:115-185): the clamped tile is the padding
                int band_ = (int)((uint32_t)px >> (bitdepth - cp.max_band_log2));
                int idx;
                if (cp.bo_only)
                    idx = band_ & 0xff;
                else
                    idx = ((int)((ccso_score(t[coff] - px, cq, cp.edge_clf) << 5) |
                                 (ccso_score(t[-coff] - px, cq, cp.edge_clf) << 3)) |
                           band_) & 0xff;
                int bi = idx >> 1;
                int packed = bi < 64 ? cp.filter_off[bi] : 0;
                v = iclip_(v + f.tab.CCSO_OFFSET[cp.scale_idx * 8 + (7 & (packed >> (4 * (idx & 1))))], 0, bdmax);
            }
            out[k] = v;
        }
        Cy[gy * ys + gx0 + c0] = (P)out[0];
        Cy[gy * ys + gx0 + c0 + 1] = (P)out[1];
        // chroma: lane -> plane lane/16, row (lane%16)/4, column lane%4
        const int pl = lane >> 4, cr = (lane & 15) >> 2, cc = (bx0 >> 1) + (lane & 3);
        const int cgy = cy0 + cr, cgx = cx0 + cc;
        P *Cp = plane_ptr<P>(f.C[1 + pl]);
        int px = tc[pl][2 + cr][2 + cc];
        int v = px;
        if (p.active && p.uv_on) {
            v = cdef_px(&ptc[pl][2 + cr][2 + cc], p.uv_pri, p.uv_sec, p.uvoff, damping - 1, bd8);
            v = bitdepth == 8 ? (v & 0xff) : (v & 0xffff);
        }
        if (s_ccso[1 + pl]) {
            const R2gCcsoPlane &cpc = fp.ccso[1 + pl];
            bool ll = f.any_lossless && ((m.lossless_mask_uv[by_idx][sb64x_idx] >> (cc >> 2)) & 1);
            if (!ll) {
                // co-located luma of the chroma sample (ccso_prep, 4:2:0)
                const int16_t *t = &ty[2 + 2 * cr][2 + 2 * cc];
                int cl = t[0];
                int band_ = (int)((uint32_t)cl >> (bitdepth - cpc.max_band_log2));
                int idx;
                if (cpc.bo_only) {
                    idx = band_ & 0xff;
                } else {
                    const int q = f.tab.CCSO_QUANT_SZ[cpc.scale_idx * 4 + cpc.quant_idx];
                    const int o = c_ccso_pos[cpc.ext_filter_support][0] * TW + c_ccso_pos[cpc.ext_filter_support][1];
                    idx = ((int)((ccso_score(t[o] - cl, q, cpc.edge_clf) << 5) |
                                 (ccso_score(t[-o] - cl, q, cpc.edge_clf) << 3)) |
                           band_) & 0xff;
                }
                int bi = idx >> 1;
                int packed = bi < 64 ? cpc.filter_off[bi] : 0;
                v = iclip_(v + f.tab.CCSO_OFFSET[cpc.scale_idx * 8 + (7 & (packed >> (4 * (idx & 1))))], 0, bdmax);
            }
        }
        Cp[cgy * uvs + cgx] = (P)v;
    }
}

template <typename P>
__global__ void __launch_bounds__(256) cdef_ccso_kernel(const DevFrame f) {
    __shared__ CdefSmem sm;
    cdef_band<P>(f, sm, blockIdx.x, blockIdx.y);
}

// Persistent kernel over a cross-frame work list: item = frame << 22 | band
// * sb64w + sbx.
__global__ void __launch_bounds__(256) cdef_batch_kernel(BatchArgs a) {
    __shared__ CdefSmem sm;
    const int n = a.count[1];
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const uint32_t it = a.work[1][w];
        const DevFrame &f = a.frames[it >> 22];
        const int b = it & 0x3fffff, sb64w = (f.w + 63) >> 6;
        if (f.bitdepth > 8)
            cdef_band<uint16_t>(f, sm, b % sb64w, b / sb64w);
        else
            cdef_band<uint8_t>(f, sm, b % sb64w, b / sb64w);
        __syncthreads();
    }
}

}  // namespace

void r2g_batch_launch_cdef(const BatchArgs &a, int grid, cudaStream_t s) { cdef_batch_kernel<<<grid, 256, 0, s>>>(a); }
int r2g_batch_occupancy_cdef() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, cdef_batch_kernel, 256, 0);
    return nb;
}
int r2g_cdef_items(const DevFrame &f) { return f.cdef_stage_on ? ((f.w + 63) >> 6) * (f.h >> 3) : 0; }

int r2g_launch_cdef(const DevFrame &f, cudaStream_t s) {
    if (!f.cdef_stage_on) return 0;
    dim3 grid((f.w + 63) / 64, f.h / 8);
    if (f.bitdepth > 8)
        cdef_ccso_kernel<uint16_t><<<grid, 256, 0, s>>>(f);
    else
        cdef_ccso_kernel<uint8_t><<<grid, 256, 0, s>>>(f);
    return 1;
}
