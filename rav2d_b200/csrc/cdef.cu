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

// cdef_filter_block (cdef.rs:320-458) for one sample.  `tap(dy, dx)`
// returns the padded neighbour value.
template <typename TapF>
R2G_D int cdef_px(int px, int pri, int sec, int dir, int damping, int bd8, const DevTables &tab, TapF tap) {
    const int8_t *D = tab.CDEF_DIRECTIONS;
    if (pri != 0) {
        int pri_tap = 4 - ((pri >> bd8) & 1);
        int pri_shift = imax_(0, damping - ulog2_((uint32_t)pri));
        int sum = 0, mx = px, mn = px, tk = pri_tap;
        if (sec != 0) {
            int sec_shift = damping - ulog2_((uint32_t)sec);
#pragma unroll
            for (int k = 0; k < 2; k++) {
                int dy, dx;
                dir_off(D[(dir + 2) * 2 + k], dy, dx);
                int p0 = tap(dy, dx), p1 = tap(-dy, -dx);
                sum += tk * constrain(p0 - px, pri, pri_shift);
                sum += tk * constrain(p1 - px, pri, pri_shift);
                tk = (tk & 3) | 2;
                mn = imin_(p0, mn);
                mx = imax_(p0, mx);
                mn = imin_(p1, mn);
                mx = imax_(p1, mx);
                int ay, ax, by, bx;
                dir_off(D[(dir + 4) * 2 + k], ay, ax);
                dir_off(D[dir * 2 + k], by, bx);
                int s0 = tap(ay, ax), s1 = tap(-ay, -ax), s2 = tap(by, bx), s3 = tap(-by, -bx);
                int st = 2 - k;
                sum += st * constrain(s0 - px, sec, sec_shift);
                sum += st * constrain(s1 - px, sec, sec_shift);
                sum += st * constrain(s2 - px, sec, sec_shift);
                sum += st * constrain(s3 - px, sec, sec_shift);
                mn = imin_(s0, mn);
                mx = imax_(s0, mx);
                mn = imin_(s1, mn);
                mx = imax_(s1, mx);
                mn = imin_(s2, mn);
                mx = imax_(s2, mx);
                mn = imin_(s3, mn);
                mx = imax_(s3, mx);
            }
            return iclip_(px + ((sum - (sum < 0) + 8) >> 4), mn, mx);
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            int dy, dx;
            dir_off(D[(dir + 2) * 2 + k], dy, dx);
            int p0 = tap(dy, dx), p1 = tap(-dy, -dx);
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
        int ay, ax, by, bx;
        dir_off(D[(dir + 4) * 2 + k], ay, ax);
        dir_off(D[dir * 2 + k], by, bx);
        int s0 = tap(ay, ax), s1 = tap(-ay, -ax), s2 = tap(by, bx), s3 = tap(-by, -bx);
        int st = 2 - k;
        sum += st * constrain(s0 - px, sec, sec_shift);
        sum += st * constrain(s1 - px, sec, sec_shift);
        sum += st * constrain(s2 - px, sec, sec_shift);
        sum += st * constrain(s3 - px, sec, sec_shift);
    }
    return px + ((sum - (sum < 0) + 8) >> 4);
}

// ccso_score (ccso.rs:16-24)
R2G_D uint32_t ccso_score(int diff, int q, uint32_t clf) {
    if (diff > q && clf == 0) return 2;
    if (diff < -q) return 0;
    return 1;
}

template <typename P>
__global__ void __launch_bounds__(256) cdef_ccso_kernel(const DevFrame f) {
    __shared__ int16_t ty[TH][TW];
    __shared__ int16_t tc[2][CH][CW];
    __shared__ int bins[8][96];
    __shared__ BlockParams bp[8];
    __shared__ int s_ccso[3];

    const int sbx = blockIdx.x;
    const int band = blockIdx.y;  // 8-row luma band
    const int gx0 = sbx * 64, gy0 = band * 8;
    const int cx0 = gx0 >> 1, cy0 = gy0 >> 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int bd8 = f.bitdepth - 8;
    const P *Dy = plane_ptr<const P>(f.R[0]);
    const P *Du = plane_ptr<const P>(f.R[1]);
    const P *Dv = plane_ptr<const P>(f.R[2]);
    const int64_t ys = f.stride[0], uvs = f.stride[1];

    // ---- stage the band (clamped coordinates) ----
    for (int i = tid; i < TH * TW; i += 256) {
        int r = i / TW, c = i % TW;
        int gy = iclip_(gy0 - 2 + r, 0, f.h - 1), gx = iclip_(gx0 - 2 + c, 0, f.w - 1);
        ty[r][c] = (int16_t)Dy[gy * ys + gx];
    }
    for (int i = tid; i < 2 * CH * CW; i += 256) {
        int pl = i / (CH * CW), j = i % (CH * CW);
        int r = j / CW, c = j % CW;
        int gy = iclip_(cy0 - 2 + r, 0, f.ch - 1), gx = iclip_(cx0 - 2 + c, 0, f.cw - 1);
        tc[pl][r][c] = (int16_t)(pl ? Dv : Du)[gy * uvs + gx];
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
            }
            bp[warp] = p;
        }
    }
    __syncthreads();

    // ---- phase 2: filter + CCSO, row-contiguous ----
    const int bitdepth = f.bitdepth, bdmax = f.bdmax;
    // luma: thread -> row tid/32, samples 2*(tid%32) and +1
    {
        int r = tid >> 5, c0 = (tid & 31) * 2;
        P *Cy = plane_ptr<P>(f.C[0]);
        int gy = gy0 + r;
        int out[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            int c = c0 + k, gx = gx0 + c;
            int px = ty[2 + r][2 + c];
            const BlockParams &p = bp[c >> 3];
            int v = px;
            if (p.active && p.y_on) {
                auto tap = [&](int dy, int dx) -> int {
                    int yy = gy + dy, xx = gx + dx;
                    if (yy < 0 || yy >= f.h || xx < 0 || xx >= f.w) return INT16_MIN;
                    return ty[2 + r + dy][2 + c + dx];
                };
                v = cdef_px(px, p.y_pri, p.y_sec, p.y_dir, damping, bd8, f.tab, tap);
                v = bitdepth == 8 ? (v & 0xff) : (v & 0xffff);
            }
            if (s_ccso[0]) {
                const R2gCcsoPlane &cp = fp.ccso[0];
                int cl = px;
                int band_ = (int)((uint32_t)cl >> (bitdepth - cp.max_band_log2));
                int idx;
                if (cp.bo_only) {
                    idx = band_;
                } else {
                    int dy = c_ccso_pos[cp.ext_filter_support][0], dx = c_ccso_pos[cp.ext_filter_support][1];
                    int q = f.tab.CCSO_QUANT_SZ[cp.scale_idx * 4 + cp.quant_idx];
                    int a = ty[iclip_(gy + dy, 0, f.h - 1) - gy0 + 2][iclip_(gx + dx, 0, f.w - 1) - gx0 + 2];
                    int b = ty[iclip_(gy - dy, 0, f.h - 1) - gy0 + 2][iclip_(gx - dx, 0, f.w - 1) - gx0 + 2];
                    idx = (int)((ccso_score(a - cl, q, cp.edge_clf) << 5) | (ccso_score(b - cl, q, cp.edge_clf) << 3)) | band_;
                    idx &= 0xff;
                }
                bool ll = false;
                if (f.any_lossless) ll = (m.lossless_mask_y[2 * by_idx + (r >> 2)][sb64x_idx] >> (c >> 2)) & 1;
                if (!ll) {
                    int bi = idx >> 1;
                    int packed = bi < 64 ? cp.filter_off[bi] : 0;
                    int oi = 7 & (packed >> (4 * (idx & 1)));
                    v = iclip_(v + f.tab.CCSO_OFFSET[cp.scale_idx * 8 + oi], 0, bdmax);
                }
            }
            out[k] = v;
        }
        if (gx0 + c0 < f.w) {
            Cy[gy * ys + gx0 + c0] = (P)out[0];
            Cy[gy * ys + gx0 + c0 + 1] = (P)out[1];
        }
    }
    // chroma: thread -> plane tid/128, row (tid%128)/32, column tid%32
    {
        int pl = tid >> 7, r = (tid & 127) >> 5, c = tid & 31;
        int gy = cy0 + r, gx = cx0 + c;
        if (gx < f.cw) {
            P *Cp = plane_ptr<P>(f.C[1 + pl]);
            int px = tc[pl][2 + r][2 + c];
            const BlockParams &p = bp[c >> 2];
            int v = px;
            if (p.active && p.uv_on) {
                auto tap = [&](int dy, int dx) -> int {
                    int yy = gy + dy, xx = gx + dx;
                    if (yy < 0 || yy >= f.ch || xx < 0 || xx >= f.cw) return INT16_MIN;
                    return tc[pl][2 + r + dy][2 + c + dx];
                };
                v = cdef_px(px, p.uv_pri, p.uv_sec, p.uv_dir, damping - 1, bd8, f.tab, tap);
                v = bitdepth == 8 ? (v & 0xff) : (v & 0xffff);
            }
            if (s_ccso[1 + pl]) {
                const R2gCcsoPlane &cp = fp.ccso[1 + pl];
                int lx = gx << 1, ly = gy << 1;  // co-located luma
                int cl = ty[ly - gy0 + 2][lx - gx0 + 2];
                int band_ = (int)((uint32_t)cl >> (bitdepth - cp.max_band_log2));
                int idx;
                if (cp.bo_only) {
                    idx = band_;
                } else {
                    int dy = c_ccso_pos[cp.ext_filter_support][0], dx = c_ccso_pos[cp.ext_filter_support][1];
                    int q = f.tab.CCSO_QUANT_SZ[cp.scale_idx * 4 + cp.quant_idx];
                    int a = ty[iclip_(ly + dy, 0, f.h - 1) - gy0 + 2][iclip_(lx + dx, 0, f.w - 1) - gx0 + 2];
                    int b = ty[iclip_(ly - dy, 0, f.h - 1) - gy0 + 2][iclip_(lx - dx, 0, f.w - 1) - gx0 + 2];
                    idx = (int)((ccso_score(a - cl, q, cp.edge_clf) << 5) | (ccso_score(b - cl, q, cp.edge_clf) << 3)) | band_;
                    idx &= 0xff;
                }
                bool ll = false;
                if (f.any_lossless) ll = (m.lossless_mask_uv[by_idx][sb64x_idx] >> (c >> 2)) & 1;
                if (!ll) {
                    int bi = idx >> 1;
                    int packed = bi < 64 ? cp.filter_off[bi] : 0;
                    int oi = 7 & (packed >> (4 * (idx & 1)));
                    v = iclip_(v + f.tab.CCSO_OFFSET[cp.scale_idx * 8 + oi], 0, bdmax);
                }
            }
            Cp[gy * uvs + gx] = (P)v;
        }
    }
}

}  // namespace

int r2g_launch_cdef(const DevFrame &f, cudaStream_t s) {
    if (!f.cdef_stage_on) return 0;
    dim3 grid((f.w + 63) / 64, f.h / 8);
    if (f.bitdepth > 8)
        cdef_ccso_kernel<uint16_t><<<grid, 256, 0, s>>>(f);
    else
        cdef_ccso_kernel<uint8_t><<<grid, 256, 0, s>>>(f);
    return 1;
}
