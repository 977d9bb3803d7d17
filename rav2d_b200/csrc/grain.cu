// Film-grain synthesis and apply on the GPU: filtered frame L -> display
// copy G.
//
// Reference: crates/rav2d/src/filmgrain.rs (get_random_number :11,
// generate_scaling_* :22/:59, generate_grain_y/uv :115/:160, fgy_32x32xn
// :248, fguv_32x32xn :409, prep_grain :617, apply_grain_row :688) and
// decode.rs:4641-4775.
//
// The reference's serial parts are re-scheduled, not approximated:
// * the 16-bit LFSR is maximal-length, so every nonzero state lies on one
//   cycle of 65535 states; the host tabulates the cycle and each state's
//   position on it, and a thread jumps k steps with two look-ups;
// * the auto-regressive filter reads rows y-lag..y-1 at x-lag..x+lag and row
//   y at x-lag..x-1, so every sample on the line x + 4y = t depends only on
//   lines < t: the template is filled as a wavefront over t, one warp per
//   plane;
// * block offsets of row band r and block b are draws 8b + 4n + 1 of the
//   band's seed, evaluated directly by jump-ahead in the apply kernel.
#include <cstring>
#include <atomic>
#include <mutex>

#include "r2g_common.cuh"
#include "r2g_runtime.h"

namespace {

constexpr int GW = 82, GH = 73, SGW = 44, SGH = 38;

// The LFSR of filmgrain.rs:11-16 (taps 16, 15, 13, 4) is maximal-length:
// every nonzero state lies on one cycle of 65535 states.  g_lfsr_cycle[i] is
// the state i steps after state 1 and g_lfsr_pos its inverse, so a jump of k
// steps is two look-ups.  Both are built on the host once per device.
__device__ uint16_t g_lfsr_cycle[65536];
__device__ uint16_t g_lfsr_pos[65536];

// one LFSR step (filmgrain.rs:11-16)
R2G_HD uint32_t lfsr_step(uint32_t r) {
    uint32_t bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1;
    return (r >> 1) | (bit << 15);
}

// state after k steps from s (16-bit state)
R2G_D uint32_t lfsr_jump(uint32_t s, uint32_t k) {
    s &= 0xffff;  // seeds are 16-bit (checked at the boundary)
    if (!s) return 0;  // the all-zero state stays zero
    uint32_t i = (uint32_t)__ldg(&g_lfsr_pos[s]) + k % 65535u;
    if (i >= 65535u) i -= 65535u;
    return __ldg(&g_lfsr_cycle[i]);
}

R2G_D int round2(int x, int shift) { return (x + ((1 << shift) >> 1)) >> shift; }

// Templates: luma 73x82, chroma 38x44 (stored in 73x82 arrays as the
// reference's GrainLut does); scaling LUTs per plane (1 << bitdepth).
struct GrainTplSmem {
    int16_t ly[GH][GW];
    int16_t lc[2][SGH][SGW];
    uint32_t sc[3 * 1024 / 4];  // scaling LUTs, built here (zero-initialised) and copied out
};

// Barrier of warps 0-2, which run the auto-regressive filters; warps 6-7
// build the scaling LUTs meanwhile.
R2G_D void ar_sync() { asm volatile("bar.sync 1, 96;\n" ::: "memory"); }

// One front of the auto-regressive filter of generate_grain_y
// (filmgrain.rs:134-157) or generate_grain_uv (:183-228), lag >= 1, for the
// calling lane.  Cell (y, x) reads rows y - LAG .. y - 1 over x - LAG .. x +
// LAG and row y over x - LAG .. x - 1, so the cells with equal x + 4y (a
// front) depend only on earlier fronts.  Lane l owns rows 3 + l + 32k; a
// row is active for 78 fronts and rows 32 apart are 128 fronts apart, so a
// lane has at most one active cell per front and one set of registers: the
// windows of the rows above (win) and its own last outputs (own).  At x == 2
// the lane loads the windows of column 3; at each cell it loads one new value
// (row y - 1, column x + LAG: the previous front's output of the lane
// above), finishes the cell and slides the windows.
template <int LAG>
R2G_D void ar_front(int16_t *base, int stride, int nrows, int xlim, int t, const int *cf, int (&win)[LAG][2 * LAG + 1],
                    int (&own)[LAG], int &g0, int sh, int gmin, int gmax, const int16_t (*luma)[GW], int lcoef) {
    constexpr int W = 2 * LAG + 1;
    const int lane = threadIdx.x & 31;
    const int rel = t - 14 - 4 * lane;  // column - 2 of row 3 + lane at front t
    if (rel < 0) return;
    const int k = rel >> 7;
    const int y = 3 + lane + 32 * k, x = 2 + rel - 128 * k;
    if (y >= nrows || x >= xlim) return;
    if (x == 2) {
#pragma unroll
        for (int r = 0; r < LAG; r++)
#pragma unroll
            for (int j = 0; j < W; j++)
                if (r < LAG - 1 || j < W - 1) win[r][j] = base[(y - LAG + r) * stride + 3 - LAG + j];
#pragma unroll
        for (int j = 0; j < LAG; j++) own[j] = base[y * stride + 3 - LAG + j];
        g0 = base[y * stride + 3];
        return;
    }
    const int v = base[(y - 1) * stride + x + LAG];
    int acc0 = 0, acc1 = 0;
#pragma unroll
    for (int r = 0; r < LAG; r++)
#pragma unroll
        for (int j = 0; j < W; j++) {
            if (r == LAG - 1 && j == W - 1) continue;
            if ((r * W + j) & 1)
                acc1 += cf[r * W + j] * win[r][j];
            else
                acc0 += cf[r * W + j] * win[r][j];
        }
#pragma unroll
    for (int j = 0; j < LAG; j++) acc1 += cf[LAG * W + j] * own[j];
    int sum = acc0 + acc1 + cf[LAG * W - 1] * v;
    if (luma) {
        const int lx = ((x - 3) << 1) + 3, lyy = ((y - 3) << 1) + 3;
        const int l4 = luma[lyy][lx] + luma[lyy][lx + 1] + luma[lyy + 1][lx] + luma[lyy + 1][lx + 1];
        sum += ((l4 + 2) >> 2) * lcoef;
    }
    const int out = iclip_(g0 + ((sum + ((1 << sh) >> 1)) >> sh), gmin, gmax);
    base[y * stride + x] = (int16_t)out;
    if (x + 1 < xlim) {
#pragma unroll
        for (int r = 0; r < LAG; r++) {
#pragma unroll
            for (int j = 0; j < W - 1; j++) win[r][j] = win[r][j + 1];
            if (r < LAG - 1) win[r][W - 1] = base[(y - LAG + r) * stride + x + 1 + LAG];
        }
        win[LAG - 1][W - 2] = v;
#pragma unroll
        for (int j = 0; j < LAG - 1; j++) own[j] = own[j + 1];
        own[LAG - 1] = out;
        g0 = base[y * stride + x + 1];
    }
}

// The filters of both templates for lag >= 1: warp 0 luma (fronts 14 ..
// 381, 8 per round), warp 1 chroma U and warp 2 chroma V (fronts 8 .. 191, 4
// per round).  Fronts are ordered inside a warp by __syncwarp; a barrier of
// the three warps ends each round.  Chroma front t reads luma fronts up to
// 2t - 10 (its luma term); in round r chroma runs fronts 4r + 8 .. 4r + 11,
// which read luma fronts up to 8r + 12, all finished in rounds before r.
template <int LAG>
R2G_D void ar_wave(const GrainParams &gp, GrainTplSmem &sm, bool gen_u, bool gen_v, int gmin, int gmax) {
    constexpr int W = 2 * LAG + 1, NT = LAG * W + LAG;
    const R2gFilmGrainData &d = gp.d;
    const int warp = threadIdx.x >> 5, sh = (int)d.ar_coeff_shift;
    const bool gen = warp == 0 || (warp == 1 ? gen_u : gen_v);
    int16_t *base = warp == 0 ? &sm.ly[0][0] : &sm.lc[warp - 1][0][0];
    const int stride = warp == 0 ? GW : SGW, nrows = warp == 0 ? GH : SGH;
    const int16_t(*luma)[GW] = (warp > 0 && d.num_points[0] > 0) ? sm.ly : nullptr;
    int cf[NT + 1];
#pragma unroll
    for (int i = 0; i <= NT; i++) cf[i] = d.ar_coeffs[warp][i];
    int win[LAG][W], own[LAG], g0 = 0;
#pragma unroll
    for (int r = 0; r < LAG; r++)
#pragma unroll
        for (int j = 0; j < W; j++) win[r][j] = 0;
#pragma unroll
    for (int j = 0; j < LAG; j++) own[j] = 0;
    for (int round = 0; round < 46; round++) {
        if (warp == 0) {
            for (int i = 0; i < 8; i++) {
                ar_front<LAG>(base, stride, nrows, GW - 3, 14 + 8 * round + i, cf, win, own, g0, sh, gmin, gmax,
                              nullptr, 0);
                __syncwarp();
            }
        } else if (gen) {
            for (int i = 0; i < 4; i++) {
                ar_front<LAG>(base, stride, nrows, SGW - 3, 4 * round + 8 + i, cf, win, own, g0, sh, gmin, gmax, luma,
                              cf[NT]);
                __syncwarp();
            }
        }
        ar_sync();
    }
}

// Lag 0: no neighbour taps.  Luma cells are only clipped; a chroma cell adds
// the luma term, which reads the finished luma template.
R2G_D void ar_lag0(const GrainParams &gp, GrainTplSmem &sm, bool gen_u, bool gen_v, int gmin, int gmax) {
    const R2gFilmGrainData &d = gp.d;
    const int tid = threadIdx.x, sh = (int)d.ar_coeff_shift, rnd = (1 << sh) >> 1;
    for (int i = tid; i < (GH - 3) * (GW - 6); i += 96) {
        int16_t &g = sm.ly[3 + i / (GW - 6)][3 + i % (GW - 6)];
        g = (int16_t)iclip_(g, gmin, gmax);
    }
    ar_sync();
    const bool with_luma = d.num_points[0] > 0;
    for (int i = tid; i < 2 * (SGH - 3) * (SGW - 6); i += 96) {
        const int uv = i / ((SGH - 3) * (SGW - 6)), j = i % ((SGH - 3) * (SGW - 6));
        if (!(uv ? gen_v : gen_u)) continue;
        const int y = 3 + j / (SGW - 6), x = 3 + j % (SGW - 6);
        int sum = 0;
        if (with_luma) {
            const int lx = ((x - 3) << 1) + 3, lyy = ((y - 3) << 1) + 3;
            const int l4 = sm.ly[lyy][lx] + sm.ly[lyy][lx + 1] + sm.ly[lyy + 1][lx] + sm.ly[lyy + 1][lx + 1];
            sum = ((l4 + 2) >> 2) * d.ar_coeffs[1 + uv][0];
        }
        sm.lc[uv][y][x] = (int16_t)iclip_(sm.lc[uv][y][x] + ((sum + rnd) >> sh), gmin, gmax);
    }
}

// Scaling LUT of one plane (generate_scaling_8bpc / _hbd, filmgrain.rs:
// 22-113) into a zeroed shared-memory LUT: the interpolation pass reads back
// what the first pass wrote, which in shared memory costs a few cycles.
R2G_D void scaling_lut(const GrainParams &gp, int pl, uint8_t *scaling) {
    const R2gFilmGrainData &d = gp.d;
    uint8_t *sc = scaling + pl * 1024;
    const int size = 1 << gp.bitdepth, sx = gp.bitdepth - 8;
    const int num = d.num_points[pl];
    const bool wanted = pl == 0 || !d.chroma_scaling_from_luma;
    if (!wanted || num == 0) {
        for (int i = 0; i < size; i++) sc[i] = 0;
        return;
    }
    const uint8_t(*pts)[2] = d.points[pl];
    for (int i = 0; i < (pts[0][0] << sx); i++) sc[i] = pts[0][1];
    for (int i = 0; i < num - 1; i++) {
        int bx = pts[i][0], by = pts[i][1], ex = pts[i + 1][0], ey = pts[i + 1][1];
        int dx = ex - bx, dyv = ey - by;
        if (dx <= 0) continue;
        int delta = dyv * ((0x10000 + (dx >> 1)) / dx);
        int dd = 0x8000;
        for (int x = 0; x < dx; x++) {
            sc[(bx + x) << sx] = (uint8_t)(by + (dd >> 16));
            dd += delta;
        }
    }
    for (int i = pts[num - 1][0] << sx; i < size; i++) sc[i] = pts[num - 1][1];
    if (sx > 0) {
        int pad = 1 << sx, rnd = pad >> 1;
        for (int i = 0; i < num - 1; i++) {
            int bx = pts[i][0] << sx, ex = pts[i + 1][0] << sx;
            for (int x = 0; x < ex - bx; x += pad) {
                int b0 = sc[bx + x], range = sc[bx + x + pad] - b0, r = rnd;
                for (int n2 = 1; n2 < pad; n2++) {
                    r += range;
                    sc[bx + x + n2] = (uint8_t)(b0 + (r >> sx));
                }
            }
        }
    }
}

R2G_D void grain_template(const GrainParams &gp, const DevTables &tab, int16_t *lut, uint8_t *scaling,
                          GrainTplSmem &sm) {
    auto &ly = sm.ly;
    auto &lc = sm.lc;
    const int tid = threadIdx.x;
    const R2gFilmGrainData &d = gp.d;
    const int b8 = gp.bitdepth - 8;
    const int shift = 4 - b8 + d.grain_scale_shift;
    const int gmin = -(128 << b8), gmax = (128 << b8) - 1;
    const bool gen_u = d.num_points[1] > 0 || d.chroma_scaling_from_luma;
    const bool gen_v = d.num_points[2] > 0 || d.chroma_scaling_from_luma;

    // Gaussian fills: value k uses the state after k + 1 steps
    {
        const int n = GH * GW;
        const int chunk = (n + 255) / 256;
        int k0 = tid * chunk;
        if (k0 < n) {
            uint32_t st = lfsr_jump(gp.seed & 0xffff, (uint32_t)k0);
            for (int k = k0; k < k0 + chunk && k < n; k++) {
                st = lfsr_step(st);
                ly[k / GW][k % GW] = (int16_t)round2(tab.GAUSSIAN_SEQUENCE[(st >> 5) & 2047], shift);
            }
        }
        const int nc = SGH * SGW;
        const int cchunk = (nc + 127) / 128;
        int uv = tid >> 7, t = tid & 127;
        int c0 = t * cchunk;
        if (c0 < nc) {
            uint32_t s0 = (gp.seed ^ (uv ? 0x49d8 : 0xb524)) & 0xffff;
            uint32_t st = lfsr_jump(s0, (uint32_t)c0);
            for (int k = c0; k < c0 + cchunk && k < nc; k++) {
                st = lfsr_step(st);
                lc[uv][k / SGW][k % SGW] = (int16_t)round2(tab.GAUSSIAN_SEQUENCE[(st >> 5) & 2047], shift);
            }
        }
    }
    for (int i = tid; i < 3 * 1024 / 4; i += 256) sm.sc[i] = 0;
    __syncthreads();
    if (tid < 96) {
        switch (d.ar_coeff_lag) {
            case 0: ar_lag0(gp, sm, gen_u, gen_v, gmin, gmax); break;
            case 1: ar_wave<1>(gp, sm, gen_u, gen_v, gmin, gmax); break;
            case 2: ar_wave<2>(gp, sm, gen_u, gen_v, gmin, gmax); break;
            default: ar_wave<3>(gp, sm, gen_u, gen_v, gmin, gmax); break;
        }
    } else if (tid >= 192 && tid < 195) {
        scaling_lut(gp, tid - 192, reinterpret_cast<uint8_t *>(sm.sc));
    }
    __syncthreads();
    for (int i = tid; i < 3 * 1024 / 4; i += 256) reinterpret_cast<uint32_t *>(scaling)[i] = sm.sc[i];
    // write templates (zero where a plane's template is not generated)
    for (int i = tid; i < GH * GW; i += 256) {
        int y = i / GW, x = i % GW;
        lut[i] = ly[y][x];
        lut[GH * GW + i] = (gen_u && y < SGH && x < SGW) ? lc[0][y][x] : 0;
        lut[2 * GH * GW + i] = (gen_v && y < SGH && x < SGW) ? lc[1][y][x] : 0;
    }
}

__global__ void __launch_bounds__(256) grain_template_kernel(const GrainParams gp, const DevTables tab,
                                                             int16_t *lut, uint8_t *scaling) {
    __shared__ GrainTplSmem sm;
    grain_template(gp, tab, lut, scaling, sm);
}

// Offsets of block b for row band `row` and seed index i (filmgrain.rs:
// 274-305): draws 8b + 4n + 1 of the band's seed.
R2G_D int block_offset(uint32_t in_seed, int row, int i, int b, int n, int block_size) {
    uint32_t s = in_seed;
    s ^= (uint32_t)((((row - i) * 37 + 178) & 0xFF)) << 8;
    s ^= (uint32_t)(((row - i) * 173 + 105) & 0xFF);
    uint32_t st = lfsr_jump(s, (uint32_t)(8 * b + 4 * n + 1));
    return (int)(((uint32_t)(3 - block_size) * ((st >> 7) & 511)) >> 6);
}

template <int BYTES>
struct RawRun;
template <>
struct RawRun<2> {
    using T = unsigned short;
};
template <>
struct RawRun<4> {
    using T = unsigned int;
};
template <>
struct RawRun<8> {
    using T = uint2;
};

// N consecutive samples at p: one aligned vector load / store when `vec`,
// else sample by sample over the first n (the part inside the plane).
template <typename P, int N>
R2G_D void load_run(const P *p, int n, bool vec, int (&v)[N]) {
    if (vec) {
        using T = typename RawRun<N * sizeof(P)>::T;
        const T raw = __ldg(reinterpret_cast<const T *>(p));
        P s[N];
        memcpy(s, &raw, sizeof(raw));
#pragma unroll
        for (int k = 0; k < N; k++) v[k] = s[k];
    } else {
#pragma unroll
        for (int k = 0; k < N; k++) v[k] = k < n ? (int)__ldg(p + k) : 0;
    }
}

template <typename P, int N>
R2G_D void store_run(P *p, int n, bool vec, const int (&v)[N]) {
    if (vec) {
        using T = typename RawRun<N * sizeof(P)>::T;
        P s[N];
#pragma unroll
        for (int k = 0; k < N; k++) s[k] = (P)v[k];
        T raw;
        memcpy(&raw, s, sizeof(raw));
        *reinterpret_cast<T *>(p) = raw;
    } else {
#pragma unroll
        for (int k = 0; k < N; k++)
            if (k < n) p[k] = (P)v[k];
    }
}

// Luma samples of a band covered by one CTA (a segment): 4 blocks of 32 or
// 8 blocks of 16.
constexpr int SEG_W = 128;

// Offsets (filmgrain.rs:274-305) of blocks b0 - 1 .. b0 + NB - 1 of a
// segment: v[j][i][n] for block b0 - 1 + j, seed row i, coordinate n.
template <int BS>
struct SegOffsets {
    int v[SEG_W / BS + 1][2][2];
};

// Overlap blend of two grain values (filmgrain.rs:560-600 / :760-800).
R2G_D int blend(int a, int wa, int b, int wb, int gmin, int gmax) {
    return iclip_((a * wa + b * wb + 16) >> 5, gmin, gmax);
}

// One CTA per segment of a row band: luma BS rows x SEG_W samples and both
// chroma planes' BS/2 x SEG_W/2 (fgy_32x32xn / fguv_32x32xn, 4:2:0).  Thread
// t takes luma columns 4 (t % 32) .. +3 over rows (t / 32) * BS/8 .. +BS/8-1
// and chroma columns 2 (t % 32) .. +1 over rows (t / 32) * BS/16 .. of both
// planes: the luma samples that chroma scaling averages are the thread's own
// even rows, a warp moves whole rows, and every plane sample is requested
// before the first template or scaling look-up.  Overlap: the blend of the
// first two rows of a band is uniform per warp; the first two columns of a
// block are a fix-up of the runs that start a block.
template <typename P, int BS>
R2G_D void grain_segment(const DevFrame &f, const GrainParams &gp, const int16_t *lut, const uint8_t *scaling, int row,
                         int seg, SegOffsets<BS> &so) {
    constexpr int NB = SEG_W / BS, RL = BS / 8, RC = BS / 16, CB = BS / 2;
    const int tid = threadIdx.x;
    const R2gFilmGrainData &d = gp.d;
    const int rows = 1 + (d.overlap_flag && row > 0);
    const int b0 = seg * NB;
    if (tid < 4 * (NB + 1)) {
        const int j = tid >> 2, i = (tid >> 1) & 1, n = tid & 1, bb = b0 - 1 + j;
        so.v[j][i][n] = (i < rows && bb >= 0) ? block_offset(gp.seed, row, i, bb, n, d.block_size) : 0;
    }
    // the filtered planes may come from the previous kernel (programmatic
    // dependent launch): wait for it
    pdl_wait();
    const int b8 = f.bitdepth - 8, bdmax = f.bdmax;
    const int gmin = -(128 << b8), gmax = (128 << b8) - 1;
    const int64_t ys = f.stride[0], uvs = f.stride[1];
    const bool vec = gp.vec;
    const int c32 = tid & 31, r0 = tid >> 5;
    const int bl = (4 * c32) / BS;  // block of the segment

    // ---- plane loads ----
    const int X = seg * SEG_W + 4 * c32, Y0 = row * BS + r0 * RL;
    const int bh = imin_(BS, f.h - row * BS);
    const int ln = f.w - X;  // luma samples of the run inside the plane
    const P *Ly = plane_ptr<const P>(f.L[0]) + (int64_t)Y0 * ys + X;
    int sy[RL][4];
#pragma unroll
    for (int k = 0; k < RL; k++) {
        if (ln > 0 && r0 * RL + k < bh)
            load_run<P, 4>(Ly + k * ys, ln, vec && ln >= 4, sy[k]);
        else
            sy[k][0] = sy[k][1] = sy[k][2] = sy[k][3] = 0;
    }
    const int CX = seg * (SEG_W / 2) + 2 * c32, CY0 = row * CB + r0 * RC;
    const int cbh = (bh + 1) >> 1;
    const int cn = ((f.w + 1) >> 1) - CX;
    int sc[2][RC][2];
#pragma unroll
    for (int uv = 0; uv < 2; uv++) {
        const P *Lc = plane_ptr<const P>(f.L[1 + uv]) + (int64_t)CY0 * uvs + CX;
#pragma unroll
        for (int k = 0; k < RC; k++) {
            if (cn > 0 && r0 * RC + k < cbh)
                load_run<P, 2>(Lc + k * uvs, cn, vec && cn >= 2, sc[uv][k]);
            else
                sc[uv][k][0] = sc[uv][k][1] = 0;
        }
    }
    __syncthreads();  // offsets

    const int bb = b0 + bl;
    const bool ovx = d.overlap_flag && bb > 0, ovy = d.overlap_flag && row > 0;
    const int sshift = d.scaling_shift, srnd = (1 << sshift) >> 1;

    // ---- chroma (uses the luma samples before grain) ----
    if (cn > 0) {
        const int cx0 = (2 * c32) % CB;  // block-relative column of the run
        const int cbw = imin_(CB, ((f.w + 1) >> 1) - bb * CB);
        const int ystart = ovy ? imin_(1, cbh) : 0;
        const bool hfix = ovx && cx0 == 0 && cbw >= 1;  // column 0 blends with the block to the left
        int minv = 0, maxv = bdmax;
        if (d.clip_to_restricted_range) {
            minv = 16 << b8;
            maxv = (d.mc_identity ? 235 : 240) << b8;
        }
        int cbase[2][2];  // template index of block-relative (0, 0)
#pragma unroll
        for (int bxs = 0; bxs < 2; bxs++)
#pragma unroll
            for (int bys = 0; bys < 2; bys++) {
                const int *of = so.v[bl + 1 - bxs][bys];
                cbase[bxs][bys] = (3 + (3 + of[0]) + CB * bys) * GW + 3 + (3 + of[1]) + CB * bxs + cx0;
            }
#pragma unroll
        for (int uv = 0; uv < 2; uv++) {
            const bool has = uv ? gp.has_v : gp.has_u;
            const int16_t *cl = lut + (1 + uv) * GH * GW;
            const uint8_t *scl = scaling + (d.chroma_scaling_from_luma ? 0 : (1 + uv)) * 1024;
            const int lm = d.uv_luma_mult[uv], m = d.uv_mult[uv], o = d.uv_offset[uv] * (1 << b8);
            P *Gc = plane_ptr<P>(f.G[1 + uv]) + (int64_t)CY0 * uvs + CX;
#pragma unroll
            for (int k = 0; k < RC; k++) {
                const int cy = r0 * RC + k;
                if (cy >= cbh) continue;
                int out[2] = {sc[uv][k][0], sc[uv][k][1]};
                if (has) {
                    int g[2];
#pragma unroll
                    for (int e = 0; e < 2; e++) g[e] = __ldg(&cl[cbase[0][0] + cy * GW + e]);
                    if (hfix) g[0] = blend(__ldg(&cl[cbase[1][0] + cy * GW]), 23, g[0], 22, gmin, gmax);
                    if (cy < ystart) {
                        int t[2];
#pragma unroll
                        for (int e = 0; e < 2; e++) t[e] = __ldg(&cl[cbase[0][1] + cy * GW + e]);
                        if (hfix) t[0] = blend(__ldg(&cl[cbase[1][1] + cy * GW]), 23, t[0], 22, gmin, gmax);
#pragma unroll
                        for (int e = 0; e < 2; e++) g[e] = blend(t[e], 23, g[e], 22, gmin, gmax);
                    }
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        // luma row 2 cy of the band is the thread's row 2 k
                        const int avg = (sy[2 * k][2 * e] + sy[2 * k][2 * e + 1] + 1) >> 1;
                        int val = avg;
                        if (!d.chroma_scaling_from_luma) val = clip_px_(((avg * lm + sc[uv][k][e] * m) >> 6) + o, bdmax);
                        const int noise = ((int)__ldg(&scl[val]) * g[e] + srnd) >> sshift;
                        out[e] = iclip_(sc[uv][k][e] + noise, minv, maxv);
                    }
                }
                store_run<P, 2>(Gc + k * uvs, cn, vec && cn >= 2, out);
            }
        }
    }

    // ---- luma ----
    if (ln > 0) {
        const int lx0 = (4 * c32) % BS;
        const int bw = imin_(BS, f.w - bb * BS);
        const int ystart = ovy ? imin_(2, bh) : 0, xstart = ovx && lx0 == 0 ? imin_(2, bw) : 0;
        int minv = 0, maxv = bdmax;
        if (d.clip_to_restricted_range) {
            minv = 16 << b8;
            maxv = 235 << b8;
        }
        int obase[2][2];
#pragma unroll
        for (int bxs = 0; bxs < 2; bxs++)
#pragma unroll
            for (int bys = 0; bys < 2; bys++) {
                const int *of = so.v[bl + 1 - bxs][bys];
                obase[bxs][bys] = (3 + 2 * (3 + of[0]) + BS * bys) * GW + 3 + 2 * (3 + of[1]) + BS * bxs + lx0;
            }
        P *Gy = plane_ptr<P>(f.G[0]) + (int64_t)Y0 * ys + X;
#pragma unroll
        for (int k = 0; k < RL; k++) {
            const int y = r0 * RL + k;
            if (y >= bh) continue;
            int out[4] = {sy[k][0], sy[k][1], sy[k][2], sy[k][3]};
            if (gp.has_y) {
                int g[4];
#pragma unroll
                for (int e = 0; e < 4; e++) g[e] = __ldg(&lut[obase[0][0] + y * GW + e]);
                if (xstart > 0) g[0] = blend(__ldg(&lut[obase[1][0] + y * GW]), 27, g[0], 17, gmin, gmax);
                if (xstart > 1) g[1] = blend(__ldg(&lut[obase[1][0] + y * GW + 1]), 17, g[1], 27, gmin, gmax);
                if (y < ystart) {  // uniform per warp
                    int t[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) t[e] = __ldg(&lut[obase[0][1] + y * GW + e]);
                    if (xstart > 0) t[0] = blend(__ldg(&lut[obase[1][1] + y * GW]), 27, t[0], 17, gmin, gmax);
                    if (xstart > 1) t[1] = blend(__ldg(&lut[obase[1][1] + y * GW + 1]), 17, t[1], 27, gmin, gmax);
                    const int wt = y ? 17 : 27, wc = y ? 27 : 17;
#pragma unroll
                    for (int e = 0; e < 4; e++) g[e] = blend(t[e], wt, g[e], wc, gmin, gmax);
                }
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int noise = ((int)__ldg(&scaling[sy[k][e]]) * g[e] + srnd) >> sshift;
                    out[e] = iclip_(sy[k][e] + noise, minv, maxv);
                }
            }
            store_run<P, 4>(Gy + k * ys, ln, vec && ln >= 4, out);
        }
    }
}

template <typename P, int BS>
__global__ void __launch_bounds__(256, 4) grain_apply_kernel(const DevFrame f, const GrainParams gp, const int16_t *lut,
                                                          const uint8_t *scaling) {
    __shared__ SegOffsets<BS> so;
    grain_segment<P, BS>(f, gp, lut, scaling, blockIdx.y, blockIdx.x, so);
}

template <typename P>
void launch_grain_apply(const DevFrame &d, const GrainParams &gp, const int16_t *lut, const uint8_t *scaling,
                        cudaStream_t s) {
    const int bs = 16 << gp.d.block_size;
    const dim3 grid((d.w + SEG_W - 1) / SEG_W, (d.h + bs - 1) / bs);
    if (bs == 32)
        r2g_launch_pdl(grain_apply_kernel<P, 32>, grid, dim3(256), s, d, gp, lut, scaling);
    else
        r2g_launch_pdl(grain_apply_kernel<P, 16>, grid, dim3(256), s, d, gp, lut, scaling);
}

// Persistent kernels of the batched path: one template set per grained
// frame, then the apply over (grained frame << 22 | row * blocks_w + block).
__global__ void __launch_bounds__(256) grain_template_batch_kernel(BatchArgs a) {
    __shared__ GrainTplSmem sm;
    const int n = a.count[4];
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const GrainBatch &g = a.grain[i];
        if (g.any) grain_template(g.gp, a.frames[g.frame].tab, g.lut, g.scaling, sm);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256, 3) grain_apply_batch_kernel(BatchArgs a) {
    __shared__ union {
        SegOffsets<32> s32;
        SegOffsets<16> s16;
    } so;
    const int n = a.count[3];
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const uint32_t it = a.work[3][w];
        const GrainBatch &g = a.grain[it >> 22];
        const DevFrame &f = a.frames[g.frame];
        const int b = it & 0x3fffff, sw = (f.w + SEG_W - 1) / SEG_W;
        const bool hbd = f.bitdepth > 8;
        if (g.gp.d.block_size) {
            if (hbd)
                grain_segment<uint16_t, 32>(f, g.gp, g.lut, g.scaling, b / sw, b % sw, so.s32);
            else
                grain_segment<uint8_t, 32>(f, g.gp, g.lut, g.scaling, b / sw, b % sw, so.s32);
        } else {
            if (hbd)
                grain_segment<uint16_t, 16>(f, g.gp, g.lut, g.scaling, b / sw, b % sw, so.s16);
            else
                grain_segment<uint8_t, 16>(f, g.gp, g.lut, g.scaling, b / sw, b % sw, so.s16);
        }
        __syncthreads();
    }
}

// per device: the LFSR cycle tables have been copied (set with release
// order after the copies, read with acquire order)
std::atomic<bool> g_lfsr_ready[64];

}  // namespace

void r2g_batch_launch_grain_template(const BatchArgs &a, int grid, cudaStream_t s) {
    grain_template_batch_kernel<<<grid, 256, 0, s>>>(a);
}
void r2g_batch_launch_grain_apply(const BatchArgs &a, int grid, cudaStream_t s) {
    r2g_launch_pdl(grain_apply_batch_kernel, dim3(grid), dim3(256), s, a);
}
int r2g_batch_occupancy_grain_apply() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, grain_apply_batch_kernel, 256, 0);
    return nb;
}

// Per-context grain scratch: templates (3 x 73 x 82 int16) + scaling LUTs.
struct GrainCtx {
    int16_t *lut = nullptr;
    uint8_t *scaling = nullptr;
    cudaEvent_t ready = nullptr;  // templates written (side stream)
    cudaEvent_t freed = nullptr;  // last apply that read them (main stream)
    bool used = false;
};

void r2g_grain_ctx_free(R2gCtx *ctx) {
    if (!ctx->grain) return;
    r2g_dev_free(ctx, ctx->grain->lut, 3 * GH * GW * sizeof(int16_t));
    r2g_dev_free(ctx, ctx->grain->scaling, 3 * 1024);
    if (ctx->grain->ready) cudaEventDestroy(ctx->grain->ready);
    if (ctx->grain->freed) cudaEventDestroy(ctx->grain->freed);
    delete ctx->grain;
    ctx->grain = nullptr;
}

// The LFSR cycle and its inverse (see g_lfsr_cycle), for the current device.
// Host threads may reach this concurrently (contexts, batches, the DSP slot
// and the allocation-free entry point): the check-and-copy runs under one
// mutex, and the per-device flag is atomic for the lock-free fast path.
static cudaError_t init_lfsr_pow(int device) {
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (g_lfsr_ready[device].load(std::memory_order_acquire)) return cudaSuccess;
    static uint16_t cyc[65536], pos[65536];
    static bool built = false;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (g_lfsr_ready[device].load(std::memory_order_relaxed)) return cudaSuccess;
    if (!built) {
        uint32_t st = 1;
        pos[0] = 0;
        for (uint32_t i = 0; i < 65535u; i++) {
            cyc[i] = (uint16_t)st;
            pos[st] = (uint16_t)i;
            st = lfsr_step(st);
        }
        cyc[65535] = 1;
        if (st != 1) return cudaErrorInvalidValue;  // not one cycle: refuse
        built = true;
    }
    cudaError_t e = cudaMemcpyToSymbol(g_lfsr_cycle, cyc, sizeof(cyc));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_lfsr_pos, pos, sizeof(pos));
    if (e == cudaSuccess) g_lfsr_ready[device].store(true, std::memory_order_release);
    return e;
}

// decode.rs:4641-4650 picture_has_grain + filmgrain.rs:688-830 plane gating
static void grain_planes(const R2gFilmGrainData &d, int &has_y, int &has_u, int &has_v, bool &any) {
    any = d.num_points[0] || d.num_points[1] || d.num_points[2] ||
          (d.clip_to_restricted_range && d.chroma_scaling_from_luma);
    has_y = any && d.num_points[0] > 0;
    bool luma_lut = d.num_points[0] > 0;
    has_u = any && (d.num_points[1] > 0 || d.chroma_scaling_from_luma) && (!d.chroma_scaling_from_luma || luma_lut);
    has_v = any && (d.num_points[2] > 0 || d.chroma_scaling_from_luma) && (!d.chroma_scaling_from_luma || luma_lut);
}

void r2g_grain_params(const R2gFilmGrainData &fgd, uint32_t seed, int bitdepth, GrainBatch &g) {
    g.gp.d = fgd;
    g.gp.seed = seed;
    g.gp.bitdepth = bitdepth;
    g.gp.vec = 1;
    bool any;
    grain_planes(fgd, g.gp.has_y, g.gp.has_u, g.gp.has_v, any);
    g.any = any;
}

int r2g_grain_items(int width, int height, int block_size) {
    const int bs = 16 << block_size;
    return ((width + SEG_W - 1) / SEG_W) * ((height + bs - 1) / bs);
}

int r2g_grain_ready(int device) { return init_lfsr_pow(device) == cudaSuccess ? R2G_OK : R2G_E_DEVICE; }

int r2g_grain_enqueue(R2gCtx *ctx, R2gFrame *f, const R2gFilmGrainData *fgd, uint32_t seed) {
    if (init_lfsr_pow(ctx->device) != cudaSuccess) return R2G_E_DEVICE;
    if (!ctx->grain) {
        ctx->grain = new GrainCtx();
        int rc = r2g_dev_alloc(ctx, (void **)&ctx->grain->lut, 3 * GH * GW * sizeof(int16_t));
        if (rc == R2G_OK) rc = r2g_dev_alloc(ctx, (void **)&ctx->grain->scaling, 3 * 1024);
        if (rc != R2G_OK) return rc;
        if (cudaEventCreateWithFlags(&ctx->grain->ready, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->grain->freed, cudaEventDisableTiming) != cudaSuccess)
            return R2G_E_DEVICE;
    }
    GrainParams gp;
    gp.d = *fgd;
    gp.seed = seed;
    gp.bitdepth = f->bd;
    gp.vec = 1;  // frames of this library: aligned planes and strides
    bool any;
    grain_planes(*fgd, gp.has_y, gp.has_u, gp.has_v, any);
    DevFrame d = f->desc;
    void *p[3];
    char *base = (char *)f->buf[4];
    p[0] = base;
    p[1] = base + f->plane_bytes[0];
    p[2] = base + f->plane_bytes[0] + f->plane_bytes[1];
    for (int i = 0; i < 3; i++) d.G[i] = p[i];
    if (any) {
        // the templates do not depend on the frame: build them on the side
        // stream (after the previous apply stopped reading them), then join
        // before this apply
        if (ctx->grain->used && cudaStreamWaitEvent(ctx->side_stream, ctx->grain->freed, 0) != cudaSuccess)
            return R2G_E_DEVICE;
        grain_template_kernel<<<1, 256, 0, ctx->side_stream>>>(gp, ctx->tab, ctx->grain->lut, ctx->grain->scaling);
        if (cudaEventRecord(ctx->grain->ready, ctx->side_stream) != cudaSuccess) return R2G_E_DEVICE;
        if (cudaStreamWaitEvent(ctx->stream, ctx->grain->ready, 0) != cudaSuccess) return R2G_E_DEVICE;
    }
    r2g_prof_stage(ctx, 3, true, 0);
    // programmatic dependent launch: the block offsets are drawn while the
    // previous kernel of the frame drains
    if (f->bd > 8)
        launch_grain_apply<uint16_t>(d, gp, ctx->grain->lut, ctx->grain->scaling, ctx->stream);
    else
        launch_grain_apply<uint8_t>(d, gp, ctx->grain->lut, ctx->grain->scaling, ctx->stream);
    r2g_prof_stage(ctx, 3, false, 1 + (any ? 1 : 0));
    if (cudaGetLastError() != cudaSuccess) return R2G_E_DEVICE;
    if (cudaEventRecord(ctx->grain->freed, ctx->stream) != cudaSuccess) return R2G_E_DEVICE;
    ctx->grain->used = true;
    f->grain_buf = 4;
    return R2G_OK;
}

extern "C" int r2g_frame_grain(R2gCtx *ctx, R2gFrame *f, const R2gFilmGrainData *fgd, uint32_t seed) {
    if (!ctx || !f || !fgd) return R2G_E_INVALID;
    if (f->out_buf < 0) {
        ctx->err = "frame not filtered";
        return R2G_E_INVALID;
    }
    if (r2g_grain_validate(fgd, seed) != R2G_OK) {
        ctx->err = "film-grain parameters out of range";
        return R2G_E_INVALID;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return R2G_E_DEVICE;
    int rc = r2g_frame_before_compute(ctx, f);
    if (rc == R2G_OK) rc = r2g_grain_enqueue(ctx, f, fgd, seed);
    if (rc == R2G_OK) rc = r2g_frame_after_compute(ctx, f);
    return rc;
}

// ---------------------------------------------------------------------------
// Film grain without any device allocation.
//
// Some callers cannot call cudaMalloc: a decoder embedded in a host framework
// whose device memory is owned by that framework's own allocator or by a
// fixed-size pool, or a latency-critical output thread that must not block in
// the driver's allocator.  This entry point takes the caller's input and
// output planes and keeps its only scratch (the three grain templates and the
// three scaling LUTs) in a file-scope device array of fixed size, resident on
// every GPU that loads this library until the process exits.
//
// * The first call on a device (made with that device current) looks up the
//   array's device address and the constant tables; make that first call
//   before any stream capture.  Later calls do no set-up.
// * Every call on a device shares the one array, and each call rewrites every
//   scratch byte it later reads, so nothing has to start at zero.  Calls whose
//   GPU work overlaps (for example on two streams) race on the array; callers
//   must serialise them, e.g. by issuing them on one stream.
// * The array holds scaling LUTs of at most 1024 entries, i.e. bit depths up
//   to 10; larger bit depths are rejected with R2G_E_TOO_LARGE.


#define R2G_NOALLOC_LUT_BYTES (3 * GH * GW * 2)
#define R2G_NOALLOC_SCALING_BYTES (3 * 1024)
#define R2G_NOALLOC_SCRATCH_BYTES (40 * 1024)
static_assert(R2G_NOALLOC_LUT_BYTES + R2G_NOALLOC_SCALING_BYTES <= R2G_NOALLOC_SCRATCH_BYTES, "scratch too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[R2G_NOALLOC_SCRATCH_BYTES];

namespace {
struct NoallocDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch
    DevTables tab{};
};
NoallocDevice g_noalloc[64];
std::mutex g_noalloc_mu;
}  // namespace

extern "C" int r2g_film_grain_apply_noalloc(const void *src_y, const void *src_u, const void *src_v, void *dst_y,
                                            void *dst_u, void *dst_v, int64_t y_stride, int64_t uv_stride, int width,
                                            int height, int bitdepth, const R2gFilmGrainData *fgd, uint32_t seed,
                                            void *stream) {
    if (!src_y || !src_u || !src_v || !dst_y || !dst_u || !dst_v || !fgd) return R2G_E_INVALID;
    if (bitdepth > 10) return R2G_E_TOO_LARGE;  // scaling LUTs would not fit the scratch
    if (bitdepth != 8 && bitdepth != 10) return R2G_E_INVALID;
    if (width <= 0 || height <= 0 || (width & 1) || (height & 1)) return R2G_E_INVALID;
    if (r2g_grain_validate(fgd, seed) != R2G_OK) return R2G_E_INVALID;
    const int bps = bitdepth > 8 ? 2 : 1;
    if (y_stride < (int64_t)width * bps || uv_stride < (int64_t)((width + 1) >> 1) * bps || (y_stride % bps) ||
        (uv_stride % bps))
        return R2G_E_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return R2G_E_DEVICE;
    NoallocDevice &nd = g_noalloc[dev];
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!nd.ready) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return R2G_E_DEVICE;
            if (r2g_get_tables(&nd.tab) != cudaSuccess) return R2G_E_DEVICE;
            if (init_lfsr_pow(dev) != cudaSuccess) return R2G_E_DEVICE;
            nd.scratch = (unsigned char *)p;
            nd.ready = true;
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    int16_t *lut = (int16_t *)nd.scratch;
    uint8_t *scaling = nd.scratch + R2G_NOALLOC_LUT_BYTES;

    GrainParams gp;
    gp.d = *fgd;
    gp.seed = seed;
    gp.bitdepth = bitdepth;
    // runs of samples move as one vector access when every plane and stride
    // is 16-byte aligned; otherwise sample by sample
    const void *planes[6] = {src_y, src_u, src_v, dst_y, dst_u, dst_v};
    gp.vec = (y_stride % 16) == 0 && (uv_stride % 16) == 0;
    for (const void *pl : planes) gp.vec = gp.vec && ((uintptr_t)pl % 16) == 0;
    bool any;
    grain_planes(*fgd, gp.has_y, gp.has_u, gp.has_v, any);
    DevFrame d;
    memset(&d, 0, sizeof(d));
    d.w = width;
    d.h = height;
    d.cw = (width + 1) >> 1;
    d.ch = (height + 1) >> 1;
    d.bitdepth = bitdepth;
    d.bdmax = (1 << bitdepth) - 1;
    d.stride[0] = y_stride / bps;
    d.stride[1] = uv_stride / bps;
    d.L[0] = (void *)src_y;
    d.L[1] = (void *)src_u;
    d.L[2] = (void *)src_v;
    d.G[0] = dst_y;
    d.G[1] = dst_u;
    d.G[2] = dst_v;
    if (any) grain_template_kernel<<<1, 256, 0, s>>>(gp, nd.tab, lut, scaling);
    if (bitdepth > 8)
        launch_grain_apply<uint16_t>(d, gp, lut, scaling, s);
    else
        launch_grain_apply<uint8_t>(d, gp, lut, scaling, s);
    return cudaGetLastError() == cudaSuccess ? R2G_OK : R2G_E_DEVICE;
}

// DSP-context slot (r2g_dsp_generate_grain): the three grain templates of a
// parameter set on stream `s`.
void r2g_dsp_launch_grain_template(const GrainParams &gp, const DevTables &tab, int16_t *lut, uint8_t *scaling,
                                   cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    init_lfsr_pow(dev);
    grain_template_kernel<<<1, 256, 0, s>>>(gp, tab, lut, scaling);
}

// ---------------------------------------------------------------- DSP slots
// FilmGrainDSPContext.fgy_32x32xn / fguv_32x32xn[] (dsp.rs:9-16): one row
// band of blocks, as filmgrain.rs:248-407 (luma) and :409-598 (chroma) apply
// it: the per-block template offsets are drawn in order along the band by one
// thread into shared memory (seeds of this band and, with overlap, of the
// band above), then every sample takes its grain (blended across the block's
// top / left overlap) and noise from the staged template and scaling LUT.
// Planes are staged as u16 (`pitch` samples per row); `luma` holds the
// band's luma rows for chroma (NULL for luma).
namespace {
constexpr int FG_MAX_BLOCKS = 512;
__global__ void dsp_fg_band_kernel(uint16_t *dst, const uint16_t *src, int pitch, const uint16_t *luma, int lpitch,
                                   const R2gFilmGrainData data, uint32_t in_seed, int pw, const uint8_t *scaling,
                                   const int16_t *lut, int bh, int row_num, int uv, int is_id, int sx, int sy,
                                   int bitdepth) {
    __shared__ int8_t offs[FG_MAX_BLOCKS][2][2];  // [block][row of seeds][y, x]
    const int rows = 1 + (data.overlap_flag && row_num > 0);
    const int bs = 16 << data.block_size, bsx = bs >> sx;
    const int nb = (pw + bsx - 1) / bsx;
    if (threadIdx.x == 0) {
        uint32_t seed[2] = {0, 0};
        for (int i = 0; i < rows; i++) {
            seed[i] = in_seed;
            seed[i] ^= (uint32_t)((((row_num - i) * 37 + 178) & 0xff)) << 8;
            seed[i] ^= (uint32_t)(((row_num - i) * 173 + 105) & 0xff);
        }
        for (int b = 0; b < nb; b++)
            for (int i = 0; i < 2; i++)
                for (int n = 0; n < 2; n++) {
                    int v = 0;
                    if (i < rows) {
                        seed[i] = lfsr_step(seed[i]);
                        v = (int)(((uint32_t)(3 - data.block_size) * ((seed[i] >> 7) & 0x1ff)) >> 6);
                        for (int k = 0; k < 3; k++) seed[i] = lfsr_step(seed[i]);
                    }
                    offs[b][i][n] = (int8_t)v;
                }
    }
    __syncthreads();
    const int b8 = bitdepth - 8;
    const int grain_ctr = 128 << b8, grain_min = -grain_ctr, grain_max = grain_ctr - 1;
    int min_value = 0, max_value = (1 << bitdepth) - 1;
    if (data.clip_to_restricted_range) {
        min_value = 16 << b8;
        max_value = (luma && !is_id ? 240 : 235) << b8;
    }
    // blending weights: w[x] for the 2-wide overlap (27, 17 / 17, 27), or one
    // column / row when subsampled (23, 22)
    auto wgt = [](int sub, int i, int k) -> int {
        return sub ? (k == 0 ? 23 : 22) : ((i == 0) == (k == 0) ? 27 : 17);
    };
    // sample_lut (filmgrain.rs:231-246): block column `prev` (the previous
    // block) and seed row `above`
    auto grain_at = [&](int b, int prev, int above, int x, int y) -> int {
        const int ob = prev ? b - 1 : b;
        const int offx = 3 + (2 >> sx) * (3 + offs[ob][above][1]);
        const int offy = 3 + (2 >> sy) * (3 + offs[ob][above][0]);
        return lut[(offy + y + (bs >> sy) * above) * GW + offx + x + bsx * prev];
    };
    for (int i = threadIdx.x; i < pw * bh; i += blockDim.x) {
        const int y = i / pw, X = i - y * pw, b = X / bsx, x = X - b * bsx;
        const int bw = imin_(bsx, pw - b * bsx);
        const int ystart = (data.overlap_flag && row_num > 0) ? imin_(2 >> sy, bh) : 0;
        const int xstart = (data.overlap_flag && b > 0) ? imin_(2 >> sx, bw) : 0;
        int g = grain_at(b, 0, 0, x, y);
        if (x < xstart) {
            const int old = grain_at(b, 1, 0, x, y);
            g = iclip_(round2(old * wgt(sx, x, 0) + g * wgt(sx, x, 1), 5), grain_min, grain_max);
        }
        if (y < ystart) {
            int top = grain_at(b, 0, 1, x, y);
            if (x < xstart) {
                const int old = grain_at(b, 1, 1, x, y);
                top = iclip_(round2(old * wgt(sx, x, 0) + top * wgt(sx, x, 1), 5), grain_min, grain_max);
            }
            g = iclip_(round2(top * wgt(sy, y, 0) + g * wgt(sy, y, 1), 5), grain_min, grain_max);
        }
        const int sv = src[y * pitch + X];
        int val = sv;
        if (luma) {
            const int lx = X << sx, ly = y << sy;
            const int l0 = luma[ly * lpitch + lx];
            const int avg = sx ? (l0 + luma[ly * lpitch + lx + 1] + 1) >> 1 : l0;
            if (!data.chroma_scaling_from_luma) {
                const int combined = avg * data.uv_luma_mult[uv] + sv * data.uv_mult[uv];
                val = iclip_((combined >> 6) + data.uv_offset[uv] * (1 << b8), 0, (1 << bitdepth) - 1);
            } else {
                val = avg;
            }
        }
        const int noise = round2(scaling[val] * g, data.scaling_shift);
        dst[y * pitch + X] = (uint16_t)iclip_(sv + noise, min_value, max_value);
    }
}
}  // namespace

int r2g_dsp_fg_band_max_width(int block_size, int sx) { return FG_MAX_BLOCKS * ((16 << block_size) >> sx); }

void r2g_dsp_launch_fg_band(uint16_t *dst, const uint16_t *src, int pitch, const uint16_t *luma, int lpitch,
                            const R2gFilmGrainData &data, uint32_t in_seed, int pw, const uint8_t *scaling,
                            const int16_t *lut, int bh, int row_num, int uv, int is_id, int sx, int sy, int bitdepth,
                            cudaStream_t s) {
    dsp_fg_band_kernel<<<1, 256, 0, s>>>(dst, src, pitch, luma, lpitch, data, in_seed, pw, scaling, lut, bh, row_num,
                                         uv, is_id, sx, sy, bitdepth);
}
