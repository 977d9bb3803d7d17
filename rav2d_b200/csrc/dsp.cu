// DSP-context slot entry points: per-block functions with the reference's
// argument meaning and order, for the slots of DSPContext (crates/rav2d/src/
// dsp.rs:9-122) that are self-contained per call — CdefDSPContext dir / fb,
// CcsoDSPContext prep / add, LoopRestorationDSPContext gdf_add and the film
// grain template generators.  The reference declares these slots but never
// fills or calls them; its filters run through the per-frame path, which is
// this library's performance boundary too.  These entry points exist so a
// caller (or a test) can drive one block at a time: each call copies the
// block and the neighbour samples the reference would read to the GPU, runs
// one small kernel that applies the reference's padding rule and arithmetic,
// and copies the result back.  Each call is synchronous on a non-blocking
// stream the library owns on the current device, so it neither waits for nor
// delays work the caller has queued on other streams; calls are serialised
// with one another by a mutex (they share that device's scratch).  Host buffers hold u8 samples for bitdepth 8 and u16
// samples otherwise; strides count samples.
#include <cstring>
#include <mutex>
#include <vector>

#include "r2g_runtime.h"

namespace {

// Per-device scratch for the per-block calls (allocated on a device's first
// call and kept until exit) and the device tables.
struct DspDevice {
    bool ready = false;
    char *buf = nullptr;
    char *big = nullptr;  // grows for the row-band slots (film grain)
    size_t big_bytes = 0;
    cudaStream_t st = nullptr;  // non-blocking: no implicit sync with the legacy stream
    DevTables tab{};
};
constexpr size_t kScratch = 128 * 1024;
DspDevice g_dsp[64];
std::mutex g_dsp_mu;

// (called with g_dsp_mu held: every entry point holds it for its whole
// call, since the scratch of a device is shared)
int dsp_device(DspDevice **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return R2G_E_DEVICE;
    DspDevice &d = g_dsp[dev];
    if (!d.ready) {
        if (cudaMalloc((void **)&d.buf, kScratch) != cudaSuccess || r2g_get_tables(&d.tab) != cudaSuccess ||
            cudaStreamCreateWithFlags(&d.st, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return R2G_E_DEVICE;
        }
        d.ready = true;
    }
    *out = &d;
    return R2G_OK;
}

// The block (W x H) and its 2-sample ring as the reference's padding
// functions read them: rows -2, -1 from `top` (row -2 first), rows H, H + 1
// from `bottom`, columns -2, -1 of the block rows from `left` ([H][2]); only
// what the edge flags make available (1 left, 2 right, 4 top, 8 bottom) is
// read, the rest is left 0 and never used by the kernels.
template <typename P>
void gather(std::vector<uint16_t> &tile, int W, int H, const P *src, int64_t stride, const P *left, const P *top,
            const P *bottom, int edges) {
    const bool L = edges & 1, R = edges & 2, T = edges & 4, B = edges & 8;
    tile.assign((size_t)(W + 4) * (H + 4), 0);
    for (int y = -2; y < H + 2; y++)
        for (int x = -2; x < W + 2; x++) {
            const bool xin = (x >= 0 && x < W) || (x < 0 && L) || (x >= W && R);
            uint16_t v = 0;
            if (y < 0) {
                if (T && xin) v = top[(y + 2) * stride + x];
            } else if (y >= H) {
                if (B && xin) v = bottom[(y - H) * stride + x];
            } else if (x < 0) {
                if (L) v = left[y * 2 + x + 2];
            } else if (x < W || R) {
                v = src[y * stride + x];
            }
            tile[(size_t)(y + 2) * (W + 4) + x + 2] = v;
        }
}

template <typename P>
void load_block(std::vector<uint16_t> &v, const P *src, int64_t stride, int w, int h) {
    v.resize((size_t)w * h);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) v[(size_t)y * w + x] = src[y * stride + x];
}

template <typename P>
void store_block(P *dst, int64_t stride, const std::vector<uint16_t> &v, int w, int h) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) dst[y * stride + x] = (P)v[(size_t)y * w + x];
}

bool ok_bd(int bd) { return bd == 8 || bd == 10; }

int finish(const DspDevice *d, int rc);

// (called with g_dsp_mu held)
int big_scratch(DspDevice *d, size_t bytes) {
    if (d->big_bytes >= bytes) return R2G_OK;
    if (d->big) cudaFree(d->big);
    d->big = nullptr;
    d->big_bytes = 0;
    if (cudaMalloc((void **)&d->big, bytes) != cudaSuccess) {
        cudaGetLastError();
        return R2G_E_OOM;
    }
    d->big_bytes = bytes;
    return R2G_OK;
}

// rows x w samples of a plane (u8 or u16) as u16, or false if one exceeds
// the bit depth's range (the scaling LUT has 1 << bitdepth entries)
bool stage_rows(std::vector<uint16_t> &v, const void *src, int64_t stride, int w, int rows, int bitdepth) {
    v.resize((size_t)w * rows);
    const int bdmax = (1 << bitdepth) - 1;
    for (int y = 0; y < rows; y++)
        for (int x = 0; x < w; x++) {
            const int s = bitdepth > 8 ? ((const uint16_t *)src)[y * stride + x] : ((const uint8_t *)src)[y * stride + x];
            if (s > bdmax) return false;
            v[(size_t)y * w + x] = (uint16_t)s;
        }
    return true;
}

// One row band of film grain (fgy_32x32xn / fguv_32x32xn): stage, run, and
// write the band back.
int fg_band(void *dst, const void *src, int64_t stride, const R2gFilmGrainData *data, uint32_t in_seed, int pw,
            const uint8_t *scaling, const int16_t *grain_lut, int bh, int row_num, const void *luma_row,
            int64_t luma_stride, int uv, int is_id, int sx, int sy, int bitdepth) {
    if (!dst || !src || !data || !scaling || !grain_lut || !ok_bd(bitdepth) || pw <= 0 || bh <= 0 || row_num < 0 ||
        in_seed > 0xffff || data->block_size < 0 || data->block_size > 1 || data->scaling_shift < 8 ||
        data->scaling_shift > 11 || bh > ((16 << data->block_size) >> sy) || sx < 0 || sx > 1 || sy < 0 || sy > 1 ||
        (luma_row && uv > 1) || pw > r2g_dsp_fg_band_max_width(data->block_size, sx) ||
        (luma_row == nullptr) != (uv < 0))
        return R2G_E_INVALID;
    std::vector<uint16_t> s16, l16;
    if (!stage_rows(s16, src, stride, pw, bh, bitdepth)) return R2G_E_INVALID;
    const int lw = pw << sx, lh = bh << sy;
    if (luma_row && !stage_rows(l16, luma_row, luma_stride, lw, lh, bitdepth)) return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    const size_t plane = s16.size() * 2, lbytes = l16.size() * 2, lut_bytes = 73 * 82 * 2, sc = (size_t)1 << bitdepth;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    if ((rc = big_scratch(d, 2 * al(plane) + al(lbytes) + al(lut_bytes) + al(sc))) != R2G_OK) return rc;
    uint16_t *dsrc = (uint16_t *)d->big, *ddst = (uint16_t *)(d->big + al(plane));
    uint16_t *dl = (uint16_t *)(d->big + 2 * al(plane));
    int16_t *dlut = (int16_t *)(d->big + 2 * al(plane) + al(lbytes));
    uint8_t *dsc = (uint8_t *)(d->big + 2 * al(plane) + al(lbytes) + al(lut_bytes));
    if (cudaMemcpyAsync(dsrc, s16.data(), plane, cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        (lbytes && cudaMemcpyAsync(dl, l16.data(), lbytes, cudaMemcpyHostToDevice, d->st) != cudaSuccess) ||
        cudaMemcpyAsync(dlut, grain_lut, lut_bytes, cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(dsc, scaling, sc, cudaMemcpyHostToDevice, d->st) != cudaSuccess)
        return R2G_E_DEVICE;
    r2g_dsp_launch_fg_band(ddst, dsrc, pw, luma_row ? dl : nullptr, lw, *data, in_seed, pw, dsc, dlut, bh, row_num,
                           uv < 0 ? 0 : uv, is_id, sx, sy, bitdepth, d->st);
    if (cudaMemcpyAsync(s16.data(), ddst, plane, cudaMemcpyDeviceToHost, d->st) != cudaSuccess) return R2G_E_DEVICE;
    if ((rc = finish(d, R2G_OK)) != R2G_OK) return rc;
    if (bitdepth > 8)
        store_block((uint16_t *)dst, stride, s16, pw, bh);
    else
        store_block((uint8_t *)dst, stride, s16, pw, bh);
    return R2G_OK;
}

int finish(const DspDevice *d, int rc) {
    if (rc != R2G_OK) return rc;
    return cudaStreamSynchronize(d->st) == cudaSuccess && cudaGetLastError() == cudaSuccess ? R2G_OK : R2G_E_DEVICE;
}

}  // namespace

// DeblockDSPContext.deblock_sb[vert ? 0 : 1][luma ? 0 : 1]: deblock_{h,v}_
// sb64{y,uv}_bd (deblock.rs:303-548).  `dst` is the first positive-side
// sample of line 0 (the reference's dst + dst_off); with `vert` the edge is
// vertical and its lines run down the rows, else horizontal along the
// columns.  The lines of every segment up to the highest class bit, and the
// samples across the edge the filters can reach (8 per side for luma, 6 for
// chroma), are staged, filtered and written back.
extern "C" int r2g_dsp_deblock_sb64(void *dst, int64_t stride, const uint16_t *vmask, const uint16_t *ll_mask,
                                    const uint16_t *q_thr, const uint16_t *side_thr, int edge, int luma, int vert,
                                    int bitdepth) {
    if (!dst || !vmask || !ll_mask || !q_thr || !side_thr || stride <= 0 || !ok_bd(bitdepth)) return R2G_E_INVALID;
    const uint32_t vm = (uint32_t)vmask[0] | vmask[1] | vmask[2] | (luma ? vmask[3] : 0);
    if (!vm) return R2G_OK;
    const int nseg = 32 - __builtin_clz(vm), nlines = 4 * nseg;
    const int reach = luma ? 8 : 6;
    const int64_t along = vert ? stride : 1, across = vert ? 1 : stride;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    std::vector<int16_t> strip((size_t)nlines * 16, 0);
    for (int l = 0; l < nlines; l++)
        for (int j = -reach; j < reach; j++) {
            const int64_t o = l * along + j * across;
            strip[(size_t)l * 16 + 8 + j] = (int16_t)(bitdepth > 8 ? ((const uint16_t *)dst)[o] : ((const uint8_t *)dst)[o]);
        }
    uint16_t thr[32];
    for (int i = 0; i < 16; i++) {
        thr[i] = i < nseg ? q_thr[i] : 0;
        thr[16 + i] = i < nseg ? side_thr[i] : 0;
    }
    int16_t *dstrip = (int16_t *)d->buf;
    uint16_t *dthr = (uint16_t *)(d->buf + 4096);
    if (cudaMemcpyAsync(dstrip, strip.data(), strip.size() * 2, cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(dthr, thr, sizeof(thr), cudaMemcpyHostToDevice, d->st) != cudaSuccess)
        return R2G_E_DEVICE;
    r2g_dsp_launch_deblock_sb64(dstrip, vmask, ll_mask, dthr, edge != 0, luma != 0, bitdepth, d->st);
    if (cudaMemcpyAsync(strip.data(), dstrip, strip.size() * 2, cudaMemcpyDeviceToHost, d->st) != cudaSuccess)
        return R2G_E_DEVICE;
    rc = finish(d, R2G_OK);
    if (rc != R2G_OK) return rc;
    for (int l = 0; l < nlines; l++)
        for (int j = -reach; j < reach; j++) {
            const int64_t o = l * along + j * across;
            const int16_t v = strip[(size_t)l * 16 + 8 + j];
            if (bitdepth > 8)
                ((uint16_t *)dst)[o] = (uint16_t)v;
            else
                ((uint8_t *)dst)[o] = (uint8_t)v;
        }
    return R2G_OK;
}

// FilmGrainDSPContext.fgy_32x32xn (filmgrain.rs:248-407) and fguv_32x32xn
// (:409-598) on one row band of the caller's planes.
extern "C" int r2g_dsp_fgy_32x32xn(void *dst, const void *src, int64_t stride, const R2gFilmGrainData *data,
                                   uint32_t in_seed, int pw, const uint8_t *scaling, const int16_t *grain_lut, int bh,
                                   int row_num, int bitdepth) {
    return fg_band(dst, src, stride, data, in_seed, pw, scaling, grain_lut, bh, row_num, nullptr, 0, -1, 0, 0, 0,
                   bitdepth);
}
extern "C" int r2g_dsp_fguv_32x32xn(void *dst, const void *src, int64_t stride, const R2gFilmGrainData *data,
                                    uint32_t in_seed, int pw, const uint8_t *scaling, const int16_t *grain_lut, int bh,
                                    int row_num, const void *luma_row, int64_t luma_stride, int uv, int is_id, int sx,
                                    int sy, int bitdepth) {
    if (uv < 0 || !luma_row) return R2G_E_INVALID;
    return fg_band(dst, src, stride, data, in_seed, pw, scaling, grain_lut, bh, row_num, luma_row, luma_stride, uv,
                   is_id, sx, sy, bitdepth);
}

extern "C" int r2g_dsp_cdef_dir(const void *img, int64_t stride, uint32_t *var, int bitdepth) {
    if (!img || !var || !ok_bd(bitdepth)) return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    std::vector<uint16_t> blk;
    if (bitdepth > 8)
        load_block(blk, (const uint16_t *)img, stride, 8, 8);
    else
        load_block(blk, (const uint8_t *)img, stride, 8, 8);
    uint16_t *dblk = (uint16_t *)d->buf;
    uint32_t *dout = (uint32_t *)(d->buf + 256);
    if (cudaMemcpyAsync(dblk, blk.data(), 128, cudaMemcpyHostToDevice, d->st) != cudaSuccess) return R2G_E_DEVICE;
    r2g_dsp_launch_cdef_dir(dblk, bitdepth, dout, d->st);
    uint32_t out[2];
    if (cudaMemcpyAsync(out, dout, sizeof(out), cudaMemcpyDeviceToHost, d->st) != cudaSuccess) return R2G_E_DEVICE;
    *var = out[1];
    return (int)out[0];
}

extern "C" int r2g_dsp_cdef_filter(void *dst, int64_t stride, const void *left, const void *top, const void *bottom,
                                   int pri, int sec, int dir, int damping, int w, int h, int edges, int bitdepth) {
    if (!dst || !ok_bd(bitdepth) || !((w == 8 && h == 8) || (w == 4 && h == 8) || (w == 4 && h == 4)) || dir < 0 ||
        dir > 7 || ((edges & 1) && !left) || ((edges & 4) && !top) || ((edges & 8) && !bottom))
        return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    std::vector<uint16_t> tile;
    if (bitdepth > 8)
        gather(tile, w, h, (const uint16_t *)dst, stride, (const uint16_t *)left, (const uint16_t *)top,
               (const uint16_t *)bottom, edges);
    else
        gather(tile, w, h, (const uint8_t *)dst, stride, (const uint8_t *)left, (const uint8_t *)top,
               (const uint8_t *)bottom, edges);
    uint16_t *dtile = (uint16_t *)d->buf, *dout = (uint16_t *)(d->buf + 1024);
    if (cudaMemcpyAsync(dtile, tile.data(), tile.size() * 2, cudaMemcpyHostToDevice, d->st) != cudaSuccess) return R2G_E_DEVICE;
    r2g_dsp_launch_cdef_filter(dtile, w, h, edges, pri, sec, dir, damping, bitdepth, d->tab, dout, d->st);
    std::vector<uint16_t> out((size_t)w * h);
    if (cudaMemcpyAsync(out.data(), dout, out.size() * 2, cudaMemcpyDeviceToHost, d->st) != cudaSuccess) return R2G_E_DEVICE;
    if (bitdepth > 8)
        store_block((uint16_t *)dst, stride, out, w, h);
    else
        store_block((uint8_t *)dst, stride, out, w, h);
    return finish(d, R2G_OK);
}

extern "C" int r2g_dsp_ccso_prep(uint8_t *dst, int64_t dst_stride, const void *src, int64_t stride, const void *left,
                                 const void *top, const void *bottom, int max_band_log2, int ext_filter,
                                 int quant_step, int edge_clf, int bo_only, int edges, int w, int h, int ss_hor,
                                 int ss_ver, int bitdepth) {
    const int W = w << ss_hor, H = h << ss_ver;
    if (!dst || !src || !ok_bd(bitdepth) || w <= 0 || h <= 0 || W > 64 || H > 32 || ss_hor < 0 || ss_hor > 1 ||
        ss_ver < 0 || ss_ver > 1 || ext_filter < 0 || ext_filter > 6 || max_band_log2 < 0 ||
        max_band_log2 > bitdepth || ((edges & 1) && !left) || ((edges & 4) && !top) || ((edges & 8) && !bottom))
        return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    std::vector<uint16_t> tile;
    if (bitdepth > 8)
        gather(tile, W, H, (const uint16_t *)src, stride, (const uint16_t *)left, (const uint16_t *)top,
               (const uint16_t *)bottom, edges);
    else
        gather(tile, W, H, (const uint8_t *)src, stride, (const uint8_t *)left, (const uint8_t *)top,
               (const uint8_t *)bottom, edges);
    uint16_t *dtile = (uint16_t *)d->buf;
    uint8_t *dout = (uint8_t *)(d->buf + 32 * 1024);
    if (cudaMemcpyAsync(dtile, tile.data(), tile.size() * 2, cudaMemcpyHostToDevice, d->st) != cudaSuccess) return R2G_E_DEVICE;
    r2g_dsp_launch_ccso_prep(dtile, w, h, ss_hor, ss_ver, edges, max_band_log2, ext_filter, quant_step, edge_clf,
                             bo_only, bitdepth, dout, d->st);
    std::vector<uint8_t> out((size_t)w * h);
    if (cudaMemcpyAsync(out.data(), dout, out.size(), cudaMemcpyDeviceToHost, d->st) != cudaSuccess) return R2G_E_DEVICE;
    for (int y = 0; y < h; y++) memcpy(dst + y * dst_stride, &out[(size_t)y * w], (size_t)w);
    return finish(d, R2G_OK);
}

extern "C" int r2g_dsp_ccso_add(void *dst, int64_t dst_stride, const uint8_t *idx, int64_t idx_stride,
                                const uint8_t *offset_idxs, const int8_t *offset_lut, int w, int h,
                                const uint16_t *ll_mask, int bitdepth) {
    if (!dst || !idx || !offset_idxs || !offset_lut || !ll_mask || !ok_bd(bitdepth) || w <= 0 || h <= 0 || w > 64 ||
        h > 64 || (w & 3) || (h & 3))
        return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    std::vector<uint16_t> px;
    if (bitdepth > 8)
        load_block(px, (const uint16_t *)dst, dst_stride, w, h);
    else
        load_block(px, (const uint8_t *)dst, dst_stride, w, h);
    std::vector<uint8_t> id((size_t)w * h);
    for (int y = 0; y < h; y++) memcpy(&id[(size_t)y * w], idx + y * idx_stride, (size_t)w);
    uint16_t *dpx = (uint16_t *)d->buf;
    uint8_t *did = (uint8_t *)(d->buf + 8192), *doffs = (uint8_t *)(d->buf + 12288);
    int8_t *dlut = (int8_t *)(d->buf + 12416);
    uint16_t *dllm = (uint16_t *)(d->buf + 12544);
    if (cudaMemcpyAsync(dpx, px.data(), px.size() * 2, cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(did, id.data(), id.size(), cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(doffs, offset_idxs, 64, cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(dlut, offset_lut, 8, cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(dllm, ll_mask, (size_t)(h / 4) * 4 * sizeof(uint16_t), cudaMemcpyHostToDevice, d->st) != cudaSuccess)
        return R2G_E_DEVICE;
    r2g_dsp_launch_ccso_add(dpx, did, doffs, dlut, w, h, dllm, (1 << bitdepth) - 1, d->st);
    if (cudaMemcpyAsync(px.data(), dpx, px.size() * 2, cudaMemcpyDeviceToHost, d->st) != cudaSuccess) return R2G_E_DEVICE;
    if (bitdepth > 8)
        store_block((uint16_t *)dst, dst_stride, px, w, h);
    else
        store_block((uint8_t *)dst, dst_stride, px, w, h);
    return finish(d, R2G_OK);
}

extern "C" int r2g_dsp_gdf_add(void *p, int64_t stride, const int8_t *err, int64_t err_stride, int w, int h,
                               int scale, const uint16_t *ll_mask, int bitdepth) {
    if (!p || !err || !ll_mask || !ok_bd(bitdepth) || w <= 0 || h <= 0 || w > 64 || h > 64) return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    std::vector<uint16_t> px;
    if (bitdepth > 8)
        load_block(px, (const uint16_t *)p, stride, w, h);
    else
        load_block(px, (const uint8_t *)p, stride, w, h);
    std::vector<int8_t> e((size_t)w * h);
    for (int y = 0; y < h; y++) memcpy(&e[(size_t)y * w], err + y * err_stride, (size_t)w);
    uint16_t *dpx = (uint16_t *)d->buf;
    int8_t *derr = (int8_t *)(d->buf + 8192);
    uint16_t *dllm = (uint16_t *)(d->buf + 12288);
    if (cudaMemcpyAsync(dpx, px.data(), px.size() * 2, cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(derr, e.data(), e.size(), cudaMemcpyHostToDevice, d->st) != cudaSuccess ||
        cudaMemcpyAsync(dllm, ll_mask, (size_t)(h / 4) * 4 * sizeof(uint16_t), cudaMemcpyHostToDevice, d->st) != cudaSuccess)
        return R2G_E_DEVICE;
    r2g_dsp_launch_gdf_add(dpx, derr, w, h, scale, dllm, bitdepth, d->st);
    if (cudaMemcpyAsync(px.data(), dpx, px.size() * 2, cudaMemcpyDeviceToHost, d->st) != cudaSuccess) return R2G_E_DEVICE;
    if (bitdepth > 8)
        store_block((uint16_t *)p, stride, px, w, h);
    else
        store_block((uint8_t *)p, stride, px, w, h);
    return finish(d, R2G_OK);
}

extern "C" int r2g_dsp_generate_grain(int16_t *buf_y, int16_t *buf_u, int16_t *buf_v, const R2gFilmGrainData *fgd,
                                      uint32_t seed, int bitdepth) {
    if (!fgd || !ok_bd(bitdepth) || fgd->ar_coeff_lag < 0 || fgd->ar_coeff_lag > 3 || seed > 0xffff)
        return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    // generate_grain_uv is computed for both chroma planes whatever the
    // scaling points (the template does not depend on them)
    GrainParams gp;
    gp.d = *fgd;
    gp.d.chroma_scaling_from_luma = 1;
    gp.seed = seed;
    gp.bitdepth = bitdepth;
    gp.has_y = gp.has_u = gp.has_v = 1;
    gp.vec = 0;
    const size_t plane = 73 * 82;
    int16_t *lut = (int16_t *)d->buf;
    uint8_t *scaling = (uint8_t *)(d->buf + 3 * plane * sizeof(int16_t));
    r2g_dsp_launch_grain_template(gp, d->tab, lut, scaling, d->st);
    int16_t *dst[3] = {buf_y, buf_u, buf_v};
    for (int pl = 0; pl < 3; pl++)
        if (dst[pl] && cudaMemcpyAsync(dst[pl], lut + pl * plane, plane * sizeof(int16_t), cudaMemcpyDeviceToHost, d->st) !=
                           cudaSuccess)
            return R2G_E_DEVICE;
    return finish(d, R2G_OK);
}

// ---------------------------------------------------------------------------
// Typed loop-restoration slots (WienerFilterFn / GdfPrepFn,
// looprestoration.rs:1716-1768).  The reference's per-block functions keep a
// ring of backed-up rows (each row with edge_len samples of left / right
// context, filled from `left`, the unit to the right, the saved deblocked
// rows or by replication) and move ring pointers as they walk down the
// block.  The host stages every row the ring would hold, in the order the
// reference builds them, and records which staged row each ring slot points
// at for every output row; the GPU then does all the arithmetic.

namespace {

enum { LRE_LEFT = 1, LRE_RIGHT = 2, LRE_TOP = 4, LRE_BOTTOM = 8 };

// Staged rows: `n` rows of (w + 2e) samples, column 0 of the block at e.
struct RowStage {
    int w = 0, e = 0, rs = 0, n = 0;
    std::vector<uint16_t> data;
    RowStage(int w_, int e_) : w(w_), e(e_), rs(w_ + 2 * e_) {}
    int add() {
        data.resize(data.size() + rs, 0);
        return n++;
    }
    uint16_t *row(int id) { return &data[(size_t)id * rs + e]; }
};

// backup_row (looprestoration.rs:54-80): src row at column 0, left[6]
template <typename P>
int stage_row(RowStage &st, const P *src, const P *left6, int edge_len, int edges) {
    const int id = st.add();
    uint16_t *d = st.row(id);
    for (int x = 0; x < edge_len; x++) d[x - edge_len] = (edges & LRE_LEFT) ? left6[6 - edge_len + x] : src[0];
    for (int x = 0; x < st.w; x++) d[x] = src[x];
    for (int x = 0; x < edge_len; x++) d[st.w + x] = (edges & LRE_RIGHT) ? src[st.w + x] : src[st.w - 1];
    return id;
}

// backup_row_lpf (:85-108): a saved row, its own left / right context
template <typename P>
int stage_row_lpf(RowStage &st, const P *src, int edge_len, int edges) {
    const int id = st.add();
    uint16_t *d = st.row(id);
    for (int x = 0; x < edge_len; x++) d[x - edge_len] = (edges & LRE_LEFT) ? src[x - edge_len] : src[0];
    for (int x = 0; x < st.w; x++) d[x] = src[x];
    for (int x = 0; x < edge_len; x++) d[st.w + x] = (edges & LRE_RIGHT) ? src[st.w + x] : src[st.w - 1];
    return id;
}

// backup_row_luma (:408-522, 4:2:0 and 4:4:4 arms): one downsampled luma
// row from rows src and src + src_stride (st.w = the luma width)
template <typename P>
int stage_row_luma(RowStage &st, const P *src, int64_t src_stride, int edges, int ss_hor, int ss_ver, int ds) {
    if (ss_ver == 0) return stage_row_lpf(st, src, 4, edges);
    const int id = st.add();
    uint16_t *d = st.row(id);
    const int w = st.w;
    const P *s2 = src + src_stride;
    auto sample = [&](int x) -> int {
        if (ds == 0) return ((int)src[x] + s2[x] + src[x + 1] + s2[x + 1]) >> 2;
        if (ds == 1) return ((int)src[x] + s2[x]) >> 1;
        return src[x];
    };
    if (ds == 0) {
        for (int x = 0; x < w; x += 1 + ss_hor) d[x] = (uint16_t)sample(x);
    } else {
        for (int x = 0; x < w; x++) d[x] = (uint16_t)sample(x);
    }
    for (int i = 0; i < 4; i++) d[i - 4] = (edges & LRE_LEFT) ? (uint16_t)sample(i - 4) : d[0];
    for (int i = 0; i < 4; i++) d[w + i] = (edges & LRE_RIGHT) ? (uint16_t)sample(w + i) : d[w - 2];
    return id;
}

// ns_wiener_single_y / wiener_multi row walk (:524-713, :715-1059): FIR
// ring slots [h][9] and, for the multi-class kinds, the classification
// slots [h/4][10].
template <typename P>
void stage_wiener_y(RowStage &st, const P *p, int64_t stride, const P *left, const P *top, const P *bottom, int h,
                    int edges, bool multi, std::vector<int> &ref, std::vector<int> &cref) {
    auto row = [&](int y) { return stage_row(st, p + y * stride, left + 6 * y, 4, edges); };
    int ptrs[10] = {0};
    ptrs[4] = row(0);
    if (edges & LRE_TOP) {
        ptrs[2] = stage_row_lpf(st, top, 4, edges);
        ptrs[3] = stage_row_lpf(st, top + stride, 4, edges);
        ptrs[0] = ptrs[1] = ptrs[2];
    } else {
        ptrs[0] = ptrs[1] = ptrs[2] = ptrs[3] = ptrs[4];
    }
    ptrs[5] = row(1);
    ptrs[6] = row(2);
    ptrs[7] = row(3);
    ref.assign((size_t)h * 9, 0);
    cref.assign((size_t)(h >> 2) * 10, 0);
    auto fir_row = [&](int y) {
        if (y + 4 < h)
            ptrs[8] = row(y + 4);
        else if (y + 2 < h && (edges & LRE_BOTTOM))
            ptrs[8] = stage_row_lpf(st, bottom + (y + 4 - h) * stride, 4, edges);
        else
            ptrs[8] = ptrs[7];
        for (int i = 0; i < 9; i++) ref[(size_t)y * 9 + i] = ptrs[i];
        for (int r = 0; r < 8; r++) ptrs[r] = ptrs[r + 1];
    };
    if (!multi) {
        for (int y = 0; y < h; y++) fir_row(y);
        return;
    }
    const int bh = h >> 2;
    for (int by = 0; by < bh; by++) {
        const int by4 = by << 2;
        if (by + 1 < bh) {
            ptrs[8] = row(by4 + 4);
            ptrs[9] = row(by4 + 5);
        } else if (edges & LRE_BOTTOM) {
            ptrs[8] = stage_row_lpf(st, bottom, 4, edges);
            ptrs[9] = stage_row_lpf(st, bottom + stride, 4, edges);
        } else {
            ptrs[8] = ptrs[9] = ptrs[7];
        }
        for (int i = 0; i < 10; i++) cref[(size_t)by * 10 + i] = ptrs[i];
        for (int y = by4; y < by4 + 4; y++) fir_row(y);
    }
}

// gdf_prep row walk (:1456-1560): gradient events (the initial one, then one
// per even row) and per output row slots [h][13]
template <typename P>
void stage_gdf(RowStage &st, const P *p, int64_t stride, const P *left, const P *top, const P *bottom, int h,
               int edges, std::vector<int> &gref, std::vector<int> &pref) {
    auto row = [&](int y) { return stage_row(st, p + y * stride, left + 6 * y, 6, edges); };
    int ptrs[13] = {0};
    ptrs[6] = row(0);
    if (edges & LRE_TOP) {
        ptrs[4] = stage_row_lpf(st, top, 6, edges);
        ptrs[5] = stage_row_lpf(st, top + stride, 6, edges);
        ptrs[0] = ptrs[1] = ptrs[2] = ptrs[3] = ptrs[4];
    } else {
        for (int n = 0; n < 6; n++) ptrs[n] = ptrs[6];
    }
    for (int y = 1; y < 6; y++) ptrs[6 + y] = row(y);
    gref.assign(ptrs, ptrs + 13);
    pref.assign((size_t)h * 13, 0);
    for (int y = 0; y < h; y++) {
        if (y + 6 < h)
            ptrs[12] = row(y + 6);
        else if (y + 4 < h && (edges & LRE_BOTTOM))
            ptrs[12] = stage_row_lpf(st, bottom + (y + 6 - h) * stride, 6, edges);
        else
            ptrs[12] = ptrs[11];
        if ((y & 1) == 0) gref.insert(gref.end(), ptrs, ptrs + 13);
        for (int i = 0; i < 13; i++) pref[(size_t)y * 13 + i] = ptrs[i];
        for (int r = 0; r < 12; r++) ptrs[r] = ptrs[r + 1];
    }
}

// ns_wiener_single_uv row walk (:1145-1430): chroma slots and downsampled
// luma slots [h][5]
template <typename P>
void stage_wiener_uv(RowStage &cs, RowStage &ls, const P *p, int64_t stride, const P *left, const P *top,
                     const P *bottom, int h, int edges, const R2gWienerParamsSingle &sp, std::vector<int> &cref,
                     std::vector<int> &lref) {
    const P *luma = (const P *)sp.luma, *ltop = (const P *)sp.luma_top, *lbot = (const P *)sp.luma_bottom;
    const int64_t lstride = sp.stride;
    const int ssh = sp.ss_hor, ssv = sp.ss_ver, ds = sp.ds_flt;
    auto crow = [&](int y) { return stage_row(cs, p + y * stride, left + 6 * y, 2, edges); };
    auto lrow = [&](const P *src, int64_t s2) { return stage_row_luma(ls, src, s2, edges, ssh, ssv, ds); };
    int c[5] = {0}, l[5] = {0};
    c[2] = crow(0);
    if (edges & LRE_TOP) {
        c[0] = stage_row_lpf(cs, top, 2, edges);
        c[1] = stage_row_lpf(cs, top + stride, 2, edges);
    } else {
        c[0] = c[1] = c[2];
    }
    c[3] = crow(1);
    l[2] = lrow(luma, lstride);
    if (edges & LRE_TOP) {
        l[0] = lrow(ltop, 0);
        l[1] = lrow(ltop, lstride);
    } else {
        l[0] = l[1] = l[2];
    }
    l[3] = lrow(luma + ((int64_t)1 << ssv) * lstride, lstride);
    cref.assign((size_t)h * 5, 0);
    lref.assign((size_t)h * 5, 0);
    int64_t luma_pos = 0;
    for (int y = 0; y < h; y++) {
        if (y + 2 < h)
            c[4] = crow(y + 2);
        else if (edges & LRE_BOTTOM)
            c[4] = stage_row_lpf(cs, bottom + (y + 2 - h) * stride, 2, edges);
        else
            c[4] = c[3];
        if (c[4] == c[3])
            l[4] = l[3];
        else if (y + 2 == h)
            l[4] = lrow(lbot, lstride);
        else if (y + 1 == h)
            l[4] = lrow(lbot + lstride, 0);
        else
            l[4] = lrow(luma + luma_pos + ((int64_t)2 << ssv) * lstride, lstride);
        for (int i = 0; i < 5; i++) {
            cref[(size_t)y * 5 + i] = c[i];
            lref[(size_t)y * 5 + i] = l[i];
        }
        for (int r = 0; r < 4; r++) {
            c[r] = c[r + 1];
            l[r] = l[r + 1];
        }
        luma_pos += lstride << ssv;
    }
}

// Device scratch layout of one typed-LR call, 256-byte aligned pieces.
struct Scratch {
    char *base;
    size_t off = 0, cap;
    template <typename T>
    T *take(size_t n) {
        T *p = (T *)(base + off);
        off = (off + n * sizeof(T) + 255) & ~(size_t)255;
        return off <= cap ? p : nullptr;
    }
};

bool lr_dims_ok(int w, int h, int wmul, int hmin) {
    return w >= 4 && h >= hmin && w <= 64 && h <= 64 && (w % wmul) == 0 && (h & 1) == 0;
}

template <typename P>
void load_rect(std::vector<uint16_t> &v, const P *src, int64_t stride, int w, int h) {
    v.resize((size_t)w * h);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) v[(size_t)y * w + x] = src[y * stride + x];
}

// Common path of the three luma Wiener slots.
template <typename P>
int wiener_y(DspDevice *d, void *dst, int64_t stride, const void *left, const void *top, const void *bottom, int w,
             int h, const R2gWienerParams *params, int edges, const uint16_t *ll_mask, int bitdepth, int kind) {
    RowStage st(w, 4);
    std::vector<int> ref, cref;
    stage_wiener_y<P>(st, (const P *)dst, stride, (const P *)left, (const P *)top, (const P *)bottom, h, edges,
                      kind != 1, ref, cref);
    const int bh = h >> 2;
    // classes the multi-class kinds can select: the largest value in the
    // subclass LUT bounds the caller's filter table
    int nclass = 1;
    std::vector<uint8_t> lut(256, 0);
    std::vector<uint16_t> noskip(bh, 0);
    if (kind != 1) {
        memcpy(lut.data(), params->multi.subclass_lut, 256);
        for (uint8_t v : lut) nclass = v + 1 > nclass ? v + 1 : nclass;
        memcpy(noskip.data(), params->multi.noskip_mask, sizeof(uint16_t) * bh);
    }
    Scratch sc{d->buf, 0, kScratch};
    uint16_t *drows = sc.take<uint16_t>(st.data.size());
    int *dref = sc.take<int>(ref.size()), *dcref = sc.take<int>(cref.size() + 1);
    int8_t *dtaps = sc.take<int8_t>(16 * 18);
    int16_t *dpcf = sc.take<int16_t>(64 * 13);
    uint8_t *dlut = sc.take<uint8_t>(256);
    uint16_t *dns = sc.take<uint16_t>(bh + 1), *dllm = sc.take<uint16_t>((bh + 1) * 4);
    uint16_t *dout = sc.take<uint16_t>((size_t)w * h);
    if (!dout) return R2G_E_TOO_LARGE;
    int taps_stride = 18;
    cudaStream_t s = d->st;
    bool ok = cudaMemcpyAsync(drows, st.data.data(), st.data.size() * 2, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(dref, ref.data(), ref.size() * 4, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(dllm, ll_mask, (bh + 1) * 4 * 2, cudaMemcpyHostToDevice, s) == cudaSuccess;
    if (kind == 1) {
        ok = ok && cudaMemcpyAsync(dtaps, params->single.filter, 16, cudaMemcpyHostToDevice, s) == cudaSuccess;
    } else {
        ok = ok && cudaMemcpyAsync(dcref, cref.data(), cref.size() * 4, cudaMemcpyHostToDevice, s) == cudaSuccess &&
             cudaMemcpyAsync(dlut, lut.data(), 256, cudaMemcpyHostToDevice, s) == cudaSuccess &&
             cudaMemcpyAsync(dns, noskip.data(), bh * 2, cudaMemcpyHostToDevice, s) == cudaSuccess;
        if (kind == 2)
            ok = ok && nclass <= 16 &&
                 cudaMemcpyAsync(dtaps, params->multi.filters, (size_t)nclass * 18, cudaMemcpyHostToDevice, s) ==
                     cudaSuccess;
        else
            ok = ok && nclass <= 64 &&
                 cudaMemcpyAsync(dpcf, params->multi.filters, (size_t)nclass * 13 * 2, cudaMemcpyHostToDevice, s) ==
                     cudaSuccess;
    }
    if (!ok) return R2G_E_INVALID;
    r2g_dsp_launch_wiener_y(drows, st.rs, st.e, dref, dcref, w, h, kind, dtaps, taps_stride, dpcf, dlut, dns,
                            kind == 1 ? 0 : params->multi.base_q, dllm, bitdepth, d->tab, dout, s);
    std::vector<uint16_t> out((size_t)w * h);
    if (cudaMemcpyAsync(out.data(), dout, out.size() * 2, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return R2G_E_DEVICE;
    store_block((P *)dst, stride, out, w, h);
    return R2G_OK;
}

template <typename P>
int wiener_uv(DspDevice *d, void *dst, int64_t stride, const void *left, const void *top, const void *bottom, int w,
              int h, const R2gWienerParams *params, int edges, const uint16_t *ll_mask, int bitdepth) {
    const R2gWienerParamsSingle &sp = params->single;
    RowStage cs(w, 2), ls(w << sp.ss_hor, 4);
    std::vector<int> cref, lref;
    stage_wiener_uv<P>(cs, ls, (const P *)dst, stride, (const P *)left, (const P *)top, (const P *)bottom, h, edges,
                       sp, cref, lref);
    const int bh = h >> 2;
    Scratch sc{d->buf, 0, kScratch};
    uint16_t *dc = sc.take<uint16_t>(cs.data.size()), *dl = sc.take<uint16_t>(ls.data.size());
    int *dcr = sc.take<int>(cref.size()), *dlr = sc.take<int>(lref.size());
    int8_t *df = sc.take<int8_t>(18);
    uint16_t *dllm = sc.take<uint16_t>((bh + 1) * 4), *dout = sc.take<uint16_t>((size_t)w * h);
    if (!dout) return R2G_E_TOO_LARGE;
    cudaStream_t s = d->st;
    if (cudaMemcpyAsync(dc, cs.data.data(), cs.data.size() * 2, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dl, ls.data.data(), ls.data.size() * 2, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dcr, cref.data(), cref.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dlr, lref.data(), lref.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(df, sp.filter, 18, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dllm, ll_mask, (bh + 1) * 4 * 2, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return R2G_E_INVALID;
    r2g_dsp_launch_wiener_uv(dc, cs.rs, dl, ls.rs, dcr, dlr, w, h, sp.ss_hor, df, dllm, bitdepth, dout, s);
    std::vector<uint16_t> out((size_t)w * h);
    if (cudaMemcpyAsync(out.data(), dout, out.size() * 2, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return R2G_E_DEVICE;
    store_block((P *)dst, stride, out, w, h);
    return R2G_OK;
}

template <typename P>
int gdf_prep(DspDevice *d, int8_t *dst, int64_t dst_stride, const void *p, int64_t stride, const void *left,
             const void *top, const void *bottom, int w, int h, int ref_dst_idx, int qp_idx, int edges, int bitdepth) {
    RowStage st(w, 6);
    std::vector<int> gref, pref;
    stage_gdf<P>(st, (const P *)p, stride, (const P *)left, (const P *)top, (const P *)bottom, h, edges, gref, pref);
    const int ng = (int)(gref.size() / 13);
    Scratch sc{d->buf, 0, kScratch};
    uint16_t *drows = sc.take<uint16_t>(st.data.size());
    int *dg = sc.take<int>(gref.size()), *dp = sc.take<int>(pref.size());
    int8_t *dout = sc.take<int8_t>((size_t)w * h);
    if (!dout) return R2G_E_TOO_LARGE;
    cudaStream_t s = d->st;
    if (cudaMemcpyAsync(drows, st.data.data(), st.data.size() * 2, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dg, gref.data(), gref.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dp, pref.data(), pref.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return R2G_E_DEVICE;
    r2g_dsp_launch_gdf_prep(drows, st.rs, st.e, dg, ng, dp, w, h, ref_dst_idx, qp_idx, bitdepth, d->tab, dout, s);
    std::vector<int8_t> out((size_t)w * h);
    if (cudaMemcpyAsync(out.data(), dout, out.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return R2G_E_DEVICE;
    for (int y = 0; y < h; y++) memcpy(dst + y * dst_stride, &out[(size_t)y * w], (size_t)w);
    return R2G_OK;
}

bool lr_edges_ok(int edges) { return (edges & ~15) == 0; }

int wiener_y_entry(void *dst, int64_t stride, const void *left, const void *top, const void *bottom, int w, int h,
                   const R2gWienerParams *params, int edges, const uint16_t *ll_mask, int bitdepth, int kind) {
    if (!dst || !params || !ll_mask || !ok_bd(bitdepth) || !lr_dims_ok(w, h, 4, 4) || (h & 3) ||
        !lr_edges_ok(edges) || ((edges & LRE_LEFT) && !left) || ((edges & LRE_TOP) && !top) ||
        ((edges & LRE_BOTTOM) && !bottom))
        return R2G_E_INVALID;
    if (kind == 1 ? !params->single.filter
                  : (!params->multi.filters || !params->multi.subclass_lut || !params->multi.noskip_mask))
        return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    rc = bitdepth > 8 ? wiener_y<uint16_t>(d, dst, stride, left, top, bottom, w, h, params, edges, ll_mask, bitdepth, kind)
                      : wiener_y<uint8_t>(d, dst, stride, left, top, bottom, w, h, params, edges, ll_mask, bitdepth, kind);
    return finish(d, rc);
}

}  // namespace

extern "C" int r2g_dsp_ns_wiener_single_y(void *dst, int64_t dst_stride, const void *left, const void *top,
                                          const void *bottom, int w, int h, const R2gWienerParams *params, int edges,
                                          const uint16_t *ll_mask, int bitdepth) {
    return wiener_y_entry(dst, dst_stride, left, top, bottom, w, h, params, edges, ll_mask, bitdepth, 1);
}
extern "C" int r2g_dsp_ns_wiener_multi(void *dst, int64_t dst_stride, const void *left, const void *top,
                                       const void *bottom, int w, int h, const R2gWienerParams *params, int edges,
                                       const uint16_t *ll_mask, int bitdepth) {
    return wiener_y_entry(dst, dst_stride, left, top, bottom, w, h, params, edges, ll_mask, bitdepth, 2);
}
extern "C" int r2g_dsp_pc_wiener(void *dst, int64_t dst_stride, const void *left, const void *top, const void *bottom,
                                 int w, int h, const R2gWienerParams *params, int edges, const uint16_t *ll_mask,
                                 int bitdepth) {
    return wiener_y_entry(dst, dst_stride, left, top, bottom, w, h, params, edges, ll_mask, bitdepth, 3);
}
extern "C" int r2g_dsp_ns_wiener_single_uv(void *dst, int64_t dst_stride, const void *left, const void *top,
                                           const void *bottom, int w, int h, const R2gWienerParams *params, int edges,
                                           const uint16_t *ll_mask, int bitdepth) {
    if (!dst || !params || !ll_mask || !ok_bd(bitdepth) || !lr_dims_ok(w, h, 4, 2) || !lr_edges_ok(edges) ||
        ((edges & LRE_LEFT) && !left) || ((edges & LRE_TOP) && (!top || !params->single.luma_top)) ||
        ((edges & LRE_BOTTOM) && (!bottom || !params->single.luma_bottom)) || !params->single.filter ||
        !params->single.luma || params->single.ss_hor < 0 || params->single.ss_hor > 1 ||
        params->single.ss_ver < 0 || params->single.ss_ver > 1 || params->single.ds_flt < 0 ||
        params->single.ds_flt > 2)
        return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    rc = bitdepth > 8 ? wiener_uv<uint16_t>(d, dst, dst_stride, left, top, bottom, w, h, params, edges, ll_mask, bitdepth)
                      : wiener_uv<uint8_t>(d, dst, dst_stride, left, top, bottom, w, h, params, edges, ll_mask, bitdepth);
    return finish(d, rc);
}
extern "C" int r2g_dsp_gdf_prep(int8_t *dst, int64_t dst_stride, const void *p, int64_t stride, const void *left,
                                const void *top, const void *bottom, int w, int h, int ref_dst_idx, int qp_idx,
                                int edges, int bitdepth) {
    if (!dst || !p || !ok_bd(bitdepth) || !lr_dims_ok(w, h, 2, 6) || !lr_edges_ok(edges) || ref_dst_idx < 0 ||
        ref_dst_idx > 5 || qp_idx < 0 || qp_idx > 5 || ((edges & LRE_LEFT) && !left) || ((edges & LRE_TOP) && !top) ||
        ((edges & LRE_BOTTOM) && !bottom))
        return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(g_dsp_mu);
    DspDevice *d;
    int rc = dsp_device(&d);
    if (rc != R2G_OK) return rc;
    rc = bitdepth > 8 ? gdf_prep<uint16_t>(d, dst, dst_stride, p, stride, left, top, bottom, w, h, ref_dst_idx, qp_idx,
                                           edges, bitdepth)
                      : gdf_prep<uint8_t>(d, dst, dst_stride, p, stride, left, top, bottom, w, h, ref_dst_idx, qp_idx,
                                          edges, bitdepth);
    return finish(d, rc);
}
