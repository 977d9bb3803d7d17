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
    cudaStream_t st = nullptr;  // non-blocking: no implicit sync with the legacy stream
    DevTables tab{};
};
constexpr size_t kScratch = 64 * 1024;
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

int finish(const DspDevice *d, int rc) {
    if (rc != R2G_OK) return rc;
    return cudaStreamSynchronize(d->st) == cudaSuccess && cudaGetLastError() == cudaSuccess ? R2G_OK : R2G_E_DEVICE;
}

}  // namespace

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
