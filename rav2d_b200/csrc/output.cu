// Output formatting and partial downloads.
//
// r2g_download_y4m packs a frame's planes on the device the way rav2d-cli
// writes a Y4M frame (crates/rav2d-cli/src/main.rs:114-149 pack_plane /
// write_picture, y4m.rs:36-45 write_frame): "FRAME\n", then the luma plane
// and the two chroma planes, each tightly packed (width samples per row,
// little-endian 16-bit samples above 8 bits).  One kernel packs into a device
// buffer of the frame and one copy brings the payload back.  Optionally the
// samples are reduced to 8 bits on the device for display ((v + 2) >> 2,
// clipped; an addition of this library, the reference writes the native depth).
//
// r2g_download_rows copies a band of rows (the part of a reference frame the
// next frame's reconstruction needs) instead of the whole frame.
#include <cstdio>
#include <cstring>

#include "r2g_runtime.h"

namespace {

// One thread per output sample pair position; planes in order Y, U, V.
template <typename P, typename O>
__global__ void __launch_bounds__(256) pack_kernel(const P *y, const P *u, const P *v, int64_t ys, int64_t uvs,
                                                   int w, int h, int shift, O *out) {
    const int cw = w >> 1, ch = h >> 1;
    const int64_t ny = (int64_t)w * h, nc = (int64_t)cw * ch;
    const int maxv = (1 << (8 * (int)sizeof(O))) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ny + 2 * nc;
         i += (int64_t)gridDim.x * blockDim.x) {
        int s;
        if (i < ny) {
            s = y[(i / w) * ys + i % w];
        } else {
            const int64_t j = (i - ny) % nc;
            const P *p = i - ny < nc ? u : v;
            s = p[(j / cw) * uvs + j % cw];
        }
        if (shift) {
            s = (s + (1 << (shift - 1))) >> shift;
            s = s > maxv ? maxv : s;
        }
        out[i] = (O)s;
    }
}

}  // namespace

extern "C" int r2g_y4m_header(int width, int height, int fps_num, int fps_den, int bitdepth, char *buf, int cap) {
    if (!buf || cap <= 0 || width <= 0 || height <= 0 || fps_num <= 0 || fps_den <= 0 ||
        (bitdepth != 8 && bitdepth != 10))
        return R2G_E_INVALID;
    // y4m_colorspace (crates/rav2d-cli/src/main.rs:98-111) for 4:2:0
    char cs[16];
    if (bitdepth == 8)
        snprintf(cs, sizeof(cs), "420jpeg");
    else
        snprintf(cs, sizeof(cs), "420p%d", bitdepth);
    int n = snprintf(buf, (size_t)cap, "YUV4MPEG2 W%d H%d F%d:%d Ip C%s\n", width, height, fps_num, fps_den, cs);
    return n < cap ? n : R2G_E_INVALID;
}

extern "C" int64_t r2g_y4m_frame_bytes(int width, int height, int out_bitdepth) {
    if (width <= 0 || height <= 0 || (out_bitdepth != 8 && out_bitdepth != 10)) return R2G_E_INVALID;
    const int64_t samples = (int64_t)width * height + 2 * (int64_t)(width >> 1) * (height >> 1);
    return 6 + samples * (out_bitdepth > 8 ? 2 : 1);
}

extern "C" int r2g_download_y4m(R2gCtx *ctx, R2gFrame *f, int which, int out_bitdepth, void *dst, int64_t dst_size) {
    if (!ctx || !f || !dst || (which != 0 && which != 1)) return R2G_E_INVALID;
    if (out_bitdepth == 0) out_bitdepth = f->bd;
    if (out_bitdepth != 8 && out_bitdepth != f->bd) {
        ctx->err = "output bit depth must be 8 or the frame's own";
        return R2G_E_INVALID;
    }
    const int64_t need = r2g_y4m_frame_bytes(f->w, f->h, out_bitdepth);
    if (need < 0 || dst_size < need) {
        ctx->err = "destination smaller than the Y4M frame";
        return R2G_E_INVALID;
    }
    const int buf = which == 0 ? f->out_buf : f->grain_buf;
    if (buf < 0) {
        ctx->err = which ? "frame has no grained copy" : "frame not filtered";
        return R2G_E_INVALID;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return R2G_E_DEVICE;
    const size_t payload = (size_t)(need - 6);
    if (f->pack_bytes < payload) {
        r2g_dev_free(ctx, f->pack_buf, f->pack_bytes);
        f->pack_buf = nullptr;
        f->pack_bytes = 0;
        int rc = r2g_dev_alloc(ctx, &f->pack_buf, payload);
        if (rc != R2G_OK) return rc;
        f->pack_bytes = payload;
    }
    // order: after this frame's kernels, on the download stream when copies
    // overlap (the packing is part of the download)
    cudaStream_t st = ctx->stream;
    if (ctx->overlap) {
        st = ctx->down_stream;
        if (f->pend_comp && cudaStreamWaitEvent(st, f->ev_comp, 0) != cudaSuccess) return R2G_E_DEVICE;
    }
    const char *b = (const char *)f->buf[buf];
    const int bps = f->bd > 8 ? 2 : 1;
    const int64_t ys = f->stride[0] / bps, uvs = f->stride[1] / bps;
    const int shift = f->bd - out_bitdepth;
    const int grid = 148 * 4;
    if (bps == 2) {
        const uint16_t *y = (const uint16_t *)b, *u = (const uint16_t *)(b + f->plane_bytes[0]),
                       *v = (const uint16_t *)(b + f->plane_bytes[0] + f->plane_bytes[1]);
        if (out_bitdepth > 8)
            pack_kernel<uint16_t, uint16_t><<<grid, 256, 0, st>>>(y, u, v, ys, uvs, f->w, f->h, 0,
                                                                  (uint16_t *)f->pack_buf);
        else
            pack_kernel<uint16_t, uint8_t><<<grid, 256, 0, st>>>(y, u, v, ys, uvs, f->w, f->h, shift,
                                                                 (uint8_t *)f->pack_buf);
    } else {
        const uint8_t *y = (const uint8_t *)b, *u = (const uint8_t *)(b + f->plane_bytes[0]),
                      *v = (const uint8_t *)(b + f->plane_bytes[0] + f->plane_bytes[1]);
        pack_kernel<uint8_t, uint8_t><<<grid, 256, 0, st>>>(y, u, v, ys, uvs, f->w, f->h, 0, (uint8_t *)f->pack_buf);
    }
    ctx->launches += 1;
    memcpy(dst, "FRAME\n", 6);
    if (cudaMemcpyAsync((char *)dst + 6, f->pack_buf, payload, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return R2G_E_DEVICE;
    if (ctx->overlap) {
        if (cudaEventRecord(f->ev_down, st) != cudaSuccess) return R2G_E_DEVICE;
        f->pend_down = true;
    }
    return cudaGetLastError() == cudaSuccess ? R2G_OK : R2G_E_DEVICE;
}

extern "C" int r2g_download_rows(R2gCtx *ctx, R2gFrame *f, int which, int row0, int nrows, void *y, int64_t y_stride,
                                 void *u, void *v, int64_t uv_stride) {
    if (!ctx || !f || (which != 0 && which != 1) || row0 < 0 || nrows <= 0 || row0 + nrows > f->h || (row0 & 1) ||
        (nrows & 1))
        return R2G_E_INVALID;
    const int buf = which == 0 ? f->out_buf : f->grain_buf;
    if (buf < 0) {
        ctx->err = which ? "frame has no grained copy" : "frame not filtered";
        return R2G_E_INVALID;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return R2G_E_DEVICE;
    cudaStream_t st = ctx->stream;
    if (ctx->overlap) {
        st = ctx->down_stream;
        if (f->pend_comp && cudaStreamWaitEvent(st, f->ev_comp, 0) != cudaSuccess) return R2G_E_DEVICE;
    }
    const int bps = f->bd > 8 ? 2 : 1;
    const char *b = (const char *)f->buf[buf];
    const char *src[3] = {b, b + f->plane_bytes[0], b + f->plane_bytes[0] + f->plane_bytes[1]};
    void *dst[3] = {y, u, v};
    for (int pl = 0; pl < 3; pl++) {
        if (!dst[pl]) continue;
        const int64_t ds = pl ? uv_stride : y_stride, ss = f->stride[pl ? 1 : 0];
        const int64_t wb = (int64_t)(pl ? f->w / 2 : f->w) * bps;
        const int r0 = pl ? row0 / 2 : row0, nr = pl ? nrows / 2 : nrows;
        if (ds < wb) {
            ctx->err = "host stride smaller than the plane width";
            return R2G_E_INVALID;
        }
        if (cudaMemcpy2DAsync(dst[pl], ds, src[pl] + r0 * ss, ss, wb, nr, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return R2G_E_DEVICE;
    }
    if (ctx->overlap) {
        if (cudaEventRecord(f->ev_down, st) != cudaSuccess) return R2G_E_DEVICE;
        f->pend_down = true;
    }
    return R2G_OK;
}
