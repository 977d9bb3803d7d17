// Host runtime of the C ABI declared in include/rav2d_gpu.h: contexts,
// device-resident frames, side-info staging, stage gating and launch order.
//
// The per-frame pipeline replaces the reference's Phase-B loop of
// filter_sbrow (decode.rs:3597-3625, :3718-4058) with whole-frame stages:
//   deblock (in place on the recon: vertical edges, then horizontal edges)
//   -> CDEF+CCSO (deblocked -> C) -> loop restoration (C, deblocked -> L)
//   -> film grain (L -> display copy G).
// A disabled stage aliases its output to its input, as the reference simply
// skips it.
#include <chrono>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "r2g_common.cuh"
#include "r2g_runtime.h"

#define R2G_VERSION 1

static void set_err(R2gCtx *ctx, const char *fmt, const char *a = "") {
    if (!ctx) return;
    char buf[512];
    snprintf(buf, sizeof(buf), fmt, a);
    ctx->err = buf;
}

#define CK(call)                                                                    \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            set_err(ctx, "CUDA error: %s", cudaGetErrorString(e_));                 \
            return R2G_E_DEVICE;                                                    \
        }                                                                           \
    } while (0)

extern "C" int r2g_version(void) { return R2G_VERSION; }

bool r2g_pdl_enabled() {
    static const bool on = [] {
        const char *e = getenv("R2G_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

extern "C" int r2g_plane_geometry(int width, int height, int bitdepth, int64_t *y_stride, int64_t *uv_stride,
                                  int64_t *y_rows, int64_t *uv_rows) {
    if (width <= 0 || height <= 0 || (bitdepth != 8 && bitdepth != 10)) return R2G_E_INVALID;
    int hbd = bitdepth > 8;
    int64_t aw = (width + 127) & ~127, ah = (height + 127) & ~127;
    int64_t ys = aw << hbd, uvs = ys >> 1;
    if ((ys & 1023) == 0) ys += 64;
    if ((uvs & 1023) == 0) uvs += 64;
    if (y_stride) *y_stride = ys;
    if (uv_stride) *uv_stride = uvs;
    if (y_rows) *y_rows = ah;
    if (uv_rows) *uv_rows = ah >> 1;
    return R2G_OK;
}

extern "C" int r2g_struct_sizes(int32_t *sizes, int n) {
    const int32_t v[] = {(int32_t)sizeof(R2gAv2Filter), (int32_t)sizeof(R2gAv2RestorationUnit),
                         (int32_t)sizeof(R2gAv2Restoration), (int32_t)sizeof(R2gFrameParams),
                         (int32_t)sizeof(R2gFilmGrainData), (int32_t)sizeof(R2gSideInfo),
                         (int32_t)sizeof(R2gBatchItem), (int32_t)sizeof(R2gServeConfig),
                         (int32_t)sizeof(R2gServeRequest), (int32_t)sizeof(R2gServeResult),
                         (int32_t)sizeof(R2gServeStats), (int32_t)sizeof(R2gWienerParams),
                         (int32_t)sizeof(R2gDbBlock), (int32_t)sizeof(R2gDbMaskInput)};
    int m = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < m; i++) sizes[i] = v[i];
    return m;
}

// ---------------------------------------------------------------- context
extern "C" int r2g_ctx_create(int device, int64_t mem_budget, R2gCtx **out) {
    if (!out) return R2G_E_INVALID;
    *out = nullptr;
    R2gCtx *ctx = new R2gCtx();
    ctx->device = device;
    ctx->budget = mem_budget;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        delete ctx;
        return R2G_E_DEVICE;
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
        r2g_get_tables(&ctx->tab) != cudaSuccess) {
        delete ctx;
        return R2G_E_DEVICE;
    }
    void *ctl = nullptr;
    if (cudaMalloc(&ctl, R2G_CTL_BYTES) != cudaSuccess || cudaMemset(ctl, 0, R2G_CTL_BYTES) != cudaSuccess) {
        cudaGetLastError();
        if (ctl) cudaFree(ctl);
        cudaStreamDestroy(ctx->stream);
        cudaStreamDestroy(ctx->side_stream);
        delete ctx;
        return R2G_E_DEVICE;
    }
    ctx->sched = (StageSched *)ctl;
    ctx->fault = (unsigned *)((char *)ctl + 128);
    ctx->bad_blocks = (unsigned *)((char *)ctl + 132);
    *out = ctx;
    return R2G_OK;
}

extern "C" int r2g_ctx_device_faults(R2gCtx *ctx, uint32_t *count) {
    if (!ctx || !count) return R2G_E_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess ||
        cudaMemcpy(count, ctx->fault, sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return R2G_E_DEVICE;
    return R2G_OK;
}

extern "C" int r2g_ctx_destroy(R2gCtx *ctx) {
    if (!ctx) return R2G_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->side_stream);
    for (auto &t : ctx->tickets) cudaEventDestroy(t.ev);
    ctx->tickets.clear();
    r2g_grain_ctx_free(ctx);
    r2g_batch_free(ctx);
    r2g_ctx_profile(ctx, 0);
    for (cudaStream_t st : {ctx->up_stream, ctx->down_stream, ctx->side_up_stream})
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    for (cudaEvent_t e : ctx->fence_ev)
        if (e) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->own_stream ? ctx->own_stream : ctx->stream);
    cudaStreamDestroy(ctx->side_stream);
    if (ctx->sched) cudaFree(ctx->sched);
    delete ctx;
    return R2G_OK;
}

extern "C" const char *r2g_last_error(R2gCtx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int r2g_dev_alloc(R2gCtx *ctx, void **p, size_t bytes) {
    if (ctx->budget > 0 && ctx->used + (int64_t)bytes > ctx->budget) {
        set_err(ctx, "device-memory budget exhausted");
        return R2G_E_OOM;
    }
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_err(ctx, "cudaMalloc failed");
        return R2G_E_OOM;
    }
    ctx->used += (int64_t)bytes;
    return R2G_OK;
}

void r2g_dev_free(R2gCtx *ctx, void *p, size_t bytes) {
    if (!p) return;
    cudaFree(p);
    ctx->used -= (int64_t)bytes;
}

// ---------------------------------------------------------------- frames
// Device bytes r2g_frame_alloc takes for one frame (five plane sets and the
// side-info records), plus the batched film-grain scratch.
size_t r2g_frame_device_bytes(int width, int height, int bitdepth) {
    int64_t ys, uvs, yr, uvr;
    if (r2g_plane_geometry(width, height, bitdepth, &ys, &uvs, &yr, &uvr) != R2G_OK) return 0;
    size_t buf = (size_t)(ys * yr + 2 * uvs * uvr);
    int bw4 = ((width + 7) >> 3) << 1, bh4 = ((height + 7) >> 3) << 1;
    size_t nsb = (size_t)((bw4 + 63) >> 6) * ((bh4 + 63) >> 6);
    return 5 * buf + nsb * (sizeof(R2gAv2Filter) + sizeof(LrPacked)) + R2G_GRAIN_SCRATCH;
}

extern "C" int r2g_frame_alloc(R2gCtx *ctx, int width, int height, int bitdepth, R2gFrame **out) {
    if (!ctx || !out) return R2G_E_INVALID;
    *out = nullptr;
    if ((width & 7) || (height & 7) || width <= 0 || height <= 0 || (bitdepth != 8 && bitdepth != 10)) {
        set_err(ctx, "unsupported frame geometry");
        return R2G_E_INVALID;
    }
    CK(cudaSetDevice(ctx->device));
    R2gFrame *f = new R2gFrame();
    f->w = width;
    f->h = height;
    f->bd = bitdepth;
    r2g_plane_geometry(width, height, bitdepth, &f->stride[0], &f->stride[1], &f->rows[0], &f->rows[1]);
    f->plane_bytes[0] = (size_t)(f->stride[0] * f->rows[0]);
    f->plane_bytes[1] = (size_t)(f->stride[1] * f->rows[1]);
    f->buf_bytes = f->plane_bytes[0] + 2 * f->plane_bytes[1];
    int bw4 = ((width + 7) >> 3) << 1, bh4 = ((height + 7) >> 3) << 1;
    f->n_sb256 = ((bw4 + 63) >> 6) * ((bh4 + 63) >> 6);
    f->side_bytes = (size_t)f->n_sb256 * (sizeof(R2gAv2Filter) + sizeof(LrPacked));
    int rc;
    for (int i = 0; i < 5; i++)
        if ((rc = r2g_dev_alloc(ctx, &f->buf[i], f->buf_bytes)) != R2G_OK) {
            r2g_frame_free(ctx, f);
            return rc;
        }
    if ((rc = r2g_dev_alloc(ctx, &f->side_dev, f->side_bytes)) != R2G_OK) {
        r2g_frame_free(ctx, f);
        return rc;
    }
    if (cudaMallocHost(&f->side_host, f->side_bytes) != cudaSuccess) {
        cudaGetLastError();
        r2g_frame_free(ctx, f);
        set_err(ctx, "pinned allocation failed");
        return R2G_E_OOM;
    }
    // the display copy starts as a copy of whatever is filtered; zero it so
    // downloads of an ungrained frame are deterministic
    for (int i = 0; i < 5; i++) CK(cudaMemsetAsync(f->buf[i], 0, f->buf_bytes, ctx->stream));
    *out = f;
    return R2G_OK;
}

extern "C" int r2g_frame_free(R2gCtx *ctx, R2gFrame *f) {
    if (!ctx || !f) return R2G_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (cudaStream_t st : {ctx->up_stream, ctx->down_stream, ctx->side_up_stream})
        if (st) cudaStreamSynchronize(st);
    for (cudaEvent_t e : {f->ev_up, f->ev_comp, f->ev_down, f->ev_side})
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < 5; i++) r2g_dev_free(ctx, f->buf[i], f->buf_bytes);
    r2g_dev_free(ctx, f->side_dev, f->side_bytes);
    r2g_dev_free(ctx, f->seg_dev, f->seg_bytes);
    r2g_dev_free(ctx, f->grain_scratch, R2G_GRAIN_SCRATCH);
    r2g_dev_free(ctx, f->pack_buf, f->pack_bytes);
    if (f->side_host) cudaFreeHost(f->side_host);
    if (f->seg_host) cudaFreeHost(f->seg_host);
    if (f->side_done) cudaEventDestroy(f->side_done);
    r2g_dev_free(ctx, f->dbm_dev, f->dbm_bytes);
    if (f->dbm_host) cudaFreeHost(f->dbm_host);
    for (cudaEvent_t e : f->ev_dbm)
        if (e) cudaEventDestroy(e);
    delete f;
    return R2G_OK;
}

static void plane_ptrs(const R2gFrame *f, int buf, void *p[3]) {
    char *b = (char *)f->buf[buf];
    p[0] = b;
    p[1] = b + f->plane_bytes[0];
    p[2] = b + f->plane_bytes[0] + f->plane_bytes[1];
}

int r2g_copy_planes(R2gCtx *ctx, const R2gFrame *f, int buf, const void *y, int64_t ys, const void *u,
                    const void *v, int64_t uvs, bool upload, cudaStream_t st) {
    void *p[3];
    plane_ptrs(f, buf, p);
    int bps = f->bd > 8 ? 2 : 1;
    const void *hs[3] = {y, u, v};
    for (int i = 0; i < 3; i++) {
        int64_t hstride = i ? uvs : ys;
        int64_t dstride = f->stride[i ? 1 : 0];
        int64_t wbytes = (int64_t)(i ? f->w / 2 : f->w) * bps;
        int64_t rows = i ? f->h / 2 : f->h;
        if (!hs[i]) continue;
        if (hstride < wbytes) {
            set_err(ctx, "host stride smaller than the plane width");
            return R2G_E_INVALID;
        }
        if (hstride == wbytes && dstride == wbytes) {
            // rows back to back on both sides: one linear copy
            if (upload)
                CK(cudaMemcpyAsync(p[i], hs[i], (size_t)(wbytes * rows), cudaMemcpyHostToDevice, st));
            else
                CK(cudaMemcpyAsync((void *)hs[i], p[i], (size_t)(wbytes * rows), cudaMemcpyDeviceToHost, st));
        } else if (upload) {
            CK(cudaMemcpy2DAsync(p[i], dstride, hs[i], hstride, wbytes, rows, cudaMemcpyHostToDevice, st));
        } else {
            CK(cudaMemcpy2DAsync((void *)hs[i], hstride, p[i], dstride, wbytes, rows, cudaMemcpyDeviceToHost, st));
        }
    }
    return R2G_OK;
}

// ---- copy overlap: per-frame ordering across the three streams
static int ensure_events(R2gCtx *ctx, R2gFrame *f) {
    for (cudaEvent_t *e : {&f->ev_up, &f->ev_comp, &f->ev_down, &f->ev_side})
        if (!*e) CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return R2G_OK;
}

// The stream a frame's upload / staging goes on.  With overlap, the copy
// must not overwrite the recon or side-info while earlier kernels of this
// frame may still read them.
static int upload_stream(R2gCtx *ctx, R2gFrame *f, cudaStream_t *st) {
    *st = ctx->stream;
    if (!ctx->overlap) return R2G_OK;
    int rc = ensure_events(ctx, f);
    if (rc != R2G_OK) return rc;
    if (f->pend_comp) CK(cudaStreamWaitEvent(ctx->up_stream, f->ev_comp, 0));
    *st = ctx->up_stream;
    return R2G_OK;
}

static int upload_done(R2gCtx *ctx, R2gFrame *f) {
    if (!ctx->overlap) return R2G_OK;
    CK(cudaEventRecord(f->ev_up, ctx->up_stream));
    f->pend_up = true;
    return R2G_OK;
}

int r2g_frame_before_compute(R2gCtx *ctx, R2gFrame *f) {
    if (f->pend_dbm) CK(cudaStreamWaitEvent(ctx->stream, f->ev_dbm[1], 0));
    if (!ctx->overlap || !f->ev_up) return R2G_OK;
    // the kernels read this frame's uploads and overwrite planes a pending
    // download may still read
    if (f->pend_up) CK(cudaStreamWaitEvent(ctx->stream, f->ev_up, 0));
    if (f->pend_side) CK(cudaStreamWaitEvent(ctx->stream, f->ev_side, 0));
    if (f->pend_down) CK(cudaStreamWaitEvent(ctx->stream, f->ev_down, 0));
    return R2G_OK;
}

int r2g_frame_after_compute(R2gCtx *ctx, R2gFrame *f) {
    if (!ctx->overlap) return R2G_OK;
    int rc = ensure_events(ctx, f);
    if (rc != R2G_OK) return rc;
    CK(cudaEventRecord(f->ev_comp, ctx->stream));
    f->pend_comp = true;
    return R2G_OK;
}

extern "C" int r2g_ctx_overlap_copies(R2gCtx *ctx, int enable) {
    if (!ctx) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    if (enable && !ctx->up_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->up_stream, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&ctx->down_stream, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&ctx->side_up_stream, cudaStreamNonBlocking));
        for (cudaEvent_t &e : ctx->fence_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (!enable && ctx->up_stream) {
        // later work goes on the context stream again: order it after every
        // copy issued so far
        int rc = r2g_ctx_fence(ctx);
        if (rc != R2G_OK) return rc;
    }
    ctx->overlap = enable != 0;
    return R2G_OK;
}

extern "C" int r2g_ctx_fence(R2gCtx *ctx) {
    if (!ctx) return R2G_E_INVALID;
    if (!ctx->up_stream) return R2G_OK;
    CK(cudaSetDevice(ctx->device));
    CK(cudaEventRecord(ctx->fence_ev[0], ctx->up_stream));
    CK(cudaEventRecord(ctx->fence_ev[1], ctx->down_stream));
    CK(cudaEventRecord(ctx->fence_ev[2], ctx->side_up_stream));
    for (cudaEvent_t e : ctx->fence_ev) CK(cudaStreamWaitEvent(ctx->stream, e, 0));
    return R2G_OK;
}

extern "C" int r2g_frame_upload_recon(R2gCtx *ctx, R2gFrame *f, const void *y, int64_t y_stride, const void *u,
                                      const void *v, int64_t uv_stride) {
    if (!ctx || !f || !y || !u || !v) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st;
    int rc = upload_stream(ctx, f, &st);
    if (rc == R2G_OK) rc = r2g_copy_planes(ctx, f, 0, y, y_stride, u, v, uv_stride, true, st);
    if (rc == R2G_OK) rc = upload_done(ctx, f);
    return rc;
}

extern "C" int r2g_download(R2gCtx *ctx, R2gFrame *f, int which, void *y, int64_t y_stride, void *u, void *v,
                            int64_t uv_stride) {
    if (!ctx || !f || (which != 0 && which != 1)) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    int buf = which == 0 ? f->out_buf : f->grain_buf;
    if (buf < 0) {
        set_err(ctx, which ? "frame has no grained copy" : "frame not filtered");
        return R2G_E_INVALID;
    }
    if (!ctx->overlap) return r2g_copy_planes(ctx, f, buf, y, y_stride, u, v, uv_stride, false, ctx->stream);
    int rc = ensure_events(ctx, f);
    if (rc != R2G_OK) return rc;
    if (f->pend_comp) CK(cudaStreamWaitEvent(ctx->down_stream, f->ev_comp, 0));
    rc = r2g_copy_planes(ctx, f, buf, y, y_stride, u, v, uv_stride, false, ctx->down_stream);
    if (rc != R2G_OK) return rc;
    CK(cudaEventRecord(f->ev_down, ctx->down_stream));
    f->pend_down = true;
    return R2G_OK;
}

extern "C" int r2g_sync(R2gCtx *ctx) {
    if (!ctx) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->side_stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (cudaStream_t st : {ctx->up_stream, ctx->down_stream, ctx->side_up_stream})
        if (st) CK(cudaStreamSynchronize(st));
    // a stage kernel whose bounded wait ran out left its work incomplete
    uint32_t faults[2] = {0, 0};
    CK(cudaMemcpy(faults, ctx->fault, sizeof(faults), cudaMemcpyDeviceToHost));
    if (faults[0]) {
        set_err(ctx, "%s", (std::to_string(faults[0]) + " device-side waits ran out; the filtered output is incomplete").c_str());
        return R2G_E_DEVICE;
    }
    // a block record the reference could not have produced was skipped
    if (faults[1]) {
        CK(cudaMemset(ctx->bad_blocks, 0, sizeof(unsigned)));  // reported once
        set_err(ctx, "%s", (std::to_string(faults[1]) + " deblock block records were invalid and skipped").c_str());
        return R2G_E_INVALID;
    }
    return R2G_OK;
}

// ---------------------------------------------------------------- filtering
// decode.rs:27-57 init_wiener, :59-65 compute_restore_planes, :67-80
// compute_gdf_ref_dst_idx, dq_lookup (quantizer.rs:31)
static int host_dq_lookup(int qidx) {
    static const uint8_t T[24] = {40, 41, 43, 44, 45, 47, 48, 49, 51, 52, 54, 55,
                                  57, 59, 60, 62, 64, 66, 68, 70, 72, 74, 76, 78};
    qidx = qidx < 0 ? 0 : (qidx > 255 ? 255 : qidx);
    if (qidx == 0) return 64;
    qidx -= 1;
    return (int)T[qidx % 24] << (qidx / 24);
}

int r2g_validate(R2gCtx *ctx, const R2gFrame *f, const R2gFrameParams *fp, const R2gSideInfo *side) {
    if (!fp || !side || !side->masks || !side->lr) {
        set_err(ctx, "missing frame parameters or side-info");
        return R2G_E_INVALID;
    }
    if (fp->width != f->w || fp->height != f->h || fp->bitdepth != f->bd) {
        set_err(ctx, "frame parameters do not match the frame buffer");
        return R2G_E_INVALID;
    }
    if (fp->layout != 1 || fp->sb128 != 0) {
        set_err(ctx, "only 4:2:0 with 64x64 superblocks is supported");
        return R2G_E_INVALID;
    }
    if (fp->tile_rows > 64) {
        set_err(ctx, "more than 64 tile rows");
        return R2G_E_INVALID;
    }
    for (int i = 1; i < fp->tile_rows; i++)
        if (fp->tile_row_start_sb[i] <= fp->tile_row_start_sb[i - 1]) {
            set_err(ctx, "tile row starts are not increasing");
            return R2G_E_INVALID;
        }
    if (fp->tile_rows > 1 && ((fp->height + 63) >> 6) > 128) {
        set_err(ctx, "tile rows are supported up to 128 superblock rows");
        return R2G_E_INVALID;
    }
    if (side->n_sb256 != f->n_sb256) {
        set_err(ctx, "side-info count does not match the frame size");
        return R2G_E_INVALID;
    }
    for (int pl = 1; pl < 3; pl++)
        if (fp->restoration[pl].frame_filters_on && fp->restoration[pl].num_classes != 1) {
            set_err(ctx, "multi-class chroma restoration is not supported");
            return R2G_E_INVALID;
        }
    for (int i = 0; i < side->n_sb256; i++)
        for (int pl = 1; pl < 3; pl++)
            for (int u = 0; u < 16; u++)
                if (side->lr[i].lr[pl][u].restoration_type == R2G_RESTORE_PC_WIENER) {
                    set_err(ctx, "PC-Wiener on a chroma unit is not supported");
                    return R2G_E_INVALID;
                }
    if (fp->restoration_unit_size[0] < 5 || fp->restoration_unit_size[0] > 9 ||
        fp->restoration_unit_size[1] < 5 || fp->restoration_unit_size[1] > 9) {
        set_err(ctx, "restoration unit size out of range");
        return R2G_E_INVALID;
    }
    if (const R2gDbMaskInput *m = side->db_masks) {
        const int bw4 = ((f->w + 7) >> 3) << 1, bh4 = ((f->h + 7) >> 3) << 1;
        if (m->n_blocks < 0 || (m->n_blocks > 0 && !m->blocks) || m->n_tile_cols < 1 || m->n_tile_cols > 64 ||
            m->n_tile_rows < 1 || m->n_tile_rows > 64 || bw4 > 2048 || bh4 > 2048) {
            set_err(ctx, "invalid deblock block records");
            return R2G_E_INVALID;
        }
        for (int i = 0; i < m->n_tile_cols; i++)
            if (m->tile_col_start4[i] >= bw4 || (i && m->tile_col_start4[i] <= m->tile_col_start4[i - 1])) {
                set_err(ctx, "tile column starts out of order or outside the frame");
                return R2G_E_INVALID;
            }
        for (int i = 0; i < m->n_tile_rows; i++)
            if (m->tile_row_start4[i] >= bh4 || (i && m->tile_row_start4[i] <= m->tile_row_start4[i - 1])) {
                set_err(ctx, "tile row starts out of order or outside the frame");
                return R2G_E_INVALID;
            }
    }
    // segmentation enabled without a map is accepted: the kernels read
    // segment 0 for every block when the map pointer is NULL
    return R2G_OK;
}

// Stage the frame's block records and build its deblock masks on the device
// (r2g_launch_db_masks) after the side-info copies on `cs`: records go
// straight from page-locked caller memory in copy-overlap mode, else through
// the frame's pinned staging copy.  The build runs on the side stream,
// forked from and joined back to `cs` by events, so a stage kernel launched
// with programmatic serialisation after it never overlaps the build.
static int stage_db_masks(R2gCtx *ctx, R2gFrame *f, const R2gFrameParams *fp, const R2gDbMaskInput &m,
                          const DevFrame &d, cudaStream_t cs) {
    const size_t rb = (size_t)m.n_blocks * sizeof(R2gDbBlock);
    const size_t lb = r2g_db_levels_bytes(d.bw4, d.bh4);
    const size_t need = ((rb + 255) & ~(size_t)255) + lb;
    if (f->dbm_bytes < need) {
        r2g_dev_free(ctx, f->dbm_dev, f->dbm_bytes);
        f->dbm_dev = nullptr;
        f->dbm_bytes = 0;
        int rc = r2g_dev_alloc(ctx, &f->dbm_dev, need);
        if (rc != R2G_OK) return rc;
        f->dbm_bytes = need;
    }
    bool direct = false;
    if (ctx->overlap && rb) {
        cudaPointerAttributes am;
        direct = cudaPointerGetAttributes(&am, m.blocks) == cudaSuccess && am.type == cudaMemoryTypeHost;
        cudaGetLastError();
    }
    if (rb && !direct && f->dbm_host_bytes < rb) {
        if (f->dbm_host) cudaFreeHost(f->dbm_host);
        f->dbm_host = nullptr;
        f->dbm_host_bytes = 0;
        if (cudaMallocHost(&f->dbm_host, rb) != cudaSuccess) {
            cudaGetLastError();
            set_err(ctx, "pinned allocation failed");
            return R2G_E_OOM;
        }
        f->dbm_host_bytes = rb;
    }
    // a deferred build of this frame's previous staging still reads the
    // records and writes the masks: order this staging after it
    if (f->pend_dbm) CK(cudaStreamWaitEvent(cs, f->ev_dbm[1], 0));
    if (rb) {
        const void *src = m.blocks;
        if (!direct) {
            memcpy(f->dbm_host, m.blocks, rb);
            src = f->dbm_host;
        }
        CK(cudaMemcpyAsync(f->dbm_dev, src, rb, cudaMemcpyHostToDevice, cs));
    }
    for (cudaEvent_t &e : f->ev_dbm)
        if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaEventRecord(f->ev_dbm[0], cs));
    CK(cudaStreamWaitEvent(ctx->side_stream, f->ev_dbm[0], 0));
    uint8_t lossless[8];
    for (int i = 0; i < 8; i++) lossless[i] = fp->seg_lossless[i];
    ctx->launches += r2g_launch_db_masks(m, (const R2gDbBlock *)f->dbm_dev, (R2gAv2Filter *)f->side_dev, f->n_sb256,
                                         d.sb256w, d.bw4, d.bh4,
                                         (uint8_t *)f->dbm_dev + ((rb + 255) & ~(size_t)255), lossless, ctx->tab,
                                         ctx->bad_blocks, ctx->side_stream);
    CK(cudaGetLastError());
    CK(cudaEventRecord(f->ev_dbm[1], ctx->side_stream));
    if (ctx->defer_mask_join && cs != ctx->stream) {
        // the upload stream goes on with the next copies; the frame's
        // kernels wait for the build (r2g_frame_before_compute)
        f->pend_dbm = true;
    } else {
        CK(cudaStreamWaitEvent(cs, f->ev_dbm[1], 0));
        f->pend_dbm = false;
    }
    return R2G_OK;
}

int r2g_prepare(R2gCtx *ctx, R2gFrame *f, const R2gFrameParams *fp, const R2gSideInfo *side, uint32_t inloop,
                DevFrame &d, cudaStream_t cs) {
    if (!cs) cs = ctx->stream;
    int rc = r2g_validate(ctx, f, fp, side);
    if (rc != R2G_OK) return rc;
    memset(&d, 0, sizeof(d));
    d.w = f->w;
    d.h = f->h;
    d.cw = f->w >> 1;
    d.ch = f->h >> 1;
    d.bw4 = ((f->w + 7) >> 3) << 1;
    d.bh4 = ((f->h + 7) >> 3) << 1;
    d.sb256w = (d.bw4 + 63) >> 6;
    d.sb256h = (d.bh4 + 63) >> 6;
    d.sbh = (d.bh4 + 15) / 16;
    d.bitdepth = f->bd;
    d.hbd = (f->bd - 8) >> 1;
    d.bdmax = (1 << f->bd) - 1;
    int bps = f->bd > 8 ? 2 : 1;
    d.stride[0] = f->stride[0] / bps;
    d.stride[1] = f->stride[1] / bps;
    d.fp = *fp;
    d.tab = ctx->tab;
    d.sched = ctx->sched;
    d.fault = ctx->fault;
    d.inloop = inloop;
    d.deblock_on = (inloop & R2G_INLOOP_DEBLOCK) && (fp->deblock_level_y[0] || fp->deblock_level_y[1]);
    d.cdef_stage_on = fp->seq_cdef && (inloop & (R2G_INLOOP_CDEF | R2G_INLOOP_CCSO));
    d.ccso_on = (inloop & R2G_INLOOP_CCSO) && (fp->ccso[0].enabled || fp->ccso[1].enabled || fp->ccso[2].enabled);
    d.cdef_on = (inloop & R2G_INLOOP_CDEF) != 0;
    d.any_lossless = 0;
    if (fp->seg_enabled)
        for (int i = 0; i < 8; i++) d.any_lossless |= fp->seg_lossless[i] != 0;
    d.restore_planes = (fp->restoration[0].restoration_type != R2G_RESTORE_NONE || fp->gdf_enabled != 0) |
                       ((fp->restoration[1].restoration_type != R2G_RESTORE_NONE) << 1) |
                       ((fp->restoration[2].restoration_type != R2G_RESTORE_NONE) << 2);
    d.lr_on = d.restore_planes != 0 && (inloop & (R2G_INLOOP_WIENER | R2G_INLOOP_GDF));
    d.lr_rows = 32;
    // tile rows: init_start_of_tile_row (decode.rs:99-120) over sbh rows
    d.n_tr = 0;
    if (fp->tile_rows > 1)
        for (int tr = 0, sby = 0; tr < fp->tile_rows && sby < d.sbh; tr++) {
            if (sby > 0) {
                d.tr_first[sby >> 5] |= 1u << (sby & 31);
                d.tr_sby[d.n_tr++] = (int16_t)sby;
            }
            sby++;
            const int end = imin_(fp->tile_row_start_sb[tr + 1], d.sbh);
            while (sby < end) sby++;
        }
    d.base_q = 0;
    d.wiener_idx = 0;
    d.ns_ci = -1;
    int rtype = fp->restoration[0].restoration_type;
    if (rtype != R2G_RESTORE_NONE) {
        int q = fp->quant_yac;
        d.base_q = host_dq_lookup(q);
        d.wiener_idx = q < 130 ? 0 : q < 190 ? 1 : q < 220 ? 2 : 3;
        if (rtype == R2G_RESTORE_NS_WIENER || rtype == R2G_RESTORE_SWITCHABLE) {
            int nci = fp->restoration[0].num_classes_idx;
            d.ns_ci = nci > 0 ? nci - 1 : -1;
        }
    }
    d.gdf_ref_dst_idx = 0;
    if (fp->gdf_enabled && (fp->frame_type & 1)) {
        static const int TBL[12] = {5, 1, 2, 3, 3, 3, 4, 4, 4, 4, 4, 5};
        int md = 0;
        int nr = fp->n_ref_frames < 2 ? fp->n_ref_frames : 2;
        for (int i = 0; i < nr; i++) md = md > fp->absrefdist[i] ? md : fp->absrefdist[i];
        d.gdf_ref_dst_idx = TBL[md < 11 ? md : 11];
    }

    // stage side-info: masks, restoration records packed to the fields the
    // filters read (LrPacked), then segmaps.  The deblock kernel applies the
    // reference's bottom-edge crop as it reads the masks.  With copy overlap,
    // masks in page-locked memory go straight to the device (asynchronously:
    // the caller keeps them unchanged until the frame's work completes);
    // otherwise they go through the frame's pinned staging buffer, which is
    // reused, so wait for its previous upload first.
    if (!f->side_done) CK(cudaEventCreateWithFlags(&f->side_done, cudaEventDisableTiming));
    size_t mbytes = (size_t)f->n_sb256 * sizeof(R2gAv2Filter);
    size_t lbytes = (size_t)f->n_sb256 * sizeof(LrPacked);
    bool direct = false;
    if (ctx->overlap) {
        cudaPointerAttributes am;
        direct = cudaPointerGetAttributes(&am, side->masks) == cudaSuccess && am.type == cudaMemoryTypeHost;
        cudaGetLastError();
    }
    CK(cudaEventSynchronize(f->side_done));
    LrPacked *pk = (LrPacked *)((char *)f->side_host + mbytes);
    for (int i = 0; i < f->n_sb256; i++)
        for (int pl = 0; pl < 3; pl++)
            for (int u = 0; u < 16; u++) {
                const R2gAv2RestorationUnit &src = side->lr[i].lr[pl][u];
                LrUnitPacked &dst = pk[i].lr[pl][u];
                dst.type = src.restoration_type;
                memcpy(dst.f, src.ns_filter[0], sizeof(dst.f));
                dst.pad = 0;
            }
    if (side->db_masks) {
        // the edge masks are built on the device: upload the rest of each
        // SB256 record only
        const size_t head = offsetof(R2gAv2Filter, qidx), tail = sizeof(R2gAv2Filter) - head;
        const char *src = (const char *)side->masks;
        if (!direct) {
            for (int i = 0; i < f->n_sb256; i++)
                memcpy((char *)f->side_host + i * sizeof(R2gAv2Filter) + head, src + i * sizeof(R2gAv2Filter) + head,
                       tail);
            src = (const char *)f->side_host;
        }
        CK(cudaMemcpy2DAsync((char *)f->side_dev + head, sizeof(R2gAv2Filter), src + head, sizeof(R2gAv2Filter),
                             tail, f->n_sb256, cudaMemcpyHostToDevice, cs));
        CK(cudaMemcpyAsync((char *)f->side_dev + mbytes, pk, lbytes, cudaMemcpyHostToDevice, cs));
        int rc2 = stage_db_masks(ctx, f, fp, *side->db_masks, d, cs);
        if (rc2 != R2G_OK) return rc2;
    } else if (direct) {
        CK(cudaMemcpyAsync(f->side_dev, side->masks, mbytes, cudaMemcpyHostToDevice, cs));
        CK(cudaMemcpyAsync((char *)f->side_dev + mbytes, pk, lbytes, cudaMemcpyHostToDevice, cs));
    } else {
        memcpy(f->side_host, side->masks, mbytes);
        CK(cudaMemcpyAsync(f->side_dev, f->side_host, mbytes + lbytes, cudaMemcpyHostToDevice, cs));
    }
    d.masks = (const R2gAv2Filter *)f->side_dev;
    d.lr = (const LrPacked *)((char *)f->side_dev + mbytes);
    size_t seg_y = side->segmap ? (size_t)side->segmap_stride * d.bh4 : 0;
    size_t seg_uv = side->segmap_uv ? (size_t)side->segmap_uv_stride * (d.bh4 >> 1) : 0;
    if (seg_y + seg_uv) {
        if (f->seg_bytes < seg_y + seg_uv) {
            r2g_dev_free(ctx, f->seg_dev, f->seg_bytes);
            if (f->seg_host) cudaFreeHost(f->seg_host);
            f->seg_dev = nullptr;
            f->seg_host = nullptr;
            f->seg_bytes = 0;
            int rc2 = r2g_dev_alloc(ctx, &f->seg_dev, seg_y + seg_uv);
            if (rc2 != R2G_OK) return rc2;
            CK(cudaMallocHost(&f->seg_host, seg_y + seg_uv));
            f->seg_bytes = seg_y + seg_uv;
        }
        if (seg_y) memcpy(f->seg_host, side->segmap, seg_y);
        if (seg_uv) memcpy((char *)f->seg_host + seg_y, side->segmap_uv, seg_uv);
        CK(cudaMemcpyAsync(f->seg_dev, f->seg_host, seg_y + seg_uv, cudaMemcpyHostToDevice, cs));
        d.segmap = seg_y ? (const uint8_t *)f->seg_dev : nullptr;
        d.segmap_uv = seg_uv ? (const uint8_t *)f->seg_dev + seg_y : nullptr;
        d.segmap_stride = side->segmap_stride;
        d.segmap_uv_stride = side->segmap_uv_stride;
    }
    CK(cudaEventRecord(f->side_done, cs));

    // buffers: 0 = recon (preserved), 1 = deblocked, 2 = CDEF out,
    // 3 = LR out, 4 = grain display copy
    void *p[5][3];
    for (int i = 0; i < 5; i++) plane_ptrs(f, i, p[i]);
    for (int i = 0; i < 3; i++) {
        d.R[i] = p[0][i];
        d.D[i] = d.deblock_on ? p[1][i] : p[0][i];
        d.C[i] = d.cdef_stage_on ? p[2][i] : d.D[i];
        d.L[i] = d.lr_on ? p[3][i] : d.C[i];
        d.G[i] = p[4][i];
    }
    f->out_buf = d.lr_on ? 3 : (d.cdef_stage_on ? 2 : (d.deblock_on ? 1 : 0));
    f->grain_buf = -1;
    return R2G_OK;
}

// ---------------------------------------------------------------- profiling
void r2g_prof_stage(R2gCtx *ctx, int stage, bool begin, int launches) {
    ctx->launches += launches;
    if (!ctx->profiling) return;
    if (begin) {
        if (stage == 0 || ctx->prof.empty()) {
            ProfRun r;
            for (int i = 0; i <= R2G_N_STAGES; i++) r.ev[i] = nullptr;
            for (int i = 0; i < R2G_N_STAGES; i++) r.have[i] = 0;
            ctx->prof.push_back(r);
        }
        ProfRun &r = ctx->prof.back();
        if (!r.ev[stage]) {
            cudaEventCreate(&r.ev[stage]);
            cudaEventRecord(r.ev[stage], ctx->stream);
        }
    } else {
        ProfRun &r = ctx->prof.back();
        if (!r.ev[stage + 1]) cudaEventCreate(&r.ev[stage + 1]);
        cudaEventRecord(r.ev[stage + 1], ctx->stream);
        r.have[stage] = launches;
    }
}

extern "C" int r2g_ctx_profile(R2gCtx *ctx, int enable) {
    if (!ctx) return R2G_E_INVALID;
    ctx->profiling = enable != 0;
    for (auto &r : ctx->prof)
        for (int i = 0; i <= R2G_N_STAGES; i++)
            if (r.ev[i]) cudaEventDestroy(r.ev[i]);
    ctx->prof.clear();
    for (int i = 0; i < R2G_N_STAGES; i++) {
        ctx->prof_ms[i] = 0;
        ctx->prof_launches[i] = 0;
    }
    return R2G_OK;
}

extern "C" int r2g_ctx_profile_read(R2gCtx *ctx, double *stage_ms, int64_t *stage_launches, int n) {
    if (!ctx) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    for (auto &r : ctx->prof) {
        for (int i = 0; i < R2G_N_STAGES; i++) {
            if (!r.have[i] || !r.ev[i] || !r.ev[i + 1]) continue;
            float ms = 0;
            if (cudaEventElapsedTime(&ms, r.ev[i], r.ev[i + 1]) == cudaSuccess) {
                ctx->prof_ms[i] += ms;
                ctx->prof_launches[i] += r.have[i];
            }
        }
        for (int i = 0; i <= R2G_N_STAGES; i++)
            if (r.ev[i]) cudaEventDestroy(r.ev[i]);
    }
    ctx->prof.clear();
    for (int i = 0; i < n && i < R2G_N_STAGES; i++) {
        if (stage_ms) stage_ms[i] = ctx->prof_ms[i];
        if (stage_launches) stage_launches[i] = ctx->prof_launches[i];
    }
    return R2G_OK;
}

extern "C" int64_t r2g_ctx_launch_count(R2gCtx *ctx) { return ctx ? ctx->launches : -1; }

extern "C" int r2g_ctx_set_stream(R2gCtx *ctx, void *stream) {
    if (!ctx) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    if (!ctx->own_stream) ctx->own_stream = ctx->stream;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return R2G_OK;
}

void r2g_launch_pipeline(R2gCtx *ctx, const DevFrame &d) {
    cudaStream_t s = ctx->stream;
    r2g_prof_stage(ctx, 0, true, 0);
    int n = r2g_launch_deblock(d, s);
    r2g_prof_stage(ctx, 0, false, n);
    r2g_prof_stage(ctx, 1, true, 0);
    n = r2g_launch_cdef(d, s);
    r2g_prof_stage(ctx, 1, false, n);
    r2g_prof_stage(ctx, 2, true, 0);
    n = r2g_launch_lr(d, s);
    r2g_prof_stage(ctx, 2, false, n);
}

extern "C" int r2g_frame_stage(R2gCtx *ctx, R2gFrame *f, const R2gFrameParams *fp, const R2gSideInfo *side,
                               uint32_t inloop_mask) {
    if (!ctx || !f) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (ctx->overlap) {
        // the side-info copies go on their own stream (the kernels of this
        // frame's previous run may still read what they overwrite)
        int rc = ensure_events(ctx, f);
        if (rc != R2G_OK) return rc;
        if (f->pend_comp) CK(cudaStreamWaitEvent(ctx->side_up_stream, f->ev_comp, 0));
        st = ctx->side_up_stream;
    }
    ctx->defer_mask_join = true;
    int rc = r2g_prepare(ctx, f, fp, side, inloop_mask, f->desc, st);
    ctx->defer_mask_join = false;
    if (rc != R2G_OK) return rc;
    f->staged = true;
    if (ctx->overlap) {
        CK(cudaEventRecord(f->ev_side, ctx->side_up_stream));
        f->pend_side = true;
    }
    return R2G_OK;
}

extern "C" int r2g_frame_run(R2gCtx *ctx, R2gFrame *f) {
    if (!ctx || !f) return R2G_E_INVALID;
    if (!f->staged) {
        set_err(ctx, "frame has no staged side-info");
        return R2G_E_INVALID;
    }
    CK(cudaSetDevice(ctx->device));
    int rc = r2g_frame_before_compute(ctx, f);
    if (rc != R2G_OK) return rc;
    r2g_launch_pipeline(ctx, f->desc);
    CK(cudaGetLastError());
    return r2g_frame_after_compute(ctx, f);
}

extern "C" int r2g_frame_read_masks(R2gCtx *ctx, R2gFrame *f, R2gAv2Filter *out, int n) {
    if (!ctx || !f || !out || n != f->n_sb256) return R2G_E_INVALID;
    if (!f->staged) {
        set_err(ctx, "frame has no staged side-info");
        return R2G_E_INVALID;
    }
    CK(cudaSetDevice(ctx->device));
    int rc = r2g_sync(ctx);
    if (rc != R2G_OK) return rc;
    CK(cudaMemcpy(out, f->side_dev, (size_t)n * sizeof(R2gAv2Filter), cudaMemcpyDeviceToHost));
    return R2G_OK;
}

extern "C" int r2g_frame_filter(R2gCtx *ctx, R2gFrame *f, const R2gFrameParams *fp, const R2gSideInfo *side,
                                uint32_t inloop_mask) {
    int rc = r2g_frame_stage(ctx, f, fp, side, inloop_mask);
    if (rc != R2G_OK) return rc;
    return r2g_frame_run(ctx, f);
}

extern "C" int r2g_filter_frame_host(R2gCtx *ctx, const R2gFrameParams *fp, const R2gSideInfo *side,
                                     uint32_t inloop_mask, const R2gFilmGrainData *fgd, uint32_t grain_seed,
                                     const void *src_y, const void *src_u, const void *src_v, int64_t y_stride,
                                     int64_t uv_stride, void *dst_y, void *dst_u, void *dst_v, void *grain_y,
                                     void *grain_u, void *grain_v) {
    if (!ctx || !fp) return R2G_E_INVALID;
    R2gFrame *f = nullptr;
    int rc = r2g_frame_alloc(ctx, fp->width, fp->height, fp->bitdepth, &f);
    if (rc != R2G_OK) return rc;
    if ((rc = r2g_frame_upload_recon(ctx, f, src_y, y_stride, src_u, src_v, uv_stride)) == R2G_OK &&
        (rc = r2g_frame_filter(ctx, f, fp, side, inloop_mask)) == R2G_OK &&
        (rc = r2g_download(ctx, f, 0, dst_y, y_stride, dst_u, dst_v, uv_stride)) == R2G_OK) {
        if (fgd && grain_y) {
            if ((rc = r2g_frame_grain(ctx, f, fgd, grain_seed)) == R2G_OK)
                rc = r2g_download(ctx, f, 1, grain_y, y_stride, grain_u, grain_v, uv_stride);
        }
        if (rc == R2G_OK) rc = r2g_sync(ctx);
    }
    r2g_frame_free(ctx, f);
    return rc;
}

// ---------------------------------------------------------------- tickets
int r2g_ticket_record(R2gCtx *ctx, uint64_t *ticket) {
    Ticket t;
    CK(cudaEventCreateWithFlags(&t.ev, cudaEventDisableTiming));
    CK(cudaEventRecord(t.ev, ctx->stream));
    t.id = ++ctx->next_ticket;
    ctx->tickets.push_back(t);
    *ticket = t.id;
    return R2G_OK;
}

extern "C" int r2g_wait(R2gCtx *ctx, uint64_t ticket, int timeout_ms) {
    if (!ctx) return R2G_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    size_t i = 0;
    for (; i < ctx->tickets.size(); i++)
        if (ctx->tickets[i].id == ticket) break;
    if (i == ctx->tickets.size()) {
        set_err(ctx, "unknown or already completed ticket");
        return R2G_E_INVALID;
    }
    cudaEvent_t ev = ctx->tickets[i].ev;
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) {
            set_err(ctx, "CUDA error: %s", cudaGetErrorString(q));
            return R2G_E_DEVICE;
        }
        if (timeout_ms == 0) return R2G_E_NOTREADY;
        if (timeout_ms > 0) {
            auto el = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0);
            if (el.count() >= timeout_ms) {
                set_err(ctx, "wait timed out");
                return R2G_E_TIMEOUT;
            }
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    cudaEventDestroy(ev);
    ctx->tickets.erase(ctx->tickets.begin() + i);
    return R2G_OK;
}
