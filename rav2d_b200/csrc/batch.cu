// Batched submission: many frames, one ticket.
#include "r2g_runtime.h"

int r2g_grain_enqueue(R2gCtx *ctx, R2gFrame *f, const R2gFilmGrainData *fgd, uint32_t seed);

extern "C" int r2g_batch_submit(R2gCtx *ctx, const R2gBatchItem *items, int n, uint64_t *ticket) {
    if (!ctx || (!items && n > 0) || n < 0 || !ticket) return R2G_E_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return R2G_E_DEVICE;
    for (int i = 0; i < n; i++) {
        R2gFrame *f = items[i].frame;
        if (!f) return R2G_E_INVALID;
        int rc = r2g_prepare(ctx, f, items[i].fp, items[i].side, items[i].inloop_mask, f->desc);
        if (rc != R2G_OK) return rc;
        f->staged = true;
        r2g_launch_pipeline(ctx, f->desc);
        if (items[i].fgd) {
            if (items[i].grain_seed > 0xffff) return R2G_E_INVALID;
            rc = r2g_grain_enqueue(ctx, f, items[i].fgd, items[i].grain_seed);
            if (rc != R2G_OK) return rc;
        }
    }
    if (cudaGetLastError() != cudaSuccess) return R2G_E_DEVICE;
    return r2g_ticket_record(ctx, ticket);
}
