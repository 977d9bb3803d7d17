// Host-side definitions of the opaque ABI handles, shared by the runtime,
// the batch scheduler and the film-grain stage.
#pragma once

#include <string>
#include <vector>

#include "r2g_common.cuh"

struct Ticket {
    uint64_t id;
    cudaEvent_t ev;
};

struct GrainCtx;    // grain.cu
struct BatchState;  // batch.cu

// Per-frame film-grain scratch of the batched path: three 82x73 templates and
// three 1024-entry scaling LUTs.
#define R2G_GRAIN_SCRATCH (3 * 73 * 82 * 2 + 3 * 1024)

enum { R2G_N_STAGES = 4 };

// Per-run profiling events: ev[i] .. ev[i+1] brackets stage i.
struct ProfRun {
    cudaEvent_t ev[R2G_N_STAGES + 1];
    int have[R2G_N_STAGES];
};

struct R2gCtx {
    int device = 0;
    int64_t budget = 0, used = 0;
    cudaStream_t stream = nullptr;       // filter stages
    cudaStream_t side_stream = nullptr;  // grain templates (frame-independent)
    DevTables tab{};
    std::string err;
    std::vector<Ticket> tickets;
    uint64_t next_ticket = 0;
    GrainCtx *grain = nullptr;
    BatchState *batch = nullptr;
    cudaStream_t own_stream = nullptr;
    // copy overlap (r2g_ctx_overlap_copies): per-frame uploads / staging on
    // up_stream, downloads on down_stream, ordered by per-frame events
    bool overlap = false;
    cudaStream_t up_stream = nullptr, down_stream = nullptr;
    // side-info staging of r2g_frame_stage: its own stream, so its small
    // copies (each bound by PCIe latency while downloads run) overlap the
    // recon upload instead of queueing behind it
    cudaStream_t side_up_stream = nullptr;
    cudaEvent_t fence_ev[3] = {nullptr, nullptr, nullptr};
    int64_t launches = 0;
    bool profiling = false;
    std::vector<ProfRun> prof;
    double prof_ms[R2G_N_STAGES] = {0};
    int64_t prof_launches[R2G_N_STAGES] = {0};
    // device control block: work counters of the per-frame persistent stage
    // kernels, then the fault word (bounded waits that ran out)
    StageSched *sched = nullptr;
    unsigned *fault = nullptr;
    unsigned *bad_blocks = nullptr;  // block records the mask builder skipped
    // set while r2g_frame_stage stages on the upload stream: the device mask
    // build is then joined by the frame's kernels, not by the upload stream
    bool defer_mask_join = false;
};
// bytes of the context's device control block
#define R2G_CTL_BYTES 256

struct R2gFrame {
    int w = 0, h = 0, bd = 8;
    int64_t stride[2] = {0, 0};  // bytes
    int64_t rows[2] = {0, 0};
    size_t plane_bytes[2] = {0, 0};
    size_t buf_bytes = 0;
    void *buf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // R, D, C, L, G
    int n_sb256 = 0;
    size_t side_bytes = 0;
    void *side_dev = nullptr;
    void *side_host = nullptr;  // pinned staging
    cudaEvent_t side_done = nullptr;  // last upload out of side_host finished
    void *seg_dev = nullptr;
    void *seg_host = nullptr;
    size_t seg_bytes = 0;
    int out_buf = -1, grain_buf = -1;
    bool staged = false;
    void *grain_scratch = nullptr;  // batched film grain (R2G_GRAIN_SCRATCH)
    DevFrame desc{};
    void *pack_buf = nullptr;  // packed Y4M payload (r2g_download_y4m)
    size_t pack_bytes = 0;
    // copy-overlap ordering: last upload / staging (up stream), last kernels
    // (context stream), last download (down stream) of this frame
    cudaEvent_t ev_up = nullptr, ev_comp = nullptr, ev_down = nullptr, ev_side = nullptr;
    bool pend_up = false, pend_comp = false, pend_down = false, pend_side = false;
    // device-built deblock masks (R2gSideInfo.db_masks): block records and
    // level maps on the device, a pinned staging copy of the records, and
    // the events that fork the build onto the side stream and join it back
    void *dbm_dev = nullptr, *dbm_host = nullptr;
    size_t dbm_bytes = 0, dbm_host_bytes = 0;
    cudaEvent_t ev_dbm[2] = {nullptr, nullptr};
    bool pend_dbm = false;  // the kernels must wait for ev_dbm[1]
};

// Device mask build (dbmask.cu): zero the frame's filter_y / filter_uv and
// build them from the block records; returns the kernels launched.
int r2g_launch_db_masks(const R2gDbMaskInput &in, const R2gDbBlock *dev_blocks, R2gAv2Filter *dev_masks,
                        int n_sb256, int sb256w, int bw4, int bh4, void *dev_levels, const uint8_t lossless[8],
                        const DevTables &tab, unsigned *bad, cudaStream_t s);
size_t r2g_db_levels_bytes(int bw4, int bh4);

int r2g_dev_alloc(R2gCtx *ctx, void **p, size_t bytes);
void r2g_dev_free(R2gCtx *ctx, void *p, size_t bytes);
// Validate and stage one frame's side-info (copies on `cs`, or the context
// stream when null) and fill its stage descriptor.
int r2g_prepare(R2gCtx *ctx, R2gFrame *f, const R2gFrameParams *fp, const R2gSideInfo *side, uint32_t inloop,
                DevFrame &d, cudaStream_t cs);
// 2-D plane copies between host planes and plane set `buf` of a frame.
int r2g_copy_planes(R2gCtx *ctx, const R2gFrame *f, int buf, const void *y, int64_t ys, const void *u,
                    const void *v, int64_t uvs, bool upload, cudaStream_t st);
size_t r2g_frame_device_bytes(int width, int height, int bitdepth);
// Parameter checks of r2g_prepare / r2g_frame_grain (no device work).
int r2g_validate(R2gCtx *ctx, const R2gFrame *f, const R2gFrameParams *fp, const R2gSideInfo *side);
int r2g_grain_validate(const R2gFilmGrainData *fgd, uint32_t seed);
// Stage and launch a batch: side-info copies on `copy_stream` (null = the
// context stream), kernels on the context stream after them.
int r2g_batch_enqueue(R2gCtx *ctx, const R2gBatchItem *items, int n, cudaStream_t copy_stream);
void r2g_launch_pipeline(R2gCtx *ctx, const DevFrame &d);
// Copy-overlap ordering of one frame's kernels on the context stream: wait
// for its pending upload and download before, record after (no-ops unless
// the context overlaps copies).
int r2g_frame_before_compute(R2gCtx *ctx, R2gFrame *f);
int r2g_frame_after_compute(R2gCtx *ctx, R2gFrame *f);
// Profiling hooks around one stage (no-ops unless profiling is enabled).
void r2g_prof_stage(R2gCtx *ctx, int stage, bool begin, int launches);
int r2g_ticket_record(R2gCtx *ctx, uint64_t *ticket);
void r2g_grain_ctx_free(R2gCtx *ctx);
void r2g_batch_free(R2gCtx *ctx);
