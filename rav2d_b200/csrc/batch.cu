// Batched execution: many frames, one persistent launch per stage.
//
// Every frame of a batch is staged as in the per-frame path (side-info on
// the device, DevFrame descriptor); then one staging blob carries the
// descriptors, the film-grain parameters and a work list per stage (item =
// frame << 22 | the frame's own item index) to the device, and a CUDA graph
// runs the persistent stage kernels over those lists:
//   deblock -> CDEF+CCSO -> loop restoration -> grain apply, with the grain
//   templates on a forked branch (they depend only on the grain parameters)
//   joined before the apply.
// The graph's kernels read the item counts from device memory, so one
// instantiated graph serves every batch that fits the slot's capacity.  Two
// slots alternate, so the host can stage batch k+1 while batch k runs.
//
// The grid of each persistent kernel (CTAs per SM, or one CTA per work
// item) and the tile shape of the stages that have a choice (loop
// restoration: 32 or 16 luma rows per work item) are chosen by a small
// autotuner: on the first batch of a given bit-depth mix it times every
// (shape, grid) pair per stage and keeps the fastest; the choice is cached
// per device in a text file ($R2G_TUNE_CACHE, default
// $HOME/.cache/rav2d_b200/autotune-v3.txt).  R2G_AUTOTUNE=0 skips tuning and
// uses the occupancy limit and the default shapes.
#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "r2g_runtime.h"

int r2g_grain_ready(int device);
int r2g_grain_enqueue(R2gCtx *ctx, R2gFrame *f, const R2gFilmGrainData *fgd, uint32_t seed);

namespace {

enum { N_BSTAGES = 4 };  // deblock, cdef, lr, grain apply
// Tuned grid choice meaning "one CTA per work item" (grid = the batch's item
// count; the hardware then hands items to SMs as CTAs finish) rather than a
// persistent grid of CTAs-per-SM x SMs.
constexpr int PER_ITEM = 255;
// Frames of at least this many luma samples skip the batch's persistent
// kernels and run through the per-frame pipeline (measured on a B200: 1080p
// and 4K frames filter faster per frame, 720p and smaller faster batched).
constexpr int64_t R2G_BATCH_DIRECT_PIX = 1500000;

struct Layout {
    int max_frames = 0;
    int max_items[N_BSTAGES] = {0, 0, 0, 0};
    size_t off_frames = 0, off_grain = 0, off_work[N_BSTAGES] = {0, 0, 0, 0}, bytes = 0;
};

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

static Layout make_layout(int frames, const int *items) {
    Layout L;
    L.max_frames = frames;
    size_t o = 256;  // counts
    L.off_frames = o;
    o = align256(o + sizeof(DevFrame) * frames);
    L.off_grain = o;
    o = align256(o + sizeof(GrainBatch) * frames);
    for (int k = 0; k < N_BSTAGES; k++) {
        L.max_items[k] = items[k];
        L.off_work[k] = o;
        o = align256(o + sizeof(uint32_t) * items[k]);
    }
    L.bytes = o;
    return L;
}

struct Slot {
    Layout L;
    char *host = nullptr;
    char *dev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int grids[N_BSTAGES + 1] = {0, 0, 0, 0, 0};
    cudaEvent_t done = nullptr;
    bool used = false;
};

}  // namespace

struct BatchState {
    Slot slot[2];
    int next = 0;
    int num_sms = 0;
    int occ[N_BSTAGES] = {0, 0, 0, 0};
    int tuned[3][N_BSTAGES] = {{0}};  // [8-bit, 10-bit, mixed][stage] CTAs per SM
    int shape[3][N_BSTAGES] = {{0}};  // tile shape (luma rows per work item; 0: the stage's fixed shape)
    int last[N_BSTAGES] = {0, 0, 0, 0};
    int last_rows[N_BSTAGES] = {0, 0, 0, 0};  // luma rows per work item of the last batch
    bool cache_loaded = false;
    std::string dev_name;
    cudaEvent_t fork = nullptr, join = nullptr, copied = nullptr, t0 = nullptr, t1 = nullptr;
};

static std::string cache_path() {
    const char *p = getenv("R2G_TUNE_CACHE");
    if (p && *p) return p;
    const char *h = getenv("HOME");
    return std::string(h ? h : "/tmp") + "/.cache/rav2d_b200/autotune-v3.txt";
}

static void load_cache(BatchState &b) {
    b.cache_loaded = true;
    FILE *fp = fopen(cache_path().c_str(), "r");
    if (!fp) return;
    char line[512];
    while (fgets(line, sizeof(line), fp)) {
        char name[256];
        int cls, k, v, shape;
        if (sscanf(line, "%255[^|]|%d|%d|%d|%d", name, &cls, &k, &v, &shape) == 5 && b.dev_name == name &&
            cls >= 0 && cls < 3 && k >= 0 && k < N_BSTAGES && v > 0 && (v <= b.occ[k] || v == PER_ITEM) &&
            (shape == 0 || (k == 2 && (shape == 16 || shape == 32)))) {
            b.tuned[cls][k] = v;
            b.shape[cls][k] = shape;
        }
    }
    fclose(fp);
}

static void save_cache(const BatchState &b, int cls) {
    std::string path = cache_path();
    std::string dir = path.substr(0, path.find_last_of('/'));
    std::string mk = dir;
    for (size_t i = 1; i <= mk.size(); i++)
        if (i == mk.size() || mk[i] == '/') mkdir(mk.substr(0, i).c_str(), 0755);
    FILE *fp = fopen(path.c_str(), "a");
    if (!fp) return;
    for (int k = 0; k < N_BSTAGES; k++)
        if (b.tuned[cls][k] > 0)
            fprintf(fp, "%s|%d|%d|%d|%d\n", b.dev_name.c_str(), cls, k, b.tuned[cls][k], b.shape[cls][k]);
    fclose(fp);
}

static void launch_stage(int k, const BatchArgs &a, int grid, cudaStream_t s) {
    switch (k) {
        case 0: r2g_batch_launch_deblock(a, grid, s); break;
        case 1: r2g_batch_launch_cdef(a, grid, s); break;
        case 2: r2g_batch_launch_lr(a, grid, s); break;
        default: r2g_batch_launch_grain_apply(a, grid, s); break;
    }
}

// The first 256 bytes of a slot's blob: item counts (ints 0..7), then the
// stage kernels' work counters at byte 64 (zeroed with each batch's upload;
// the kernels leave them zero after every launch).
static BatchArgs args_of(const R2gCtx *ctx, const Slot &s) {
    BatchArgs a;
    a.count = (const int *)s.dev;
    a.sched = (StageSched *)(s.dev + 64);
    a.fault = ctx->fault;
    a.frames = (const DevFrame *)(s.dev + s.L.off_frames);
    a.grain = (const GrainBatch *)(s.dev + s.L.off_grain);
    for (int k = 0; k < N_BSTAGES; k++) a.work[k] = (const uint32_t *)(s.dev + s.L.off_work[k]);
    return a;
}

void r2g_batch_free(R2gCtx *ctx) {
    BatchState *b = ctx->batch;
    if (!b) return;
    for (auto &s : b->slot) {
        if (s.exec) cudaGraphExecDestroy(s.exec);
        if (s.graph) cudaGraphDestroy(s.graph);
        if (s.host) cudaFreeHost(s.host);
        if (s.dev) r2g_dev_free(ctx, s.dev, s.L.bytes);
        if (s.done) cudaEventDestroy(s.done);
    }
    for (cudaEvent_t e : {b->fork, b->join, b->copied, b->t0, b->t1})
        if (e) cudaEventDestroy(e);
    delete b;
    ctx->batch = nullptr;
}

static int ensure_state(R2gCtx *ctx) {
    if (ctx->batch) return R2G_OK;
    BatchState *b = new BatchState();
    ctx->batch = b;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) return R2G_E_DEVICE;
    b->num_sms = prop.multiProcessorCount;
    b->dev_name = prop.name;
    b->occ[0] = r2g_batch_occupancy_deblock();
    b->occ[1] = r2g_batch_occupancy_cdef();
    b->occ[2] = r2g_batch_occupancy_lr();
    b->occ[3] = r2g_batch_occupancy_grain_apply();
    for (int k = 0; k < N_BSTAGES; k++)
        if (b->occ[k] < 1) b->occ[k] = 1;
    for (cudaEvent_t *e : {&b->fork, &b->join, &b->copied})
        if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return R2G_E_DEVICE;
    if (cudaEventCreate(&b->t0) != cudaSuccess || cudaEventCreate(&b->t1) != cudaSuccess) return R2G_E_DEVICE;
    for (auto &s : b->slot)
        if (cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) return R2G_E_DEVICE;
    return R2G_OK;
}

// Loop-restoration tile shapes the autotuner tries (luma rows per item).
constexpr int LR_SHAPES[2] = {32, 16};

// Sets every frame's loop-restoration item height to `rows` and rewrites the
// LR work list and its count in the slot's host blob; returns the count.
static int stage_lr_shape(Slot &s, std::vector<DevFrame> &frames, int rows, int *counts) {
    const int n = (int)frames.size();
    DevFrame *hf = (DevFrame *)(s.host + s.L.off_frames);
    uint32_t *w2 = (uint32_t *)(s.host + s.L.off_work[2]);
    int c2 = 0;
    for (int i = 0; i < n; i++) {
        frames[i].lr_rows = rows;
        hf[i].lr_rows = rows;
        for (int j = 0, e = r2g_lr_items(frames[i]); j < e; j++) w2[c2++] = ((uint32_t)i << 22) | j;
    }
    counts[2] = c2;
    memcpy(s.host, counts, sizeof(int) * 8);
    return c2;
}

// Copies the used part of the slot's host blob to the device.
static int copy_blob(R2gCtx *ctx, const Slot &s, const int *counts) {
    size_t used = s.L.off_work[N_BSTAGES - 1] + sizeof(uint32_t) * counts[3];
    return cudaMemcpyAsync(s.dev, s.host, used, cudaMemcpyHostToDevice, ctx->stream) == cudaSuccess ? R2G_OK
                                                                                                     : R2G_E_DEVICE;
}

// Times every legal (shape, grid) pair of each stage on the staged batch
// (stage outputs are pure functions of their inputs, so re-running a stage
// is harmless).  Leaves the blob staged with the chosen LR shape.
static int autotune(R2gCtx *ctx, BatchState &b, Slot &s, std::vector<DevFrame> &frames, int *counts, int cls) {
    const char *env = getenv("R2G_AUTOTUNE");
    bool enabled = !(env && env[0] == '0');
    BatchArgs a = args_of(ctx, s);
    for (int k = 0; k < N_BSTAGES; k++) {
        if (b.tuned[cls][k] > 0) continue;
        if (!enabled || counts[k] == 0) {
            if (!enabled) b.tuned[cls][k] = b.occ[k];
            if (k == 3 && counts[4] > 0)
                r2g_batch_launch_grain_template(a, counts[4] < b.num_sms ? counts[4] : b.num_sms, ctx->stream);
            continue;
        }
        if (k == 3 && counts[4] > 0)
            r2g_batch_launch_grain_template(a, counts[4] < b.num_sms ? counts[4] : b.num_sms, ctx->stream);
        float best = 1e30f;
        int best_v = b.occ[k], best_shape = 0;
        const int nshapes = k == 2 ? 2 : 1;
        for (int si = 0; si < nshapes; si++) {
            const int shape = k == 2 ? LR_SHAPES[si] : 0;
            if (k == 2) {
                stage_lr_shape(s, frames, shape, counts);
                if (copy_blob(ctx, s, counts) != R2G_OK) return R2G_E_DEVICE;
            }
            for (int v = 1; v <= b.occ[k] + 1; v++) {
                const int vv = v <= b.occ[k] ? v : PER_ITEM;
                const int grid = vv == PER_ITEM ? counts[k] : v * b.num_sms;
                launch_stage(k, a, grid, ctx->stream);  // warm
                cudaEventRecord(b.t0, ctx->stream);
                launch_stage(k, a, grid, ctx->stream);
                launch_stage(k, a, grid, ctx->stream);
                cudaEventRecord(b.t1, ctx->stream);
                if (cudaEventSynchronize(b.t1) != cudaSuccess) return R2G_E_DEVICE;
                float ms = 0;
                cudaEventElapsedTime(&ms, b.t0, b.t1);
                if (ms < best) {
                    best = ms;
                    best_v = vv;
                    best_shape = shape;
                }
            }
        }
        b.tuned[cls][k] = best_v;
        b.shape[cls][k] = best_shape;
        if (k == 2 && best_shape != LR_SHAPES[nshapes - 1]) {
            stage_lr_shape(s, frames, best_shape, counts);
            if (copy_blob(ctx, s, counts) != R2G_OK) return R2G_E_DEVICE;
        }
    }
    if (enabled) save_cache(b, cls);
    return cudaGetLastError() == cudaSuccess ? R2G_OK : R2G_E_DEVICE;
}

// Captures the batch graph with these grids.  An instantiated graph of the
// slot is updated in place when the topology allows (only grids changed),
// else re-instantiated.
static int build_graph(R2gCtx *ctx, BatchState &b, Slot &s, const int *grids, int tpl_grid) {
    if (s.graph) cudaGraphDestroy(s.graph);
    s.graph = nullptr;
    BatchArgs a = args_of(ctx, s);
    cudaStream_t st = ctx->stream;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return R2G_E_DEVICE;
    cudaEventRecord(b.fork, st);
    cudaStreamWaitEvent(ctx->side_stream, b.fork, 0);
    r2g_batch_launch_grain_template(a, tpl_grid, ctx->side_stream);
    cudaEventRecord(b.join, ctx->side_stream);
    for (int k = 0; k < 3; k++) launch_stage(k, a, grids[k], st);
    cudaStreamWaitEvent(st, b.join, 0);
    launch_stage(3, a, grids[3], st);
    if (cudaStreamEndCapture(st, &s.graph) != cudaSuccess) return R2G_E_DEVICE;
    bool updated = false;
    if (s.exec) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(s.exec, s.graph, &info) == cudaSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(s.exec);
            s.exec = nullptr;
        }
    }
    if (!updated && cudaGraphInstantiate(&s.exec, s.graph, 0) != cudaSuccess) return R2G_E_DEVICE;
    for (int k = 0; k < N_BSTAGES; k++) s.grids[k] = grids[k];
    s.grids[N_BSTAGES] = tpl_grid;
    return R2G_OK;
}

// The ranges the reference's parser admits (obu.rs:272-325): at most 14
// scaling points per plane (the kernels index points[pl][num - 1]), shifts
// from their 2-bit fields, a 16-bit seed.
int r2g_grain_validate(const R2gFilmGrainData *fgd, uint32_t seed) {
    if (fgd->block_size < 0 || fgd->block_size > 1 || fgd->ar_coeff_lag < 0 || fgd->ar_coeff_lag > 3 ||
        fgd->scaling_shift < 8 || fgd->scaling_shift > 11 || fgd->ar_coeff_shift < 6 || fgd->ar_coeff_shift > 9 ||
        fgd->grain_scale_shift < 0 || fgd->grain_scale_shift > 3 || seed > 0xffff)
        return R2G_E_INVALID;
    for (int pl = 0; pl < 3; pl++)
        if (fgd->num_points[pl] < 0 || fgd->num_points[pl] > 14) return R2G_E_INVALID;
    return R2G_OK;
}

int r2g_batch_enqueue(R2gCtx *ctx, const R2gBatchItem *items, int n, cudaStream_t copy_stream) {
    if (!ctx || (!items && n > 0) || n < 0 || n > 1023) return R2G_E_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return R2G_E_DEVICE;
    int rc = ensure_state(ctx);
    if (rc != R2G_OK) return rc;
    BatchState &b = *ctx->batch;
    if (!b.cache_loaded) load_cache(b);
    if (r2g_grain_ready(ctx->device) != R2G_OK) return R2G_E_DEVICE;

    // stage every frame; collect descriptors and grain parameters of the
    // frames the batch's persistent kernels take.  A frame of at least
    // R2G_BATCH_DIRECT_PIX luma samples fills the GPU by itself: it runs
    // through the per-frame pipeline instead (its stages overlap the next
    // frame's by programmatic dependent launch, which a batch's stage
    // barriers do not allow), before the batch on the same stream.
    std::vector<DevFrame> frames;
    frames.reserve(n);
    std::vector<int> direct, batched;
    std::vector<GrainBatch> grains;
    int counts[8] = {0};
    bool any8 = false, any10 = false;
    for (int i = 0; i < n; i++) {
        R2gFrame *f = items[i].frame;
        if (!f) return R2G_E_INVALID;
        if (items[i].fp || items[i].side) {
            rc = r2g_prepare(ctx, f, items[i].fp, items[i].side, items[i].inloop_mask, f->desc, copy_stream);
            if (rc != R2G_OK) return rc;
            f->staged = true;
        } else if (!f->staged) {
            ctx->err = "batch item without side-info on a frame that was never staged";
            return R2G_E_INVALID;
        }
        if (items[i].fgd && r2g_grain_validate(items[i].fgd, items[i].grain_seed) != R2G_OK) {
            ctx->err = "film-grain parameters out of range";
            return R2G_E_INVALID;
        }
        if ((int64_t)f->w * f->h >= R2G_BATCH_DIRECT_PIX) {
            direct.push_back(i);
            continue;
        }
        batched.push_back(i);
        frames.push_back(f->desc);
        (f->bd > 8 ? any10 : any8) = true;
        counts[0] += r2g_deblock_items(f->desc);
        counts[1] += r2g_cdef_items(f->desc);
        if (items[i].fgd) {
            if (!f->grain_scratch) {
                rc = r2g_dev_alloc(ctx, &f->grain_scratch, R2G_GRAIN_SCRATCH);
                if (rc != R2G_OK) return rc;
            }
            GrainBatch g;
            memset(&g, 0, sizeof(g));
            r2g_grain_params(*items[i].fgd, items[i].grain_seed, f->bd, g);
            g.frame = (int)frames.size() - 1;
            g.lut = (int16_t *)f->grain_scratch;
            g.scaling = (uint8_t *)f->grain_scratch + 3 * 73 * 82 * 2;
            counts[3] += r2g_grain_items(f->w, f->h, items[i].fgd->block_size);
            grains.push_back(g);
            f->grain_buf = 4;
        }
    }
    counts[4] = (int)grains.size();
    if (copy_stream && copy_stream != ctx->stream) {
        // the kernels wait for this batch's side-info (and any recon uploads
        // the caller enqueued before) on the copy stream
        if (cudaEventRecord(b.copied, copy_stream) != cudaSuccess ||
            cudaStreamWaitEvent(ctx->stream, b.copied, 0) != cudaSuccess)
            return R2G_E_DEVICE;
    }
    for (int i : direct) {
        R2gFrame *f = items[i].frame;
        rc = r2g_frame_before_compute(ctx, f);
        if (rc != R2G_OK) return rc;
        r2g_launch_pipeline(ctx, f->desc);
        if (cudaGetLastError() != cudaSuccess) return R2G_E_DEVICE;
        f->out_buf = f->desc.lr_on ? 3 : (f->desc.cdef_stage_on ? 2 : (f->desc.deblock_on ? 1 : 0));
        if (items[i].fgd) {
            rc = r2g_grain_enqueue(ctx, f, items[i].fgd, items[i].grain_seed);
            if (rc != R2G_OK) return rc;
        }
        rc = r2g_frame_after_compute(ctx, f);
        if (rc != R2G_OK) return rc;
    }
    if (batched.empty()) return R2G_OK;
    const int nb = (int)batched.size();
    const int cls = any8 && any10 ? 2 : (any10 ? 1 : 0);
    // loop-restoration tile shape: the tuned one, else the default; while
    // the stage is still to be tuned, room for the largest item count
    const int lr_shape = b.shape[cls][2] > 0 ? b.shape[cls][2] : LR_SHAPES[0];
    int lr_cap = 0;
    for (int rows : LR_SHAPES) {
        int c = 0;
        for (DevFrame &fr : frames) {
            fr.lr_rows = rows;
            c += r2g_lr_items(fr);
        }
        if (rows == lr_shape) counts[2] = c;
        if (b.tuned[cls][2] == 0 && c > lr_cap) lr_cap = c;
    }
    for (DevFrame &fr : frames) fr.lr_rows = lr_shape;

    // slot and capacity
    Slot &s = b.slot[b.next];
    b.next ^= 1;
    if (s.used && cudaEventSynchronize(s.done) != cudaSuccess) return R2G_E_DEVICE;
    int need[N_BSTAGES];
    for (int k = 0; k < N_BSTAGES; k++) need[k] = k == 2 && lr_cap > counts[2] ? lr_cap : counts[k];
    bool fits = nb <= s.L.max_frames;
    for (int k = 0; k < N_BSTAGES; k++) fits = fits && need[k] <= s.L.max_items[k];
    if (!fits) {
        int want_items[N_BSTAGES];
        for (int k = 0; k < N_BSTAGES; k++)
            want_items[k] = need[k] > s.L.max_items[k] ? need[k] + need[k] / 2 + 64 : s.L.max_items[k];
        Layout L = make_layout(nb > s.L.max_frames ? nb + nb / 2 + 4 : s.L.max_frames, want_items);
        if (s.host) cudaFreeHost(s.host);
        if (s.dev) r2g_dev_free(ctx, s.dev, s.L.bytes);
        s.host = nullptr;
        s.dev = nullptr;
        if (s.exec) cudaGraphExecDestroy(s.exec);
        if (s.graph) cudaGraphDestroy(s.graph);
        s.exec = nullptr;
        s.graph = nullptr;
        s.L = Layout();
        if (cudaMallocHost((void **)&s.host, L.bytes) != cudaSuccess) return R2G_E_OOM;
        rc = r2g_dev_alloc(ctx, (void **)&s.dev, L.bytes);
        if (rc != R2G_OK) return rc;
        s.L = L;
    }
    // fill the staging blob
    memset(s.host, 0, 256);
    memcpy(s.host, counts, sizeof(counts));
    memcpy(s.host + s.L.off_frames, frames.data(), sizeof(DevFrame) * nb);
    if (!grains.empty()) memcpy(s.host + s.L.off_grain, grains.data(), sizeof(GrainBatch) * grains.size());
    {
        uint32_t *w0 = (uint32_t *)(s.host + s.L.off_work[0]);
        uint32_t *w1 = (uint32_t *)(s.host + s.L.off_work[1]);
        uint32_t *w2 = (uint32_t *)(s.host + s.L.off_work[2]);
        int c0 = 0, c1 = 0, c2 = 0;
        for (int i = 0; i < nb; i++) {
            uint32_t hi = (uint32_t)i << 22;
            for (int j = 0, e = r2g_deblock_items(frames[i]); j < e; j++) w0[c0++] = hi | j;
            for (int j = 0, e = r2g_cdef_items(frames[i]); j < e; j++) w1[c1++] = hi | j;
            for (int j = 0, e = r2g_lr_items(frames[i]); j < e; j++) w2[c2++] = hi | j;
        }
        uint32_t *w3 = (uint32_t *)(s.host + s.L.off_work[3]);
        int c3 = 0;
        for (size_t gi = 0; gi < grains.size(); gi++) {
            const DevFrame &f = frames[grains[gi].frame];
            int e = r2g_grain_items(f.w, f.h, grains[gi].gp.d.block_size);
            for (int j = 0; j < e; j++) w3[c3++] = ((uint32_t)gi << 22) | j;
        }
    }
    rc = copy_blob(ctx, s, counts);
    if (rc != R2G_OK) return rc;

    // grid and tile-shape choice (autotuned per bit-depth mix), graph
    // (re)build, launch
    rc = autotune(ctx, b, s, frames, counts, cls);
    if (rc != R2G_OK) return rc;
    int grids[N_BSTAGES];
    b.last_rows[0] = 64;
    b.last_rows[1] = 32;
    b.last_rows[2] = frames.empty() ? 0 : frames[0].lr_rows;
    b.last_rows[3] = 0;
    for (const GrainBatch &g : grains) b.last_rows[3] = 16 << g.gp.d.block_size;
    for (int k = 0; k < N_BSTAGES; k++) {
        int v = b.tuned[cls][k] > 0 ? b.tuned[cls][k] : b.occ[k];
        b.last[k] = v == PER_ITEM ? 0 : v;
        grids[k] = v == PER_ITEM ? (counts[k] > 0 ? counts[k] : 1) : v * b.num_sms;
    }
    const int tpl_grid = b.num_sms;
    bool same = s.exec != nullptr && s.grids[N_BSTAGES] == tpl_grid;
    for (int k = 0; k < N_BSTAGES; k++) same = same && s.grids[k] == grids[k];
    if (!same) {
        rc = build_graph(ctx, b, s, grids, tpl_grid);
        if (rc != R2G_OK) return rc;
    }
    for (int i : batched) {
        rc = r2g_frame_before_compute(ctx, items[i].frame);
        if (rc != R2G_OK) return rc;
    }
    if (cudaGraphLaunch(s.exec, ctx->stream) != cudaSuccess) return R2G_E_DEVICE;
    for (int i : batched) {
        rc = r2g_frame_after_compute(ctx, items[i].frame);
        if (rc != R2G_OK) return rc;
    }
    ctx->launches += 5;
    if (cudaEventRecord(s.done, ctx->stream) != cudaSuccess) return R2G_E_DEVICE;
    s.used = true;
    for (int i : batched) {
        R2gFrame *f = items[i].frame;
        f->out_buf = f->desc.lr_on ? 3 : (f->desc.cdef_stage_on ? 2 : (f->desc.deblock_on ? 1 : 0));
    }
    if (cudaGetLastError() != cudaSuccess) return R2G_E_DEVICE;
    return R2G_OK;
}

extern "C" int r2g_batch_submit(R2gCtx *ctx, const R2gBatchItem *items, int n, uint64_t *ticket) {
    if (!ticket) return R2G_E_INVALID;
    int rc = r2g_batch_enqueue(ctx, items, n, nullptr);
    if (rc != R2G_OK) return rc;
    return r2g_ticket_record(ctx, ticket);
}

extern "C" int r2g_batch_tile_rows(R2gCtx *ctx, int32_t *rows, int n) {
    if (!ctx || !rows) return R2G_E_INVALID;
    if (!ctx->batch) return 0;
    for (int k = 0; k < n && k < N_BSTAGES; k++) rows[k] = ctx->batch->last_rows[k];
    return N_BSTAGES;
}

extern "C" int r2g_batch_config(R2gCtx *ctx, int32_t *ctas_per_sm, int n) {
    if (!ctx || !ctas_per_sm) return R2G_E_INVALID;
    if (!ctx->batch) return 0;
    for (int k = 0; k < n && k < N_BSTAGES; k++) ctas_per_sm[k] = ctx->batch->last[k];
    return ctx->batch->num_sms;
}
