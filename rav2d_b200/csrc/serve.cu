// Serving: continuous batching of frames from many concurrent streams.
//
// Requests (one decoded frame of one stream: its recon planes and side-info
// in host memory, and where to put the output) are queued by
// r2g_server_submit from any thread.  One worker thread owns all CUDA work:
//
//   admit    take queued requests in arrival order (a stream's frames stay in
//            order) and bind each to one of its stream's device-resident
//            frames; frames are allocated on first use under the server's
//            device-memory budget, evicting the least-recently-used idle
//            stream when the budget is full; a request that cannot fit even
//            in an empty budget fails with R2G_E_OOM, one that must wait for
//            memory stays queued;
//   issue    every admitted request goes into the next batch at once
//            (continuous batching: requests that arrived while earlier
//            batches run join the next one): recon uploads and side-info
//            staging on the upload stream, the batched stage kernels on the
//            context stream, output downloads on the download stream.  Up to
//            two batches are in flight, so the uploads of batch k+1, the
//            kernels of batch k and the downloads of batch k-1 overlap;
//   retire   a host callback after each batch's downloads wakes the worker,
//            which completes the batch's requests (latency = submit ->
//            output in host memory) and frees their frames for reuse.
//
// The stream's filtered frames stay resident on the device after a request
// completes (the reference frames of a decoder), until the stream is closed
// or evicted.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "r2g_runtime.h"

namespace {

using Clock = std::chrono::steady_clock;

struct StreamRes;

struct Req {
    uint64_t id = 0;
    R2gServeRequest r{};
    R2gFrameParams fp{};
    R2gSideInfo side{};
    R2gFilmGrainData fgd{};
    bool has_fgd = false;
    Clock::time_point t_submit, t_issue, t_done;
    int status = R2G_OK;
    bool done = false;
    int batch_frames = 0;
    StreamRes *sr = nullptr;
    int slot = -1;
};

struct StreamRes {
    int id = 0;
    int w = 0, h = 0, bd = 0;
    std::vector<R2gFrame *> frames;
    std::vector<bool> busy;
    int64_t bytes = 0;
    uint64_t last_use = 0;
    int inflight = 0;
};

struct Batch {
    std::vector<Req *> reqs;
    cudaEvent_t done = nullptr;
    std::atomic<bool> complete{false};  // set by the host callback, lock-free
};

}  // namespace

struct R2gServer {
    R2gCtx *ctx = nullptr;
    R2gServeConfig cfg{};
    int64_t budget = 0, resident = 0;
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t computed = nullptr;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> pending;
    std::map<uint64_t, Req *> reqs;
    std::map<int, StreamRes *> streams;
    std::deque<Batch *> inflight;
    std::vector<Batch *> free_batches;
    uint64_t next_id = 1, use_clock = 0;
    bool stop = false;
    bool fresh_frames = false;      // frames allocated since the last issue
    std::vector<int> to_close;      // streams whose frames the worker frees
    std::thread worker;
    // statistics
    std::vector<double> lat_us;
    int64_t completed = 0, failed = 0, batches = 0, batch_frames = 0, evictions = 0;
    double mpix = 0, busy_s = 0;
    Clock::time_point t_first, t_last;
    bool any = false;
};

// Runs on the driver's callback thread after a batch's downloads.  It must
// not take the server mutex: the worker may hold it inside a CUDA call that
// waits for this very callback (cudaFree synchronises the device), so it only
// sets a flag and wakes the worker (which also re-checks on a short timer, in
// case this wake-up lands between its check and its wait).
static void CUDART_CB batch_done_cb(void *p) {
    auto *pair = (std::pair<R2gServer *, Batch *> *)p;
    R2gServer *s = pair->first;
    pair->second->complete.store(true, std::memory_order_release);
    s->cv_work.notify_one();
    delete pair;
}

static void free_stream_frames(R2gServer *s, StreamRes *sr) {
    for (R2gFrame *f : sr->frames) r2g_frame_free(s->ctx, f);
    sr->frames.clear();
    sr->busy.clear();
    s->resident -= sr->bytes;
    sr->bytes = 0;
}

static bool any_busy(const R2gServer *s) {
    for (auto &kv : s->streams)
        if (kv.second->inflight) return true;
    return false;
}

// Finds a free resident frame of the request's stream, allocating one when
// the stream has fewer than frames_per_stream and the budget allows (after
// evicting idle streams).  Returns 1 bound, 0 wait, <0 fail.
static int bind_frame(R2gServer *s, Req *q) {
    const int w = q->fp.width, h = q->fp.height, bd = q->fp.bitdepth;
    {
        // reject a bad frame alone, before it can fail a whole batch
        if ((w & 7) || (h & 7) || w <= 0 || h <= 0 || (bd != 8 && bd != 10)) return R2G_E_INVALID;
        R2gFrame probe;
        probe.w = w;
        probe.h = h;
        probe.bd = bd;
        int bw4 = ((w + 7) >> 3) << 1, bh4 = ((h + 7) >> 3) << 1;
        probe.n_sb256 = ((bw4 + 63) >> 6) * ((bh4 + 63) >> 6);
        if (r2g_validate(s->ctx, &probe, &q->fp, &q->side) != R2G_OK) return R2G_E_INVALID;
        if (q->has_fgd && r2g_grain_validate(&q->fgd, q->r.grain_seed) != R2G_OK) return R2G_E_INVALID;
    }
    StreamRes *&sr = s->streams[q->r.stream_id];
    if (!sr) {
        sr = new StreamRes();
        sr->id = q->r.stream_id;
    }
    if (!sr->frames.empty() && (sr->w != w || sr->h != h || sr->bd != bd)) {
        // the stream changed format: drop its frames once they are idle
        if (sr->inflight) return 0;
        free_stream_frames(s, sr);
    }
    sr->w = w;
    sr->h = h;
    sr->bd = bd;
    for (size_t i = 0; i < sr->frames.size(); i++)
        if (!sr->busy[i]) {
            sr->busy[i] = true;
            q->sr = sr;
            q->slot = (int)i;
            return 1;
        }
    if ((int)sr->frames.size() >= s->cfg.frames_per_stream) return 0;
    const int64_t fb = (int64_t)r2g_frame_device_bytes(w, h, bd);
    if (fb <= 0) return R2G_E_INVALID;
    if (fb > s->budget) return R2G_E_OOM;
    while (s->resident + fb > s->budget) {
        StreamRes *victim = nullptr;
        for (auto &kv : s->streams) {
            StreamRes *o = kv.second;
            if (o == sr || o->inflight || o->frames.empty()) continue;
            if (!victim || o->last_use < victim->last_use) victim = o;
        }
        if (!victim) return any_busy(s) ? 0 : R2G_E_OOM;
        free_stream_frames(s, victim);
        s->evictions++;
    }
    R2gFrame *f = nullptr;
    int rc = r2g_frame_alloc(s->ctx, w, h, bd, &f);
    if (rc != R2G_OK) return rc == R2G_E_OOM && any_busy(s) ? 0 : rc;
    s->fresh_frames = true;
    sr->frames.push_back(f);
    sr->busy.push_back(true);
    sr->bytes += fb;
    s->resident += fb;
    q->sr = sr;
    q->slot = (int)sr->frames.size() - 1;
    return 1;
}

static void finish(R2gServer *s, Req *q, int status) {
    q->status = status;
    q->done = true;
    q->t_done = Clock::now();
    if (status == R2G_OK) {
        double us = std::chrono::duration<double, std::micro>(q->t_done - q->t_submit).count();
        s->lat_us.push_back(us);
        s->completed++;
        s->mpix += (double)q->fp.width * q->fp.height / 1e6;
        if (!s->any || q->t_submit < s->t_first) s->t_first = q->t_submit;
        s->t_last = q->t_done;
        s->any = true;
    } else {
        s->failed++;
    }
    if (q->sr) {
        q->sr->busy[q->slot] = false;
        q->sr->inflight--;
        q->sr->last_use = ++s->use_clock;
    }
}

// Enqueues one batch; called without the lock (the worker is the only thread
// that touches CUDA or the resident frames).
static int issue(R2gServer *s, Batch *b, bool fresh) {
    R2gCtx *ctx = s->ctx;
    if (fresh) {
        // new frames are zero-filled on the context stream: order the
        // uploads into them after that
        if (cudaEventRecord(s->computed, ctx->stream) != cudaSuccess ||
            cudaStreamWaitEvent(s->up, s->computed, 0) != cudaSuccess)
            return R2G_E_DEVICE;
    }
    std::vector<R2gBatchItem> items(b->reqs.size());
    for (size_t i = 0; i < b->reqs.size(); i++) {
        Req *q = b->reqs[i];
        R2gFrame *f = q->sr->frames[q->slot];
        int rc = r2g_copy_planes(ctx, f, 0, q->r.src_y, q->r.src_y_stride, q->r.src_u, q->r.src_v,
                                 q->r.src_uv_stride, true, s->up);
        if (rc != R2G_OK) return rc;
        items[i].frame = f;
        items[i].fp = &q->fp;
        items[i].side = &q->side;
        items[i].inloop_mask = q->r.inloop_mask;
        items[i].fgd = q->has_fgd ? &q->fgd : nullptr;
        items[i].grain_seed = q->r.grain_seed;
    }
    int rc = r2g_batch_enqueue(ctx, items.data(), (int)items.size(), s->up);
    if (rc != R2G_OK) return rc;
    if (cudaEventRecord(s->computed, ctx->stream) != cudaSuccess ||
        cudaStreamWaitEvent(s->down, s->computed, 0) != cudaSuccess)
        return R2G_E_DEVICE;
    for (Req *q : b->reqs) {
        R2gFrame *f = q->sr->frames[q->slot];
        int disp = q->has_fgd && f->grain_buf >= 0 ? f->grain_buf : f->out_buf;
        rc = r2g_copy_planes(ctx, f, disp, q->r.dst_y, q->r.dst_y_stride, q->r.dst_u, q->r.dst_v,
                             q->r.dst_uv_stride, false, s->down);
        if (rc != R2G_OK) return rc;
        if (q->r.ref_y) {
            rc = r2g_copy_planes(ctx, f, f->out_buf, q->r.ref_y, q->r.dst_y_stride, q->r.ref_u, q->r.ref_v,
                                 q->r.dst_uv_stride, false, s->down);
            if (rc != R2G_OK) return rc;
        }
    }
    if (cudaEventRecord(b->done, s->down) != cudaSuccess) return R2G_E_DEVICE;
    auto *pair = new std::pair<R2gServer *, Batch *>(s, b);
    if (cudaLaunchHostFunc(s->down, batch_done_cb, pair) != cudaSuccess) {
        delete pair;
        return R2G_E_DEVICE;
    }
    return R2G_OK;
}

static void worker_main(R2gServer *s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // retire completed batches (in order)
        bool retired = false;
        while (!s->inflight.empty() && s->inflight.front()->complete.load(std::memory_order_acquire)) {
            Batch *b = s->inflight.front();
            s->inflight.pop_front();
            for (Req *q : b->reqs) finish(s, q, R2G_OK);
            b->reqs.clear();
            b->complete.store(false, std::memory_order_relaxed);
            s->free_batches.push_back(b);
            retired = true;
        }
        if (retired) s->cv_done.notify_all();
        // streams closed by the caller, once idle
        for (size_t i = 0; i < s->to_close.size();) {
            auto it = s->streams.find(s->to_close[i]);
            bool queued = false;
            for (Req *q : s->pending) queued = queued || q->r.stream_id == s->to_close[i];
            if (it != s->streams.end() && (it->second->inflight || queued)) {
                i++;
                continue;
            }
            if (it != s->streams.end()) {
                free_stream_frames(s, it->second);
                delete it->second;
                s->streams.erase(it);
            }
            s->to_close.erase(s->to_close.begin() + i);
        }
        if (s->stop && s->pending.empty() && s->inflight.empty()) break;
        // admit and issue
        Batch *b = nullptr;
        if (!s->pending.empty() && (int)s->inflight.size() < 2) {
            std::vector<Req *> take;
            std::vector<int> blocked_streams;
            bool failed_any = false;
            for (auto it = s->pending.begin(); it != s->pending.end() && (int)take.size() < s->cfg.max_batch;) {
                Req *q = *it;
                if (std::find(blocked_streams.begin(), blocked_streams.end(), q->r.stream_id) !=
                    blocked_streams.end()) {
                    ++it;
                    continue;
                }
                int rc = bind_frame(s, q);
                if (rc == 1) {
                    q->sr->inflight++;
                    take.push_back(q);
                    it = s->pending.erase(it);
                } else if (rc == 0) {
                    blocked_streams.push_back(q->r.stream_id);
                    ++it;
                } else {
                    finish(s, q, rc);
                    failed_any = true;
                    it = s->pending.erase(it);
                }
            }
            if (failed_any) s->cv_done.notify_all();
            if (!take.empty()) {
                if (s->free_batches.empty()) {
                    Batch *nb = new Batch();
                    cudaEventCreateWithFlags(&nb->done, cudaEventDisableTiming);
                    s->free_batches.push_back(nb);
                }
                b = s->free_batches.back();
                s->free_batches.pop_back();
                b->reqs = take;
                auto now = Clock::now();
                for (Req *q : take) {
                    q->t_issue = now;
                    q->batch_frames = (int)take.size();
                }
            }
        }
        if (b) {
            const bool fresh = s->fresh_frames;
            s->fresh_frames = false;
            lk.unlock();
            auto t0 = Clock::now();
            int rc = issue(s, b, fresh);
            auto t1 = Clock::now();
            lk.lock();
            s->busy_s += std::chrono::duration<double>(t1 - t0).count();
            if (rc == R2G_OK) {
                s->inflight.push_back(b);
                s->batches++;
                s->batch_frames += (int64_t)b->reqs.size();
            } else {
                // nothing of a failed batch is trusted: wait for what was
                // enqueued, then fail its requests
                lk.unlock();
                cudaStreamSynchronize(s->up);
                cudaStreamSynchronize(s->ctx->stream);
                cudaStreamSynchronize(s->down);
                lk.lock();
                for (Req *q : b->reqs) finish(s, q, rc);
                b->reqs.clear();
                s->free_batches.push_back(b);
                s->cv_done.notify_all();
            }
            continue;
        }
        if (s->inflight.empty())
            s->cv_work.wait(lk);
        else
            s->cv_work.wait_for(lk, std::chrono::microseconds(500));
    }
}

extern "C" int r2g_server_create(R2gCtx *ctx, const R2gServeConfig *cfg, R2gServer **out) {
    if (!ctx || !out) return R2G_E_INVALID;
    *out = nullptr;
    R2gServer *s = new R2gServer();
    s->ctx = ctx;
    if (cfg) s->cfg = *cfg;
    if (s->cfg.max_batch <= 0 || s->cfg.max_batch > 1023) s->cfg.max_batch = 64;
    if (s->cfg.frames_per_stream <= 0) s->cfg.frames_per_stream = 2;
    s->budget = s->cfg.mem_budget > 0 ? s->cfg.mem_budget : (ctx->budget > 0 ? ctx->budget : INT64_MAX / 2);
    if (cudaSetDevice(ctx->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->computed, cudaEventDisableTiming) != cudaSuccess) {
        delete s;
        return R2G_E_DEVICE;
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return R2G_OK;
}

extern "C" int r2g_server_submit(R2gServer *s, const R2gServeRequest *req, uint64_t *id) {
    if (!s || !req || !id || !req->fp || !req->side || !req->src_y || !req->src_u || !req->src_v || !req->dst_y ||
        !req->dst_u || !req->dst_v)
        return R2G_E_INVALID;
    Req *q = new Req();
    q->r = *req;
    q->fp = *req->fp;
    q->side = *req->side;
    if (req->fgd) {
        q->fgd = *req->fgd;
        q->has_fgd = true;
    }
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete q;
            return R2G_E_INVALID;
        }
        q->id = s->next_id++;
        s->reqs[q->id] = q;
        s->pending.push_back(q);
    }
    *id = q->id;
    s->cv_work.notify_one();
    return R2G_OK;
}

extern "C" int r2g_server_wait(R2gServer *s, uint64_t id, int timeout_ms, R2gServeResult *res) {
    if (!s) return R2G_E_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return R2G_E_INVALID;
    Req *q = it->second;
    if (!q->done) {
        if (timeout_ms == 0) return R2G_E_NOTREADY;
        if (timeout_ms < 0)
            s->cv_done.wait(lk, [&] { return q->done; });
        else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return q->done; }))
            return R2G_E_TIMEOUT;
    }
    if (res) {
        res->status = q->status;
        res->batch_frames = q->batch_frames;
        res->queue_us = q->status == R2G_OK
                            ? std::chrono::duration<double, std::micro>(q->t_issue - q->t_submit).count()
                            : 0.0;
        res->latency_us = std::chrono::duration<double, std::micro>(q->t_done - q->t_submit).count();
    }
    s->reqs.erase(it);
    delete q;
    return R2G_OK;
}

extern "C" int r2g_server_close_stream(R2gServer *s, int32_t stream_id) {
    if (!s) return R2G_E_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->to_close.push_back(stream_id);
    }
    s->cv_work.notify_one();
    return R2G_OK;
}

// nearest-rank percentile
static double pct(std::vector<double> v, double p) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    size_t n = v.size(), k = (size_t)std::ceil(p / 100.0 * (double)n);
    k = k < 1 ? 1 : (k > n ? n : k);
    return v[k - 1];
}

extern "C" int r2g_server_stats(R2gServer *s, R2gServeStats *st, int reset) {
    if (!s || !st) return R2G_E_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    memset(st, 0, sizeof(*st));
    st->completed = s->completed;
    st->failed = s->failed;
    st->batches = s->batches;
    st->mean_batch = s->batches ? (double)s->batch_frames / s->batches : 0;
    st->mpix = s->mpix;
    st->p50_us = pct(s->lat_us, 50);
    st->p99_us = pct(s->lat_us, 99);
    double sum = 0, mx = 0;
    for (double v : s->lat_us) {
        sum += v;
        mx = std::max(mx, v);
    }
    st->mean_us = s->lat_us.empty() ? 0 : sum / s->lat_us.size();
    st->max_us = mx;
    st->span_s = s->any ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0;
    st->issue_s = s->busy_s;
    st->evictions = s->evictions;
    st->resident_bytes = s->resident;
    st->pending = (int64_t)s->pending.size();
    if (reset) {
        s->lat_us.clear();
        s->completed = s->failed = s->batches = s->batch_frames = s->evictions = 0;
        s->mpix = s->busy_s = 0;
        s->any = false;
    }
    return R2G_OK;
}

extern "C" int r2g_server_destroy(R2gServer *s) {
    if (!s) return R2G_E_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_one();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->down);
    for (auto &kv : s->streams) {
        free_stream_frames(s, kv.second);
        delete kv.second;
    }
    for (auto &kv : s->reqs) delete kv.second;
    for (Batch *b : s->free_batches) {
        cudaEventDestroy(b->done);
        delete b;
    }
    cudaEventDestroy(s->computed);
    cudaStreamDestroy(s->up);
    cudaStreamDestroy(s->down);
    delete s;
    return R2G_OK;
}
