// Shared device-side definitions of the B200 in-loop filter library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rav2d_gpu.h"

#define R2G_HD __host__ __device__ __forceinline__
#define R2G_D __device__ __forceinline__

// Per-stage work counters of the persistent stage kernels (two words: the
// next dynamic item, and CTAs finished).  A CTA takes blockIdx.x first, then
// gridDim.x + atomicAdd(next); the last CTA to finish resets both words, so
// every launch starts from zero without a memset.
struct StageSched {
    unsigned next, done;
};

// Device addresses of the AV2 constant tables (defined once in tables.cu).
struct DevTables {
    const int8_t *CDEF_DIRECTIONS;          // [12][2]
    const uint16_t *CCSO_QUANT_SZ;          // [4][4]
    const int8_t *CCSO_OFFSET;              // [4][8]
    const int16_t *DEBLOCK_SIDE_THRESHOLDS; // [296]
    const int16_t *PC_WIENER_FILTERS;       // [4][64][13]
    const uint8_t *PC_WIENER_SUB_CLASSIFY;  // [4][256]
    const uint8_t *PC_WIENER_SUB_CLASSIFY_NS;  // [4][7][256]
    const int16_t *GAUSSIAN_SEQUENCE;       // [2048]
    const uint8_t *PC_WIENER_LUT_TO_CLASS;  // [4096]
    const uint16_t *GDF_ALPHA;              // [3168]
    const int16_t *GDF_WEIGHT;              // [9504]
    const int16_t *GDF_BIAS;                // [36][3]
    const int8_t *GDF_INTRA_ERROR;          // [24576]
    const int8_t *GDF_INTER_ERROR;          // [30000]
    const uint8_t *BLOCK_DIMENSIONS;        // [31][4]
    const uint8_t *TXFM_DIMENSIONS;         // [25][8]
    const uint8_t *MAX_TXFM_SIZE_FOR_BS;    // [31][4]
    const int8_t *TX_PART_TBL;              // [31][8]
};
// Fills `t` with this device's table addresses (the current device).
cudaError_t r2g_get_tables(DevTables *t);

// Frame descriptor handed to every stage kernel (by value, or from a device
// array in batched launches).  All derived per-frame scalars of the
// reference's LoopFilterState are computed once on the host.
// Staged form of one R2gAv2RestorationUnit: its type and the (at most 18)
// NS-Wiener taps the filters read; a SB256's 3 x 16 units take 960 bytes on
// the device instead of 24624.
struct LrUnitPacked {
    uint8_t type;
    int8_t f[18];
    uint8_t pad;
};
struct LrPacked {
    LrUnitPacked lr[3][16];
};

struct DevFrame {
    int w, h;          // luma size in samples
    int cw, ch;        // chroma size in samples (4:2:0)
    int bw4, bh4;      // luma size in 4x4 units (bw, bh of the reference)
    int sb256w, sb256h, sbh;
    int bitdepth, hbd, bdmax;
    int64_t stride[2];  // in samples: luma, chroma
    void *R[3];         // recon (input, preserved)
    void *D[3];         // deblocked frame
    void *C[3];         // CDEF+CCSO output
    void *L[3];         // loop-restoration output (the filtered frame)
    void *G[3];         // film-grain display copy
    const R2gAv2Filter *masks;
    const LrPacked *lr;  // packed restoration records, one per SB256
    const uint8_t *segmap;
    const uint8_t *segmap_uv;
    int segmap_stride, segmap_uv_stride;
    uint32_t inloop;
    int deblock_on, cdef_stage_on, ccso_on, cdef_on, lr_on, any_lossless;
    int restore_planes, base_q, wiener_idx, ns_ci, gdf_ref_dst_idx;
    // tile shape of the loop-restoration work items: luma rows per item (32,
    // or 16 for four lighter items per stripe); set by the batch autotuner
    int lr_rows;
    // tile rows (loop restoration only): bit sby of tr_first is set when
    // superblock row sby > 0 starts a tile row; tr_sby lists those rows, one
    // extra 8-row stripe each (decode.rs:99-120, looprestoration.rs:2401-2548)
    uint32_t tr_first[4];
    int n_tr;
    int16_t tr_sby[64];
    // per-stage work counters of the persistent kernels (per-frame launches;
    // the batched path keeps its own) and the context's device fault word
    // (bounded waits that ran out)
    StageSched *sched;
    unsigned *fault;
    DevTables tab;
    R2gFrameParams fp;
};

R2G_HD int imin_(int a, int b) { return a < b ? a : b; }
R2G_HD int imax_(int a, int b) { return a > b ? a : b; }
R2G_HD int iclip_(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
// clip to [0, hi] (hi >= 0): max(min(v, hi), 0) as one fused instruction
R2G_D int clip_px_(int v, int hi) { return __vimin_s32_relu(v, hi); }
R2G_HD int apply_sign_(int v, int s) { return s < 0 ? -v : v; }
R2G_D int ulog2_(uint32_t v) { return 31 - __clz((int)v); }

template <typename P>
R2G_D P *plane_ptr(void *base) {
    return reinterpret_cast<P *>(base);
}

// Launch helpers implemented per stage (deblock.cu, cdef.cu, lr.cu, grain.cu).
// Arguments of the batched persistent kernels: a device array of frame
// descriptors, per-stage work lists (item = frame index << 22 | per-frame
// item index) and the per-stage item counts in device memory, so one CUDA
// graph serves every batch.  Stages: 0 deblock, 1 CDEF+CCSO, 2 loop
// restoration, 3 film-grain apply.
// Film-grain parameters of one frame (R2gFilmGrainData + seed + the planes
// the reference grains, decode.rs:4641 / filmgrain.rs:688-830).
struct GrainParams {
    R2gFilmGrainData d;
    uint32_t seed;
    int bitdepth;
    int has_y, has_u, has_v;
    // planes 16-byte aligned with 16-byte multiple strides: runs of samples
    // move with one vector access each
    int vec;
};
// One grained frame of a batch: its parameters, its frame index in the
// batch and its template / scaling-LUT scratch.
struct GrainBatch {
    GrainParams gp;
    int frame;
    int any;  // some plane is grained: the templates must be generated
    int16_t *lut;
    uint8_t *scaling;
};
struct BatchArgs {
    const DevFrame *frames;
    const uint32_t *work[4];
    const int *count;  // [0..3] items per stage, [4] grained frames
    const GrainBatch *grain;
    StageSched *sched;  // [4] work counters of the batch's stage kernels
    unsigned *fault;
};
void r2g_batch_launch_grain_template(const BatchArgs &a, int grid, cudaStream_t s);
void r2g_batch_launch_grain_apply(const BatchArgs &a, int grid, cudaStream_t s);
int r2g_batch_occupancy_grain_apply();
// Sets the grain fields of a GrainBatch from the frame's parameters.
void r2g_grain_params(const R2gFilmGrainData &fgd, uint32_t seed, int bitdepth, GrainBatch &g);
// Work items (band segments of 256 luma columns) of a grained frame.
int r2g_grain_items(int width, int height, int block_size);
void r2g_batch_launch_deblock(const BatchArgs &a, int grid, cudaStream_t s);
void r2g_batch_launch_cdef(const BatchArgs &a, int grid, cudaStream_t s);
void r2g_batch_launch_lr(const BatchArgs &a, int grid, cudaStream_t s);
int r2g_batch_occupancy_deblock();
int r2g_batch_occupancy_cdef();
int r2g_batch_occupancy_lr();
// Work-item counts of one frame per stage (0 when the stage is off).
int r2g_deblock_items(const DevFrame &f);
int r2g_cdef_items(const DevFrame &f);
int r2g_lr_items(const DevFrame &f);

// Each returns the number of kernels it launched.
int r2g_launch_deblock(const DevFrame &f, cudaStream_t s);
int r2g_launch_cdef(const DevFrame &f, cudaStream_t s);
int r2g_launch_lr(const DevFrame &f, cudaStream_t s);

struct GrainDev;  // grain.cu

// DSP-context slot launchers (dsp.cu): one block per call, on stream `s`.
void r2g_dsp_launch_cdef_filter(const uint16_t *tile, int w, int h, int edges, int pri, int sec, int dir, int damping,
                                int bitdepth, const DevTables &tab, uint16_t *out, cudaStream_t s);
void r2g_dsp_launch_cdef_dir(const uint16_t *blk, int bitdepth, uint32_t *out, cudaStream_t s);
int r2g_dsp_fg_band_max_width(int block_size, int sx);
void r2g_dsp_launch_fg_band(uint16_t *dst, const uint16_t *src, int pitch, const uint16_t *luma, int lpitch,
                            const R2gFilmGrainData &data, uint32_t in_seed, int pw, const uint8_t *scaling,
                            const int16_t *lut, int bh, int row_num, int uv, int is_id, int sx, int sy, int bitdepth,
                            cudaStream_t s);
void r2g_dsp_launch_deblock_sb64(int16_t *strip, const uint16_t vmask[4], const uint16_t ll_mask[2],
                                 const uint16_t *thr, int edge, int luma, int bitdepth, cudaStream_t s);
void r2g_dsp_launch_ccso_prep(const uint16_t *tile, int w, int h, int ss_hor, int ss_ver, int edges, int max_band_log2,
                              int ext, int quant_step, int edge_clf, int bo_only, int bitdepth, uint8_t *out,
                              cudaStream_t s);
void r2g_dsp_launch_ccso_add(uint16_t *dst, const uint8_t *idx, const uint8_t *offs, const int8_t *lut, int w, int h,
                             const uint16_t *llm, int bdmax, cudaStream_t s);
void r2g_dsp_launch_gdf_add(uint16_t *p, const int8_t *err, int w, int h, int scale, const uint16_t *llm, int bitdepth,
                            cudaStream_t s);
void r2g_dsp_launch_grain_template(const GrainParams &gp, const DevTables &tab, int16_t *lut, uint8_t *scaling,
                                   cudaStream_t s);
// Typed LR slots: staged row tables (see dsp.cu) -> one block.
void r2g_dsp_launch_wiener_y(const uint16_t *rows, int rs, int e, const int *ref, const int *cref, int w, int h,
                             int kind, const int8_t *taps, int taps_stride, const int16_t *pcf, const uint8_t *sub_lut,
                             const uint16_t *noskip, int base_q, const uint16_t *llm, int bitdepth,
                             const DevTables &tab, uint16_t *out, cudaStream_t s);
void r2g_dsp_launch_wiener_uv(const uint16_t *crows, int crs, const uint16_t *lrows, int lrs, const int *cref,
                              const int *lref, int w, int h, int ss_hor, const int8_t *f, const uint16_t *llm,
                              int bitdepth, uint16_t *out, cudaStream_t s);
void r2g_dsp_launch_gdf_prep(const uint16_t *rows, int rs, int e, const int *gref, int ng, const int *pref, int w,
                             int h, int ref_dst_idx, int qp_idx, int bitdepth, const DevTables &tab, int8_t *out,
                             cudaStream_t s);

// ---- asynchronous staging: bulk copies (TMA engine) + mbarriers ----
// A producer warp copies each work item's rows from global memory into
// shared memory with cp.async.bulk (one instruction per row, 16-byte aligned
// addresses and sizes), completing on an mbarrier that counts the bytes;
// consumer warps wait on that barrier and release the buffer through a
// second one.  Every wait is bounded (R2G_WAIT_NS): a wait that runs out
// reports failure so the kernel can record a fault and stop instead of
// spinning forever.
constexpr unsigned long long R2G_WAIT_NS = 1000000000ull;  // 1 s

R2G_D uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
R2G_D void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// makes the initialised barriers visible to the other threads and to the
// asynchronous proxy (before the CTA-wide barrier that follows it)
R2G_D void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
R2G_D void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
R2G_D void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
R2G_D bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
R2G_D uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Waits for the phase of `bar` with the given parity to complete; false when
// it has not completed within R2G_WAIT_NS.
R2G_D bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 32; i++)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > R2G_WAIT_NS) return false;
    }
}
// global -> shared bulk copy of `bytes` (multiple of 16; both addresses
// 16-byte aligned) completing on `bar`; never multicast
R2G_D void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// orders this thread's earlier shared-memory accesses before its later
// asynchronous-proxy (bulk copy) accesses
R2G_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// barrier among the first `n` threads (the consumer warps) on named barrier
// 1; returns whether `pred` was true in any of them
R2G_D bool bar_or(int pred, int n) {
    uint32_t any;
    asm volatile(
        "{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\nbar.red.or.pred q, 1, %2, p;\nselp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(any)
        : "r"(pred), "r"(n)
        : "memory");
    return any != 0;
}
R2G_D void bar_sync_n(int n) { asm volatile("bar.sync 1, %0;\n" ::"r"(n) : "memory"); }

// (StageSched: see the definition near DevFrame.)
R2G_D void sched_retire(StageSched *s) {
    __threadfence();
    if (atomicAdd(&s->done, 1u) == gridDim.x - 1) {
        atomicExch(&s->next, 0u);
        atomicExch(&s->done, 0u);
    }
}

// ---- programmatic dependent launch (per-frame kernels) ----
// A per-frame kernel is launched so that it may start while the previous
// kernel on the stream finishes: it does its prologue (work that reads only
// side-info, tables or the recon, which no kernel writes), then waits for the
// previous grid (griddepcontrol.wait: a hardware dependency, complete and
// memory-visible) before reading or writing any plane a kernel produces.
// Each of these kernels lets its own dependents launch as soon as all its
// CTAs are resident.  R2G_PDL=0 in the environment launches them plainly.
R2G_D void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
R2G_D void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::); }

bool r2g_pdl_enabled();

template <typename... Exp, typename... Act>
inline cudaError_t r2g_launch_pdl_smem(void (*kern)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                       Act &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = r2g_pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<Act &&>(args)...);
}

template <typename... Exp, typename... Act>
inline cudaError_t r2g_launch_pdl(void (*kern)(Exp...), dim3 grid, dim3 block, cudaStream_t s, Act &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = r2g_pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<Act &&>(args)...);
}
